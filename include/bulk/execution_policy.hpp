// bulk/execution_policy.hpp -- the execution-agent hierarchy of the Bulk
// programming model, mapped onto B200 (sm_100a) hardware.
//
// Same names, template signatures and meaning as the reference's
// bulk/execution_policy.hpp (agent :60-89, group_base :103-182,
// parallel_group :189-234, par :237-253 / :302-324, async_launch :256-299,
// concurrent_group :327-436, con :439-466, bounded / bound :469-521,
// cursor / root :524-625, grid :628-675), so functor code written against
// Bulk compiles unchanged.  The mapping is this library's own:
//   agent                       one CUDA thread (grainsize is a hint)
//   concurrent_group<A, S>      one CTA of S threads; wait() is a CTA barrier;
//                               the heap is the CTA's dynamic shared memory
//   concurrent_group<concurrent_group<A, S>, C>
//                               a thread-block cluster of C CTAs (C <= 16);
//                               wait() is a cluster barrier; each CTA's heap
//                               falls back to its peers' shared memory
//                               (distributed shared memory)
//   parallel_group<A>           independent agents: a grid-stride launch
//   parallel_group<concurrent_group<...>>  a grid of CTAs (or of clusters)
#pragma once

#include <climits>
#include <cstddef>
#include <type_traits>

#include <cuda_runtime.h>

namespace bulk {

static const int invalid_index = INT_MAX;
static const int use_default = INT_MAX;
static const int dynamic_group_size = 0;

template <typename T>
class future;

// A sequential execution agent: an index within its group and a static
// grainsize hint (how many elements it processes).
template <std::size_t grainsize_ = 1>
class agent {
 public:
  typedef int size_type;
  static const size_type static_grainsize = grainsize_;

  __host__ __device__ agent(size_type i = invalid_index) : m_index(i) {}
  __host__ __device__ size_type index() const { return m_index; }
  __host__ __device__ size_type grainsize() const { return static_grainsize; }

 private:
  size_type m_index;
};

namespace detail {

template <typename ExecutionAgent, std::size_t size_>
class group_base {
 public:
  typedef ExecutionAgent agent_type;
  typedef int size_type;
  static const size_type static_size = size_;

  __host__ __device__ group_base(agent_type exec = agent_type(), size_type i = invalid_index)
      : this_exec(exec), m_index(i) {}
  __host__ __device__ size_type index() const { return m_index; }
  __host__ __device__ size_type size() const { return static_size; }
  __host__ __device__ size_type global_index() const { return index() * size() + this_exec.index(); }

  agent_type this_exec;

 private:
  size_type m_index;
};

template <typename ExecutionAgent>
class group_base<ExecutionAgent, dynamic_group_size> {
 public:
  typedef ExecutionAgent agent_type;
  typedef int size_type;

  __host__ __device__ group_base(size_type sz, agent_type exec = agent_type(), size_type i = invalid_index)
      : this_exec(exec), m_size(sz), m_index(i) {}
  __host__ __device__ size_type index() const { return m_index; }
  __host__ __device__ size_type size() const { return m_size; }
  __host__ __device__ size_type global_index() const { return index() * size() + this_exec.index(); }

  agent_type this_exec;

 private:
  size_type m_size;
  size_type m_index;
};

int sm_count();  // defined in bulk/async.hpp (host only)

}  // namespace detail

// A group of independent agents.
template <typename ExecutionAgent = agent<>, std::size_t size_ = dynamic_group_size>
class parallel_group : public detail::group_base<ExecutionAgent, size_> {
  typedef detail::group_base<ExecutionAgent, size_> super_t;

 public:
  typedef typename super_t::agent_type agent_type;
  typedef typename super_t::size_type size_type;
  __host__ __device__ parallel_group(agent_type exec = agent_type(), size_type i = invalid_index)
      : super_t(exec, i) {}
};

template <typename ExecutionAgent>
class parallel_group<ExecutionAgent, dynamic_group_size>
    : public detail::group_base<ExecutionAgent, dynamic_group_size> {
  typedef detail::group_base<ExecutionAgent, dynamic_group_size> super_t;

 public:
  typedef typename super_t::agent_type agent_type;
  typedef typename super_t::size_type size_type;
  __host__ __device__ parallel_group(size_type size, agent_type exec = agent_type(), size_type i = invalid_index)
      : super_t(size, exec, i) {}
};

inline __host__ __device__ parallel_group<> par(size_t size) {
  return parallel_group<>(static_cast<parallel_group<>::size_type>(size));
}

template <typename ExecutionAgent>
inline __host__ __device__ parallel_group<ExecutionAgent> par(ExecutionAgent exec, size_t size) {
  return parallel_group<ExecutionAgent>(static_cast<int>(size), exec);
}

// A policy bound to a stream, or ordered after an event.
template <typename ExecutionGroup>
class async_launch {
 public:
  __host__ __device__ async_launch(ExecutionGroup exec, cudaStream_t s, cudaEvent_t be = 0)
      : stream_valid(true), e(exec), s(s), be(be) {}
  __host__ async_launch(ExecutionGroup exec, cudaEvent_t be) : stream_valid(false), e(exec), s(0), be(be) {}
  __host__ __device__ ExecutionGroup exec() const { return e; }
  __host__ __device__ cudaStream_t stream() const { return s; }
  __host__ __device__ cudaEvent_t before_event() const { return be; }
  __host__ __device__ bool is_stream_valid() const { return stream_valid; }

 private:
  bool stream_valid;
  ExecutionGroup e;
  cudaStream_t s;
  cudaEvent_t be;
};

inline __host__ __device__ async_launch<parallel_group<>> par(cudaStream_t s, size_t num_threads) {
  return async_launch<parallel_group<>>(par(num_threads), s);
}

template <typename ExecutionAgent>
inline __host__ __device__ async_launch<parallel_group<ExecutionAgent>> par(cudaStream_t s, ExecutionAgent exec,
                                                                           size_t num_groups) {
  return async_launch<parallel_group<ExecutionAgent>>(par(exec, num_groups), s);
}

inline async_launch<parallel_group<>> par(future<void> &before, size_t num_threads);  // bulk/future.hpp

// A group of agents that may synchronise with wait(): one CTA.
template <typename ExecutionAgent = agent<>, std::size_t size_ = dynamic_group_size>
class concurrent_group : public parallel_group<ExecutionAgent, size_> {
  typedef parallel_group<ExecutionAgent, size_> super_t;

 public:
  typedef typename super_t::agent_type agent_type;
  typedef typename super_t::size_type size_type;

  __host__ __device__ concurrent_group(size_type heap_size = use_default, agent_type exec = agent_type(),
                                       size_type i = invalid_index)
      : super_t(exec, i), m_heap_size(heap_size) {}

  // all agents of the group reach this point before any continues
  __device__ void wait() const { __syncthreads(); }

  __host__ __device__ size_type heap_size() const { return m_heap_size; }

  // number of SMs: groups that run at once, one per SM
  __host__ static size_type hardware_concurrency() { return detail::sm_count(); }

 private:
  size_type m_heap_size;
};

template <typename ExecutionAgent>
class concurrent_group<ExecutionAgent, dynamic_group_size>
    : public parallel_group<ExecutionAgent, dynamic_group_size> {
  typedef parallel_group<ExecutionAgent, dynamic_group_size> super_t;

 public:
  typedef typename super_t::agent_type agent_type;
  typedef typename super_t::size_type size_type;

  __host__ __device__ concurrent_group(size_type size, size_type heap_size = use_default,
                                       agent_type exec = agent_type(), size_type i = invalid_index)
      : super_t(size, exec, i), m_heap_size(heap_size) {}

  __device__ void wait() const { __syncthreads(); }
  __host__ __device__ size_type heap_size() const { return m_heap_size; }
  __host__ static size_type hardware_concurrency() { return detail::sm_count(); }

 private:
  size_type m_heap_size;
};

namespace detail {
// Barrier over every thread of the thread-block cluster, with release /
// acquire semantics (shared and distributed shared memory writes before it
// are visible after it).
__device__ inline void cluster_barrier() {
#ifdef __CUDA_ARCH__
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
#endif
}
__device__ inline unsigned int cluster_ctarank() {
  unsigned int r = 0;
#ifdef __CUDA_ARCH__
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
#endif
  return r;
}
__device__ inline unsigned int cluster_nctarank() {
  unsigned int r = 1;
#ifdef __CUDA_ARCH__
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
#endif
  return r;
}
}  // namespace detail

// A concurrent group of C concurrent groups: one thread-block cluster of C
// CTAs, each CTA one inner group.  this_exec is the executing CTA's group
// (its index() is the CTA's rank in the cluster), index() is the cluster's
// index in its grid, wait() synchronises every agent of every CTA.
template <typename InnerAgent, std::size_t inner_size, std::size_t size_>
class concurrent_group<concurrent_group<InnerAgent, inner_size>, size_>
    : public parallel_group<concurrent_group<InnerAgent, inner_size>, size_> {
  typedef parallel_group<concurrent_group<InnerAgent, inner_size>, size_> super_t;
  static_assert(size_ >= 1 && size_ <= 16, "a cluster holds 1 to 16 CTAs");

 public:
  typedef typename super_t::agent_type agent_type;
  typedef typename super_t::size_type size_type;

  __host__ __device__ concurrent_group(agent_type exec = agent_type(), size_type i = invalid_index)
      : super_t(exec, i) {}

  __device__ void wait() const { detail::cluster_barrier(); }
  // the heap of each CTA (its dynamic shared memory)
  __host__ __device__ size_type heap_size() const { return this->this_exec.heap_size(); }
  // clusters of this size that run at once on the whole GPU (occupancy)
  __host__ static size_type hardware_concurrency() { return detail::sm_count() / size_; }
};

inline __host__ __device__ concurrent_group<> con(size_t size, size_t heap_size = use_default) {
  return concurrent_group<>(static_cast<int>(size), static_cast<int>(heap_size));
}

template <typename ExecutionAgent>
inline __host__ __device__ concurrent_group<ExecutionAgent> con(ExecutionAgent exec, size_t size,
                                                                size_t heap_size = use_default) {
  return concurrent_group<ExecutionAgent>(static_cast<int>(size), static_cast<int>(heap_size), exec);
}

template <std::size_t groupsize, std::size_t grainsize>
inline __host__ __device__ concurrent_group<agent<grainsize>, groupsize> con(size_t heap_size) {
  return concurrent_group<agent<grainsize>, groupsize>(static_cast<int>(heap_size));
}

// A view of an execution agent or group with a static upper bound on the
// work it does (enables fully unrolled, register-resident loops).
// A cluster of C concurrent groups (CTAs) of `inner` agents each.
template <std::size_t C, typename InnerAgent, std::size_t S>
inline __host__ __device__ concurrent_group<concurrent_group<InnerAgent, S>, C> cluster(
    concurrent_group<InnerAgent, S> inner) {
  return concurrent_group<concurrent_group<InnerAgent, S>, C>(inner);
}

template <std::size_t bound_, typename ExecutionAgent>
class bounded : public ExecutionAgent {
 public:
  typedef typename ExecutionAgent::size_type size_type;
  static const size_type static_bound = bound_;
  __host__ __device__ size_type bound() const { return static_bound; }
  __host__ __device__ ExecutionAgent &unbound() { return *this; }
  __host__ __device__ const ExecutionAgent &unbound() const { return *this; }

 private:
  bounded();
  bounded(const bounded &);
};

template <std::size_t bound_, typename ExecutionAgent>
__host__ __device__ bounded<bound_, ExecutionAgent> &bound(ExecutionAgent &exec) {
  return static_cast<bounded<bound_, ExecutionAgent> &>(exec);
}
template <std::size_t bound_, typename ExecutionAgent>
__host__ __device__ const bounded<bound_, ExecutionAgent> &bound(const ExecutionAgent &exec) {
  return static_cast<const bounded<bound_, ExecutionAgent> &>(exec);
}

namespace detail {

template <unsigned int depth, typename ExecutionAgent>
struct agent_at_depth {
  typedef typename agent_at_depth<depth - 1, ExecutionAgent>::type::agent_type type;
};
template <typename ExecutionAgent>
struct agent_at_depth<0, ExecutionAgent> {
  typedef ExecutionAgent type;
};

// Placeholders for the live execution hierarchy inside bulk::async:
// root is the launched group, root.this_exec its agent, and so on.
template <unsigned int d>
struct cursor {
  static const unsigned int depth = d;
  __host__ __device__ cursor() {}
  cursor<d + 1> this_exec;
  template <typename ExecutionGroup>
  static __host__ __device__ typename agent_at_depth<d, ExecutionGroup>::type &get(ExecutionGroup &root) {
    return cursor<d - 1>::get(root.this_exec);
  }
};
template <>
struct cursor<3> {
  static const unsigned int depth = 3;
  __host__ __device__ cursor() {}
  template <typename ExecutionGroup>
  static __host__ __device__ typename agent_at_depth<3, ExecutionGroup>::type &get(ExecutionGroup &root) {
    return cursor<2>::get(root.this_exec);
  }
};
template <>
struct cursor<0> {
  static const unsigned int depth = 0;
  __host__ __device__ cursor() {}
  cursor<1> this_exec;
  template <typename ExecutionGroup>
  static __host__ __device__ ExecutionGroup &get(ExecutionGroup &root) {
    return root;
  }
};

template <typename T>
struct is_cursor : std::false_type {};
template <unsigned int d>
struct is_cursor<cursor<d>> : std::true_type {};

}  // namespace detail

#ifdef __CUDA_ARCH__
static const __device__ detail::cursor<0> root;
#else
static const detail::cursor<0> root;
#endif

inline __host__ __device__ parallel_group<concurrent_group<>> grid(size_t num_groups = use_default,
                                                                  size_t group_size = use_default,
                                                                  size_t heap_size = use_default) {
  return par(con(group_size, heap_size), num_groups);
}

inline __host__ __device__ async_launch<parallel_group<concurrent_group<>>> grid(size_t num_groups, size_t group_size,
                                                                                size_t heap_size, cudaStream_t stream) {
  return async_launch<parallel_group<concurrent_group<>>>(grid(num_groups, group_size, heap_size), stream);
}

template <std::size_t groupsize, std::size_t grainsize>
inline __host__ __device__ parallel_group<concurrent_group<agent<grainsize>, groupsize>> grid(
    size_t num_groups, size_t heap_size = use_default) {
  return par(con<groupsize, grainsize>(heap_size), num_groups);
}

template <std::size_t groupsize, std::size_t grainsize>
inline __host__ __device__ async_launch<parallel_group<concurrent_group<agent<grainsize>, groupsize>>> grid(
    size_t num_groups, size_t heap_size, cudaStream_t stream) {
  return async_launch<parallel_group<concurrent_group<agent<grainsize>, groupsize>>>(
      grid<groupsize, grainsize>(num_groups, heap_size), stream);
}

}  // namespace bulk
