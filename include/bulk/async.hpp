// bulk/async.hpp -- bulk::async(policy, f, args...): launch f across an
// execution hierarchy and return a future.
//
// Interface of the reference's bulk::async (bulk/async.hpp:31-83,
// bulk/detail/async.inl:32-190): placeholders among args (bulk::root,
// bulk::root.this_exec, ...) are replaced inside the kernel by the live
// group / agent, other args are passed by value; a stream policy launches
// into that stream, a future policy into a new stream ordered after the
// future, anything else into the legacy default stream.  The launch layer is
// this library's own (in place of cuda_launcher / choose_sizes):
//   parallel_group<agent<G>> of n agents   grid-stride loop, 256-thread CTAs,
//                                          at most as many CTAs as are resident
//                                          at once
//   concurrent_group<agent<G>, S>          one CTA of S threads
//   parallel_group<concurrent_group<...>>  n CTAs of S threads; an unspecified
//                                          n is the number resident at once
// "Resident at once" is the CUDA runtime's occupancy model of the kernel as
// compiled for this functor (its registers, static and dynamic shared
// memory) times the SM count, so grids follow each kernel instead of a fixed
// table (the reference sizes them by a pre-Maxwell occupancy calculator,
// bulk/detail/cuda_launcher/cuda_launch_config.hpp:240-379).
// Concurrent groups get a dynamic shared-memory heap (bulk/malloc.hpp): the
// requested heap size, or by default the share of an SM's shared memory that
// keeps every group that fits by threads resident (opted in above 48 KB).
// Device properties are cached once per device (thread-safe).
#pragma once

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <tuple>

#include <cuda/std/tuple>
#include <type_traits>
#include <utility>

#include <cuda_runtime.h>

#include "execution_policy.hpp"
#include "future.hpp"
#include "malloc.hpp"

namespace bulk {
namespace detail {

struct device_props {
  int sm_count;
  int max_smem_optin;  // bytes per CTA
  int smem_per_sm;
  int max_threads_per_sm;
};

inline device_props device_properties() {
  static std::once_flag once[64];
  static device_props props[64];
  int dev = 0;
  throw_on_error(cudaGetDevice(&dev), "bulk: cudaGetDevice");
  if (dev < 0 || dev >= 64) throw_on_error(cudaErrorInvalidDevice, "bulk: device index out of range");
  std::call_once(once[dev], [dev]() {
    device_props p{};
    cudaDeviceGetAttribute(&p.sm_count, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&p.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&p.smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&p.max_threads_per_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    props[dev] = p;
  });
  return props[dev];
}

inline int sm_count() { return device_properties().sm_count; }

// ---- placeholder substitution --------------------------------------------
template <typename Root, typename T>
__device__ __forceinline__ decltype(auto) substitute(Root &root, T &arg) {
  if constexpr (is_cursor<std::remove_cv_t<T>>::value) {
    return std::remove_cv_t<T>::get(root);
  } else {
    return (arg);
  }
}

template <typename Root, typename F, typename Tuple, std::size_t... I>
__device__ __forceinline__ void invoke(Root &root, F &f, Tuple &args, std::index_sequence<I...>) {
  f(substitute(root, cuda::std::get<I>(args))...);
}

// ---- group construction helpers ---------------------------------------------
template <typename A, std::size_t S>
__host__ __device__ concurrent_group<A, S> make_group(const concurrent_group<A, S> &proto, A exec, int index) {
  if constexpr (S == dynamic_group_size) return concurrent_group<A, S>(proto.size(), proto.heap_size(), exec, index);
  else return concurrent_group<A, S>(proto.heap_size(), exec, index);
}

template <typename T>
struct is_concurrent_group : std::false_type {};
template <typename A, std::size_t S>
struct is_concurrent_group<concurrent_group<A, S>> : std::true_type {};

template <typename A, std::size_t S>
__host__ __device__ concurrent_group<A, S> make_group_size(const concurrent_group<A, S> &g, int size, int heap) {
  if constexpr (S == dynamic_group_size) return concurrent_group<A, S>(size, heap, g.this_exec, g.index());
  else return concurrent_group<A, S>(heap, g.this_exec, g.index());
}


// ---- kernels ---------------------------------------------------------------
template <typename Agent, typename F, typename... Args>
__global__ void async_parallel_agents(int n, F f, Args... args) {
  cuda::std::tuple<Args...> a(args...);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    parallel_group<Agent> g(n, Agent(i), 0);
    invoke(g, f, a, std::index_sequence_for<Args...>());
  }
}

template <typename Group, typename F, typename... Args>
__global__ void async_concurrent_group(Group proto, unsigned int heap_bytes, F f, Args... args) {
  if (threadIdx.x == 0) heap_init(heap_bytes);
  __syncthreads();
  cuda::std::tuple<Args...> a(args...);
  typedef typename Group::agent_type agent_type;
  Group g = make_group(proto, agent_type(threadIdx.x), 0);
  invoke(g, f, a, std::index_sequence_for<Args...>());
}

template <typename Group, typename F, typename... Args>
__global__ void async_grid_of_groups(int num_groups, Group proto, unsigned int heap_bytes, F f, Args... args) {
  if (threadIdx.x == 0) heap_init(heap_bytes);
  __syncthreads();
  cuda::std::tuple<Args...> a(args...);
  typedef typename Group::agent_type agent_type;
  parallel_group<Group> root(num_groups, make_group(proto, agent_type(threadIdx.x), blockIdx.x), 0);
  invoke(root, f, a, std::index_sequence_for<Args...>());
}

template <typename T>
struct is_cluster_group : std::false_type {};
template <typename A, std::size_t S, std::size_t C>
struct is_cluster_group<concurrent_group<concurrent_group<A, S>, C>> : std::true_type {};

// A grid of clusters (AS_GRID: the root is parallel_group<Cluster> of
// num_clusters clusters) or one cluster (the cluster group is the root).
// Every CTA initialises its heap and the cluster meets once before the
// functor runs (a peer may allocate from this CTA's heap) and once after it
// (no CTA leaves while a peer may still use its shared memory).
template <bool AS_GRID, typename Cluster, typename F, typename... Args>
__global__ void async_cluster_groups(int num_clusters, Cluster proto, unsigned int heap_bytes, F f, Args... args) {
  if (threadIdx.x == 0) heap_init(heap_bytes);
  cluster_barrier();
  {
    cuda::std::tuple<Args...> a(args...);
    typedef typename Cluster::agent_type cta_type;
    typedef typename cta_type::agent_type agent_type;
    const int rank = (int)cluster_ctarank();
    const int cluster_index = (int)(blockIdx.x / cluster_nctarank());
    cta_type cta = make_group(proto.this_exec, agent_type(threadIdx.x), rank);
    Cluster cl(cta, cluster_index);
    if constexpr (AS_GRID) {
      parallel_group<Cluster> root(num_clusters, cl, 0);
      invoke(root, f, a, std::index_sequence_for<Args...>());
    } else {
      invoke(cl, f, a, std::index_sequence_for<Args...>());
    }
  }
  cluster_barrier();
}

// Default heap: the share of an SM's shared memory that keeps every group
// that fits by thread count resident.
inline unsigned int choose_heap(int group_size, int requested) {
  const device_props p = device_properties();
  if (requested != use_default) return (unsigned int)requested;
  const int per_sm = std::max(1, std::min(32, p.max_threads_per_sm / std::max(group_size, 1)));
  int bytes = (p.smem_per_sm - 1024 * per_sm) / per_sm;
  bytes = std::min(bytes, p.max_smem_optin);
  return (unsigned int)(std::max(bytes, 0) / 1024 * 1024);
}

template <typename Kernel>
inline void opt_in_smem(Kernel k, unsigned int bytes) {
  if (bytes > 48 * 1024)
    throw_on_error(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
                   "bulk::async: shared memory opt-in");
}

inline int default_group_size(int requested) { return requested == use_default ? 256 : requested; }

// CTAs of kernel k one SM holds at once with `threads` threads and `smem`
// bytes of dynamic shared memory (at least 1).
template <typename Kernel>
inline int resident_per_sm(Kernel k, int threads, size_t smem) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem) != cudaSuccess || per_sm < 1) {
    (void)cudaGetLastError();  // a failed query leaves no sticky error behind
    per_sm = 1;
  }
  return per_sm;
}

// Launches `num_clusters` clusters of C CTAs (grid = num_clusters * C) with
// cudaLaunchKernelEx and a cluster dimension; above 8 CTAs per cluster the
// kernel is opted into non-portable cluster sizes.  num_clusters == 0 asks
// for the number of clusters resident at once (occupancy of this kernel).
template <bool AS_GRID, typename Cluster, typename F, typename... Args>
void launch_clusters(int num_clusters, const Cluster &g_in, cudaStream_t s, F f, Args... args) {
  constexpr int C = (int)Cluster::static_size;
  typedef typename Cluster::agent_type cta_type;
  const cta_type &inner = g_in.this_exec;
  const int size = default_group_size(inner.size());
  const unsigned int heap = choose_heap(size, inner.heap_size());
  Cluster proto(make_group_size(inner, size, (int)heap), 0);
  auto k = async_cluster_groups<AS_GRID, Cluster, F, Args...>;
  opt_in_smem(k, heap);
  if (C > 8)
    throw_on_error(cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1),
                   "bulk::async: non-portable cluster size");
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(size);
  cfg.dynamicSmemBytes = heap;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (num_clusters == use_default) {
    cfg.gridDim = dim3(C);
    int resident = 0;
    throw_on_error(cudaOccupancyMaxActiveClusters(&resident, k, &cfg), "bulk::async: cluster occupancy");
    num_clusters = resident > 0 ? resident : 1;
  }
  if (num_clusters <= 0) return;
  cfg.gridDim = dim3((unsigned)num_clusters * C);
  throw_on_error(cudaLaunchKernelEx(&cfg, k, num_clusters, proto, heap, f, args...),
                 "bulk::async: cluster launch");
}

// ---- launch into a stream ----------------------------------------------------
template <typename Agent, std::size_t N, typename F, typename... Args>
void launch(const parallel_group<Agent, N> &g, cudaStream_t s, F f, Args... args) {
  if constexpr (is_cluster_group<Agent>::value) {
    // a grid of clusters
    launch_clusters<true>(g.size(), g.this_exec, s, f, args...);
    return;
  } else if constexpr (is_concurrent_group<Agent>::value) {
    // a grid of concurrent groups (one CTA each)
    const Agent &proto_in = g.this_exec;
    const int size = default_group_size(proto_in.size());
    const unsigned int heap = choose_heap(size, proto_in.heap_size());
    Agent proto = make_group_size(proto_in, size, (int)heap);
    auto k = async_grid_of_groups<Agent, F, Args...>;
    opt_in_smem(k, heap);
    int num_groups = g.size();
    if (num_groups == use_default) num_groups = device_properties().sm_count * resident_per_sm(k, size, heap);
    if (num_groups > 0) k<<<num_groups, size, heap, s>>>(num_groups, proto, heap, f, args...);
  } else {
    const int n = g.size();
    const int threads = 256;
    auto k = async_parallel_agents<Agent, F, Args...>;
    const int resident = device_properties().sm_count * resident_per_sm(k, threads, 0);
    const int blocks = std::max(1, std::min((n + threads - 1) / threads, resident));
    if (n > 0) k<<<blocks, threads, 0, s>>>(n, f, args...);
  }
  throw_on_error(cudaGetLastError(), "bulk::async: launch");
}

// one cluster of C CTAs
template <typename A, std::size_t S, std::size_t C, typename F, typename... Args>
void launch(const concurrent_group<concurrent_group<A, S>, C> &g, cudaStream_t s, F f, Args... args) {
  launch_clusters<false>(1, g, s, f, args...);
}

template <typename A, std::size_t S, typename F, typename... Args>
void launch(const concurrent_group<A, S> &g_in, cudaStream_t s, F f, Args... args) {
  const int size = default_group_size(g_in.size());
  const unsigned int heap = choose_heap(size, g_in.heap_size());
  concurrent_group<A, S> g = make_group_size(g_in, size, (int)heap);
  auto k = async_concurrent_group<concurrent_group<A, S>, F, Args...>;
  opt_in_smem(k, heap);
  k<<<1, size, heap, s>>>(g, heap, f, args...);
  throw_on_error(cudaGetLastError(), "bulk::async: launch");
}

}  // namespace detail

// Launch f(args...) across the agents of `g` in the legacy default stream.
template <typename ExecutionGroup, typename F, typename... Args>
future<void> async(ExecutionGroup g, F f, Args... args) {
  detail::launch(g, cudaStream_t(0), f, args...);
  return detail::future_core_access::create(cudaStream_t(0), false);
}

// Launch into a stream, or after a future (into a new stream the future owns).
template <typename ExecutionGroup, typename F, typename... Args>
future<void> async(async_launch<ExecutionGroup> policy, F f, Args... args) {
  cudaStream_t s = policy.stream();
  bool owns = false;
  if (!policy.is_stream_valid()) {
    detail::throw_on_error(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "bulk::async: stream");
    owns = true;
  }
  if (policy.before_event()) detail::throw_on_error(cudaStreamWaitEvent(s, policy.before_event(), 0),
                                                    "bulk::async: wait event");
  detail::launch(policy.exec(), s, f, args...);
  return detail::future_core_access::create(s, owns);
}

// The group count and size bulk::async would choose for a grid of
// concurrent groups running f(args...) (replaces the reference's
// occupancy-based choose_sizes, bulk/choose_sizes.hpp:29-75): an unspecified
// size becomes 256 threads per group, an unspecified count the number of
// such groups resident at once under the runtime's occupancy model of this
// kernel with its heap.
template <typename F, typename... Args>
std::pair<int, int> choose_sizes(parallel_group<concurrent_group<>> g, F, Args...) {
  const int size = detail::default_group_size(g.this_exec.size());
  int num = g.size();
  if (num == use_default) {
    const unsigned int heap = detail::choose_heap(size, g.this_exec.heap_size());
    auto k = detail::async_grid_of_groups<concurrent_group<>, F, Args...>;
    detail::opt_in_smem(k, heap);
    num = detail::device_properties().sm_count * detail::resident_per_sm(k, size, heap);
  }
  return std::make_pair(num, size);
}

}  // namespace bulk
