// ref_group.cpp -- TEST INFRASTRUCTURE ONLY.  The reference's cooperative
// group algorithms (concurrent_group<agent<3>, 4>) run on the host with one
// std::thread per agent and a std::barrier standing in for wait()
// (__syncthreads), so the group code executes exactly as written.  Used to pin
// the oracle against the reference's own group reduce, scan, block sort,
// merge_by_key and reduce_by_key.  Built by oracle/ref/build_ref.py (which
// compiles this file with __shared__ mapped to static storage: groups run one
// at a time, so static storage plays the part of a CTA's shared memory).
//
// Reference pieces used (jaredhoberock/bulk):
//   concurrent_group                      bulk/execution_policy.hpp:327-436
//   bulk::reduce(group, ...)              bulk/algorithm/reduce.hpp:110-219
//   bulk::inclusive_scan(group, ...)      bulk/algorithm/scan.hpp:455-486
//   bulk::stable_sort_by_key(bounded g)   bulk/algorithm/sort.hpp:152-166
//   bulk::merge_by_key(bounded g, ...)    bulk/algorithm/merge.hpp:507-607
//   bulk::reduce_by_key(group, ...)       bulk/algorithm/reduce_by_key.hpp:115-216
#include <barrier>
#include <cstdint>
#include <thread>
#include <vector>

#include <bulk/execution_policy.hpp>

static std::barrier<> *g_bar = nullptr;

BULK_NAMESPACE_PREFIX
namespace bulk {
// The host stand-in for a CTA of 4 agents: wait() is a std::barrier.
template <>
class concurrent_group<agent<3>, 4> : public parallel_group<agent<3>, 4> {
 public:
  typedef parallel_group<agent<3>, 4> super_t;
  typedef super_t::agent_type agent_type;
  typedef super_t::size_type size_type;
  concurrent_group(size_type heap = use_default, agent_type e = agent_type(), size_type i = invalid_index)
      : super_t(e, i), m_heap(heap) {}
  void wait() const { g_bar->arrive_and_wait(); }
  size_type heap_size() const { return m_heap; }
  static size_type hardware_concurrency() { return 1; }

 private:
  size_type m_heap;
};
}  // namespace bulk
BULK_NAMESPACE_SUFFIX

#include <bulk/bulk.hpp>
#include <thrust/functional.h>

namespace bulk {
namespace detail {
int s_data_segment_begin[1 << 16];  // the "dynamic shared memory" heap of the group
}
}  // namespace bulk

namespace {

typedef bulk::concurrent_group<bulk::agent<3>, 4> group_t;
constexpr int kGroup = 4;

template <typename F>
void run_group(F f) {
  std::barrier<> bar(kGroup);
  g_bar = &bar;
  bulk::detail::init_on_chip_malloc(sizeof(bulk::detail::s_data_segment_begin));
  std::vector<std::thread> ts;
  for (int t = 0; t < kGroup; ++t)
    ts.emplace_back([&, t] {
      group_t g(sizeof(bulk::detail::s_data_segment_begin), bulk::agent<3>(t), 0);
      f(g);
    });
  for (auto &t : ts) t.join();
  g_bar = nullptr;
}

}  // namespace

#define BKREF_API extern "C" __attribute__((visibility("default")))

BKREF_API int32_t bkref_group_reduce_i32(const int32_t *x, int64_t n, int32_t init) {
  int32_t r = 0;
  run_group([&](group_t &g) {
    const int32_t s = bulk::reduce(g, x, x + n, init, thrust::plus<int32_t>());
    if (g.this_exec.index() == 0) r = s;
  });
  return r;
}

BKREF_API void bkref_group_inclusive_scan_i32(const int32_t *x, int64_t n, int32_t init, int32_t *out) {
  run_group([&](group_t &g) { bulk::inclusive_scan(g, x, x + n, out, init, thrust::plus<int32_t>()); });
}

// A single-interval reduce_by_key_kernel (reduce_by_key.cu:16-130): the first
// pair seeds the carry, the group reduces the rest, and the final carry is the
// last run.  Returns the number of runs.
BKREF_API int64_t bkref_group_reduce_by_key_i32_i32(const int32_t *keys, const int32_t *vals, int64_t n,
                                                    int32_t *out_keys, int32_t *out_vals) {
  if (n <= 0) return 0;
  int64_t count = 0;
  run_group([&](group_t &g) {
    auto r = bulk::reduce_by_key(g, keys + 1, keys + n, vals + 1, out_keys, out_vals, keys[0], vals[0],
                                 thrust::equal_to<int32_t>(), thrust::plus<int32_t>());
    if (g.this_exec.index() == 0) {
      int32_t *k_end = thrust::get<0>(r);
      int32_t *v_end = thrust::get<1>(r);
      *k_end = thrust::get<2>(r);
      *v_end = thrust::get<3>(r);
      count = (k_end - out_keys) + 1;
    }
  });
  return count;
}

// The bounded group block sort of one tile (n <= 12).
BKREF_API void bkref_group_stable_sort_by_key_i32_i32(int32_t *keys, int32_t *vals, int64_t n) {
  run_group([&](group_t &g) {
    bulk::stable_sort_by_key(bulk::bound<12>(g), keys, keys + n, vals, thrust::less<int32_t>());
  });
}

// The bounded group merge_by_key of two sorted runs (na + nb <= 12).
BKREF_API void bkref_group_merge_by_key_i32_i32(const int32_t *ak, const int32_t *av, int64_t na,
                                                const int32_t *bk, const int32_t *bv, int64_t nb, int32_t *ok,
                                                int32_t *ov) {
  run_group([&](group_t &g) {
    bulk::merge_by_key(bulk::bound<12>(g), ak, ak + na, bk, bk + nb, av, bv, ok, ov, thrust::less<int32_t>());
  });
}
