// ref_agent.cpp -- TEST INFRASTRUCTURE ONLY.  The reference's own sequential
// (agent-level) algorithms, compiled for the host from the reference's headers,
// driven over the decompositions the reference's device-wide drivers use.  It
// serves as the timed CPU baseline ("the reference's algorithms compiled for
// the host") and as a second check of the oracle.  Built by oracle/ref/build_ref.py
// into oracle/_ref/libbulkref.so; nothing in the product loads it.
//
// Reference pieces used (jaredhoberock/bulk):
//   bulk::reduce(bounded<B, agent<G>>, ...)          bulk/algorithm/reduce.hpp:33-58
//   bulk::inclusive_scan(bounded<B, agent<G>>, ...)  bulk/algorithm/scan.hpp:35-56
//   bulk::merge_path / bulk::merge(bounded agent)    bulk/algorithm/merge.hpp:35-170
//   aligned_decomposition                            decomposition.hpp:142-210
// The partition structure follows my_reduce (reduce.cu:58-97: the partition's
// last element is its init, partial sums folded with the last partial as init)
// and the three-pass ::inclusive_scan (scan.cu:87-148).
#include <bulk/bulk.hpp>
#include <thrust/functional.h>

#include <cstdint>
#include <thread>
#include <vector>

#include "decomposition.hpp"

namespace {

constexpr std::size_t kTile = 896;  // 128 x 7, the drivers' reduce tile

template <typename T>
T agent_reduce(const T *first, const T *last, T init) {
  bulk::agent<7> a(0);
  while (first < last) {
    const T *e = last - first > (std::ptrdiff_t)kTile ? first + kTile : last;
    init = bulk::reduce(bulk::bound<kTile>(a), first, e, init, thrust::plus<T>());
    first = e;
  }
  return init;
}

template <typename T>
void agent_inclusive_scan(const T *first, const T *last, T *result, T init) {
  bulk::agent<7> a(0);
  while (first < last) {
    const T *e = last - first > (std::ptrdiff_t)kTile ? first + kTile : last;
    bulk::inclusive_scan(bulk::bound<kTile>(a), first, e, result, init, thrust::plus<T>());
    init = result[(e - first) - 1];
    result += e - first;
    first = e;
  }
}

template <typename F>
void parallel_for(int parts, F f) {
  std::vector<std::thread> ts;
  for (int p = 1; p < parts; ++p) ts.emplace_back(f, p);
  f(0);
  for (auto &t : ts) t.join();
}

// my_reduce on host threads: partition p folds [first, last) of its aligned
// range (p > 0 uses its last element as init), then the partials are folded
// with the last partial as init.
template <typename T>
T cpu_reduce(const T *x, int64_t n, T init, int threads) {
  if (n <= 0) return init;
  const int64_t tiles = (n + kTile - 1) / kTile;
  const int64_t parts = std::min<int64_t>(threads, tiles);
  aligned_decomposition<int64_t> decomp(n, parts, kTile);
  std::vector<T> partial(parts);
  parallel_for((int)parts, [&](int p) {
    auto r = decomp[p];
    const T *first = x + r.first, *last = x + r.second;
    T in = init;
    if (p != 0) in = *--last;
    partial[p] = agent_reduce(first, last, in);
  });
  if (parts == 1) return partial[0];
  return agent_reduce(partial.data(), partial.data() + parts - 1, partial[parts - 1]);
}

// ::inclusive_scan on host threads: upsweep (partition sums), spine
// (exclusive scan of the sums seeded with init), downsweep (rescan each
// partition with its carry).
template <typename T>
void cpu_inclusive_scan(const T *x, int64_t n, T init, T *out, int threads) {
  if (n <= 0) return;
  const int64_t tiles = (n + kTile - 1) / kTile;
  const int64_t parts = std::min<int64_t>(threads, tiles);
  aligned_decomposition<int64_t> decomp(n, parts, kTile);
  std::vector<T> carries(parts);
  parallel_for((int)parts, [&](int p) {
    auto r = decomp[p];
    const T *first = x + r.first, *last = x + r.second;
    carries[p] = agent_reduce(first, last - 1, last[-1]);
  });
  T c = init;
  for (int64_t p = 0; p < parts; ++p) {
    const T s = carries[p];
    carries[p] = c;
    c = c + s;
  }
  parallel_for((int)parts, [&](int p) {
    auto r = decomp[p];
    agent_inclusive_scan(x + r.first, x + r.second, out + r.first, carries[p]);
  });
}

// my_merge (merge.cu:127-162): merge_path at every tile diagonal, then each
// tile merged by the agent-level merge (tile = 256 x 9 for 4-byte keys).
template <typename K>
void cpu_merge(const K *a, int64_t na, const K *b, int64_t nb, K *out) {
  constexpr int kT = 256 * 9;
  const int64_t n = na + nb;
  bulk::agent<kT> ag(0);
  for (int64_t d0 = 0; d0 < n; d0 += kT) {
    const int64_t d1 = std::min<int64_t>(d0 + kT, n);
    const int64_t a0 = bulk::merge_path(a, na, b, nb, d0, thrust::less<K>());
    const int64_t a1 = bulk::merge_path(a, na, b, nb, d1, thrust::less<K>());
    const int64_t b0 = d0 - a0, b1 = d1 - a1;
    bulk::merge(bulk::bound<kT>(ag), a + a0, a + a1, b + b0, b + b1, out + d0, thrust::less<K>());
  }
}

}  // namespace

#define BKREF_API extern "C" __attribute__((visibility("default")))

BKREF_API int32_t bkref_cpu_reduce_i32(const int32_t *x, int64_t n, int32_t init, int threads) {
  return cpu_reduce(x, n, init, threads);
}
BKREF_API float bkref_cpu_reduce_f32(const float *x, int64_t n, float init, int threads) {
  return cpu_reduce(x, n, init, threads);
}
BKREF_API double bkref_cpu_reduce_f64(const double *x, int64_t n, double init, int threads) {
  return cpu_reduce(x, n, init, threads);
}
BKREF_API void bkref_cpu_inclusive_scan_i32(const int32_t *x, int64_t n, int32_t init, int32_t *out, int threads) {
  cpu_inclusive_scan(x, n, init, out, threads);
}
BKREF_API void bkref_cpu_inclusive_scan_f32(const float *x, int64_t n, float init, float *out, int threads) {
  cpu_inclusive_scan(x, n, init, out, threads);
}
BKREF_API void bkref_cpu_inclusive_scan_f64(const double *x, int64_t n, double init, double *out, int threads) {
  cpu_inclusive_scan(x, n, init, out, threads);
}
BKREF_API void bkref_merge_i32(const int32_t *a, int64_t na, const int32_t *b, int64_t nb, int32_t *out) {
  cpu_merge(a, na, b, nb, out);
}
BKREF_API void bkref_merge_f32(const float *a, int64_t na, const float *b, int64_t nb, float *out) {
  cpu_merge(a, na, b, nb, out);
}
BKREF_API int64_t bkref_merge_path_i32(const int32_t *a, int64_t na, const int32_t *b, int64_t nb, int64_t diag) {
  return bulk::merge_path(a, na, b, nb, diag, thrust::less<int32_t>());
}
