// bulk/algorithm.hpp -- agent-level and group-level algorithms.
//
// The names, template signatures and semantics of the reference's
// bulk/algorithm/*.hpp: every algorithm has an agent-level overload taking
// bounded<B, agent<G>> (a sequential, register-resident loop of at most B
// steps) and a group-level overload taking a concurrent_group (all agents of
// the group call it together).  Reference citations per function below.
// The group implementations are this library's own, for one CTA on sm_100a:
// ordered warp-shuffle scans and reductions (so non-commutative operators keep
// their order), a 32-slot shared-memory exchange between warps, and the
// merge-path stable order of bulk/algorithm/merge.hpp:35-60.
//
// Deviation: the reference's bounded-group exclusive_scan computes an
// inclusive scan (bulk/algorithm/scan.hpp:539-550); here exclusive_scan is
// exclusive in every overload.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <iterator>
#include <type_traits>

#include <cuda/std/tuple>
#include <cuda/std/utility>
#include <thrust/tuple.h>

#include "execution_policy.hpp"
#include "malloc.hpp"

namespace bulk {
namespace detail {

template <typename It>
using value_t = typename std::iterator_traits<It>::value_type;

// ---- warp / CTA collectives over any trivially copyable T -------------------
template <typename T>
__device__ __forceinline__ T shfl_up_t(unsigned mask, T v, int d) {
  constexpr int W = (sizeof(T) + 3) / 4;
  uint32_t w[W] = {};
  memcpy(w, &v, sizeof(T));
#pragma unroll
  for (int i = 0; i < W; ++i) w[i] = __shfl_up_sync(mask, w[i], d);
  T r;
  memcpy(&r, w, sizeof(T));
  return r;
}

// A value that may be empty (no element yet): keeps operators without an
// identity element usable in scans.
template <typename T>
struct opt {
  T v;
  bool has;
};
template <typename T, typename Op>
__device__ __forceinline__ opt<T> combine(const opt<T> &a, const opt<T> &b, Op &op) {
  if (!a.has) return b;
  if (!b.has) return a;
  return opt<T>{op(a.v, b.v), true};
}

// Ordered CTA-wide scan of one optional value per thread (threads 0..n-1 of
// the CTA, n = blockDim.x).  Returns the exclusive prefix; *total receives the
// fold of all values.  Every thread of the CTA calls it.
template <typename T, typename Op>
__device__ opt<T> cta_exclusive_scan(opt<T> x, Op op, opt<T> *total) {
  __shared__ opt<T> s_warp[33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = (blockDim.x + 31) >> 5;
  // the last warp of a CTA whose size is not a multiple of 32 is partial
  const int in_warp = min(32, (int)blockDim.x - warp * 32);
  const unsigned mask = in_warp == 32 ? 0xffffffffu : ((1u << in_warp) - 1u);
  opt<T> incl = x;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    opt<T> o;
    o.v = shfl_up_t(mask, incl.v, d);
    o.has = __shfl_up_sync(mask, (int)incl.has, d) != 0;
    if (lane >= d) incl = combine(o, incl, op);
  }
  // every lane named in the mask executes each shuffle (no short-circuit)
  opt<T> excl;
  excl.v = shfl_up_t(mask, incl.v, 1);
  const int prev_has = __shfl_up_sync(mask, (int)incl.has, 1);
  excl.has = lane > 0 && prev_has != 0;
  __syncthreads();
  if (lane == 31 || (int)threadIdx.x == (int)blockDim.x - 1) s_warp[warp] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    opt<T> run{T(), false};
    for (int w = 0; w < nwarps; ++w) {
      const opt<T> t = s_warp[w];
      s_warp[w] = run;  // exclusive prefix of warp w
      run = combine(run, t, op);
    }
    s_warp[32] = run;
  }
  __syncthreads();
  const opt<T> r = combine(s_warp[warp], excl, op);
  *total = s_warp[32];
  __syncthreads();
  return r;
}

template <typename T>
__host__ __device__ __forceinline__ T min_(T a, T b) { return b < a ? b : a; }

template <typename It>
struct value_or_char {
  typedef value_t<It> type;
};
template <>
struct value_or_char<std::nullptr_t> {
  typedef char type;
};

}  // namespace detail

// ============================================================================
// copy_n / gather / scatter_if            bulk/algorithm/copy.hpp:31-276,
//                                         gather.hpp:31-81, scatter.hpp:27-197
// ============================================================================
template <std::size_t bound, std::size_t grainsize, typename InputIt, typename Size, typename OutputIt>
__host__ __device__ OutputIt copy_n(const bounded<bound, agent<grainsize>> &, InputIt first, Size n, OutputIt result) {
  for (Size i = 0; i < (Size)bound; ++i)
    if (i < n) result[i] = first[i];
  return result + n;
}

template <typename A, std::size_t S, typename InputIt, typename Size, typename OutputIt>
__device__ OutputIt copy_n(concurrent_group<A, S> &g, InputIt first, Size n, OutputIt result) {
  for (Size i = g.this_exec.index(); i < n; i += g.size()) result[i] = first[i];
  g.wait();
  return result + n;
}

template <std::size_t bound, std::size_t grainsize, typename MapIt, typename InputIt, typename OutputIt>
__host__ __device__ OutputIt gather(const bounded<bound, agent<grainsize>> &, MapIt map_first, MapIt map_last,
                                    InputIt input, OutputIt result) {
  const auto n = map_last - map_first;
  for (decltype(n + 0) i = 0; i < (decltype(n + 0))bound; ++i)
    if (i < n) result[i] = input[map_first[i]];
  return result + n;
}

template <typename A, std::size_t S, typename MapIt, typename InputIt, typename OutputIt>
__device__ OutputIt gather(concurrent_group<A, S> &g, MapIt map_first, MapIt map_last, InputIt input,
                           OutputIt result) {
  const auto n = map_last - map_first;
  for (decltype(n + 0) i = g.this_exec.index(); i < n; i += g.size()) result[i] = input[map_first[i]];
  g.wait();
  return result + n;
}

template <std::size_t bound, std::size_t grainsize, typename InputIt, typename MapIt, typename StencilIt,
          typename OutputIt>
__host__ __device__ void scatter_if(const bounded<bound, agent<grainsize>> &, InputIt first, InputIt last, MapIt map,
                                    StencilIt stencil, OutputIt result) {
  const auto n = last - first;
  for (decltype(n + 0) i = 0; i < (decltype(n + 0))bound; ++i)
    if (i < n && stencil[i]) result[map[i]] = first[i];
}

template <typename A, std::size_t S, typename InputIt, typename MapIt, typename StencilIt, typename OutputIt>
__device__ void scatter_if(concurrent_group<A, S> &g, InputIt first, InputIt last, MapIt map, StencilIt stencil,
                           OutputIt result) {
  const auto n = last - first;
  for (decltype(n + 0) i = g.this_exec.index(); i < n; i += g.size())
    if (stencil[i]) result[map[i]] = first[i];
  g.wait();
}

// ============================================================================
// for_each_n                              bulk/algorithm/for_each.hpp:28-70
// ============================================================================
template <std::size_t bound, std::size_t grainsize, typename It, typename Size, typename F>
__host__ __device__ It for_each_n(bounded<bound, agent<grainsize>> &, It first, Size n, F f) {
  for (Size i = 0; i < (Size)bound; ++i)
    if (i < n) f(first[i]);
  return first + n;
}

template <typename A, std::size_t S, typename It, typename Size, typename F>
__device__ It for_each_n(concurrent_group<A, S> &g, It first, Size n, F f) {
  for (Size i = g.this_exec.index(); i < n; i += g.size()) f(first[i]);
  g.wait();
  return first + n;
}

// ============================================================================
// adjacent_difference                     bulk/algorithm/adjacent_difference.hpp:28-140
// ============================================================================
// result[i] = op(first[i], first[i-1]), with init standing for first[-1].
template <std::size_t grainsize, typename InIt, typename OutIt, typename T, typename Op>
__host__ __device__ OutIt adjacent_difference(agent<grainsize> &, InIt first, InIt last, OutIt result, T init,
                                              Op op) {
  for (; first != last; ++first, ++result) {
    const T x = *first;
    *result = op(x, init);
    init = x;
  }
  return result;
}

// Group version; the input and output may be the same range.
template <typename A, std::size_t S, typename InIt, typename OutIt, typename T, typename Op>
__device__ OutIt adjacent_difference(concurrent_group<A, S> &g, InIt first, InIt last, OutIt result, T init, Op op) {
  const long long n = last - first;
  T *prev = static_cast<T *>(bulk::malloc(g, sizeof(T) * (n > 0 ? n : 1)));
  for (long long i = g.this_exec.index(); i < n; i += g.size()) prev[i] = i == 0 ? init : T(first[i - 1]);
  g.wait();
  for (long long i = g.this_exec.index(); i < n; i += g.size()) result[i] = op(T(first[i]), prev[i]);
  bulk::free(g, prev);
  return result + n;
}

// result[0] = first[0], then the differences of neighbours.
template <typename A, std::size_t S, typename InIt, typename OutIt, typename Op>
__device__ OutIt adjacent_difference(concurrent_group<A, S> &g, InIt first, InIt last, OutIt result, Op op) {
  if (!(first < last)) return result;
  typedef detail::value_t<InIt> T;
  const T x0 = *first;
  g.wait();  // first may equal result
  if (g.this_exec.index() == 0) *result = x0;
  return adjacent_difference(g, first + 1, last, result + 1, x0, op);
}

// ============================================================================
// reduce / accumulate                     bulk/algorithm/reduce.hpp:33-264,
//                                         accumulate.hpp:30-217
// ============================================================================
template <std::size_t bound, std::size_t grainsize, typename It, typename T, typename Op>
__host__ __device__ T reduce(const bounded<bound, agent<grainsize>> &, It first, It last, T init, Op op) {
  const auto n = last - first;
  for (decltype(n + 0) i = 0; i < (decltype(n + 0))bound; ++i)
    if (i < n) init = op(init, first[i]);
  return init;
}

// init (+) first[0] (+) ... in order (associative operators; commutativity is
// not assumed).  Every agent receives the result.
template <typename A, std::size_t S, typename It, typename T, typename Op>
__device__ T reduce(concurrent_group<A, S> &g, It first, It last, T init, Op op) {
  const long long n = last - first;
  const int size = g.size(), t = g.this_exec.index();
  const long long chunk = (n + size - 1) / size;
  const long long lo = detail::min_((long long)t * chunk, n), hi = detail::min_(lo + chunk, n);
  detail::opt<T> local{T(), false};
  for (long long i = lo; i < hi; ++i) local = detail::opt<T>{local.has ? op(local.v, first[i]) : T(first[i]), true};
  detail::opt<T> total;
  (void)detail::cta_exclusive_scan(local, op, &total);
  return total.has ? op(init, total.v) : init;
}

template <typename A, std::size_t S, typename It, typename T, typename Op>
__device__ T accumulate(concurrent_group<A, S> &g, It first, It last, T init, Op op) {
  return reduce(g, first, last, init, op);
}

// A cluster group (a concurrent group of C CTAs) reduces in order: CTA r
// folds its contiguous share of the range with the CTA-wide ordered scan and
// leaves the result in its shared memory; after a cluster barrier every
// agent folds the C results in rank order, reading the other CTAs' shared
// memory through the cluster window.  Every agent receives the result.
template <typename A, std::size_t S, std::size_t C, typename It, typename T, typename Op>
__device__ T reduce(concurrent_group<concurrent_group<A, S>, C> &g, It first, It last, T init, Op op) {
  __shared__ __align__(16) unsigned char s_part[sizeof(T)];
  __shared__ int s_part_has;
  const long long n = last - first;
  const int r = g.this_exec.index(), size = g.this_exec.size(), t = g.this_exec.this_exec.index();
  const long long share = (n + (long long)C - 1) / (long long)C;
  const long long lo = detail::min_((long long)r * share, n), hi = detail::min_(lo + share, n);
  const long long chunk = (hi - lo + size - 1) / size;
  const long long a0 = detail::min_(lo + (long long)t * chunk, hi), a1 = detail::min_(a0 + chunk, hi);
  detail::opt<T> local{T(), false};
  for (long long i = a0; i < a1; ++i) local = detail::opt<T>{local.has ? op(local.v, first[i]) : T(first[i]), true};
  detail::opt<T> total;
  (void)detail::cta_exclusive_scan(local, op, &total);
  if (t == 0) {
    memcpy(s_part, &total.v, sizeof(T));
    s_part_has = total.has ? 1 : 0;
  }
  g.wait();  // every CTA's result is in place
  T acc = init;
  for (int q = 0; q < (int)C; ++q) {
    if (*detail::cluster_map(&s_part_has, (unsigned)q)) {
      T v;
      memcpy(&v, detail::cluster_map(&s_part[0], (unsigned)q), sizeof(T));
      acc = op(acc, v);
    }
  }
  g.wait();  // every agent has read them before any CTA reuses its slot
  return acc;
}

template <typename A, std::size_t S, std::size_t C, typename It, typename T, typename Op>
__device__ T accumulate(concurrent_group<concurrent_group<A, S>, C> &g, It first, It last, T init, Op op) {
  return reduce(g, first, last, init, op);
}

// ============================================================================
// inclusive_scan / exclusive_scan          bulk/algorithm/scan.hpp:35-591
// ============================================================================
template <std::size_t bound, std::size_t grainsize, typename InIt, typename OutIt, typename T, typename Op>
__host__ __device__ OutIt inclusive_scan(const bounded<bound, agent<grainsize>> &, InIt first, InIt last,
                                         OutIt result, T init, Op op) {
  const auto n = last - first;
  for (decltype(n + 0) i = 0; i < (decltype(n + 0))bound; ++i)
    if (i < n) {
      init = op(init, first[i]);
      result[i] = init;
    }
  return result + n;
}

template <std::size_t bound, std::size_t grainsize, typename InIt, typename OutIt, typename T, typename Op>
__host__ __device__ OutIt exclusive_scan(const bounded<bound, agent<grainsize>> &, InIt first, InIt last,
                                         OutIt result, T init, Op op) {
  const auto n = last - first;
  for (decltype(n + 0) i = 0; i < (decltype(n + 0))bound; ++i)
    if (i < n) {
      const T x = first[i];
      result[i] = init;
      init = op(init, x);
    }
  return result + n;
}

namespace detail {
// Group scan: tiles of (group size x G) elements, each agent scanning G
// consecutive elements; `exclusive` selects the scan kind; has_init says
// whether `init` seeds the scan.
template <bool exclusive, typename A, std::size_t S, typename InIt, typename OutIt, typename T, typename Op>
__device__ OutIt group_scan(concurrent_group<A, S> &g, InIt first, InIt last, OutIt result, T init, bool has_init,
                            Op op) {
  constexpr int G = A::static_grainsize;
  const long long n = last - first;
  const int size = g.size(), t = g.this_exec.index();
  opt<T> carry{init, has_init};
  for (long long base = 0; base < n; base += (long long)size * G) {
    const long long my0 = base + (long long)t * G;
    T x[G];
    bool valid[G];
    opt<T> local{T(), false};
#pragma unroll
    for (int j = 0; j < G; ++j) {
      valid[j] = my0 + j < n;
      if (valid[j]) {
        x[j] = first[my0 + j];
        local = opt<T>{local.has ? op(local.v, x[j]) : x[j], true};
      }
    }
    opt<T> total;
    const opt<T> pre = combine(carry, cta_exclusive_scan(local, op, &total), op);
    opt<T> run = pre;
#pragma unroll
    for (int j = 0; j < G; ++j) {
      if (valid[j]) {
        if (exclusive) {
          result[my0 + j] = run.v;  // exclusive scans always have init
          run = opt<T>{op(run.v, x[j]), true};
        } else {
          run = opt<T>{run.has ? op(run.v, x[j]) : x[j], true};
          result[my0 + j] = run.v;
        }
      }
    }
    carry = combine(carry, total, op);
  }
  g.wait();
  return result + n;
}
}  // namespace detail

template <typename A, std::size_t S, typename InIt, typename OutIt, typename T, typename Op>
__device__ OutIt inclusive_scan(concurrent_group<A, S> &g, InIt first, InIt last, OutIt result, T init, Op op) {
  return detail::group_scan<false>(g, first, last, result, init, true, op);
}

template <typename A, std::size_t S, typename InIt, typename OutIt, typename Op>
__device__ OutIt inclusive_scan(concurrent_group<A, S> &g, InIt first, InIt last, OutIt result, Op op) {
  typedef detail::value_t<InIt> T;
  return detail::group_scan<false>(g, first, last, result, T(), false, op);
}

template <typename A, std::size_t S, typename InIt, typename OutIt, typename T, typename Op>
__device__ OutIt exclusive_scan(concurrent_group<A, S> &g, InIt first, InIt last, OutIt result, T init, Op op) {
  return detail::group_scan<true>(g, first, last, result, init, true, op);
}

// ============================================================================
// merge_path / merge / merge_by_key        bulk/algorithm/merge.hpp:35-607
// ============================================================================
// Among the first diag outputs of a stable merge, how many come from A
// (ties go to A).
template <typename It1, typename Size, typename It2, typename Compare>
__host__ __device__ Size merge_path(It1 first1, Size n1, It2 first2, Size n2, Size diag, Compare comp) {
  Size lo = diag > n2 ? diag - n2 : Size(0);
  Size hi = diag < n1 ? diag : n1;
  while (lo < hi) {
    const Size mid = (lo + hi) >> 1;
    if (comp(first2[diag - 1 - mid], first1[mid])) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

namespace detail {
// Serial stable merge of up to `count` outputs starting at A[i], B[j]; also
// moves values when ValIt1 is not std::nullptr_t.
template <typename KIt1, typename KIt2, typename VIt1, typename VIt2, typename KOut, typename VOut, typename Compare>
__host__ __device__ void serial_merge(KIt1 a, long long na, KIt2 b, long long nb, long long i, long long j,
                                      long long count, KOut ko, VIt1 av, VIt2 bv, VOut vo, Compare comp) {
  constexpr bool with_values = !std::is_same<VIt1, std::nullptr_t>::value;
  for (long long k = 0; k < count; ++k) {
    const bool take_a = (j >= nb) || (i < na && !comp(b[j], a[i]));
    if (take_a) {
      ko[k] = a[i];
      if constexpr (with_values) vo[k] = av[i];
      ++i;
    } else {
      ko[k] = b[j];
      if constexpr (with_values) vo[k] = bv[j];
      ++j;
    }
  }
}

template <typename A, std::size_t S, typename KIt1, typename KIt2, typename VIt1, typename VIt2, typename KOut,
          typename VOut, typename Compare>
__device__ void group_merge(concurrent_group<A, S> &g, KIt1 a, long long na, KIt2 b, long long nb, KOut ko, VIt1 av,
                            VIt2 bv, VOut vo, Compare comp) {
  constexpr int G = A::static_grainsize;
  const long long n = na + nb;
  const int size = g.size(), t = g.this_exec.index();
  for (long long d = (long long)t * G; d < n; d += (long long)size * G) {
    const long long i = merge_path(a, na, b, nb, d, comp);
    const long long cnt = detail::min_((long long)G, n - d);
    if constexpr (std::is_same<VIt1, std::nullptr_t>::value) {
      serial_merge(a, na, b, nb, i, d - i, cnt, ko + d, av, bv, vo, comp);
    } else {
      serial_merge(a, na, b, nb, i, d - i, cnt, ko + d, av, bv, vo + d, comp);
    }
  }
}
}  // namespace detail

// A bounded agent produces at most `bound` outputs of the merge.
template <std::size_t bound, std::size_t grainsize, typename It1, typename It2, typename OutIt, typename Compare>
__host__ __device__ OutIt merge(const bounded<bound, agent<grainsize>> &, It1 first1, It1 last1, It2 first2,
                                It2 last2, OutIt result, Compare comp) {
  const long long n1 = last1 - first1, n2 = last2 - first2;
  const long long cnt = detail::min_(n1 + n2, (long long)bound);
  detail::serial_merge(first1, n1, first2, n2, 0, 0, cnt, result, nullptr, nullptr, nullptr, comp);
  return result + cnt;
}

template <std::size_t bound, std::size_t grainsize, typename KIt1, typename KIt2, typename VIt1, typename VIt2,
          typename KOut, typename VOut, typename Compare>
__host__ __device__ cuda::std::pair<KOut, VOut> merge_by_key(const bounded<bound, agent<grainsize>> &,
                                                            KIt1 keys_first1, KIt1 keys_last1, KIt2 keys_first2,
                                                            KIt2 keys_last2, VIt1 values_first1, VIt2 values_first2,
                                                            KOut keys_result, VOut values_result, Compare comp) {
  const long long n1 = keys_last1 - keys_first1, n2 = keys_last2 - keys_first2;
  const long long cnt = detail::min_(n1 + n2, (long long)bound);
  detail::serial_merge(keys_first1, n1, keys_first2, n2, 0, 0, cnt, keys_result, values_first1, values_first2,
                       values_result, comp);
  return cuda::std::make_pair(keys_result + cnt, values_result + cnt);
}

template <typename A, std::size_t S, typename It1, typename It2, typename OutIt, typename Compare>
__device__ OutIt merge(concurrent_group<A, S> &g, It1 first1, It1 last1, It2 first2, It2 last2, OutIt result,
                       Compare comp) {
  const long long n1 = last1 - first1, n2 = last2 - first2;
  detail::group_merge(g, first1, n1, first2, n2, result, nullptr, nullptr, nullptr, comp);
  g.wait();
  return result + (n1 + n2);
}

template <typename A, std::size_t S, typename KIt1, typename KIt2, typename VIt1, typename VIt2, typename KOut,
          typename VOut, typename Compare>
__device__ cuda::std::pair<KOut, VOut> merge_by_key(concurrent_group<A, S> &g, KIt1 keys_first1, KIt1 keys_last1,
                                                    KIt2 keys_first2, KIt2 keys_last2, VIt1 values_first1,
                                                    VIt2 values_first2, KOut keys_result, VOut values_result,
                                                    Compare comp) {
  const long long n1 = keys_last1 - keys_first1, n2 = keys_last2 - keys_first2;
  detail::group_merge(g, keys_first1, n1, keys_first2, n2, keys_result, values_first1, values_first2, values_result,
                      comp);
  g.wait();
  return cuda::std::make_pair(keys_result + (n1 + n2), values_result + (n1 + n2));
}

// Merges the sorted ranges [first, middle) and [middle, last) in place
// (bulk/algorithm/merge.hpp:308-353): the merged result is staged on the
// group's heap and copied back.
template <typename A, std::size_t S, typename It, typename Compare>
__device__ void inplace_merge(concurrent_group<A, S> &g, It first, It middle, It last, Compare comp) {
  typedef detail::value_t<It> T;
  const long long n = last - first;
  T *tmp = static_cast<T *>(bulk::malloc(g, sizeof(T) * (n > 0 ? n : 1)));
  detail::group_merge(g, first, middle - first, middle, last - middle, tmp, nullptr, nullptr, nullptr, comp);
  g.wait();
  for (long long i = g.this_exec.index(); i < n; i += g.size()) first[i] = tmp[i];
  bulk::free(g, tmp);
}

// ============================================================================
// stable_sort / stable_sort_by_key         bulk/algorithm/sort.hpp:33-166
// ============================================================================
namespace detail {
// stable odd-even transposition sort of n <= B items
template <std::size_t B, typename KIt, typename VIt, typename Compare>
__host__ __device__ void agent_stable_sort(KIt keys, VIt vals, long long n, Compare comp) {
  constexpr bool with_values = !std::is_same<VIt, std::nullptr_t>::value;
  for (long long r = 0; r < n; ++r)
    for (long long i = r & 1; i + 1 < n; i += 2)
      if (comp(keys[i + 1], keys[i])) {
        auto tk = keys[i];
        keys[i] = keys[i + 1];
        keys[i + 1] = tk;
        if constexpr (with_values) {
          auto tv = vals[i];
          vals[i] = vals[i + 1];
          vals[i + 1] = tv;
        }
      }
}

// Group stable sort of n <= size * G elements in place: each agent sorts
// G consecutive elements, then runs of width w merge pairwise (merge path)
// through a heap stage until one run is left.
template <typename A, std::size_t S, typename KIt, typename VIt, typename Compare>
__device__ void group_stable_sort(concurrent_group<A, S> &g, KIt keys, VIt vals, long long n, Compare comp) {
  constexpr int G = A::static_grainsize;
  constexpr bool with_values = !std::is_same<VIt, std::nullptr_t>::value;
  typedef value_t<KIt> K;
  typedef typename value_or_char<VIt>::type V;
  const int t = g.this_exec.index();
  const long long my0 = (long long)t * G;
  const long long mine = my0 < n ? detail::min_((long long)G, n - my0) : 0;
  if (mine > 0) {
    if constexpr (with_values) agent_stable_sort<G>(keys + my0, vals + my0, mine, comp);
    else agent_stable_sort<G>(keys + my0, nullptr, mine, comp);
  }
  g.wait();
  if (n <= G) return;
  K *sk = static_cast<K *>(bulk::malloc(g, sizeof(K) * n));
  V *sv = with_values ? static_cast<V *>(bulk::malloc(g, sizeof(V) * n)) : nullptr;
  for (long long w = G; w < n; w *= 2) {
    for (long long i = t; i < n; i += g.size()) {  // stage the current runs
      sk[i] = keys[i];
      if constexpr (with_values) sv[i] = vals[i];
    }
    g.wait();
    if (mine > 0) {
      const long long p0 = my0 / (2 * w) * (2 * w);
      const long long a_end = detail::min_(p0 + w, n), b_end = detail::min_(p0 + 2 * w, n);
      const long long d = my0 - p0;
      const long long i = merge_path(sk + p0, a_end - p0, sk + a_end, b_end - a_end, d, comp);
      if constexpr (with_values)
        serial_merge(sk + p0, a_end - p0, sk + a_end, b_end - a_end, i, d - i, mine, keys + my0, sv + p0, sv + a_end,
                     vals + my0, comp);
      else
        serial_merge(sk + p0, a_end - p0, sk + a_end, b_end - a_end, i, d - i, mine, keys + my0, nullptr, nullptr,
                     nullptr, comp);
    }
    g.wait();
  }
  if constexpr (with_values) bulk::free(g, sv);
  bulk::free(g, sk);
}
}  // namespace detail

template <std::size_t bound, std::size_t grainsize, typename KIt, typename VIt, typename Compare>
__host__ __device__ void stable_sort_by_key(const bounded<bound, agent<grainsize>> &, KIt keys_first, KIt keys_last,
                                            VIt values_first, Compare comp) {
  detail::agent_stable_sort<bound>(keys_first, values_first, keys_last - keys_first, comp);
}

template <std::size_t bound, std::size_t grainsize, typename It, typename Compare>
__host__ __device__ void stable_sort(const bounded<bound, agent<grainsize>> &, It first, It last, Compare comp) {
  detail::agent_stable_sort<bound>(first, nullptr, last - first, comp);
}

// Bounded group sorts: n <= bound <= group size x grainsize.
template <std::size_t bound, typename A, std::size_t S, typename KIt, typename VIt, typename Compare>
__device__ void stable_sort_by_key(bounded<bound, concurrent_group<A, S>> &g, KIt keys_first, KIt keys_last,
                                   VIt values_first, Compare comp) {
  detail::group_stable_sort(g.unbound(), keys_first, values_first, keys_last - keys_first, comp);
}

template <std::size_t bound, typename A, std::size_t S, typename It, typename Compare>
__device__ void stable_sort(bounded<bound, concurrent_group<A, S>> &g, It first, It last, Compare comp) {
  detail::group_stable_sort(g.unbound(), first, nullptr, last - first, comp);
}

// ============================================================================
// reduce_by_key                            bulk/algorithm/reduce_by_key.hpp:115-216
// ============================================================================
// The sequence is the carried pair (init_key, init_value) followed by the
// input pairs.  Every run of equal keys (pred) that ends inside the input is
// written to the outputs in order; the last run stays open and is returned as
// the new carry: (keys_result end, values_result end, carry key, carry value).
template <typename A, std::size_t S, typename KIt, typename VIt, typename KOut, typename VOut, typename T1,
          typename T2, typename Pred, typename Op>
__device__ thrust::tuple<KOut, VOut, detail::value_t<KIt>, detail::value_t<VOut>> reduce_by_key(
    concurrent_group<A, S> &g, KIt keys_first, KIt keys_last, VIt values_first, KOut keys_result, VOut values_result,
    T1 init_key, T2 init_value, Pred pred, Op op) {
  typedef detail::value_t<KIt> K;
  typedef detail::value_t<VOut> V;
  constexpr int G = A::static_grainsize;
  struct seg {
    int c;  // run heads
    V v;    // sum since the last head
  };
  struct seg_op {
    Op op;
    __device__ seg operator()(const seg &a, const seg &b) const {
      return seg{a.c + b.c, b.c ? b.v : op(a.v, b.v)};
    }
  } sop{op};
  const long long n = keys_last - keys_first;
  const int size = g.size(), t = g.this_exec.index();
  seg carry{0, V(init_value)};
  K carry_key = K(init_key);
  long long emitted = 0;
  for (long long base = 0; base < n; base += (long long)size * G) {
    const long long my0 = base + (long long)t * G;
    K k[G];
    V v[G];
    bool head[G], valid[G];
    detail::opt<seg> local{seg{0, V()}, false};
#pragma unroll
    for (int j = 0; j < G; ++j) {
      valid[j] = my0 + j < n;
      if (valid[j]) {
        k[j] = keys_first[my0 + j];
        v[j] = values_first[my0 + j];
        const K prev = (my0 + j == 0) ? carry_key : (j > 0 ? k[j - 1] : K(keys_first[my0 + j - 1]));
        head[j] = (my0 + j == 0) ? !pred(K(init_key), k[j]) : !pred(prev, k[j]);
        const seg e{head[j] ? 1 : 0, v[j]};
        local = detail::opt<seg>{local.has ? sop(local.v, e) : e, true};
      }
    }
    detail::opt<seg> total;
    const detail::opt<seg> ex = detail::cta_exclusive_scan(local, sop, &total);
    seg run = ex.has ? sop(carry, ex.v) : carry;
#pragma unroll
    for (int j = 0; j < G; ++j) {
      if (valid[j]) {
        if (head[j]) {  // the run before this element closes
          const K pk = (my0 + j == 0) ? carry_key : (j > 0 ? k[j - 1] : K(keys_first[my0 + j - 1]));
          keys_result[emitted + run.c] = pk;
          values_result[emitted + run.c] = run.v;
        }
        run = sop(run, seg{head[j] ? 1 : 0, v[j]});
      }
    }
    if (total.has) carry = sop(carry, total.v);
    const long long last = detail::min_(base + (long long)size * G, n) - 1;
    carry_key = K(keys_first[last]);
    emitted += carry.c;
    carry.c = 0;
  }
  g.wait();
  return thrust::make_tuple(keys_result + emitted, values_result + emitted, carry_key, carry.v);
}

}  // namespace bulk
