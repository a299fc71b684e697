// bk_merge.cuh -- merge-path machinery shared by merge and the merge sort.
//
// Semantics follow the reference exactly:
//   merge_path (bulk/algorithm/merge.hpp:35-60): among the first `diag`
//     outputs of a stable merge, how many come from A; ties go to A, i.e. the
//     search moves left while comp(b[diag-1-mid], a[mid]) holds.
//   serial merge (merge.hpp:63-170): take A while !comp(b, a), so equal keys
//     keep A before B and each input's own order.
// With comp = less these produce exactly std::merge / std::stable_sort order.
//
// A merge tile is THREADS x ITEMS outputs.  Its A and B ranges are staged in
// shared memory with coalesced loads (A first, then B), each thread finds its
// own diagonal with a shared-memory merge-path search, merges ITEMS outputs
// serially (keys plus the shared-memory index of each output's source), the
// payload is gathered through those indices, and the tile leaves through
// shared memory with 16-byte coalesced stores.
#pragma once

#include "bk_common.cuh"

namespace bk {

// Opaque payload of 0, 4 or 8 bytes.
struct NoPayload {};
template <int B>
struct PayloadT;
template <>
struct PayloadT<0> { using type = NoPayload; };
template <>
struct PayloadT<4> { using type = uint32_t; };
template <>
struct PayloadT<8> { using type = unsigned long long; };

template <typename P>
constexpr bool has_payload() { return !std::is_same_v<P, NoPayload>; }
template <typename P>
constexpr int payload_bytes() {
  if constexpr (has_payload<P>()) return (int)sizeof(P);
  else return 0;
}

// Largest key value: pads a partial tile of a sort (stable sort keeps the
// real elements with that key ahead of the padding).
template <typename K>
__host__ __device__ constexpr K key_max() {
  return std::numeric_limits<K>::has_infinity ? std::numeric_limits<K>::infinity() : std::numeric_limits<K>::max();
}

// merge_path over global or shared memory (64-bit or 32-bit indices).
template <typename K, typename I>
__device__ __forceinline__ I merge_path(const K *a, I na, const K *b, I nb, I diag) {
  I lo = diag > nb ? diag - nb : I(0);
  I hi = diag < na ? diag : na;
  while (lo < hi) {
    const I mid = (lo + hi) >> 1;
    if (b[diag - 1 - mid] < a[mid]) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// Serial stable merge of ITEMS outputs from shared memory: A = s[ia..na),
// B = s[nb0 + ib .. nb0 + nb) (B stored right after A at offset nb0 = na).
// Writes keys and the shared-memory source index of each output.
template <int ITEMS, typename K>
__device__ __forceinline__ void serial_merge(const K *s, int na, int nb, int ia, int ib, K (&keys)[ITEMS],
                                             int (&src)[ITEMS], int valid) {
  K ka = ia < na ? s[ia] : K();
  K kb = ib < nb ? s[na + ib] : K();
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    if (i < valid) {
      const bool take_a = (ib >= nb) || (ia < na && !(kb < ka));
      keys[i] = take_a ? ka : kb;
      src[i] = take_a ? ia : na + ib;
      if (take_a) {
        ++ia;
        ka = s[min(ia, na - 1)];  // clamped load, like merge.hpp:117
      } else {
        ++ib;
        kb = s[na + min(ib, nb - 1)];
      }
    }
  }
}

// Coalesced copy of n elements (n <= THREADS * ITEMS) global -> shared.
template <int THREADS, int ITEMS, typename T>
__device__ __forceinline__ void stage_in(T *s, const T *g, int n) {
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const int i = j * THREADS + (int)threadIdx.x;
    if (i < n) s[i] = g[i];
  }
}

// Coalesced copy shared -> global of n elements; 16-byte vectors when the
// destination is 16-byte aligned.
template <int THREADS, typename T>
__device__ __forceinline__ void stage_out(T *g, const T *s, int n) {
  constexpr int VE = 16 / (int)sizeof(T);
  if ((reinterpret_cast<uintptr_t>(g) & 15) == 0) {
    const int nv = n / VE;
    for (int c = threadIdx.x; c < nv; c += THREADS)
      reinterpret_cast<uint4 *>(g)[c] = reinterpret_cast<const uint4 *>(s)[c];
    for (int i = nv * VE + threadIdx.x; i < n; i += THREADS) g[i] = s[i];
  } else {
    for (int i = threadIdx.x; i < n; i += THREADS) g[i] = s[i];
  }
}

// One merge tile.  The caller supplies the tile's A and B ranges (global
// pointers and lengths, la + lb <= THREADS * ITEMS) and the output position.
// Shared memory: THREADS * ITEMS keys, then THREADS * ITEMS payloads.
template <int THREADS, int ITEMS, typename K, typename P>
__device__ __forceinline__ void merge_tile(const K *ak, const P *av, int la, const K *bk, const P *bv, int lb, K *ok,
                                           P *ov, unsigned char *smem) {
  constexpr int T = THREADS * ITEMS;
  K *sk = reinterpret_cast<K *>(smem);
  const int n = la + lb;
  // stage A then B (keys and payloads)
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const int i = j * THREADS + (int)threadIdx.x;
    if (i < la) sk[i] = ak[i];
    else if (i < n) sk[i] = bk[i - la];
  }
  P *sv = nullptr;
  if constexpr (has_payload<P>()) {
    sv = reinterpret_cast<P *>(smem + align_up(sizeof(K) * T, 16));
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const int i = j * THREADS + (int)threadIdx.x;
      if (i < la) sv[i] = av[i];
      else if (i < n) sv[i] = bv[i - la];
    }
  }
  __syncthreads();
  const int d = (int)threadIdx.x * ITEMS;
  K keys[ITEMS];
  int src[ITEMS];
  const int valid = n - d;
  if (valid > 0) {
    const int ia = merge_path<K, int>(sk, la, sk + la, lb, d);
    serial_merge<ITEMS>(sk, la, lb, ia, d - ia, keys, src, valid);
  }
  P vals[ITEMS];
  if constexpr (has_payload<P>()) {
#pragma unroll
    for (int i = 0; i < ITEMS; ++i)
      if (i < valid) vals[i] = sv[src[i]];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    if (i < valid) {
      sk[d + i] = keys[i];
      if constexpr (has_payload<P>()) sv[d + i] = vals[i];
    }
  }
  __syncthreads();
  stage_out<THREADS>(ok, sk, n);
  if constexpr (has_payload<P>()) stage_out<THREADS>(ov, sv, n);
}

}  // namespace bk
