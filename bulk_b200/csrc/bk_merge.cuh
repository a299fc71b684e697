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

// Shared-memory layout with one pad element after every 32: a thread reading
// or writing its own ITEMS consecutive elements (stride ITEMS between lanes)
// and a warp reading 32 consecutive elements both hit 32 distinct banks.
__host__ __device__ constexpr int pad32(int i) { return i + (i >> 5); }
__host__ __device__ constexpr int padded_len(int n) { return n + (n >> 5) + 1; }

// A view of a padded shared-memory array starting at unpadded index `off`.
template <typename K>
struct PView {
  const K *base;
  int off;
  __device__ __forceinline__ K operator[](int i) const { return base[pad32(off + i)]; }
};

// merge_path over global or shared memory (64-bit or 32-bit indices).
template <typename K, typename I, typename A, typename B>
__device__ __forceinline__ I merge_path(A a, I na, B b, I nb, I diag) {
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
// B = s[na + ib .. na + nb) (B stored right after A).  Writes keys and the
// (unpadded) index of each output's source.  S indexes like an array.
template <int ITEMS, typename K, typename S>
__device__ __forceinline__ void serial_merge(S s, int na, int nb, int ia, int ib, K (&keys)[ITEMS],
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

// Coalesced copy of n elements from a padded shared-memory array to global
// memory: each thread gathers 16 bytes (conflict-free) and stores them as one
// vector when the destination is 16-byte aligned.
template <int THREADS, typename T>
__device__ __forceinline__ void stage_out_padded(T *g, const T *s, int n) {
  constexpr int VE = 16 / (int)sizeof(T);
  if ((reinterpret_cast<uintptr_t>(g) & 15) == 0) {
    const int nv = n / VE;
    for (int c = threadIdx.x; c < nv; c += THREADS) {
      T v[VE];
#pragma unroll
      for (int j = 0; j < VE; ++j) v[j] = s[pad32(c * VE + j)];
      uint4 q;
      memcpy(&q, v, 16);
      reinterpret_cast<uint4 *>(g)[c] = q;
    }
    for (int i = nv * VE + threadIdx.x; i < n; i += THREADS) g[i] = s[pad32(i)];
  } else {
    for (int i = threadIdx.x; i < n; i += THREADS) g[i] = s[pad32(i)];
  }
}

// One merge tile.  The caller supplies the tile's A and B ranges (global
// pointers and lengths, la + lb <= THREADS * ITEMS) and the output position.
// Shared memory (padded layout): padded_len(THREADS * ITEMS) keys, then as
// many payloads.
template <int THREADS, int ITEMS, typename K, typename P>
__device__ __forceinline__ void merge_tile(const K *ak, const P *av, int la, const K *bk, const P *bv, int lb, K *ok,
                                           P *ov, unsigned char *smem) {
  constexpr int T = THREADS * ITEMS;
  K *sk = reinterpret_cast<K *>(smem);
  const int n = la + lb;
  // stage A then B (keys and payloads, padded layout): every load is issued
  // into registers before the first shared-memory store, so all are in flight
  P *sv = nullptr;
  {
    K tk[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const int i = j * THREADS + (int)threadIdx.x;
      const K *src = i < la ? ak + i : bk + (i - la);
      tk[j] = i < n ? __ldg(src) : K();
    }
    if constexpr (has_payload<P>()) {
      sv = reinterpret_cast<P *>(smem + align_up(sizeof(K) * padded_len(T), 16));
      P tv[ITEMS];
#pragma unroll
      for (int j = 0; j < ITEMS; ++j) {
        const int i = j * THREADS + (int)threadIdx.x;
        const P *src = i < la ? av + i : bv + (i - la);
        tv[j] = i < n ? __ldg(src) : P();
      }
#pragma unroll
      for (int j = 0; j < ITEMS; ++j) {
        const int i = j * THREADS + (int)threadIdx.x;
        if (i < n) sv[pad32(i)] = tv[j];
      }
    }
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const int i = j * THREADS + (int)threadIdx.x;
      if (i < n) sk[pad32(i)] = tk[j];
    }
  }
  __syncthreads();
  const int d = (int)threadIdx.x * ITEMS;
  K keys[ITEMS];
  int src[ITEMS];
  const int valid = n - d;
  if (valid > 0) {
    const PView<K> pa{sk, 0}, pb{sk, la};  // B follows A in the unpadded numbering
    const int ia = merge_path<K, int>(pa, la, pb, lb, d);
    serial_merge<ITEMS, K>(pa, la, lb, ia, d - ia, keys, src, valid);
  }
  P vals[ITEMS];
  if constexpr (has_payload<P>()) {
#pragma unroll
    for (int i = 0; i < ITEMS; ++i)
      if (i < valid) vals[i] = sv[pad32(src[i])];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    if (i < valid) {
      sk[pad32(d + i)] = keys[i];
      if constexpr (has_payload<P>()) sv[pad32(d + i)] = vals[i];
    }
  }
  __syncthreads();
  stage_out_padded<THREADS>(ok, sk, n);
  if constexpr (has_payload<P>()) stage_out_padded<THREADS>(ov, sv, n);
}

}  // namespace bk
