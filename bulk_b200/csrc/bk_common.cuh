// bk_common.cuh -- shared device/host helpers of the sm_100a algorithm library.
//
// Contents: the workspace header every kernel shares, the associative operators
// (sum / min / max with their identities), cache-hinted vector memory access in
// inline PTX, acquire/release status-word access for cross-CTA look-back, the
// bounded-spin helper, warp/CTA reductions and scans, and the host-side device
// property cache used to size grids in multiples of the SM count.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>
#include <limits>
#include <type_traits>

#include "bk_host_cache.hpp"
#include "bulk_b200.h"

namespace bk {

// ---------------------------------------------------------------------------
// Workspace header: the first 256 bytes of every workspace.  Zero-filled once
// by the caller; every kernel that uses a counter leaves it zero on exit.
// ---------------------------------------------------------------------------
struct WsHeader {
  unsigned int tile_ticket;  // dynamic tile counter of look-back kernels
  unsigned int done_count;   // finished CTAs (last-CTA detection)
  int status;                // first device-side error (BK_OK when none)
  unsigned int err_tile;     // tile that recorded the error
  unsigned int aux[60];      // per-algorithm scratch counters
};
static_assert(sizeof(WsHeader) == 256, "header is 256 bytes");
constexpr size_t kHeaderBytes = 256;

__host__ __device__ constexpr size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// ---------------------------------------------------------------------------
// Operators.  All three are associative and commutative; identity() is the
// neutral element used to pad partial tiles.
// ---------------------------------------------------------------------------
template <typename T>
struct OpSum {
  static constexpr int kind = 0;
  __host__ __device__ __forceinline__ T operator()(T a, T b) const { return a + b; }
  __host__ __device__ static constexpr T identity() { return T(0); }
};
template <typename T>
struct OpMin {
  static constexpr int kind = 1;
  // thrust::minimum semantics: lhs < rhs ? lhs : rhs
  __host__ __device__ __forceinline__ T operator()(T a, T b) const { return a < b ? a : b; }
  __host__ __device__ static constexpr T identity() {
    return std::numeric_limits<T>::has_infinity ? std::numeric_limits<T>::infinity()
                                                : std::numeric_limits<T>::max();
  }
};
template <typename T>
struct OpMax {
  static constexpr int kind = 2;
  // thrust::maximum semantics: lhs < rhs ? rhs : lhs
  __host__ __device__ __forceinline__ T operator()(T a, T b) const { return a < b ? b : a; }
  __host__ __device__ static constexpr T identity() {
    return std::numeric_limits<T>::has_infinity ? -std::numeric_limits<T>::infinity()
                                                : std::numeric_limits<T>::lowest();
  }
};

// ---------------------------------------------------------------------------
// Memory access helpers (inline PTX).
// ---------------------------------------------------------------------------
// Streaming 16-byte load through the non-coherent path, not kept in L1.
__device__ __forceinline__ uint4 ld_stream_v4(const void *p) {
  uint4 r;
  asm("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
      : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
      : "l"(p));
  return r;
}
// 16-byte load through L1 without allocating there, with an L2 eviction
// policy (createpolicy); coherent, so the source may be written later in the
// same kernel.
__device__ __forceinline__ uint4 ld_v4_l2hint(const void *p, uint64_t policy) {
  uint4 r;
  asm("ld.global.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
      : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
      : "l"(p), "l"(policy));
  return r;
}
// Streaming 16-byte store (evict-first).
__device__ __forceinline__ void st_stream_v4(void *p, uint4 v) {
  asm volatile("st.global.cs.v4.u32 [%0], {%1,%2,%3,%4};" ::"l"(p), "r"(v.x), "r"(v.y), "r"(v.z),
               "r"(v.w)
               : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// Two adjacent 64-bit words (16-byte aligned), each single-copy atomic.
__device__ __forceinline__ void ld_relaxed_v2_u64(const unsigned long long *p, unsigned long long &a,
                                                  unsigned long long &b) {
  asm volatile("ld.relaxed.gpu.global.v2.u64 {%0,%1}, [%2];" : "=l"(a), "=l"(b) : "l"(p));
}
__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned int *p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Acquire / release on a CTA-local word (shared memory, generic address).
__device__ __forceinline__ unsigned int ld_acquire_cta_u32(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.cta.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_cta_u32(unsigned int *p, unsigned int v) {
  asm volatile("st.release.cta.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Barrier `id` (1-15; 0 is __syncthreads) over the first `threads` threads
// that reach it; every participating warp must take part with all its lanes.
__device__ __forceinline__ void named_barrier_sync(int id, int threads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}
// Barrier `id` over `threads` threads that also ORs a predicate across them:
// every participant gets the same answer.
__device__ __forceinline__ bool named_barrier_or(int id, int threads, bool pred) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.or.pred p, %2, %3, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)pred), "r"(id), "r"(threads)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ unsigned int ld_relaxed_u32(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u32(unsigned int *p, unsigned int v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_relaxed_s32(const int *p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Asks L2 to fetch [p, p + bytes) from memory ahead of its use (nothing
// reaches the SM).  The range is trimmed inward to 16-byte boundaries, so the
// prefetch never leaves the caller's array.
__device__ __forceinline__ void prefetch_l2_range(const void *p, uint64_t bytes) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  uintptr_t lo = (a + 15) & ~(uintptr_t)15;
  const uintptr_t hi = (a + bytes) & ~(uintptr_t)15;
  while (lo < hi) {
    const uint32_t s = (hi - lo) > (1u << 30) ? (1u << 30) : (uint32_t)(hi - lo);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo), "r"(s) : "memory");
    lo += s;
  }
}

// Record the first device-side error in the workspace header.
__device__ __forceinline__ void record_error(WsHeader *h, int code, unsigned int tile) {
  if (atomicCAS(&h->status, 0, code) == 0) atomicExch(&h->err_tile, tile);
}

// Bit casts between T and same-sized unsigned integers.
template <typename T>
struct Bits;
template <>
struct Bits<int32_t> { using U = uint32_t; };
template <>
struct Bits<uint32_t> { using U = uint32_t; };
template <>
struct Bits<float> { using U = uint32_t; };
template <>
struct Bits<int64_t> { using U = unsigned long long; };
template <>
struct Bits<uint64_t> { using U = unsigned long long; };
template <>
struct Bits<double> { using U = unsigned long long; };

template <typename To, typename From>
__host__ __device__ __forceinline__ To bit_cast(const From &f) {
  static_assert(sizeof(To) == sizeof(From), "size");
  To t;
  memcpy(&t, &f, sizeof(To));
  return t;
}

// ---------------------------------------------------------------------------
// Warp / CTA collectives.
// ---------------------------------------------------------------------------
// Shuffles of any trivially copyable type, moved as 32-bit words.
enum class Shfl { Xor, Up, Down, Idx };
template <Shfl M, typename T>
__device__ __forceinline__ T shfl_any(T v, int arg) {
  static_assert(sizeof(T) % 4 == 0, "shuffle of 4-byte multiples");
  constexpr int W = sizeof(T) / 4;
  uint32_t w[W];
  memcpy(w, &v, sizeof(T));
#pragma unroll
  for (int i = 0; i < W; ++i) {
    if constexpr (M == Shfl::Xor) w[i] = __shfl_xor_sync(0xffffffffu, w[i], arg);
    else if constexpr (M == Shfl::Up) w[i] = __shfl_up_sync(0xffffffffu, w[i], arg);
    else if constexpr (M == Shfl::Down) w[i] = __shfl_down_sync(0xffffffffu, w[i], arg);
    else w[i] = __shfl_sync(0xffffffffu, w[i], arg);
  }
  T r;
  memcpy(&r, w, sizeof(T));
  return r;
}
template <typename T>
__device__ __forceinline__ T shfl_xor(T v, int m) { return shfl_any<Shfl::Xor>(v, m); }
template <typename T>
__device__ __forceinline__ T shfl_up(T v, int d) { return shfl_any<Shfl::Up>(v, d); }
template <typename T>
__device__ __forceinline__ T shfl_down_any(T v, int d) { return shfl_any<Shfl::Down>(v, d); }
template <typename T>
__device__ __forceinline__ T shfl_idx_any(T v, int s) { return shfl_any<Shfl::Idx>(v, s); }

template <typename T, typename Op>
__device__ __forceinline__ T warp_reduce(T v, Op op) {
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) v = op(v, shfl_xor(v, m));
  return v;
}

// Inclusive warp scan (Kogge-Stone over shuffles).
template <typename T, typename Op>
__device__ __forceinline__ T warp_inclusive_scan(T v, Op op, int lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T o = shfl_up(v, d);
    if (lane >= d) v = op(o, v);
  }
  return v;
}

// CTA-wide exclusive scan of one value per thread.  Returns the exclusive
// prefix (identity for thread 0) and writes the CTA aggregate.  s_warp needs
// THREADS/32 + 1 slots.  Ends with a barrier, so s_warp may be reused after.
template <int THREADS, typename T, typename Op>
__device__ __forceinline__ T block_exclusive_scan(T v, Op op, T *s_warp, T &aggregate) {
  constexpr int W = THREADS / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T incl = warp_inclusive_scan(v, op, lane);
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    T w = lane < W ? s_warp[lane] : Op::identity();
    T wi = warp_inclusive_scan(w, op, lane);
    if (lane < W) s_warp[lane] = wi;  // inclusive prefix over warps
  }
  __syncthreads();
  T warp_prefix = warp == 0 ? Op::identity() : s_warp[warp - 1];
  aggregate = s_warp[W - 1];
  T excl_in_warp = shfl_up(incl, 1);
  if (lane == 0) excl_in_warp = Op::identity();
  T r = warp == 0 ? excl_in_warp : (lane == 0 ? warp_prefix : op(warp_prefix, excl_in_warp));
  __syncthreads();
  return r;
}

template <int THREADS, typename T, typename Op>
__device__ __forceinline__ T block_reduce(T v, Op op, T *s_warp) {
  constexpr int W = THREADS / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_reduce(v, op);
  if (lane == 0) s_warp[warp] = v;
  __syncthreads();
  T r = Op::identity();
  if (warp == 0) {
    T w = lane < W ? s_warp[lane] : Op::identity();
    r = warp_reduce(w, op);
  }
  __syncthreads();
  return r;  // valid in warp 0
}

}  // namespace bk

// ---------------------------------------------------------------------------
// Host-side helpers shared by the entry points.
// ---------------------------------------------------------------------------
namespace bk {
namespace host {

struct DeviceInfo {
  int sm_count;
  int cc_major;
  int cc_minor;
  int max_smem_optin;
};

// Cached per device; thread-safe (call_once per slot).
int device_info(DeviceInfo *out);

// CTAs of `kern` (threads, dynamic shared memory) resident on the whole GPU
// at once: how far ahead of itself a CTA can usefully prefetch.
template <typename Kern>
inline uint64_t resident_ctas(Kern kern, int threads, size_t smem, int sm_count) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return (uint64_t)per_sm * (uint64_t)sm_count;
}

// Debug settings (process-wide, test-only).
struct DebugFault {
  long long skip_publish_tile;        // -1: none
  unsigned long long spin_limit_ns;   // 0: default
};
DebugFault debug_fault();
constexpr unsigned long long kDefaultSpinLimitNs = 2000000000ull;  // 2 s

inline int from_cuda(cudaError_t e) { return e == cudaSuccess ? BK_OK : (int)e; }

// Describes bytes [base, base + rows * 128) as a 2-D tensor of `rows` rows
// of 128 bytes for tiled TMA loads of `box_rows` rows with the 128-byte
// swizzle (`map` points at a 64-byte-aligned, 128-byte CUtensorMap).  base
// must be 16-byte aligned and rows > 0.  The driver's encoder is looked up
// once per process.
int encode_rows_128b(void *map, const void *base, uint64_t rows, uint32_t box_rows);

inline int check_ws(void *d_ws, size_t ws_bytes, size_t need) {
  if (need > 0 && d_ws == nullptr) return BK_ERR_INVALID_ARGUMENT;
  if (ws_bytes < need) return BK_ERR_WORKSPACE_TOO_SMALL;
  if ((reinterpret_cast<uintptr_t>(d_ws) & 255) != 0) return BK_ERR_MISALIGNED;
  return BK_OK;
}

template <typename T>
inline bool aligned_to(const void *p) {
  return (reinterpret_cast<uintptr_t>(p) % sizeof(T)) == 0;
}

inline int launch_status() { return from_cuda(cudaGetLastError()); }

// Opt a kernel into `bytes` of dynamic shared memory and the largest shared
// memory carveout (the L1 / shared split), so that as many CTAs as the
// shared memory allows are resident.
template <typename Kern>
inline int set_smem_attrs(Kern kern, size_t bytes) {
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
  return from_cuda(e);
}

// Runs setup(&value) once per device for the call site `Site` (a type unique
// to the caller, such as a struct local to a function template), with that
// device current, and caches the value only when setup returns BK_OK.
// Kernel attributes and occupancy belong to a device, so the cache is keyed
// by the current device, not by host thread.
template <typename Site, typename T, typename F>
inline int once_per_device(T *out, F &&setup) {
  int dev = 0;
  const cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  return PerDevice<T, Site>::get(dev, out, setup, BK_ERR_UNSUPPORTED);
}

// One kernel's per-device launch facts.
struct KernelSetup {
  uint64_t resident_ctas;  // CTAs of it resident on the whole GPU at once
};

// Once per device for the call site `Site`: opts `kern` into `smem` bytes of
// dynamic shared memory (and the largest carveout) and finds how many CTAs
// of `threads` threads are resident on the GPU at once.
template <typename Site, typename Kern>
inline int kernel_setup(Kern kern, int threads, size_t smem, KernelSetup *out) {
  return once_per_device<Site>(out, [&](KernelSetup *k) -> int {
    DeviceInfo di;
    int st = device_info(&di);
    if (st != BK_OK) return st;
    if ((st = set_smem_attrs(kern, smem)) != BK_OK) return st;
    k->resident_ctas = resident_ctas(kern, threads, smem, di.sm_count);
    return BK_OK;
  });
}

}  // namespace host
}  // namespace bk
