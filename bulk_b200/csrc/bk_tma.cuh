// bk_tma.cuh -- bulk (TMA) copies between global and shared memory, and the
// mbarrier they complete on (sm_90+ PTX, used here for sm_100a).
//
// Two forms are used: the untiled cp.async.bulk (global->shared with an
// mbarrier complete_tx, shared->global with a bulk group), whose addresses
// must be 16-byte aligned and whose size is a multiple of 16 bytes (callers
// fetch ragged edges with plain loads); and the tiled 2-D
// cp.async.bulk.tensor load over a "row view" of a 1-D array (rows of 128
// bytes, see host::encode_rows_128b) with the 128-byte swizzle, whose x
// coordinate is always 0.  No multicast form appears anywhere in this
// library.
#pragma once

#include <cuda.h>  // CUtensorMap (type only; the encoder comes from the driver at run time)

#include "bk_common.cuh"

namespace bk {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Make the barrier initialisation and earlier generic-proxy shared-memory
// writes visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Orders this thread's earlier generic-proxy global writes before later
// async-proxy (TMA) accesses that a release / acquire chain makes depend on
// them.
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// Adds `bytes` to the transaction count bar's current phase waits for,
// without arriving (the arrival comes later, after any plain stores that the
// waiting threads must also see).
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// Bulk copy global -> shared; completes `bytes` of transaction count on bar.
__device__ __forceinline__ void tma_load_1d(void *smem_dst, const void *gmem_src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// L2 eviction-priority policies for the cache_hint forms below.
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// Bulk copy global -> shared with an L2 eviction-priority hint.
__device__ __forceinline__ void tma_load_1d_hint(void *smem_dst, const void *gmem_src, uint32_t bytes, uint64_t *bar,
                                                 uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
          "r"(smem_addr(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}

// Tiled 2-D copy global -> shared of the box at row `row` (x = 0) of the row
// view `map` (a __grid_constant__ kernel parameter), with an L2 eviction
// hint; completes the box's bytes on bar (rows past the view read as zero
// and still count).  dst must be 1024-byte aligned for the 128-byte swizzle.
__device__ __forceinline__ void tma_load_rows(void *smem_dst, const CUtensorMap *map, uint32_t row, uint64_t *bar,
                                              uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1, {%2, %3}], [%4], %5;" ::"r"(smem_addr(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(row), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}

// Tiled 2-D copy shared -> global of a box at row `row` of the row view
// `map`, tracked by the issuing thread's bulk group (rows past the view are
// not written).
__device__ __forceinline__ void tma_store_rows(const CUtensorMap *map, uint32_t row, const void *smem_src,
                                               uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.2d.global.shared::cta.bulk_group.L2::cache_hint [%0, {%1, %2}], [%3], %4;" ::"l"(
          reinterpret_cast<uint64_t>(map)),
      "r"(0), "r"(row), "r"(smem_addr(smem_src)), "l"(policy)
      : "memory");
}

// Byte offset at which a tensor copy with the 128-byte swizzle places byte
// `o` of a 1024-byte-aligned box of 128-byte rows: the 16-byte chunk index
// within each row is XORed with the row index mod 8, so eight lanes that
// read the same chunk of eight consecutive rows hit eight distinct bank
// groups.
__host__ __device__ __forceinline__ uint32_t swz128(uint32_t o) { return o ^ (((o >> 7) & 7u) << 4); }

// Bounded wait for phase `parity` of bar.  Returns false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, unsigned long long limit_ns) {
  const uint32_t a = smem_addr(bar);
  unsigned long long t0 = 0;
  for (uint32_t it = 0;; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 15u) == 15u) {
      const unsigned long long now = globaltimer_ns();
      if (t0 == 0) t0 = now;
      else if (now - t0 > limit_ns) return false;
    }
  }
}

// Plain arrival on an mbarrier (no transaction bytes).
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Bounded wait for phase `parity` of bar that also gives up as soon as
// *abort_flag is non-zero.  Returns true when the phase completed.
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t *bar, uint32_t parity, unsigned long long limit_ns,
                                                   const int *abort_flag) {
  const uint32_t a = smem_addr(bar);
  unsigned long long t0 = 0;
  for (uint32_t it = 0;; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 15u) == 15u) {
      if (*reinterpret_cast<const volatile int *>(abort_flag) != 0) return false;
      const unsigned long long now = globaltimer_ns();
      if (t0 == 0) t0 = now;
      else if (now - t0 > limit_ns) return false;
    }
  }
}

// Bulk copy shared -> global, tracked by the issuing thread's bulk group.
__device__ __forceinline__ void tma_store_1d(void *gmem_dst, const void *smem_src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gmem_dst),
               "r"(smem_addr(smem_src)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tma_store_1d_hint(void *gmem_dst, const void *smem_src, uint32_t bytes,
                                                  uint64_t policy) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group.L2::cache_hint [%0], [%1], %2, %3;" ::"l"(gmem_dst),
               "r"(smem_addr(smem_src)), "r"(bytes), "l"(policy)
               : "memory");
}
__device__ __forceinline__ void tma_store_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Wait until every committed bulk store has finished reading shared memory.
__device__ __forceinline__ void tma_store_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// Wait until every committed bulk store is complete (writes visible).
__device__ __forceinline__ void tma_store_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

}  // namespace bk
