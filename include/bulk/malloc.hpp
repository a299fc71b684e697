// bulk/malloc.hpp -- the group's on-chip heap.
//
// Interface of the reference's bulk/malloc.hpp (malloc(g, n) :584-602,
// free(g, p) :605-615, shmalloc / shfree :518-581, is_on_chip :32-35,
// on_chip_cast :39-59): a concurrent group (one CTA) allocates from its heap,
// which lives in the CTA's dynamic shared memory (up to 227 KB on B200,
// opted in by bulk::async).  The design is this library's own: a stack of
// 16-byte-aligned blocks, each preceded by a 16-byte header with its size and
// owner, so freeing the most recent block pops it and other frees are
// deferred until the blocks above them are freed.  When the CTA's heap is
// exhausted and the CTA belongs to a thread-block cluster, the request goes
// to the heaps of the other CTAs of the cluster (distributed shared memory,
// addressed through the cluster's shared window); when those are full too it
// falls back to the device heap (as the reference does).  bulk::free returns
// each block to where it came from.  A cluster group (a concurrent group of
// CTAs) allocates collectively from the cluster's heaps; its blocks are
// addressed through the cluster window, so every CTA of the cluster reaches
// them.
#pragma once

#include <cstddef>
#include <cstdint>

#include "execution_policy.hpp"

namespace bulk {
namespace detail {

extern __shared__ __align__(16) unsigned char s_bulk_heap[];
static __shared__ unsigned int s_heap_top;    // bytes in use
static __shared__ unsigned int s_heap_limit;  // heap capacity in bytes
static __shared__ void *s_malloc_result;

struct heap_block_header {
  unsigned int size;   // payload bytes (multiple of 16)
  unsigned int freed;
  unsigned int owner;  // cluster rank of the CTA whose heap holds the block
  unsigned int pad;
};

// Called by one thread of the CTA before the group runs.
__device__ inline void heap_init(unsigned int bytes) {
  s_heap_top = 0;
  s_heap_limit = bytes;
}

// The generic address of the same shared-memory location in CTA `rank` of
// this CTA's cluster (valid from every CTA of the cluster).
template <typename T>
__device__ inline T *cluster_map(T *p, unsigned int rank) {
  uint64_t r = reinterpret_cast<uint64_t>(p);
#ifdef __CUDA_ARCH__
  asm volatile("mapa.u64 %0, %1, %2;" : "=l"(r) : "l"(r), "r"(rank));
#endif
  return reinterpret_cast<T *>(r);
}

__device__ inline bool is_cluster_shared(const void *p) {
  unsigned int r = 0;
#ifdef __CUDA_ARCH__
  asm volatile("{\n\t.reg .pred q;\n\tisspacep.shared::cluster q, %1;\n\tselp.u32 %0, 1, 0, q;\n\t}"
               : "=r"(r)
               : "l"(p));
#endif
  return r != 0;
}

// Reserves `need` bytes on top of the heap whose top / limit words and base
// are given (this CTA's, or a peer's through the cluster window).  A bounded
// compare-and-swap loop: other CTAs of the cluster may allocate from the
// same heap at the same time.  Returns the block's offset, or ~0u.
__device__ inline unsigned int heap_reserve(unsigned int *top, unsigned int limit, unsigned int need) {
  unsigned int cur = *reinterpret_cast<volatile unsigned int *>(top);
  for (int tries = 0; tries < 1024; ++tries) {
    if (cur > limit || need > limit - cur) return ~0u;
    const unsigned int prev = atomicCAS(top, cur, cur + need);
    if (prev == cur) return cur;
    cur = prev;
  }
  return ~0u;
}

// Pops freed blocks off the top of the heap of cluster rank `owner` (the
// caller's own CTA when it is not in a cluster).  Blocks are contiguous from
// offset 0; a header whose size leaves the heap (overwritten by a caller, or
// still being written by a peer) stops the walk, and a top that moved while
// the walk ran (a peer allocated) is left as it is.
__device__ inline void heap_pop(unsigned int owner, bool in_cluster) {
  unsigned int *top_p = in_cluster ? cluster_map(&s_heap_top, owner) : &s_heap_top;
  const unsigned int limit = in_cluster ? *cluster_map(&s_heap_limit, owner) : s_heap_limit;
  unsigned char *base = in_cluster ? cluster_map(&s_bulk_heap[0], owner) : s_bulk_heap;
  for (int rounds = 0; rounds < 4096; ++rounds) {
    const unsigned int top = *reinterpret_cast<volatile unsigned int *>(top_p);
    if (top == 0 || top > limit) return;
    unsigned int off = 0, last = 0;
    while (off < top) {
      last = off;
      if (off + sizeof(heap_block_header) > limit) return;
      const unsigned int size = reinterpret_cast<volatile heap_block_header *>(base + off)->size;
      if (size > limit - off - sizeof(heap_block_header)) return;
      off += sizeof(heap_block_header) + size;
    }
    if (off != top) return;
    if (!reinterpret_cast<volatile heap_block_header *>(base + last)->freed) return;
    if (atomicCAS(top_p, top, last) != top) return;
  }
}

}  // namespace detail

// Whether ptr is in on-chip memory: this CTA's shared memory or, inside a
// cluster, another CTA's (distributed shared memory).
__device__ inline bool is_on_chip(void *ptr) { return __isShared(ptr) || detail::is_cluster_shared(ptr); }

template <typename T>
__device__ inline T *on_chip_cast(T *ptr) { return ptr; }

// One agent's allocation: from its CTA's heap, else (in a cluster) from the
// heaps of the other CTAs of the cluster, nearest rank first, else from the
// device heap.
__device__ inline void *shmalloc(size_t num_bytes) {
  const unsigned int need = (unsigned int)((num_bytes + 15) & ~size_t(15)) + sizeof(detail::heap_block_header);
  const unsigned int me = detail::cluster_ctarank(), ranks = detail::cluster_nctarank();
  for (unsigned int k = 0; k < ranks; ++k) {
    const unsigned int r = (me + k) % ranks;
    const bool local = r == me;
    unsigned int *top = local ? &detail::s_heap_top : detail::cluster_map(&detail::s_heap_top, r);
    const unsigned int limit = local ? detail::s_heap_limit : *detail::cluster_map(&detail::s_heap_limit, r);
    const unsigned int off = detail::heap_reserve(top, limit, need);
    if (off == ~0u) continue;
    unsigned char *base = local ? detail::s_bulk_heap : detail::cluster_map(&detail::s_bulk_heap[0], r);
    auto *h = reinterpret_cast<detail::heap_block_header *>(base + off);
    h->size = need - sizeof(detail::heap_block_header);
    h->freed = 0;
    h->owner = r;
    return h + 1;
  }
  return ::malloc(num_bytes);
}

// Frees a block from shmalloc: the top block of its heap pops (with any
// freed blocks below it); a block further down is released when the blocks
// above it are.
__device__ inline void shfree(void *ptr) {
  if (ptr == nullptr) return;
  const bool local = __isShared(ptr);
  if (!local && !detail::is_cluster_shared(ptr)) {
    ::free(ptr);
    return;
  }
  auto *h = reinterpret_cast<detail::heap_block_header *>(ptr) - 1;
  const unsigned int owner = h->owner;
  __threadfence_block();
  h->freed = 1;
  if (local) detail::heap_pop(detail::cluster_ctarank(), false);
  else detail::heap_pop(owner, true);
}

// Collective allocation: every agent of the group calls it and receives the
// same block.
template <typename ConcurrentGroup>
__device__ inline void *malloc(ConcurrentGroup &g, size_t num_bytes) {
  g.wait();
  if (g.this_exec.index() == 0) detail::s_malloc_result = shmalloc(num_bytes);
  g.wait();
  void *r = detail::s_malloc_result;
  g.wait();
  return r;
}

template <typename ConcurrentGroup>
__device__ inline void free(ConcurrentGroup &g, void *ptr) {
  g.wait();
  if (g.this_exec.index() == 0) shfree(ptr);
  g.wait();
}

// Collective allocation by a cluster group: agent 0 of CTA 0 allocates (its
// CTA's heap first, then the other CTAs'), and every agent of every CTA
// receives the block's address in the cluster's shared window.
template <typename InnerAgent, std::size_t S, std::size_t C>
__device__ inline void *malloc(concurrent_group<concurrent_group<InnerAgent, S>, C> &g, size_t num_bytes) {
  g.wait();
  if (g.this_exec.index() == 0 && g.this_exec.this_exec.index() == 0) {
    void *p = shmalloc(num_bytes);
    if (__isShared(p)) p = detail::cluster_map(p, detail::cluster_ctarank());  // reachable from every CTA
    detail::s_malloc_result = p;
  }
  g.wait();
  void *r = *detail::cluster_map(&detail::s_malloc_result, 0u);
  g.wait();
  return r;
}

template <typename InnerAgent, std::size_t S, std::size_t C>
__device__ inline void free(concurrent_group<concurrent_group<InnerAgent, S>, C> &g, void *ptr) {
  g.wait();
  if (g.this_exec.index() == 0 && g.this_exec.this_exec.index() == 0) shfree(ptr);
  g.wait();
}

}  // namespace bulk
