// bulk/malloc.hpp -- the group's on-chip heap.
//
// Interface of the reference's bulk/malloc.hpp (malloc(g, n) :584-602,
// free(g, p) :605-615, shmalloc / shfree :518-581, is_on_chip :32-35,
// on_chip_cast :39-59): a concurrent group (one CTA) allocates from its heap,
// which lives in the CTA's dynamic shared memory (up to 227 KB on B200,
// opted in by bulk::async).  The design is this library's own: a stack of
// 16-byte-aligned blocks, each preceded by a 16-byte header with its size, so
// freeing the most recent block pops it and other frees are deferred until
// the blocks above them are freed.  When the heap is exhausted the request
// falls back to the device heap (as the reference does); bulk::free returns
// such blocks to it.
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
  unsigned int size;  // payload bytes (multiple of 16)
  unsigned int freed;
  unsigned int pad[2];
};

// Called by one thread of the CTA before the group runs.
__device__ inline void heap_init(unsigned int bytes) {
  s_heap_top = 0;
  s_heap_limit = bytes;
}

}  // namespace detail

__device__ inline bool is_on_chip(void *ptr) { return __isShared(ptr); }

template <typename T>
__device__ inline T *on_chip_cast(T *ptr) { return ptr; }

// One agent's allocation from its group's heap (falls back to the device heap).
__device__ inline void *shmalloc(size_t num_bytes) {
  const unsigned int need = (unsigned int)((num_bytes + 15) & ~size_t(15)) + sizeof(detail::heap_block_header);
  unsigned int old = atomicAdd(&detail::s_heap_top, need);
  if (old + need <= detail::s_heap_limit) {
    auto *h = reinterpret_cast<detail::heap_block_header *>(detail::s_bulk_heap + old);
    h->size = need - sizeof(detail::heap_block_header);
    h->freed = 0;
    return h + 1;
  }
  atomicSub(&detail::s_heap_top, need);
  return ::malloc(num_bytes);
}

// Frees a block from shmalloc: the top block pops (with any freed blocks
// below it); a block further down is released when the blocks above it are.
__device__ inline void shfree(void *ptr) {
  if (ptr == nullptr) return;
  if (!is_on_chip(ptr)) {
    ::free(ptr);
    return;
  }
  auto *h = reinterpret_cast<detail::heap_block_header *>(ptr) - 1;
  h->freed = 1;
  // pop freed blocks from the top (single-agent use, or under the group's
  // barrier).  Blocks are contiguous from offset 0; a header whose size
  // leaves the heap (overwritten by a caller) stops the walk.
  unsigned int top = detail::s_heap_top;
  const unsigned int limit = detail::s_heap_limit;
  unsigned char *base = detail::s_bulk_heap;
  while (top > 0 && top <= limit) {
    unsigned int off = 0, last = 0;
    bool sane = true;
    while (off < top) {
      last = off;
      if (off + sizeof(detail::heap_block_header) > limit) {
        sane = false;
        break;
      }
      const unsigned int size = reinterpret_cast<detail::heap_block_header *>(base + off)->size;
      if (size > limit - off - sizeof(detail::heap_block_header)) {
        sane = false;
        break;
      }
      off += sizeof(detail::heap_block_header) + size;
    }
    if (!sane || off != top) break;
    auto *lh = reinterpret_cast<detail::heap_block_header *>(base + last);
    if (!lh->freed) break;
    top = last;
  }
  detail::s_heap_top = top;
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

}  // namespace bulk
