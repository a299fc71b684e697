// bk_lookback.cuh -- single-pass decoupled look-back across CTAs.
//
// Each tile of a single-pass scan publishes its status in a per-tile word:
//   INVALID   nothing yet
//   AGGREGATE the tile's own reduction (published as soon as it is known)
//   PREFIX    the inclusive prefix through this tile
// A tile's warp 0 reads the 32 nearest predecessors at once, folds the
// aggregates up to the nearest PREFIX, and slides the window back while none
// is found.  Tiles are handed out by an atomic ticket in launch order, so every
// predecessor a tile waits on is already running: the wait always ends.  Each
// wait is still bounded (globaltimer), and on expiry the kernel records
// BK_ERR_SPIN_TIMEOUT in the workspace header and returns instead of hanging.
#pragma once

#include "bk_common.cuh"

namespace bk {

enum : unsigned int { kStInvalid = 0u, kStAggregate = 1u, kStPrefix = 2u, kStError = 3u };

// Payloads of 4 bytes share one 64-bit word with their flag (single-copy
// atomic store/load).  Larger payloads (8 or 16 bytes) use a flag array plus
// separate aggregate / prefix arrays ordered by release/acquire.
template <typename P, bool kPacked = (sizeof(P) == 4)>
struct TileStatus;

template <typename P>
struct TileStatus<P, true> {
  unsigned long long *words;

  __host__ __device__ static size_t bytes(size_t tiles) { return align_up(tiles * 8, 256); }
  __host__ __device__ static TileStatus at(void *base, size_t /*tiles*/) {
    return TileStatus{reinterpret_cast<unsigned long long *>(base)};
  }

  __device__ __forceinline__ void publish(unsigned int tile, unsigned int flag, P v) const {
    st_relaxed_u64(words + tile, ((unsigned long long)flag << 32) | (unsigned long long)bit_cast<uint32_t>(v));
  }
  __device__ __forceinline__ unsigned int read(unsigned int tile, P &v) const {
    unsigned long long w = ld_relaxed_u64(words + tile);
    v = bit_cast<P>((uint32_t)(w & 0xffffffffull));
    return (unsigned int)(w >> 32);
  }
  // Zero `tiles` words; called by the init kernel.
  __device__ __forceinline__ void clear(size_t i) const { words[i] = 0ull; }
};

template <typename P>
struct TileStatus<P, false> {
  static_assert(sizeof(P) % 8 == 0 && sizeof(P) <= 16, "payload of 8 or 16 bytes");
  static constexpr int kWords = sizeof(P) / 8;
  unsigned int *flags;
  unsigned long long *agg;
  unsigned long long *incl;

  __host__ __device__ static size_t bytes(size_t tiles) {
    return align_up(tiles * 4, 256) + 2 * align_up(tiles * sizeof(P), 256);
  }
  __host__ __device__ static TileStatus at(void *base, size_t tiles) {
    char *b = reinterpret_cast<char *>(base);
    TileStatus s;
    s.flags = reinterpret_cast<unsigned int *>(b);
    s.agg = reinterpret_cast<unsigned long long *>(b + align_up(tiles * 4, 256));
    s.incl = reinterpret_cast<unsigned long long *>(b + align_up(tiles * 4, 256) + align_up(tiles * sizeof(P), 256));
    return s;
  }
  __device__ __forceinline__ void publish(unsigned int tile, unsigned int flag, P v) const {
    unsigned long long w[kWords];
    memcpy(w, &v, sizeof(P));
    unsigned long long *dst = (flag == kStAggregate ? agg : incl) + (size_t)tile * kWords;
#pragma unroll
    for (int i = 0; i < kWords; ++i) st_relaxed_u64(dst + i, w[i]);
    st_release_u32(flags + tile, flag);  // orders the payload before the flag
  }
  __device__ __forceinline__ unsigned int read(unsigned int tile, P &v) const {
    unsigned int f = ld_acquire_u32(flags + tile);
    if (f == kStAggregate || f == kStPrefix) {
      const unsigned long long *src = (f == kStAggregate ? agg : incl) + (size_t)tile * kWords;
      unsigned long long w[kWords];
#pragma unroll
      for (int i = 0; i < kWords; ++i) w[i] = ld_relaxed_u64(src + i);
      memcpy(&v, w, sizeof(P));
    }
    return f;
  }
  __device__ __forceinline__ void clear(size_t i) const { flags[i] = 0u; }
};

// Ordered warp reduction: lane 0 receives v[31] (+) ... (+) v[1] (+) v[0]
// (higher lanes are earlier tiles), valid for non-commutative operators.
template <typename P, typename Op>
__device__ __forceinline__ P warp_reduce_ordered(P v, Op op, int lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    P o = shfl_down_any(v, d);
    if (lane + d < 32) v = op(o, v);
  }
  return v;
}

// Warp 0 of tile `tile` (> 0) computes the exclusive prefix of all earlier
// tiles.  Returns false (after recording the error) when a wait ran out or
// another tile already failed.
template <typename P, typename Op, typename Status>
__device__ __forceinline__ bool lookback_exclusive(const Status &st, unsigned int tile, Op op, P &exclusive,
                                                   WsHeader *hdr, unsigned long long limit_ns) {
  const int lane = threadIdx.x & 31;
  long long pred = (long long)tile - 1;
  P acc = Op::identity();
  unsigned long long t0 = 0;
  while (true) {
    const long long idx = pred - lane;
    P v = Op::identity();
    unsigned int f = kStPrefix;  // indices below 0 never occur: tile 0 always publishes PREFIX
    if (idx >= 0) {
      unsigned int spins = 0;
      while (true) {
        f = st.read((unsigned int)idx, v);
        if (f != kStInvalid) break;
        ++spins;
        if ((spins & 31u) == 0) {
          unsigned long long now = globaltimer_ns();
          if (t0 == 0) {
            t0 = now;
          } else if (now - t0 > limit_ns || ld_relaxed_s32(&hdr->status) != 0) {
            f = kStError;
            break;
          }
        }
        if (spins > 8) __nanosleep(spins < 256 ? 32 : 256);
      }
    }
    if (__any_sync(0xffffffffu, f == kStError)) {
      if (lane == 0) record_error(hdr, BK_ERR_SPIN_TIMEOUT, tile);
      return false;
    }
    const unsigned int pmask = __ballot_sync(0xffffffffu, f == kStPrefix);
    const int stop = pmask ? (__ffs(pmask) - 1) : 31;
    if (lane > stop) v = Op::identity();
    P w = warp_reduce_ordered(v, op, lane);
    w = shfl_idx_any(w, 0);
    acc = op(w, acc);
    if (pmask) break;
    pred -= 32;
  }
  exclusive = acc;
  return true;
}

}  // namespace bk
