// bk_lookback.cuh -- single-pass decoupled look-back across CTAs.
//
// Each tile of a single-pass scan publishes its status in a per-tile slot:
//   INVALID   nothing yet
//   AGGREGATE the tile's own reduction (published as soon as it is known)
//   PREFIX    the inclusive prefix through this tile
// A payload of W 32-bit words occupies W 64-bit status words, each holding
// (tag << 32 | data word); tag 0 = INVALID, 1 = AGGREGATE, 2 = PREFIX.  Every
// 64-bit word is stored and loaded single-copy atomically, so a reader that
// sees the same non-zero tag in all W words holds a consistent payload (each
// tag is written at most once per call); mixed tags mean a write in progress
// and the reader looks again.  A slot is therefore read in one L2 round trip,
// with no fences.
//
// Warp 0 of a tile reads kLbPerLane x 32 predecessors per round, folds the
// aggregates up to the nearest PREFIX (in order, so non-commutative operators
// work) and slides the window back while none is found.  Tiles are handed out
// by an atomic ticket in launch order, so every predecessor a tile waits on is
// already running: the wait always ends.  Each wait is still bounded
// (globaltimer); on expiry the kernel records BK_ERR_SPIN_TIMEOUT in the
// workspace header and the tile returns instead of hanging.
#pragma once

#include "bk_common.cuh"

namespace bk {

enum : unsigned int { kStInvalid = 0u, kStAggregate = 1u, kStPrefix = 2u, kStError = 3u };
constexpr int kLbPerLane = 2;  // predecessors read per lane per round (64 per warp)

template <typename P>
struct TileStatus {
  static_assert(sizeof(P) % 4 == 0 && sizeof(P) <= 16, "payload of 4, 8, 12 or 16 bytes");
  static constexpr int W = sizeof(P) / 4;  // 32-bit payload words = 64-bit status words per tile
  unsigned long long *words;

  // Rounded up to whole groups of kLbPerLane tiles (the look-back reads groups).
  __host__ __device__ static size_t bytes(size_t tiles) { return align_up(align_up(tiles, (size_t)kLbPerLane) * W * 8, 256); }
  __host__ __device__ static TileStatus at(void *base, size_t /*tiles*/) {
    return TileStatus{reinterpret_cast<unsigned long long *>(base)};
  }

  __device__ __forceinline__ void publish(unsigned int tile, unsigned int flag, P v) const {
    uint32_t d[W];
    memcpy(d, &v, sizeof(P));
    unsigned long long *dst = words + (size_t)tile * W;
    const unsigned long long tag = (unsigned long long)flag << 32;
#pragma unroll
    for (int i = 0; i < W; ++i) st_relaxed_u64(dst + i, tag | d[i]);
  }
  // Returns INVALID while the slot is empty or being written.
  __device__ __forceinline__ unsigned int read(unsigned int tile, P &v) const {
    const unsigned long long *src = words + (size_t)tile * W;
    unsigned long long w[W];
#pragma unroll
    for (int i = 0; i < W; ++i) w[i] = ld_relaxed_u64(src + i);
    const unsigned int f = (unsigned int)(w[0] >> 32);
    bool same = true;
#pragma unroll
    for (int i = 1; i < W; ++i) same &= ((unsigned int)(w[i] >> 32) == f);
    if (!same) return kStInvalid;
    uint32_t d[W];
#pragma unroll
    for (int i = 0; i < W; ++i) d[i] = (uint32_t)(w[i] & 0xffffffffull);
    memcpy(&v, d, sizeof(P));
    return f;
  }
  __device__ __forceinline__ void clear(size_t tile) const {
#pragma unroll
    for (int i = 0; i < W; ++i) words[tile * W + i] = 0ull;
  }
};

// Ordered warp reduction: lane 0 receives v[31] (+) ... (+) v[1] (+) v[0]
// (higher lanes hold earlier tiles), valid for non-commutative operators.
template <typename P, typename Op>
__device__ __forceinline__ P warp_reduce_ordered(P v, Op op, int lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    P o = shfl_down_any(v, d);
    if (lane + d < 32) v = op(o, v);
  }
  return v;
}

// Spin (bounded) until the status of `tile` is valid.  Returns the flag, or
// kStError when the wait ran out or another tile already failed.
template <typename P, typename Status>
__device__ __forceinline__ unsigned int wait_status(const Status &st, unsigned int tile, P &v, WsHeader *hdr,
                                                    unsigned long long limit_ns, unsigned long long &t0) {
  unsigned int spins = 0;
  while (true) {
    const unsigned int f = st.read(tile, v);
    if (f != kStInvalid) return f;
    ++spins;
    if ((spins & 15u) == 0) {
      const unsigned long long now = globaltimer_ns();
      if (t0 == 0) {
        t0 = now;
      } else if (now - t0 > limit_ns || ld_relaxed_s32(&hdr->status) != 0) {
        return kStError;
      }
    }
    if (spins > 4) __nanosleep(spins < 128 ? 20 : 200);
  }
}

// Warp 0 of tile `tile` (> 0) computes the exclusive prefix of all earlier
// tiles.  Returns false (after recording the error) when a wait ran out or
// another tile already failed.  All 32 lanes must call it.
//
// Lane l reads the aligned group of kLbPerLane tiles g = G - l, where G is the
// group holding tile - 1, with 16-byte vector loads issued before any result
// is used.  Window position q = kLbPerLane * l + j (j = 0 is the lane's
// nearest tile) orders the window from nearest to farthest.  Only the tiles
// nearer than the nearest PREFIX are needed, so the warp waits for those alone
// and never for a slow tile beyond a PREFIX.  Tiles at or after `tile` in the
// first group do not take part.
template <typename P, typename Op, typename Status>
__device__ __forceinline__ bool lookback_exclusive(const Status &st, unsigned int tile, Op op, P &exclusive,
                                                   WsHeader *hdr, unsigned long long limit_ns) {
  constexpr int K = kLbPerLane;
  constexpr int W = Status::W;
  constexpr int GW = K * W;  // 64-bit words per group
  static_assert(GW % 2 == 0, "group is a whole number of 16-byte vectors");
  const int lane = threadIdx.x & 31;
  long long group = ((long long)tile - 1) / K - lane;
  P acc = Op::identity();
  unsigned long long t0 = 0;
  while (true) {
    P v[K];
    unsigned int f[K];
    int first_p = 32 * K;  // window position of the nearest PREFIX (32K = none)
    for (unsigned int spins = 0;; ++spins) {
      // ---- read the group (tiles 4g .. 4g+3; j = 0 is the nearest = 4g+3)
      if (group >= 0) {
        unsigned long long w[GW];
        const unsigned long long *src = st.words + (size_t)group * GW;
#pragma unroll
        for (int i = 0; i < GW; i += 2) ld_relaxed_v2_u64(src + i, w[i], w[i + 1]);
#pragma unroll
        for (int j = 0; j < K; ++j) {
          const int t = K - 1 - j;  // position within the group
          const unsigned int tag = (unsigned int)(w[t * W] >> 32);
          bool same = true;
          uint32_t d[W];
#pragma unroll
          for (int i = 0; i < W; ++i) {
            same &= ((unsigned int)(w[t * W + i] >> 32) == tag);
            d[i] = (uint32_t)(w[t * W + i] & 0xffffffffull);
          }
          f[j] = same ? tag : kStInvalid;
          memcpy(&v[j], d, sizeof(P));
        }
      } else {
#pragma unroll
        for (int j = 0; j < K; ++j) {
          f[j] = kStPrefix;  // before tile 0: never chosen, tile 0 always publishes PREFIX
          v[j] = Op::identity();
        }
      }
#pragma unroll
      for (int j = 0; j < K; ++j) {
        if (group * K + (K - 1 - j) >= (long long)tile) {  // at or after this tile
          f[j] = kStAggregate;
          v[j] = Op::identity();
        }
      }
      // ---- nearest PREFIX, and whether any tile nearer than it is missing
      int lane_first_p = K, lane_first_inv = K;
#pragma unroll
      for (int j = K - 1; j >= 0; --j) {
        if (f[j] == kStPrefix) lane_first_p = j;
        if (f[j] == kStInvalid) lane_first_inv = j;
      }
      const unsigned int pmask = __ballot_sync(0xffffffffu, lane_first_p < K);
      first_p = pmask ? (__ffs(pmask) - 1) * K + shfl_idx_any(lane_first_p, __ffs(pmask) - 1) : 32 * K;
      const bool missing = lane_first_inv < K && (K * lane + lane_first_inv) < first_p;
      if (!__any_sync(0xffffffffu, missing)) break;
      // ---- bounded wait
      if ((spins & 15u) == 15u) {
        const unsigned long long now = globaltimer_ns();
        bool give_up = false;
        if (t0 == 0) t0 = now;
        else give_up = (now - t0 > limit_ns) || (ld_relaxed_s32(&hdr->status) != 0);
        if (__any_sync(0xffffffffu, give_up)) {
          if (lane == 0) record_error(hdr, BK_ERR_SPIN_TIMEOUT, tile);
          return false;
        }
      }
      __nanosleep(spins < 32 ? 32 : 256);
    }
    // ---- ordered fold of positions nearer than (and including) first_p
    P lv = Op::identity();
#pragma unroll
    for (int j = K - 1; j >= 0; --j)
      if (K * lane + j <= first_p) lv = op(lv, v[j]);
    P wsum = warp_reduce_ordered(lv, op, lane);
    wsum = shfl_idx_any(wsum, 0);
    acc = op(wsum, acc);
    if (first_p < 32 * K) break;
    group -= 32;
  }
  exclusive = acc;
  return true;
}

}  // namespace bk
