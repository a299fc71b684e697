// reduce_by_key.cu -- single-pass reduce_by_key (equal_to, plus), sm_100a.
//
// Replaces the reference's five-step my_reduce_by_key (reduce_by_key.cu:
// 176-272): reduce_intervals counts tail flags per interval (:240,
// reduce_intervals.hpp:6-47), a thrust::inclusive_scan turns them into output
// offsets (:243), reduce_by_key_kernel reduces each interval with
// bulk::reduce_by_key (:16-130, bulk/algorithm/reduce_by_key.hpp:115-216)
// leaving a carry per interval, thrust::inclusive_scan_by_key combines the
// carries (:255-260) and sum_tail_carries adds them in (:146-173); the keys are
// read twice and the result size comes back through a synchronous copy.
//
// Here it is one segmented scan with decoupled look-back: the input is read
// once, the output written once.  The scan element is (c, v): c counts run
// heads (a head is an element whose key differs from its predecessor's), v is
// the sum of the values since the last head.  (c1,v1) (+) (c2,v2) =
// (c1 + c2, c2 ? v2 : v1 + v2) is associative but not commutative, so every
// fold keeps data order.  At each tail (last element of a run) the inclusive
// (c, v) gives the run's output slot c - 1 and its sum v.  The tile pipeline
// is the scan's (scan.cu): persistent CTAs whose compute warps, loader lane
// and look-back warp hand over through mbarriers; three tile buffers rotate
// through prefetch (keys, values and a one-key halo on each side, by TMA),
// phase 1 (the tile aggregate, published), a re-read from L2 and phase 2
// (the tile's runs, emitted once the look-back warp has found the prefix).
#include <algorithm>

#include "bk_common.cuh"
#include "bk_tune.hpp"
#include "bk_lookback.cuh"
#include "bk_tma.cuh"

namespace bk {

template <typename V>
struct Seg {
  uint32_t c;  // run heads
  V v;         // sum since the last head
};

template <typename V>
struct OpSeg {
  __device__ __forceinline__ Seg<V> operator()(const Seg<V> &a, const Seg<V> &b) const {
    Seg<V> r;
    r.c = a.c + b.c;
    r.v = b.c ? b.v : (V)(a.v + b.v);
    return r;
  }
  __host__ __device__ static constexpr Seg<V> identity() { return Seg<V>{0u, V(0)}; }
};

constexpr int kRbkWarps = 8;                       // compute warps (0-7)
constexpr int kRbkThreads = 32 * (kRbkWarps + 2);  // + the loader warp (8; one lane works) + the look-back warp (9)
constexpr int kRbkBufs = 3;                        // tile buffers in rotation (as in scan.cu)
constexpr int kRbkQueue = 4;                       // look-back queue entries

template <typename K, typename V>
struct RbkCfg {
  // each lane owns M consecutive elements: 64 bytes of the wider of key/value
  static constexpr int M = 64 / (sizeof(K) > sizeof(V) ? sizeof(K) : sizeof(V));  // 16 or 8
  static constexpr int TILE = kRbkWarps * 32 * M;                                  // 4096 or 2048
  static constexpr uint32_t KROWS = sizeof(K) * TILE / 128;  // 128-byte rows of keys in a tile
  static constexpr uint32_t VROWS = sizeof(V) * TILE / 128;  // ... and of values
  // a buffer: the keys area, then the values area, each a whole number of
  // 1024-byte swizzle periods
  static constexpr size_t KEY_BYTES = align_up(sizeof(K) * TILE, 1024);
  static constexpr size_t VAL_BYTES = align_up(sizeof(V) * TILE, 1024);
  static constexpr size_t BUF_BYTES = KEY_BYTES + VAL_BYTES;
  static constexpr int KCH = M * (int)sizeof(K) / 16;  // 16-byte chunks of a lane's keys
  static constexpr int VCH = M * (int)sizeof(V) / 16;  // ... and of its values
  using P = Seg<V>;
  using Status = TileStatus<P>;
};

template <typename K, typename V>
size_t rbk_num_tiles(uint64_t n) {
  return (size_t)((n + RbkCfg<K, V>::TILE - 1) / RbkCfg<K, V>::TILE);
}
// Workspace: the header, one look-back status per tile, then the tail-mark
// ring: three tile-sized value slots per persistent CTA (phase 1 of a tile
// writes its running values there; the re-read for phase 2 brings them back).
constexpr size_t kRbkMaxGrid = 320;  // persistent CTAs at most (2 per SM)
template <typename K, typename V>
size_t rbk_ring_offset(size_t tiles) {
  return align_up(kHeaderBytes + RbkCfg<K, V>::Status::bytes(tiles), 256);
}
template <typename K, typename V>
size_t rbk_ws_for_tiles(size_t tiles) {
  const size_t slots = 3 * (tiles < kRbkMaxGrid ? tiles : kRbkMaxGrid);
  return rbk_ring_offset<K, V>(tiles) + slots * RbkCfg<K, V>::TILE * sizeof(V);
}
template <typename K, typename V>
size_t rbk_ws_bytes(uint64_t n) {
  return rbk_ws_for_tiles<K, V>(rbk_num_tiles<K, V>(n));
}

template <typename Status>
__global__ void rbk_init_kernel(Status st, size_t tiles, WsHeader *hdr) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t padded = align_up(tiles, (size_t)kLbPerLane);
  for (size_t t = i; t < padded; t += stride) st.clear(t);
  if (i == 0) hdr->tile_ticket = 0u;
}

template <typename V>
__global__ void write_count_kernel(uint64_t *d_num_out) { *d_num_out = 0; }

// Where one tile lives: its array (keys, values, length, outputs) and its
// index within that array.
template <typename K, typename V>
struct RbkTile {
  const K *keys;
  const V *vals;
  uint64_t n;
  uint32_t local;  // tile index within the array
  K *out_keys;
  V *out_vals;
  uint64_t *num_out;
  bool tma;        // the loader brings this tile (and its re-read) in by TMA
  __device__ __forceinline__ uint32_t count() const {
    const uint64_t base = (uint64_t)local * RbkCfg<K, V>::TILE;
    return (uint32_t)((n - base) < (uint64_t)RbkCfg<K, V>::TILE ? (n - base) : (uint64_t)RbkCfg<K, V>::TILE);
  }
  __device__ __forceinline__ bool first() const { return local == 0u; }
  __device__ __forceinline__ bool last() const { return (uint64_t)local * RbkCfg<K, V>::TILE + count() == n; }
};

// Tile source: one array.  Its keys and values are described as row views
// (rows of 128 bytes) so that a tile arrives by two tiled TMA copies with the
// 128-byte swizzle: a lane then reads its M consecutive keys and values as
// 16-byte chunks, eight lanes of each access phase on eight distinct bank
// groups, with no rearranging in registers.  Tiles past `covered` (the
// ragged end, or every tile of an array not 16-byte aligned) are staged by
// the compute warps with plain loads into the same layout.
template <typename K, typename V>
struct RbkOne {
  static constexpr bool kSwz = true;
  CUtensorMap kmap;  // keys: rows of 128 bytes, boxes of KROWS rows
  CUtensorMap vmap;  // values: boxes of VROWS rows
  const K *keys;
  const V *vals;
  uint64_t n;
  K *out_keys;
  V *out_vals;
  uint64_t *num_out;
  uint64_t covered;  // leading elements inside whole rows of both views (0: none)
  int may_stage;     // some tile has no TMA copy (covered < n)
  __device__ __forceinline__ RbkTile<K, V> tile(unsigned int t) const {
    const uint64_t base = (uint64_t)t * RbkCfg<K, V>::TILE;
    const uint64_t cnt = (n - base) < (uint64_t)RbkCfg<K, V>::TILE ? (n - base) : (uint64_t)RbkCfg<K, V>::TILE;
    return RbkTile<K, V>{keys, vals, n, t, out_keys, out_vals, num_out, base + cnt <= covered};
  }
  __device__ __forceinline__ const CUtensorMap *key_map() const { return &kmap; }
  __device__ __forceinline__ const CUtensorMap *val_map() const { return &vmap; }
};

// Tile source: a batch of independent arrays reduced by one launch.  Array i
// owns global tiles [start[i], start[i + 1]); its first tile publishes an
// inclusive prefix at once, so no look-back crosses into another array.  The
// descriptors travel in the kernel's parameters; tiles arrive by untiled
// bulk copies (linear layout), and lanes read theirs with lane-rotated
// chunk order.
constexpr int kRbkBatchMax = 256;
template <typename K, typename V>
struct RbkBatch {
  static constexpr bool kSwz = false;
  const K *keys[kRbkBatchMax];
  const V *vals[kRbkBatchMax];
  uint64_t n[kRbkBatchMax];
  K *out_keys[kRbkBatchMax];
  V *out_vals[kRbkBatchMax];
  uint64_t *num_out[kRbkBatchMax];
  uint32_t start[kRbkBatchMax + 1];
  uint32_t count;
  int may_stage;  // some array is not 16-byte aligned
  __device__ __forceinline__ RbkTile<K, V> tile(unsigned int t) const {
    int lo = 0, hi = (int)count - 1;  // the last array whose first tile is <= t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (start[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    const bool tma = ((reinterpret_cast<uintptr_t>(keys[lo]) | reinterpret_cast<uintptr_t>(vals[lo])) & 15) == 0;
    return RbkTile<K, V>{keys[lo], vals[lo], n[lo], t - start[lo], out_keys[lo], out_vals[lo], num_out[lo], tma};
  }
  __device__ __forceinline__ const CUtensorMap *key_map() const { return nullptr; }
  __device__ __forceinline__ const CUtensorMap *val_map() const { return nullptr; }
};

// Byte offset of byte o of a tile area in shared memory (and in a mark-ring
// slot, which holds an image of the values area): swizzled for tiles that
// arrive by tensor copies, linear otherwise.
template <bool SWZ>
__device__ __forceinline__ uint32_t area_off(uint32_t o) {
  if constexpr (SWZ) return swz128(o);
  else return o;
}

// Loader: bring tile `tl` (keys, values and the halo keys on either side)
// into buffer `buf`.  The halo keys arrive as the aligned 16-byte chunks that
// hold them (hb[0]: the chunk ending just before the tile, hb[1]: the chunk
// starting just after it), on the same mbarrier as the tile.  Returns whether
// a TMA copy was issued on `bar`; tiles without one are staged by the compute
// warps (the halo keys still come from here, by plain loads).
template <typename K, typename V, typename Src>
__device__ __forceinline__ bool rbk_issue_load(const Src &src, const RbkTile<K, V> &tl, unsigned char *buf,
                                               K (*hb)[16 / sizeof(K)], uint64_t *bar, uint64_t policy) {
  using C = RbkCfg<K, V>;
  constexpr uint32_t KC = 16 / sizeof(K);  // keys per 16-byte chunk
  const uint64_t base = (uint64_t)tl.local * C::TILE;
  const uint32_t count = tl.count();
  if (!tl.tma) {
    if (base > 0) hb[0][KC - 1] = tl.keys[base - 1];
    if (base + count < tl.n) hb[1][0] = tl.keys[base + count];
    return false;
  }
  const bool halo_prev = base > 0;  // base is a multiple of TILE: the chunk before it is aligned
  const bool halo_next_bulk = (count % KC) == 0 && base + count + KC <= tl.n;
  if (!halo_next_bulk && base + count < tl.n) hb[1][0] = tl.keys[base + count];  // rare: next-to-last tile
  const uint32_t halo = (halo_prev ? 16u : 0u) + (halo_next_bulk ? 16u : 0u);
  K *sk = reinterpret_cast<K *>(buf);
  V *sv = reinterpret_cast<V *>(buf + C::KEY_BYTES);
  if constexpr (Src::kSwz) {
    mbar_arrive_expect_tx(bar, (C::KROWS + C::VROWS) * 128u + halo);
    tma_load_rows(sk, src.key_map(), tl.local * C::KROWS, bar, policy);
    tma_load_rows(sv, src.val_map(), tl.local * C::VROWS, bar, policy);
  } else {
    const uint32_t bk = count & ~(KC - 1);
    const uint32_t bv = count & ~(uint32_t)(16 / sizeof(V) - 1);
    for (uint32_t i = bk; i < count; ++i) sk[i] = tl.keys[base + i];
    for (uint32_t i = bv; i < count; ++i) sv[i] = tl.vals[base + i];
    const uint32_t bytes = bk * (uint32_t)sizeof(K) + bv * (uint32_t)sizeof(V) + halo;
    if (bytes == 0) return false;
    mbar_arrive_expect_tx(bar, bytes);
    if (bk) tma_load_1d_hint(sk, tl.keys + base, bk * (uint32_t)sizeof(K), bar, policy);
    if (bv) tma_load_1d_hint(sv, tl.vals + base, bv * (uint32_t)sizeof(V), bar, policy);
  }
  if (halo_prev) tma_load_1d_hint(hb[0], tl.keys + base - KC, 16u, bar, policy);
  if (halo_next_bulk) tma_load_1d_hint(hb[1], tl.keys + base + count, 16u, bar, policy);
  return true;
}

// Loader: re-read tile `tl` for phase 2 into buffer `buf`: its keys from the
// input (L2) and, in place of its values, the running values phase 1 left in
// the mark slot `slot` (an image of the values area).  Returns whether a TMA
// copy was issued on `bar`.
template <typename K, typename V, typename Src>
__device__ __forceinline__ bool rbk_issue_reload(const Src &src, const RbkTile<K, V> &tl, const V *slot,
                                                 unsigned char *buf, uint64_t *bar, uint64_t policy) {
  using C = RbkCfg<K, V>;
  constexpr uint32_t KC = 16 / sizeof(K);
  if (!tl.tma) return false;
  const uint32_t count = tl.count();
  K *sk = reinterpret_cast<K *>(buf);
  V *sv = reinterpret_cast<V *>(buf + C::KEY_BYTES);
  if constexpr (Src::kSwz) {
    mbar_arrive_expect_tx(bar, C::KROWS * 128u + (uint32_t)(C::TILE * sizeof(V)));
    tma_load_rows(sk, src.key_map(), tl.local * C::KROWS, bar, policy);
    tma_load_1d_hint(sv, slot, (uint32_t)(C::TILE * sizeof(V)), bar, policy);
  } else {
    const uint64_t base = (uint64_t)tl.local * C::TILE;
    const uint32_t bk = count & ~(KC - 1);
    for (uint32_t i = bk; i < count; ++i) sk[i] = tl.keys[base + i];
    const uint32_t vbytes = (uint32_t)align_up(count * sizeof(V), 16);  // within the slot
    mbar_arrive_expect_tx(bar, bk * (uint32_t)sizeof(K) + vbytes);
    if (bk) tma_load_1d_hint(sk, tl.keys + base, bk * (uint32_t)sizeof(K), bar, policy);
    tma_load_1d_hint(sv, slot, vbytes, bar, policy);
  }
  return true;
}

// Compute threads: plain copy of a tile into the buffer's layout (tiles
// without a TMA copy).
template <typename K, typename V, bool SWZ>
__device__ __forceinline__ void rbk_stage_load(const RbkTile<K, V> &tl, unsigned char *buf) {
  using C = RbkCfg<K, V>;
  const uint64_t base = (uint64_t)tl.local * C::TILE;
  const uint32_t count = tl.count();
  for (uint32_t i = threadIdx.x; i < count; i += kRbkWarps * 32) {
    *reinterpret_cast<K *>(buf + area_off<SWZ>(i * (uint32_t)sizeof(K))) = tl.keys[base + i];
    *reinterpret_cast<V *>(buf + C::KEY_BYTES + area_off<SWZ>(i * (uint32_t)sizeof(V))) = tl.vals[base + i];
  }
}

// Compute threads: plain copy of a tile's keys and its mark slot (an image of
// the values area) for phase 2.
template <typename K, typename V, bool SWZ>
__device__ __forceinline__ void rbk_stage_reload(const RbkTile<K, V> &tl, const V *slot, unsigned char *buf) {
  using C = RbkCfg<K, V>;
  const uint64_t base = (uint64_t)tl.local * C::TILE;
  const uint32_t count = tl.count();
  for (uint32_t i = threadIdx.x; i < count; i += kRbkWarps * 32)
    *reinterpret_cast<K *>(buf + area_off<SWZ>(i * (uint32_t)sizeof(K))) = tl.keys[base + i];
  const uint4 *s = reinterpret_cast<const uint4 *>(slot);
  uint4 *d = reinterpret_cast<uint4 *>(buf + C::KEY_BYTES);
  for (uint32_t c = threadIdx.x; c < (uint32_t)(C::TILE * sizeof(V) / 16); c += kRbkWarps * 32) d[c] = s[c];
}

// Loads a lane's B bytes (B = 32 or 64: C = B/16 chunks of 16 bytes) starting
// at byte offset lane_off of a linear area into dst, conflict-free: eight
// lanes share one 128-byte bank period, so lane l fetches its chunks starting
// at chunk r = (l / (8 / C)) mod C, which gives the eight lanes of every
// access phase distinct banks; two select stages then rotate the chunks back
// into order.  (Used for tiles of a batch, which arrive unswizzled.)
template <int B, typename T>
__device__ __forceinline__ void load_lane_rotated(T *dst, const unsigned char *base, uint32_t lane_off, int lane) {
  constexpr int C = B / 16;
  static_assert(C == 2 || C == 4, "two or four 16-byte chunks");
  const int r = (lane / (8 / C)) & (C - 1);
  uint4 q[C];
#pragma unroll
  for (int k = 0; k < C; ++k) q[k] = *reinterpret_cast<const uint4 *>(base + lane_off + 16 * ((k + r) & (C - 1)));
  // q[k] holds chunk (k + r) mod C; rotate right by r so q[c] holds chunk c
  if (r & 1) {
    const uint4 t = q[C - 1];
#pragma unroll
    for (int k = C - 1; k > 0; --k) q[k] = q[k - 1];
    q[0] = t;
  }
  if constexpr (C == 4) {
    if (r & 2) {
      const uint4 t0 = q[0], t1 = q[1];
      q[0] = q[2];
      q[1] = q[3];
      q[2] = t0;
      q[3] = t1;
    }
  }
  memcpy(dst, q, B);
}

// A lane's 16-byte chunk offsets within the keys and values areas (the same
// for every tile: they depend on the lane's first element only).
template <typename K, typename V, bool SWZ>
struct LaneOffsets {
  uint32_t k[RbkCfg<K, V>::KCH];
  uint32_t v[RbkCfg<K, V>::VCH];
  __device__ __forceinline__ explicit LaneOffsets(uint32_t e0) {
#pragma unroll
    for (int c = 0; c < RbkCfg<K, V>::KCH; ++c) k[c] = area_off<SWZ>(e0 * (uint32_t)sizeof(K) + 16u * c);
#pragma unroll
    for (int c = 0; c < RbkCfg<K, V>::VCH; ++c) v[c] = area_off<SWZ>(e0 * (uint32_t)sizeof(V) + 16u * c);
  }
};

// Phase 1 of a lane's M consecutive elements (element index of its first:
// e0): loads them, flags run heads (a head's key differs from its
// predecessor's; the input's first element is one), folds (c, v) in order --
// c counts heads, v is the sum since the last head (or since the lane's first
// element) -- and leaves the running v of every element in vals[] (the
// "marks": at a run's last element, the run's sum from its head or from the
// lane's start).  Returns (c, v); *heads / *tails get the head and tail bit
// masks (bit j: element j starts / ends a run).  Elements past the tile's
// end (FULL = false) are neither heads nor tails and add nothing.
template <typename K, typename V, bool SWZ, bool FULL>
__device__ __forceinline__ Seg<V> rbk_phase1_lane(const unsigned char *buf, const LaneOffsets<K, V, SWZ> &lo,
                                                  const K (*hb)[16 / sizeof(K)], uint32_t count, bool first_tile,
                                                  bool last_tile, uint32_t e0, int lane, V (&val)[RbkCfg<K, V>::M],
                                                  uint32_t *heads_out, uint32_t *tails_out) {
  using C = RbkCfg<K, V>;
  constexpr int M = C::M;
  constexpr int KC = 16 / sizeof(K);
  constexpr int VC = 16 / sizeof(V);
  K key[M];
  if constexpr (SWZ) {
#pragma unroll
    for (int c = 0; c < C::KCH; ++c) {
      const uint4 q = *reinterpret_cast<const uint4 *>(buf + lo.k[c]);
      memcpy(&key[c * KC], &q, 16);
    }
#pragma unroll
    for (int c = 0; c < C::VCH; ++c) {
      const uint4 q = *reinterpret_cast<const uint4 *>(buf + C::KEY_BYTES + lo.v[c]);
      memcpy(&val[c * VC], &q, 16);
    }
  } else {
    load_lane_rotated<M * sizeof(K)>(key, buf, e0 * (uint32_t)sizeof(K), lane);
    load_lane_rotated<M * sizeof(V)>(val, buf + C::KEY_BYTES, e0 * (uint32_t)sizeof(V), lane);
  }
  const int nvalid = FULL ? M : (int)min(max((int)count - (int)e0, 0), M);
  if (!FULL && nvalid < M) {
#pragma unroll
    for (int j = 0; j < M; ++j)
      if (j >= nvalid) {
        key[j] = K();
        val[j] = V(0);
      }
  }
  // the key before the lane's first element and after its last
  K prev = shfl_up(key[M - 1], 1);
  K next = shfl_down_any(key[0], 1);
  if (lane == 0)
    prev = e0 == 0 ? hb[0][KC - 1] : *reinterpret_cast<const K *>(buf + area_off<SWZ>((e0 - 1) * (uint32_t)sizeof(K)));
  if (lane == 31)
    next = e0 + M < count ? *reinterpret_cast<const K *>(buf + area_off<SWZ>((e0 + M) * (uint32_t)sizeof(K)))
                          : hb[1][0];
  const bool force0 = first_tile && e0 == 0;
  K pk = prev;
  V v = V(0);
  uint32_t heads = 0;
#pragma unroll
  for (int j = 0; j < M; ++j) {
    bool h = !(key[j] == pk);
    if (j == 0) h = h || force0;
    if (!FULL) h = h && (j < nvalid);
    v = h ? val[j] : (V)(v + val[j]);
    val[j] = v;
    heads |= (uint32_t)h << j;
    pk = key[j];
  }
  // element j < nvalid - 1 ends a run exactly when j + 1 starts one
  uint32_t tails = 0;
  if (nvalid == M) {
    const bool tile_end = e0 + M == count;
    const bool tl = tile_end ? (last_tile || !(hb[1][0] == key[M - 1])) : !(next == key[M - 1]);
    tails = (heads >> 1) | ((uint32_t)tl << (M - 1));
  } else if (nvalid > 0) {  // the lane holding the tile's last element
    K kl = key[0];
#pragma unroll
    for (int j = 1; j < M; ++j)
      if (j == nvalid - 1) kl = key[j];
    tails = ((heads >> 1) & ((1u << (nvalid - 1)) - 1u)) |
            ((uint32_t)(last_tile || !(hb[1][0] == kl)) << (nvalid - 1));
  }
  *heads_out = heads;
  *tails_out = tails;
  return Seg<V>{(uint32_t)__popc(heads), v};
}

// Persistent two-phase reduce_by_key; the roles, buffer rotation and
// hand-over protocol are scan_kernel's (scan.cu), with these differences: a
// buffer holds a tile's keys, values and halo keys; phase 1 also writes every
// element's running value (from its run's head, or from its lane's first
// element) to the CTA's mark slot for the tile (ring slot blockIdx.x * 3 +
// iteration mod 3, an image of the values area), and the re-read for phase 2
// brings back the tile's keys with those marks in place of its values, so
// phase 2 costs one step per run, not per element; phase 2 only reads its
// buffer (the runs go straight to out_keys / out_vals), so the loader reuses
// a buffer once the compute warps are done reading it, with no store to
// drain; and tiles without a TMA copy are staged by the compute warps
// themselves between two compute-only barriers.  Barrier phase parities are
// kept as bit masks (bit b: buffer b), so no per-buffer array is indexed at
// run time.
template <typename K, typename V, typename Src>
__global__ void __launch_bounds__(kRbkThreads, 2) rbk_kernel(const __grid_constant__ Src src,
                                                             typename RbkCfg<K, V>::Status st, WsHeader *hdr,
                                                             V *ring, unsigned long long spin_limit_ns,
                                                             long long skip_publish_tile, unsigned int num_tiles) {
  using C = RbkCfg<K, V>;
  using P = typename C::P;
  constexpr bool SWZ = Src::kSwz;
  constexpr int M = C::M, TILE = C::TILE, NB = kRbkBufs, Q = kRbkQueue;
  V *const cta_ring = ring + (size_t)blockIdx.x * 3 * TILE;  // this CTA's three mark slots
  constexpr unsigned int NONE = 0xffffffffu;
  OpSeg<V> op;
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  // the tile buffers start at the first 1024-byte boundary (the swizzle's period)
  unsigned char *const smem_raw = smem_dyn + ((1024u - (smem_addr(smem_dyn) & 1023u)) & 1023u);
  __shared__ __align__(16) K s_halo[NB][2][16 / sizeof(K)];
  __shared__ __align__(8) uint64_t s_full[NB];
  __shared__ __align__(8) uint64_t s_p1[NB];
  __shared__ __align__(8) uint64_t s_p2[NB];
  __shared__ __align__(8) uint64_t s_qbar[Q];
  __shared__ unsigned int s_ticket[NB];
  __shared__ P s_wagg[4][kRbkWarps];   // per-warp (c, v) of t_i, by iteration mod 4
  __shared__ P s_wexcl[4][kRbkWarps];  // the warps before each warp, folded (thread 0)
  // phase 1's per-lane results, kept for phase 2 (each warp reads back only
  // its own lanes, so program order protects them; by iteration mod 3):
  // head flags | tail flags << 16, and the lane's exclusive (c, v) in its warp
  __shared__ uint32_t s_lflags[3][32 * kRbkWarps];
  __shared__ uint32_t s_lc[3][32 * kRbkWarps];
  __shared__ V s_lv[3][32 * kRbkWarps];
  __shared__ unsigned int s_q_tile[Q];
  __shared__ P s_q_agg[Q];
  __shared__ P s_q_prefix[Q];
  __shared__ unsigned int s_q_in;
  __shared__ int s_abort;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  auto abort_now = [&]() { *reinterpret_cast<volatile int *>(&s_abort) = 1; };
  auto aborted = [&]() -> bool { return *reinterpret_cast<volatile int *>(&s_abort) != 0; };
  auto buf = [&](int b) { return smem_raw + (size_t)b * C::BUF_BYTES; };
  auto slot = [&](int s) { return cta_ring + (size_t)s * TILE; };

  uint64_t keep = 0, stream = 0;
  uint32_t armpar = 0u, armany = 0u;  // loader: parity of the phases armed on s_full[b] / any armed
  unsigned int next_raw = NONE;
  unsigned int t_first = NONE;
  if (tid == 32 * kRbkWarps) {
    keep = l2_policy_evict_last();
    stream = l2_policy_evict_first();
    for (int b = 0; b < NB; ++b) {
      mbar_init(&s_full[b], 1);
      mbar_init(&s_p1[b], kRbkWarps);
      mbar_init(&s_p2[b], kRbkWarps);
    }
    for (int q = 0; q < Q; ++q) mbar_init(&s_qbar[q], 1);
    fence_proxy_async_smem();
    s_abort = 0;
    s_q_in = 0u;
    const unsigned int t0 = atomicAdd(&hdr->tile_ticket, 1u);
    t_first = t0 < num_tiles ? t0 : NONE;
    s_ticket[0] = t_first;
    bool tx = false;
    if (t_first != NONE) tx = rbk_issue_load<K, V>(src, src.tile(t_first), buf(0), s_halo[0], &s_full[0], keep);
    if (!tx) mbar_arrive(&s_full[0]);
    mbar_arrive(&s_full[NB - 1]);  // iteration 0's phase 2 reads buffer NB - 1: an empty phase
    armpar = 1u | (1u << (NB - 1));
    armany = armpar;
    if (t_first != NONE) next_raw = atomicAdd(&hdr->tile_ticket, 1u);
  }
  __syncthreads();

  if (warp == kRbkWarps) {
    // ================= the loader (lane 0) =================
    if (lane != 0) return;
    uint32_t p1par = 0u, p2par = 0u;
    unsigned int t = t_first, p_tile = NONE, q_tile = NONE;
    for (int it = 0;; ++it) {
      const int bt = it % NB, bp = (it + NB - 1) % NB, bn = (it + 1) % NB;
      // prefetch t_{i+1} into bn (the compute warps finished reading it last iteration)
      const unsigned int tn = (t != NONE && next_raw < num_tiles) ? next_raw : NONE;
      s_ticket[bn] = tn;
      bool tx = false;
      if (tn != NONE) tx = rbk_issue_load<K, V>(src, src.tile(tn), buf(bn), s_halo[bn], &s_full[bn], keep);
      if (!tx) mbar_arrive(&s_full[bn]);
      armpar ^= 1u << bn;
      armany |= 1u << bn;
      next_raw = (tn != NONE) ? atomicAdd(&hdr->tile_ticket, 1u) : NONE;
      // tiles are ticketed about in order, gridDim.x per iteration: ask L2 now
      // for the one some CTA will load 1 iteration(s) from now
      if (tn != NONE && tn + 1u * gridDim.x < num_tiles) {
        const RbkTile<K, V> f = src.tile(tn + 1u * gridDim.x);
        const uint64_t fb = (uint64_t)f.local * TILE;
        prefetch_l2_range(f.keys + fb, (uint64_t)f.count() * sizeof(K));
        prefetch_l2_range(f.vals + fb, (uint64_t)f.count() * sizeof(V));
      }
      // re-read t_{i-1} into t's buffer once phase 1 of t is done with it
      if (!mbar_wait_or_abort(&s_p1[bt], (p1par >> bt) & 1u, spin_limit_ns, &s_abort)) {
        record_error(hdr, BK_ERR_SPIN_TIMEOUT, t);
        abort_now();
        break;
      }
      p1par ^= 1u << bt;
      tx = false;
      if (q_tile != NONE)  // t_{it-1}: its phase 1 ran in iteration it-1
        tx = rbk_issue_reload<K, V>(src, src.tile(q_tile), slot((it + 2) % 3), buf(bt), &s_full[bt], stream);
      if (!tx) mbar_arrive(&s_full[bt]);
      armpar ^= 1u << bt;
      armany |= 1u << bt;
      // buffer bp is free once phase 2 of p has read it
      if (!mbar_wait_or_abort(&s_p2[bp], (p2par >> bp) & 1u, spin_limit_ns, &s_abort)) {
        record_error(hdr, BK_ERR_SPIN_TIMEOUT, p_tile);
        abort_now();
        break;
      }
      p2par ^= 1u << bp;
      p_tile = q_tile;
      q_tile = t;
      t = tn;
      if (t == NONE && p_tile == NONE && q_tile == NONE) break;
    }
    // every load must land before the CTA's shared memory goes away: wait for
    // the last phase armed on each buffer (phases of a barrier complete in order)
    for (int b = 0; b < NB; ++b)
      if ((armany >> b) & 1u) (void)mbar_wait(&s_full[b], ((armpar >> b) & 1u) ^ 1u, spin_limit_ns);
    return;
  }

  if (warp == kRbkWarps + 1) {
    // ================= the look-back warp =================
    auto wait_queued = [&](unsigned int count) -> bool {
      unsigned long long w0 = 0;
      bool ready = false;
      for (unsigned int spins = 0;; ++spins) {
        if (ld_acquire_cta_u32(&s_q_in) >= count) {
          ready = true;
          break;
        }
        if (aborted()) break;
        if ((spins & 15u) == 15u) {
          const unsigned long long now = globaltimer_ns();
          if (w0 == 0) w0 = now;
          else if (now - w0 > spin_limit_ns) {
            if (lane == 0) {
              record_error(hdr, BK_ERR_SPIN_TIMEOUT, NONE);
              abort_now();
            }
            break;
          }
        }
        __nanosleep(64);
      }
      return __all_sync(0xffffffffu, ready);
    };
    for (unsigned int j = 0;; ++j) {
      if (!wait_queued(j + 1u)) break;
      const unsigned int q = s_q_tile[j % Q];
      if (q == NONE) break;
      if (!wait_queued(j + 2u)) break;
      const P agg = s_q_agg[j % Q];
      const bool qfirst = src.tile(q).first();
      P excl = OpSeg<V>::identity();
      bool ok = true;
      if (!qfirst) ok = lookback_exclusive<P>(st, q, op, excl, hdr, spin_limit_ns);
      if (lane == 0) {
        if (ok) {
          if (!qfirst && (long long)q != skip_publish_tile) st.publish(q, kStPrefix, op(excl, agg));
          s_q_prefix[j % Q] = excl;
          mbar_arrive(&s_qbar[j % Q]);
        } else {
          abort_now();
        }
      }
      if (!ok) break;
    }
    return;
  }

  // ================= the compute warps =================
  const uint32_t e0 = (uint32_t)(warp * 32 + lane) * M;  // this lane's first element in every tile
  const LaneOffsets<K, V, SWZ> lo(e0);
  uint32_t fpar = 0u;  // bit b: parity of the next phase of s_full[b]
  unsigned int p_tile = NONE, q_tile = NONE;
  bool bad = false;

  for (int it = 0;; ++it) {
    const int bt = it % NB, bp = (it + NB - 1) % NB;
    const unsigned int p = p_tile;

    // ---- phase 1 of t
    unsigned int t = NONE;
    if (!mbar_wait_or_abort(&s_full[bt], (fpar >> bt) & 1u, spin_limit_ns, &s_abort)) bad = true;
    fpar ^= 1u << bt;
    // the marks this thread stored last iteration are read back by a TMA copy
    // that the loader issues once this iteration's phase 1 is done: order them
    // before it now, an iteration after the stores (fencing right after them
    // would wait for their round trip to L2)
    fence_proxy_async_global();
    bad = __any_sync(0xffffffffu, bad);
    if (!bad) t = s_ticket[bt];
    // tiles without a TMA copy: the compute warps stage them here, between
    // two barriers that every compute warp takes whenever the launch may
    // have such a tile (a flag of the launch, so a warp that saw a failure
    // still takes part; the previous iteration's readers are past the first)
    if (src.may_stage) {
      named_barrier_sync(2, 32 * kRbkWarps);
      if (t != NONE && !src.tile(t).tma) rbk_stage_load<K, V, SWZ>(src.tile(t), buf(bt));
      if (p != NONE && !bad && !src.tile(p).tma)  // phase 1 of p ran at it - 2
        rbk_stage_reload<K, V, SWZ>(src.tile(p), slot((it + 1) % 3), buf(bp));
      named_barrier_sync(2, 32 * kRbkWarps);
    }
    if (t != NONE) {
      const RbkTile<K, V> tl = src.tile(t);
      const uint32_t count = tl.count();
      V val[M];
      uint32_t heads, tails;
      P lane_agg;
      if (count == (uint32_t)TILE)  // every tile but an array's last: no bounds checks
        lane_agg = rbk_phase1_lane<K, V, SWZ, true>(buf(bt), lo, s_halo[bt], count, tl.first(), tl.last(), e0, lane,
                                                    val, &heads, &tails);
      else
        lane_agg = rbk_phase1_lane<K, V, SWZ, false>(buf(bt), lo, s_halo[bt], count, tl.first(), tl.last(), e0,
                                                     lane, val, &heads, &tails);
      // the running values go to the tile's mark slot (an image of the values area)
      unsigned char *const ms = reinterpret_cast<unsigned char *>(slot(it % 3));
#pragma unroll
      for (int c = 0; c < C::VCH; ++c) {
        uint4 q;
        memcpy(&q, &val[c * (16 / sizeof(V))], 16);
        *reinterpret_cast<uint4 *>(ms + (SWZ ? lo.v[c] : e0 * (uint32_t)sizeof(V) + 16u * c)) = q;
      }
      const P incl = warp_inclusive_scan(lane_agg, op, lane);
      if (lane == 31) s_wagg[it & 3][warp] = incl;
      P lex = shfl_up(incl, 1);
      if (lane == 0) lex = OpSeg<V>::identity();
      const int sl = it % 3, li = warp * 32 + lane;
      s_lflags[sl][li] = heads | (tails << 16);
      s_lc[sl][li] = lex.c;
      s_lv[sl][li] = lex.v;
    }
    __syncwarp();
    if (!bad && lane == 0) mbar_arrive(&s_p1[bt]);
    if (named_barrier_or(1, 32 * kRbkWarps, bad || aborted())) break;

    // ---- thread 0: publish t's aggregate and queue t for the look-back
    if (tid == 0) {
      P agg = OpSeg<V>::identity();
      if (t != NONE) {
#pragma unroll
        for (int i = 0; i < kRbkWarps; ++i) {
          s_wexcl[it & 3][i] = agg;
          agg = op(agg, s_wagg[it & 3][i]);
        }
        if ((long long)t != skip_publish_tile) st.publish(t, src.tile(t).first() ? kStPrefix : kStAggregate, agg);
      }
      s_q_tile[it % Q] = t;
      s_q_agg[it % Q] = agg;
      st_release_cta_u32(&s_q_in, (unsigned int)it + 1u);
    }

    // ---- phase 2 of p: emit its runs
    if (!mbar_wait_or_abort(&s_full[bp], (fpar >> bp) & 1u, spin_limit_ns, &s_abort)) bad = true;
    fpar ^= 1u << bp;
    if (p != NONE && !bad) {
      const unsigned int e = (unsigned int)it - 2u;
      if (!mbar_wait_or_abort(&s_qbar[e % Q], (e / Q) & 1u, spin_limit_ns, &s_abort)) bad = true;
    }
    bad = __any_sync(0xffffffffu, bad);
    if (p != NONE && !bad) {
      const unsigned int e = (unsigned int)it - 2u;
      const RbkTile<K, V> tl = src.tile(p);
      const uint32_t count = tl.count();
      const int sl = (it + 1) % 3, li = warp * 32 + lane;  // phase 1 of p ran at it - 2
      const uint32_t fl = s_lflags[sl][li];
      const uint32_t head = fl & 0xffffu, tail = fl >> 16;
      const bool holds_last = tl.last() && e0 < count && count <= e0 + M;  // the input's last element
      if (tail != 0u || holds_last) {
        P carry = op(s_q_prefix[e % Q], s_wexcl[(it + 2) & 3][warp]);
        carry = op(carry, P{s_lc[sl][li], s_lv[sl][li]});
        // each tail: its key, and its mark (the run's value from its head, or
        // from the lane's first element when the run began before the lane)
        const unsigned char *bP = buf(bp);
        for (uint32_t tb = tail; tb != 0u; tb &= tb - 1u) {
          const uint32_t j = (uint32_t)__ffs(tb) - 1u;
          const uint32_t upto = head & ((2u << j) - 1u);  // heads at or before j
          const uint32_t c = carry.c + (uint32_t)__popc(upto);
          V v = *reinterpret_cast<const V *>(bP + C::KEY_BYTES + area_off<SWZ>((e0 + j) * (uint32_t)sizeof(V)));
          if (upto == 0u) v = (V)(carry.v + v);
          tl.out_keys[c - 1] = *reinterpret_cast<const K *>(bP + area_off<SWZ>((e0 + j) * (uint32_t)sizeof(K)));
          tl.out_vals[c - 1] = v;
        }
        if (holds_last) *tl.num_out = carry.c + (uint32_t)__popc(head);
      }
    }
    __syncwarp();
    if (!bad && lane == 0) mbar_arrive(&s_p2[bp]);

    p_tile = q_tile;
    q_tile = t;
    if (t == NONE && p_tile == NONE && q_tile == NONE) break;
  }
}

// Clears the status words, then runs the persistent reduce_by_key over
// `tiles` tiles of `src` (one array or a batch).
template <typename K, typename V, typename Src>
int rbk_run(const Src &src, size_t tiles, void *d_ws, size_t ws_bytes, cudaStream_t stream) {
  using C = RbkCfg<K, V>;
  host::DeviceInfo di;
  int st = host::device_info(&di);
  if (st != BK_OK) return st;
  if (tiles >= 0x7fffffffull) return BK_ERR_TOO_LARGE;
  st = host::check_ws(d_ws, ws_bytes, rbk_ws_for_tiles<K, V>(tiles));
  if (st != BK_OK) return st;
  WsHeader *hdr = reinterpret_cast<WsHeader *>(d_ws);
  auto status = C::Status::at(reinterpret_cast<char *>(d_ws) + kHeaderBytes, tiles);
  const unsigned init_grid = (unsigned)std::min<size_t>((tiles + 255) / 256 + 1, (size_t)di.sm_count * 8);
  rbk_init_kernel<<<init_grid, 256, 0, stream>>>(status, tiles, hdr);
  if ((st = host::launch_status()) != BK_OK) return st;
  const host::DebugFault dbg = host::debug_fault();
  const unsigned long long limit = dbg.spin_limit_ns ? dbg.spin_limit_ns : host::kDefaultSpinLimitNs;
  const size_t smem = (size_t)kRbkBufs * C::BUF_BYTES + 1024;  // + room to align the buffers to 1024 bytes
  struct Site {};
  host::KernelSetup ks;
  if ((st = host::kernel_setup<Site>(rbk_kernel<K, V, Src>, kRbkThreads, smem, &ks)) != BK_OK) return st;
  const tune::Knobs kn = tune::knobs_for(tune::kReduceByKey, (int)(sizeof(K) + sizeof(V)), (uint64_t)tiles * C::TILE);
  const size_t per_sm = (size_t)std::min(std::max(kn.ctas_per_sm, 1), 2);
  const unsigned grid = (unsigned)std::min<size_t>(tiles, std::min<size_t>((size_t)di.sm_count * per_sm, kRbkMaxGrid));
  V *ring = reinterpret_cast<V *>(reinterpret_cast<char *>(d_ws) + rbk_ring_offset<K, V>(tiles));
  rbk_kernel<K, V, Src><<<grid, kRbkThreads, smem, stream>>>(src, status, hdr, ring, limit, dbg.skip_publish_tile,
                                                            (unsigned)tiles);
  return host::launch_status();
}

template <typename K, typename V>
int rbk_check_array(const K *keys, const V *vals, uint64_t n, K *out_keys, V *out_vals, uint64_t *d_num_out) {
  if (d_num_out == nullptr) return BK_ERR_INVALID_ARGUMENT;
  if (n > 0 && (keys == nullptr || vals == nullptr || out_keys == nullptr || out_vals == nullptr))
    return BK_ERR_INVALID_ARGUMENT;
  if (!host::aligned_to<K>(keys) || !host::aligned_to<V>(vals) || !host::aligned_to<K>(out_keys) ||
      !host::aligned_to<V>(out_vals) || !host::aligned_to<uint64_t>(d_num_out))
    return BK_ERR_MISALIGNED;
  if (n >= 0xffffffffull) return BK_ERR_TOO_LARGE;  // run counts are 32-bit
  return BK_OK;
}

template <typename K, typename V>
int rbk_launch(const K *keys, const V *vals, uint64_t n, K *out_keys, V *out_vals, uint64_t *d_num_out, void *d_ws,
               size_t ws_bytes, cudaStream_t stream) {
  host::DeviceInfo di;
  int st = host::device_info(&di);
  if (st != BK_OK) return st;
  if ((st = rbk_check_array(keys, vals, n, out_keys, out_vals, d_num_out)) != BK_OK) return st;
  if (n == 0) {
    write_count_kernel<V><<<1, 1, 0, stream>>>(d_num_out);
    return host::launch_status();
  }
  using C = RbkCfg<K, V>;
  RbkOne<K, V> src;
  memset(&src, 0, sizeof(src));
  src.keys = keys;
  src.vals = vals;
  src.n = n;
  src.out_keys = out_keys;
  src.out_vals = out_vals;
  src.num_out = d_num_out;
  // row views of the keys and values: the elements inside whole 128-byte
  // rows of both arrive by tensor copies, the rest is staged by plain loads
  const uint64_t krows = n * sizeof(K) / 128, vrows = n * sizeof(V) / 128;
  const bool aligned = ((reinterpret_cast<uintptr_t>(keys) | reinterpret_cast<uintptr_t>(vals)) & 15) == 0;
  if (aligned && krows > 0 && vrows > 0 && host::encode_rows_128b(&src.kmap, keys, krows, C::KROWS) == BK_OK &&
      host::encode_rows_128b(&src.vmap, vals, vrows, C::VROWS) == BK_OK)
    src.covered = std::min(krows * (128 / sizeof(K)), vrows * (128 / sizeof(V)));
  src.may_stage = src.covered < n;
  return rbk_run<K, V>(src, rbk_num_tiles<K, V>(n), d_ws, ws_bytes, stream);
}

// A batch item as the C-ABI passes it (bk_rbk_item_<key>_<value>).
template <typename K, typename V>
struct RbkItem {
  const K *keys;
  const V *vals;
  uint64_t n;
  K *out_keys;
  V *out_vals;
  uint64_t *d_num_out;
};

template <typename K, typename V>
int rbk_batch_launch(const RbkItem<K, V> *items, uint32_t count, void *d_ws, size_t ws_bytes, cudaStream_t stream) {
  host::DeviceInfo di;
  int st = host::device_info(&di);
  if (st != BK_OK) return st;
  if (count > 0 && items == nullptr) return BK_ERR_INVALID_ARGUMENT;
  if (count > (uint32_t)kRbkBatchMax) return BK_ERR_TOO_LARGE;
  RbkBatch<K, V> b;
  b.count = 0;
  b.may_stage = 0;
  size_t tiles = 0;
  for (uint32_t i = 0; i < count; ++i) {
    const RbkItem<K, V> &it = items[i];
    if ((st = rbk_check_array(it.keys, it.vals, it.n, it.out_keys, it.out_vals, it.d_num_out)) != BK_OK) return st;
    if (it.n == 0) {  // no tile: its count is written here
      write_count_kernel<V><<<1, 1, 0, stream>>>(it.d_num_out);
      if ((st = host::launch_status()) != BK_OK) return st;
      continue;
    }
    const uint32_t k = b.count++;
    b.keys[k] = it.keys;
    b.vals[k] = it.vals;
    b.n[k] = it.n;
    b.out_keys[k] = it.out_keys;
    b.out_vals[k] = it.out_vals;
    b.num_out[k] = it.d_num_out;
    b.start[k] = (uint32_t)tiles;
    if (((reinterpret_cast<uintptr_t>(it.keys) | reinterpret_cast<uintptr_t>(it.vals)) & 15) != 0) b.may_stage = 1;
    tiles += rbk_num_tiles<K, V>(it.n);
    if (tiles >= 0x7fffffffull) return BK_ERR_TOO_LARGE;
  }
  b.start[b.count] = (uint32_t)tiles;
  if (b.count == 0) return BK_OK;
  return rbk_run<K, V>(b, tiles, d_ws, ws_bytes, stream);
}

template <typename K, typename V>
size_t rbk_batch_ws(const uint64_t *sizes, uint32_t count) {
  size_t tiles = 0;
  for (uint32_t i = 0; i < count; ++i) tiles += rbk_num_tiles<K, V>(sizes[i]);
  return rbk_ws_for_tiles<K, V>(tiles);
}

size_t rbk_batch_workspace_bytes(int key_dtype, int value_dtype, const uint64_t *sizes, uint32_t count) {
  if (count > 0 && sizes == nullptr) return 0;
  const bool k4 = key_dtype == BK_DTYPE_I32 || key_dtype == BK_DTYPE_U32;
  const bool k8 = key_dtype == BK_DTYPE_I64 || key_dtype == BK_DTYPE_U64;
  const bool v4 = value_dtype == BK_DTYPE_I32 || value_dtype == BK_DTYPE_U32 || value_dtype == BK_DTYPE_F32;
  const bool v8 = value_dtype == BK_DTYPE_I64 || value_dtype == BK_DTYPE_U64 || value_dtype == BK_DTYPE_F64;
  if (k4 && v4) return rbk_batch_ws<int32_t, float>(sizes, count);
  if (k4 && v8) return rbk_batch_ws<int32_t, double>(sizes, count);
  if (k8 && v4) return rbk_batch_ws<int64_t, float>(sizes, count);
  if (k8 && v8) return rbk_batch_ws<int64_t, double>(sizes, count);
  return 0;
}

size_t rbk_workspace_bytes(int key_dtype, int value_dtype, uint64_t n) {
  const bool k4 = key_dtype == BK_DTYPE_I32 || key_dtype == BK_DTYPE_U32;
  const bool k8 = key_dtype == BK_DTYPE_I64 || key_dtype == BK_DTYPE_U64;
  const bool v4 = value_dtype == BK_DTYPE_I32 || value_dtype == BK_DTYPE_U32 || value_dtype == BK_DTYPE_F32;
  const bool v8 = value_dtype == BK_DTYPE_I64 || value_dtype == BK_DTYPE_U64 || value_dtype == BK_DTYPE_F64;
  if (k4 && v4) return rbk_ws_bytes<int32_t, float>(n);
  if (k4 && v8) return rbk_ws_bytes<int32_t, double>(n);
  if (k8 && v4) return rbk_ws_bytes<int64_t, float>(n);
  if (k8 && v8) return rbk_ws_bytes<int64_t, double>(n);
  return 0;
}

}  // namespace bk

#define BK_DEFINE_RBK(KN, K, VN, V)                                                                             \
  extern "C" int bk_reduce_by_key_##KN##_##VN(const K *keys, const V *vals, uint64_t n, K *out_keys,           \
                                              V *out_vals, uint64_t *d_num_out, void *d_ws, size_t ws_bytes, \
                                              bk_stream_t stream) {                                          \
    return bk::rbk_launch<K, V>(keys, vals, n, out_keys, out_vals, d_num_out, d_ws, ws_bytes,                  \
                                (cudaStream_t)stream);                                                        \
  }

BK_DEFINE_RBK(i32, int32_t, i32, int32_t)
BK_DEFINE_RBK(i32, int32_t, i64, int64_t)
BK_DEFINE_RBK(i32, int32_t, f32, float)
BK_DEFINE_RBK(i32, int32_t, f64, double)
BK_DEFINE_RBK(u32, uint32_t, f32, float)
BK_DEFINE_RBK(u32, uint32_t, f64, double)
BK_DEFINE_RBK(i64, int64_t, i32, int32_t)
BK_DEFINE_RBK(i64, int64_t, i64, int64_t)
BK_DEFINE_RBK(i64, int64_t, f32, float)
BK_DEFINE_RBK(i64, int64_t, f64, double)

#define BK_DEFINE_RBK_BATCH(KN, K, VN, V)                                                                      \
  static_assert(sizeof(bk_rbk_item_##KN##_##VN) == sizeof(bk::RbkItem<K, V>), "bk_rbk_item layout");        \
  extern "C" int bk_reduce_by_key_##KN##_##VN##_batch(const bk_rbk_item_##KN##_##VN *items, uint32_t count,  \
                                                      void *d_ws, size_t ws_bytes, bk_stream_t stream) {     \
    return bk::rbk_batch_launch<K, V>(reinterpret_cast<const bk::RbkItem<K, V> *>(items), count, d_ws,        \
                                      ws_bytes, (cudaStream_t)stream);                                        \
  }

BK_DEFINE_RBK_BATCH(i32, int32_t, i32, int32_t)
BK_DEFINE_RBK_BATCH(i32, int32_t, i64, int64_t)
BK_DEFINE_RBK_BATCH(i32, int32_t, f32, float)
BK_DEFINE_RBK_BATCH(i32, int32_t, f64, double)
BK_DEFINE_RBK_BATCH(u32, uint32_t, f32, float)
BK_DEFINE_RBK_BATCH(u32, uint32_t, f64, double)
BK_DEFINE_RBK_BATCH(i64, int64_t, i32, int32_t)
BK_DEFINE_RBK_BATCH(i64, int64_t, i64, int64_t)
BK_DEFINE_RBK_BATCH(i64, int64_t, f32, float)
BK_DEFINE_RBK_BATCH(i64, int64_t, f64, double)
