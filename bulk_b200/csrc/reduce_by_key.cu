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
// (c, v) gives the run's output slot c - 1 and its sum v.  Persistent CTAs
// take tiles from an atomic ticket; a loader lane brings each tile (keys,
// values and a one-key halo on each side) into shared memory by TMA, the
// compute warps reduce it (phase 1: the tile aggregate, published at once),
// compact the runs that end in it -- key and tile-local sum, in output order
// -- and copy them to a run slot of the CTA's ring in global memory, which
// frees the tile buffer for the next load; a look-back warp finds the tile's
// exclusive prefix meanwhile.  Two iterations later the compute warps copy the
// runs from the ring (L2) to the output at the prefix's run count, adding the
// prefix's sum to a run that began in an earlier tile (phase 2).  No element
// is read twice: only the runs wait for the prefix.
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
constexpr int kRbkQueue = 4;                       // look-back queue entries

template <typename K, typename V>
struct RbkCfg {
  // each lane owns M consecutive elements and reads them in passes of MP (64
  // bytes of the wider of key and value, so that a pass's keys and values fit
  // in registers).  A tile's fixed costs -- the barrier, the publication, the
  // look-back -- are paid once per tile, so tiles are as large as two CTAs
  // per SM allow: 16 elements a lane (two passes when one of key and value is
  // 8 bytes wide), or 8 when both are.  Wider lanes of 4-byte pairs (24
  // elements, 96 bytes apart) measured slower: their chunks meet in the
  // shared-memory banks.
  static constexpr int M = sizeof(K) + sizeof(V) <= 12 ? 16 : 8;
  static constexpr int MP = 64 / (sizeof(K) > sizeof(V) ? sizeof(K) : sizeof(V));  // 16 or 8
  static_assert(M % MP == 0, "whole passes");
  static constexpr int TILE = kRbkWarps * 32 * M;            // 4096 or 2048
  static constexpr uint32_t KROWS = sizeof(K) * TILE / 128;  // 128-byte rows of keys in a tile (<= 256)
  static constexpr uint32_t VROWS = sizeof(V) * TILE / 128;  // ... and of values
  // a buffer: the keys area, then the values area, each a whole number of
  // 1024-byte swizzle periods (32 or 48 KB)
  static constexpr size_t KEY_BYTES = align_up(sizeof(K) * TILE, 1024);
  static constexpr size_t VAL_BYTES = align_up(sizeof(V) * TILE, 1024);
  static constexpr size_t BUF_BYTES = KEY_BYTES + VAL_BYTES;
  // CTAs per SM: three when key and value are 4 bytes each (the kernel then
  // fits in 64 registers a thread), else two
  static constexpr int CTAS = sizeof(K) + sizeof(V) == 8 ? 3 : 2;
  // tile buffers in rotation: a tile holds one from its load, D iterations
  // before its phase 1, to the end of its phase 1, so NB = D + 1; as many as
  // CTAS CTAs per SM leave room for
  static constexpr int NB = CTAS == 3 ? 2 : (BUF_BYTES <= 32 * 1024 ? 3 : 2);
  static_assert(CTAS * NB * BUF_BYTES <= 200 * 1024, "CTAS CTAs per SM");
  static constexpr int D = NB - 1;
  static constexpr size_t RUN_SLOT_BYTES = (sizeof(K) + sizeof(V)) * TILE;  // a tile's runs, at most TILE
  using P = Seg<V>;
  using Status = TileStatus<P>;
};

template <typename K, typename V>
size_t rbk_num_tiles(uint64_t n) {
  return (size_t)((n + RbkCfg<K, V>::TILE - 1) / RbkCfg<K, V>::TILE);
}
// Workspace: the header, one look-back status per tile, then the run ring:
// kRbkRunSlots run slots per persistent CTA (a tile's runs wait there, keys
// then values, from its phase 1 to its phase 2).
constexpr int kRbkRunSlots = 4;
constexpr size_t kRbkMaxGrid = 480;  // persistent CTAs at most (3 per SM)
template <typename K, typename V>
size_t rbk_ring_offset(size_t tiles) {
  return align_up(kHeaderBytes + RbkCfg<K, V>::Status::bytes(tiles), 256);
}
template <typename K, typename V>
size_t rbk_ws_for_tiles(size_t tiles) {
  const size_t ctas = tiles < kRbkMaxGrid ? tiles : kRbkMaxGrid;
  return rbk_ring_offset<K, V>(tiles) + ctas * kRbkRunSlots * RbkCfg<K, V>::RUN_SLOT_BYTES;
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
  bool tma;        // the loader brings this tile in by TMA
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

// Byte offset of byte o of a tile area in shared memory: swizzled for tiles that
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

// Loads a lane's B bytes (C = B/16 chunks of 16 bytes, one to eight) starting
// at byte offset lane_off of a linear area into dst.  For two or four chunks,
// lane l fetches its chunks starting at chunk r = (l / (8 / C)) mod C, which
// spreads the eight lanes of an access phase over the banks when lanes are B
// bytes apart (and halves the conflicts when they are 2B apart); two select
// stages then rotate the chunks back into order.  Other counts load in order.
// (Used for tiles of a batch, which arrive unswizzled.)
template <int B, typename T>
__device__ __forceinline__ void load_lane_rotated(T *dst, const unsigned char *base, uint32_t lane_off, int lane) {
  constexpr int C = B / 16;
  static_assert(C >= 1 && C <= 8, "one to eight 16-byte chunks");
  uint4 q[C];
  if constexpr (C != 2 && C != 4) {  // no rotation: chunks in order
#pragma unroll
    for (int k = 0; k < C; ++k) q[k] = *reinterpret_cast<const uint4 *>(base + lane_off + 16 * k);
    memcpy(dst, q, B);
    return;
  }
  const int r = (lane / (8 / C)) & (C - 1);
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

// Phase 1 of a lane's M consecutive elements (element index of its first:
// e0), in passes of MP elements (so that one pass's keys and values fit in
// registers): loads them, flags run
// heads (a head's key differs from its predecessor's; the input's first
// element is one), folds (c, v) in order -- c counts heads, v is the sum since
// the last head (or since the lane's first element) -- and writes the running
// v of every element over its value in the buffer (at a run's last element:
// the run's sum from its head or from the lane's start; only this lane reads
// its values).  Returns (c, v); *heads / *tails get the head and tail bit
// masks (bit j: element j starts / ends a run).  Elements past the tile's end
// (FULL = false) are neither heads nor tails and add nothing.  Whether the
// lane's first element is a head is known only once the previous lane's last
// key has been shuffled over, after the passes; the fold does not depend on
// it (v starts at the first value either way).
template <typename K, typename V, bool SWZ, bool FULL>
__device__ __forceinline__ Seg<V> rbk_phase1_lane(unsigned char *buf, const K (*hb)[16 / sizeof(K)], uint32_t count,
                                                  bool first_tile, bool last_tile, uint32_t e0, int lane,
                                                  uint32_t *heads_out, uint32_t *tails_out) {
  using C = RbkCfg<K, V>;
  constexpr int M = C::M, MP = C::MP;
  constexpr int KC = 16 / sizeof(K);
  constexpr int VC = 16 / sizeof(V);
  const int nvalid = FULL ? M : (int)min(max((int)count - (int)e0, 0), M);
  K kfirst = K(), klast = K(), pk = K();
  V v = V(0);
  uint32_t heads = 0;
#pragma unroll
  for (int ps = 0; ps < M / MP; ++ps) {
    K key[MP];
    V val[MP];
    const uint32_t kb = (e0 + ps * MP) * (uint32_t)sizeof(K);  // byte offsets of the pass
    const uint32_t vb = (e0 + ps * MP) * (uint32_t)sizeof(V);
    if constexpr (SWZ) {
#pragma unroll
      for (int c = 0; c < MP * (int)sizeof(K) / 16; ++c) {
        const uint4 q = *reinterpret_cast<const uint4 *>(buf + swz128(kb + 16u * c));
        memcpy(&key[c * KC], &q, 16);
      }
#pragma unroll
      for (int c = 0; c < MP * (int)sizeof(V) / 16; ++c) {
        const uint4 q = *reinterpret_cast<const uint4 *>(buf + C::KEY_BYTES + swz128(vb + 16u * c));
        memcpy(&val[c * VC], &q, 16);
      }
    } else {
      load_lane_rotated<MP * sizeof(K)>(key, buf, kb, lane);
      load_lane_rotated<MP * sizeof(V)>(val, buf + C::KEY_BYTES, vb, lane);
    }
    if (!FULL) {
#pragma unroll
      for (int j = 0; j < MP; ++j)
        if (ps * MP + j >= nvalid) {
          key[j] = K();
          val[j] = V(0);
        }
    }
#pragma unroll
    for (int j = 0; j < MP; ++j) {
      const int jj = ps * MP + j;
      if (jj == 0) {
        kfirst = key[0];
        v = val[0];
      } else {
        bool h = !(key[j] == pk);
        if (!FULL) h = h && (jj < nvalid);
        v = h ? val[j] : (V)(v + val[j]);
        heads |= (uint32_t)h << jj;
      }
      val[j] = v;
      pk = key[j];
      if (!FULL && jj == nvalid - 1) klast = key[j];
    }
    if (FULL) klast = key[MP - 1];
    // the running values over the pass's values (the chunks it loaded)
#pragma unroll
    for (int c = 0; c < MP * (int)sizeof(V) / 16; ++c) {
      uint4 q;
      memcpy(&q, &val[c * VC], 16);
      *reinterpret_cast<uint4 *>(buf + C::KEY_BYTES + (SWZ ? swz128(vb + 16u * c) : vb + 16u * c)) = q;
    }
  }
  // the key before the lane's first element and after its last (a lane past
  // the tile's end shuffles a zero key that nothing reads)
  K prev = shfl_up(pk, 1);
  K next = shfl_down_any(kfirst, 1);
  if (lane == 0)
    prev = e0 == 0 ? hb[0][KC - 1] : *reinterpret_cast<const K *>(buf + area_off<SWZ>((e0 - 1) * (uint32_t)sizeof(K)));
  if (lane == 31)
    next = e0 + M < count ? *reinterpret_cast<const K *>(buf + area_off<SWZ>((e0 + M) * (uint32_t)sizeof(K)))
                          : hb[1][0];
  bool h0 = !(kfirst == prev) || (first_tile && e0 == 0);
  if (!FULL) h0 = h0 && nvalid > 0;
  heads |= (uint32_t)h0;
  // element j < nvalid - 1 ends a run exactly when j + 1 starts one
  uint32_t tails = 0;
  if (nvalid == M) {
    const bool tile_end = e0 + M == count;
    const bool tl = tile_end ? (last_tile || !(hb[1][0] == klast)) : !(next == klast);
    tails = (heads >> 1) | ((uint32_t)tl << (M - 1));
  } else if (nvalid > 0) {  // the lane holding the tile's last element
    tails = ((heads >> 1) & ((1u << (nvalid - 1)) - 1u)) |
            ((uint32_t)(last_tile || !(hb[1][0] == klast)) << (nvalid - 1));
  }
  *heads_out = heads;
  *tails_out = tails;
  return Seg<V>{(uint32_t)__popc(heads), v};
}

// Persistent single-pass reduce_by_key.  Warps 0-7 compute, warp 8 (lane 0)
// loads, warp 9 looks back.  Each CTA loops over tiles taken from an atomic
// ticket (fetched one iteration ahead).  Tile t_i, ticketed for iteration i,
// lives in buffer i mod NB and goes through:
//   iteration i-D  loader: TMA copy of its keys, values and halo keys (tiles
//                  without one -- the ragged end, or arrays not 16-byte
//                  aligned -- are staged by the compute warps in iteration i);
//   iteration i    compute: phase 1 -- each lane folds its M elements,
//                  leaving their running sums over their values, and the
//                  warps scan their lanes; after the compute warps' barrier
//                  warp 7 publishes the tile aggregate and queues the tile
//                  for the look-back warp, and each lane writes the runs
//                  that end in its elements (the key, and the run's sum from
//                  its head or from the tile's start) to the tile's run slot
//                  (ring slot i mod 4 of the CTA) at their places in the
//                  tile's output order; then the buffer is released;
//   iteration i+3  compute: phase 2 -- with the tile's exclusive prefix
//                  (c, v) from the look-back warp, the runs are copied from
//                  the run slot to the output slots from c + h0 - 1 on (h0:
//                  the tile starts a run), the first one adding v when it
//                  began in an earlier tile.
// The roles never share a barrier: they hand over through mbarriers.  full[b]:
// the loader completes one phase per use of buffer b (a TMA copy, or a plain
// arrival when there is nothing to copy) after writing the buffer's ticket;
// empty[b]: each compute warp arrives when it is done with buffer b; qbar[e]:
// the look-back warp hands over queue entry e's prefix.  The compute warps
// meet only each other, once per iteration (after phase 1's reads), in a
// barrier that also ORs their failure flags, so they all stop together; it
// also orders an iteration's run-slot writes before the phase 2 that reads
// them (whose first loads are issued at the start of its iteration, before
// phase 1) and the phase 2 reads before the slot's next writes.  Every wait is
// bounded by spin_limit_ns and gives up at once when anyone in the CTA has
// failed.  Barrier phase parities are kept as bit masks (bit b: buffer b), so
// no per-buffer array is indexed at run time.
template <typename K, typename V, typename Src>
__global__ void __launch_bounds__(kRbkThreads, RbkCfg<K, V>::CTAS) rbk_kernel(const __grid_constant__ Src src,
                                                             typename RbkCfg<K, V>::Status st, WsHeader *hdr,
                                                             unsigned char *ring, unsigned long long spin_limit_ns,
                                                             long long skip_publish_tile, unsigned int num_tiles) {
  using C = RbkCfg<K, V>;
  using P = typename C::P;
  constexpr bool SWZ = Src::kSwz;
  constexpr int M = C::M, TILE = C::TILE, NB = C::NB, D = C::D, Q = kRbkQueue;
  constexpr unsigned int NONE = 0xffffffffu;
  OpSeg<V> op;
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  // the tile buffers start at the first 1024-byte boundary (the swizzle's period)
  unsigned char *const smem_raw = smem_dyn + ((1024u - (smem_addr(smem_dyn) & 1023u)) & 1023u);
  __shared__ __align__(16) K s_halo[NB][2][16 / sizeof(K)];
  __shared__ __align__(8) uint64_t s_full[NB];
  __shared__ __align__(8) uint64_t s_empty[NB];
  __shared__ __align__(8) uint64_t s_qbar[Q];
  __shared__ unsigned int s_ticket[NB];
  // per tile, by iteration mod 2 (written in phase 1, read after the barrier
  // that follows it): each warp's (c, v) and run count, and whether the tile
  // starts with a head
  __shared__ P s_wagg[2][kRbkWarps];
  __shared__ uint32_t s_wruns[2][kRbkWarps];
  __shared__ uint32_t s_h0[2];
  __shared__ unsigned int s_q_tile[Q];
  __shared__ P s_q_agg[Q];
  __shared__ P s_q_prefix[Q];
  __shared__ unsigned int s_q_in;
  __shared__ int s_abort;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  auto abort_now = [&]() { *reinterpret_cast<volatile int *>(&s_abort) = 1; };
  auto aborted = [&]() -> bool { return *reinterpret_cast<volatile int *>(&s_abort) != 0; };
  auto buf = [&](int b) { return smem_raw + (size_t)b * C::BUF_BYTES; };
  // run slot s of this CTA: TILE keys, then TILE values
  unsigned char *const cta_ring = ring + (size_t)blockIdx.x * kRbkRunSlots * C::RUN_SLOT_BYTES;
  auto slot_keys = [&](int s) { return reinterpret_cast<K *>(cta_ring + (size_t)s * C::RUN_SLOT_BYTES); };
  auto slot_vals = [&](int s) {
    return reinterpret_cast<V *>(cta_ring + (size_t)s * C::RUN_SLOT_BYTES + sizeof(K) * TILE);
  };

  uint64_t stream = 0;
  uint32_t armpar = 0u, armany = 0u;  // loader: parity of the phases armed on s_full[b] / any armed
  unsigned int next_raw = NONE;
  bool loads_done = false;
  if (tid == 32 * kRbkWarps) {
    stream = l2_policy_evict_first();
    for (int b = 0; b < NB; ++b) {
      mbar_init(&s_full[b], 1);
      mbar_init(&s_empty[b], kRbkWarps);
    }
    for (int q = 0; q < Q; ++q) mbar_init(&s_qbar[q], 1);
    fence_proxy_async_smem();
    s_abort = 0;
    s_q_in = 0u;
    // the loads of iterations 0 .. D-1 (tickets in order; none after the first past the end)
    for (int d = 0; d < D; ++d) {
      unsigned int tk = NONE;
      if (!loads_done) {
        tk = atomicAdd(&hdr->tile_ticket, 1u);
        if (tk >= num_tiles) tk = NONE;
      }
      s_ticket[d] = tk;
      bool tx = false;
      if (tk != NONE) tx = rbk_issue_load<K, V>(src, src.tile(tk), buf(d), s_halo[d], &s_full[d], stream);
      if (!tx) mbar_arrive(&s_full[d]);
      armpar ^= 1u << d;
      armany |= 1u << d;
      if (tk == NONE) loads_done = true;
    }
    if (!loads_done) next_raw = atomicAdd(&hdr->tile_ticket, 1u);
  }
  __syncthreads();

  if (warp == kRbkWarps) {
    // ================= the loader (lane 0) =================
    if (lane != 0) return;
    uint32_t epar = 0u;
    for (int it = 0; !loads_done; ++it) {
      // the load for iteration it + D goes to the buffer of iteration it - 1,
      // free once that iteration's phase 1 is done with it
      const int bn = (it + D) % NB;
      if (it >= 1) {
        if (!mbar_wait_or_abort(&s_empty[bn], (epar >> bn) & 1u, spin_limit_ns, &s_abort)) {
          record_error(hdr, BK_ERR_SPIN_TIMEOUT, NONE);
          abort_now();
          break;
        }
        epar ^= 1u << bn;
      }
      const unsigned int tn = next_raw < num_tiles ? next_raw : NONE;
      s_ticket[bn] = tn;
      bool tx = false;
      if (tn != NONE) tx = rbk_issue_load<K, V>(src, src.tile(tn), buf(bn), s_halo[bn], &s_full[bn], stream);
      if (!tx) mbar_arrive(&s_full[bn]);
      armpar ^= 1u << bn;
      armany |= 1u << bn;
      if (tn == NONE) {
        loads_done = true;
      } else {
        next_raw = atomicAdd(&hdr->tile_ticket, 1u);
        // tiles are ticketed about in order, gridDim.x per iteration: ask L2
        // now for the one some CTA will load an iteration from now
        if (tn + gridDim.x < num_tiles) {
          const RbkTile<K, V> f = src.tile(tn + gridDim.x);
          const uint64_t fb = (uint64_t)f.local * TILE;
          prefetch_l2_range(f.keys + fb, (uint64_t)f.count() * sizeof(K));
          prefetch_l2_range(f.vals + fb, (uint64_t)f.count() * sizeof(V));
        }
      }
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
    // tiles in queue order, each once the next one is queued (its
    // predecessors have then had an iteration to publish; its phase 2 is
    // three iterations after its phase 1), so the L2 round trips of the
    // look-back mostly find aggregates and prefixes already there
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
  uint32_t fpar = 0u;  // bit b: parity of the next phase of s_full[b]
  // the tiles of the last three iterations (index: iterations ago - 1), each
  // with its run count (bits 0-12), head count (bits 13-25) and whether it
  // starts with a head (bit 26); counts are at most TILE <= 4096
  static_assert(TILE <= 4096, "13-bit counts");
  unsigned int tq[3] = {NONE, NONE, NONE};
  uint32_t iq[3] = {0u, 0u, 0u};
  bool ended = false;                 // an iteration has had no tile: no more loads
  bool bad = false;

  for (int it = 0;; ++it) {
    const int bt = it % NB, ps = it & 1;
    const unsigned int p = tq[2];  // phase 2 of t_{it-3}
    const uint32_t pr = iq[2] & 0x1fffu, pc = (iq[2] >> 13) & 0x1fffu, ph = iq[2] >> 26;

    // phase 2 of p reads its run slot (written before the last barrier):
    // start the loads of this thread's first two runs now, so that their L2
    // round trip overlaps phase 1
    K pk[2];
    V pv[2];
    if (p != NONE) {
      const K *const rk = slot_keys((it + 1) % kRbkRunSlots);  // == (it - 3) mod 4
      const V *const rv = slot_vals((it + 1) % kRbkRunSlots);
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const uint32_t i = (uint32_t)tid + 32u * kRbkWarps * k;
        if (i < pr) {
          pk[k] = rk[i];
          pv[k] = rv[i];
        }
      }
    }

    // ---- phase 1 of t
    unsigned int t = NONE;
    if (!ended) {
      if (!mbar_wait_or_abort(&s_full[bt], (fpar >> bt) & 1u, spin_limit_ns, &s_abort)) bad = true;
      fpar ^= 1u << bt;
      bad = __any_sync(0xffffffffu, bad);
      if (!bad) t = s_ticket[bt];
      // tiles without a TMA copy: the compute warps stage them here, then meet
      // (every compute warp takes that barrier whenever the launch may have
      // such a tile -- a flag of the launch, so a warp that saw a failure
      // still takes part; the buffer's previous tile was done with it before
      // the last iteration's barrier)
      if (src.may_stage) {
        if (t != NONE && !src.tile(t).tma) {
          rbk_stage_load<K, V, SWZ>(src.tile(t), buf(bt));
          fence_proxy_async_smem();  // as after phase 1's own stores below
        }
        named_barrier_sync(2, 32 * kRbkWarps);
      }
    }
    uint32_t heads = 0u, tails = 0u;
    P lex = OpSeg<V>::identity();  // the lane's exclusive (c, v) within its warp
    if (t != NONE) {
      const RbkTile<K, V> tl = src.tile(t);
      const uint32_t count = tl.count();
      P lane_agg;
      if (count == (uint32_t)TILE)  // every tile but an array's last: no bounds checks
        lane_agg = rbk_phase1_lane<K, V, SWZ, true>(buf(bt), s_halo[bt], count, tl.first(), tl.last(), e0, lane,
                                                    &heads, &tails);
      else
        lane_agg = rbk_phase1_lane<K, V, SWZ, false>(buf(bt), s_halo[bt], count, tl.first(), tl.last(), e0, lane,
                                                     &heads, &tails);
      const P incl = warp_inclusive_scan(lane_agg, op, lane);
      const uint32_t nr = __reduce_add_sync(0xffffffffu, (uint32_t)__popc(tails));
      if (lane == 31) {
        s_wagg[ps][warp] = incl;
        s_wruns[ps][warp] = nr;
      }
      lex = shfl_up(incl, 1);
      if (lane == 0) lex = OpSeg<V>::identity();
      if (tid == 0) s_h0[ps] = heads & 1u;
    }
    if (named_barrier_or(1, 32 * kRbkWarps, bad || aborted())) {
      if (lane == 0) abort_now();  // the loader and the look-back warp stop too
      break;
    }

    uint32_t h0 = 0u, nruns = 0u, aggc = 0u;
    if (t != NONE) {
      h0 = s_h0[ps];
      // lanes 0-7 scan the warps' (c, v) and run counts: lane w - 1 then holds
      // the fold of warps 0 .. w-1, lane 7 the tile's
      P a = OpSeg<V>::identity();
      uint32_t rc = 0u;
      if (lane < kRbkWarps) {
        a = s_wagg[ps][lane];
        rc = s_wruns[ps][lane];
      }
#pragma unroll
      for (int d = 1; d < kRbkWarps; d <<= 1) {
        const P o = shfl_up(a, d);
        const uint32_t ro = __shfl_up_sync(0xffffffffu, rc, d);
        if (lane >= d) {
          a = op(o, a);
          rc += ro;
        }
      }
      P wex = shfl_idx_any(a, warp > 0 ? warp - 1 : 0);
      if (warp == 0) wex = OpSeg<V>::identity();
      const P agg = shfl_idx_any(a, kRbkWarps - 1);
      nruns = __shfl_sync(0xffffffffu, rc, kRbkWarps - 1);
      aggc = agg.c;
      if (warp == kRbkWarps - 1 && lane == 0) {
        if ((long long)t != skip_publish_tile) st.publish(t, src.tile(t).first() ? kStPrefix : kStAggregate, agg);
        s_q_tile[it % Q] = t;
        s_q_agg[it % Q] = agg;
        st_release_cta_u32(&s_q_in, (unsigned int)it + 1u);
      }
      // the runs ending in this lane's elements go to the tile's run slot.
      // A run's slot within the tile counts the tile's heads up to its tail,
      // less h0; a lane's only head before its first tail can be its first
      // element, and a first tail with no head before it closes a run that
      // began before the lane, whose sum so far is the lane's exclusive v
      // (later tails' running values start at a head of the lane).
      if (tails != 0u) {
        K *const rk = slot_keys(it % kRbkRunSlots);
        V *const rv = slot_vals(it % kRbkRunSlots);
        const unsigned char *const b = buf(bt);
        const P lx = op(wex, lex);
        uint32_t r = lx.c - h0 + (heads & 1u);
        bool open = (heads & 1u) == 0u;
        for (uint32_t tb = tails; tb != 0u; tb &= tb - 1u) {
          const uint32_t e = e0 + (uint32_t)__ffs(tb) - 1u;
          const K k = *reinterpret_cast<const K *>(b + area_off<SWZ>(e * (uint32_t)sizeof(K)));
          V v = *reinterpret_cast<const V *>(b + C::KEY_BYTES + area_off<SWZ>(e * (uint32_t)sizeof(V)));
          if (open) v = (V)(lx.v + v);
          open = false;
          rk[r] = k;
          rv[r] = v;
          ++r;
        }
      }
      // the loader's next TMA copy into this buffer must land after phase 1's
      // stores to it
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&s_empty[bt]);
    } else if (!ended && warp == kRbkWarps - 1 && lane == 0) {
      s_q_tile[it % Q] = NONE;  // ends the look-back warp's loop
      st_release_cta_u32(&s_q_in, (unsigned int)it + 1u);
    }

    // ---- phase 2 of p = t_{it-3}: its runs from its run slot to the output
    if (p != NONE) {
      const unsigned int e = (unsigned int)it - 3u;
      if (!mbar_wait_or_abort(&s_qbar[e % Q], (e / Q) & 1u, spin_limit_ns, &s_abort)) bad = true;
      bad = __any_sync(0xffffffffu, bad);
      if (!bad) {
        const RbkTile<K, V> tl = src.tile(p);
        const P pre = s_q_prefix[e % Q];
        // the tile's first run goes to slot pre.c + h0 - 1 (pre.c >= 1 when h0 = 0)
        K *const ok = tl.out_keys + ((uint64_t)pre.c + ph - 1u);
        V *const ov = tl.out_vals + ((uint64_t)pre.c + ph - 1u);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const uint32_t i = (uint32_t)tid + 32u * kRbkWarps * k;
          if (i < pr) {
            V v = pv[k];
            if (i == 0u && ph == 0u) v = (V)(pre.v + v);
            ok[i] = pk[k];
            ov[i] = v;
          }
        }
        const K *const rk = slot_keys((int)(e % kRbkRunSlots));
        const V *const rv = slot_vals((int)(e % kRbkRunSlots));
        for (uint32_t i = (uint32_t)tid + 64u * kRbkWarps; i < pr; i += 32u * kRbkWarps) {
          ok[i] = rk[i];
          ov[i] = rv[i];
        }
        if (tid == 0 && tl.last()) *tl.num_out = (uint64_t)pre.c + pc;
      }
    }

    if (t == NONE) ended = true;
#pragma unroll
    for (int k = 2; k > 0; --k) {
      tq[k] = tq[k - 1];
      iq[k] = iq[k - 1];
    }
    tq[0] = t;
    iq[0] = nruns | aggc << 13 | h0 << 26;
    if (t == NONE && tq[1] == NONE && tq[2] == NONE) break;
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
  const size_t smem = (size_t)C::NB * C::BUF_BYTES + 1024;  // + room to align the buffers to 1024 bytes
  struct Site {};
  host::KernelSetup ks;
  if ((st = host::kernel_setup<Site>(rbk_kernel<K, V, Src>, kRbkThreads, smem, &ks)) != BK_OK) return st;
  const tune::Knobs kn = tune::knobs_for(tune::kReduceByKey, (int)(sizeof(K) + sizeof(V)), (uint64_t)tiles * C::TILE);
  const size_t per_sm = (size_t)std::min(std::max(kn.ctas_per_sm, 1), C::CTAS);
  const unsigned grid = (unsigned)std::min<size_t>(tiles, std::min<size_t>((size_t)di.sm_count * per_sm, kRbkMaxGrid));
  unsigned char *ring = reinterpret_cast<unsigned char *>(d_ws) + rbk_ring_offset<K, V>(tiles);
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
