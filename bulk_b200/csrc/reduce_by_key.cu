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
#include "bk_common.cuh"
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
  static constexpr size_t KEY_BYTES = align_up(sizeof(K) * TILE, 128);
  static constexpr size_t BUF_BYTES = KEY_BYTES + align_up(sizeof(V) * TILE, 128);
  using P = Seg<V>;
  using Status = TileStatus<P>;
};

template <typename K, typename V>
size_t rbk_num_tiles(uint64_t n) {
  return (size_t)((n + RbkCfg<K, V>::TILE - 1) / RbkCfg<K, V>::TILE);
}
// Workspace: the header, one look-back status per tile, then the tail-mark
// ring: three tile-sized value slots per persistent CTA (phase 1 of a tile
// writes its tails' values there; the re-read for phase 2 brings them back).
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
  bool tma;        // keys and vals 16-byte aligned
  __device__ __forceinline__ uint32_t count() const {
    const uint64_t base = (uint64_t)local * RbkCfg<K, V>::TILE;
    return (uint32_t)((n - base) < (uint64_t)RbkCfg<K, V>::TILE ? (n - base) : (uint64_t)RbkCfg<K, V>::TILE);
  }
  __device__ __forceinline__ bool first() const { return local == 0u; }
  __device__ __forceinline__ bool last() const { return (uint64_t)local * RbkCfg<K, V>::TILE + count() == n; }
};

// Tile source: one array.
template <typename K, typename V>
struct RbkOne {
  const K *keys;
  const V *vals;
  uint64_t n;
  K *out_keys;
  V *out_vals;
  uint64_t *num_out;
  int tma;
  int any_unaligned;
  __device__ __forceinline__ RbkTile<K, V> tile(unsigned int t) const {
    return RbkTile<K, V>{keys, vals, n, t, out_keys, out_vals, num_out, tma != 0};
  }
};

// Tile source: a batch of independent arrays reduced by one launch.  Array i
// owns global tiles [start[i], start[i + 1]); its first tile publishes an
// inclusive prefix at once, so no look-back crosses into another array.  The
// descriptors travel in the kernel's parameters.
constexpr int kRbkBatchMax = 256;
template <typename K, typename V>
struct RbkBatch {
  const K *keys[kRbkBatchMax];
  const V *vals[kRbkBatchMax];
  uint64_t n[kRbkBatchMax];
  K *out_keys[kRbkBatchMax];
  V *out_vals[kRbkBatchMax];
  uint64_t *num_out[kRbkBatchMax];
  uint32_t start[kRbkBatchMax + 1];
  uint32_t count;
  int any_unaligned;
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
};

// Leader: load tile `tile` (keys, values and the halo keys on either side)
// into buffer `buf`.  The halo keys arrive as the aligned 16-byte chunks that
// hold them (hb[0]: the chunk ending just before the tile, hb[1]: the chunk
// starting just after it), on the same mbarrier as the tile.  Returns whether
// a TMA copy was issued on `bar`.
template <typename K, typename V>
__device__ __forceinline__ bool rbk_issue_load(const K *keys, const V *vals, uint64_t n, unsigned int tile,
                                               unsigned char *buf, K (*hb)[16 / sizeof(K)], uint64_t *bar,
                                               uint64_t policy, bool tma_ok) {
  using C = RbkCfg<K, V>;
  constexpr uint32_t KC = 16 / sizeof(K);  // keys per 16-byte chunk
  const uint64_t base = (uint64_t)tile * C::TILE;
  const uint32_t count = (uint32_t)((n - base) < (uint64_t)C::TILE ? (n - base) : (uint64_t)C::TILE);
  K *sk = reinterpret_cast<K *>(buf);
  V *sv = reinterpret_cast<V *>(buf + C::KEY_BYTES);
  if (!tma_ok) {
    if (base > 0) hb[0][KC - 1] = keys[base - 1];
    if (base + count < n) hb[1][0] = keys[base + count];
    return false;
  }
  const uint32_t bk = count & ~(KC - 1);
  const uint32_t bv = count & ~(uint32_t)(16 / sizeof(V) - 1);
  for (uint32_t i = bk; i < count; ++i) sk[i] = keys[base + i];
  for (uint32_t i = bv; i < count; ++i) sv[i] = vals[base + i];
  const bool halo_prev = base > 0;  // base is a multiple of TILE: the chunk before it is aligned
  const bool halo_next_bulk = (count % KC) == 0 && base + count + KC <= n;
  if (!halo_next_bulk && base + count < n) hb[1][0] = keys[base + count];  // rare: next-to-last tile
  const uint32_t bytes =
      bk * (uint32_t)sizeof(K) + bv * (uint32_t)sizeof(V) + (halo_prev ? 16u : 0u) + (halo_next_bulk ? 16u : 0u);
  if (bytes == 0) return false;
  mbar_arrive_expect_tx(bar, bytes);
  if (bk) tma_load_1d_hint(sk, keys + base, bk * (uint32_t)sizeof(K), bar, policy);
  if (bv) tma_load_1d_hint(sv, vals + base, bv * (uint32_t)sizeof(V), bar, policy);
  if (halo_prev) tma_load_1d_hint(hb[0], keys + base - KC, 16u, bar, policy);
  if (halo_next_bulk) tma_load_1d_hint(hb[1], keys + base + count, 16u, bar, policy);
  return true;
}

// Compute threads: plain copy of a tile (pointers not 16-byte aligned).
template <typename K, typename V>
__device__ __forceinline__ void rbk_sync_load(const K *keys, const V *vals, uint64_t n, unsigned int tile,
                                              unsigned char *buf) {
  using C = RbkCfg<K, V>;
  const uint64_t base = (uint64_t)tile * C::TILE;
  const uint32_t count = (uint32_t)((n - base) < (uint64_t)C::TILE ? (n - base) : (uint64_t)C::TILE);
  K *sk = reinterpret_cast<K *>(buf);
  V *sv = reinterpret_cast<V *>(buf + C::KEY_BYTES);
  for (uint32_t i = threadIdx.x; i < count; i += kRbkWarps * 32) {
    sk[i] = keys[base + i];
    sv[i] = vals[base + i];
  }
}

// Leader: re-read tile `tile` for phase 2 into buffer `buf`: its keys from
// the input (L2) and its tails' values from the mark slot `marks` (TILE
// values, 16-byte aligned).  Returns whether a TMA copy was issued on `bar`;
// without TMA (keys not 16-byte aligned) the compute warps copy both.
template <typename K, typename V>
__device__ __forceinline__ bool rbk_issue_reload(const K *keys, const V *marks, uint64_t n, unsigned int tile,
                                                 unsigned char *buf, uint64_t *bar, uint64_t policy, bool tma_ok) {
  using C = RbkCfg<K, V>;
  constexpr uint32_t KC = 16 / sizeof(K);
  if (!tma_ok) return false;
  const uint64_t base = (uint64_t)tile * C::TILE;
  const uint32_t count = (uint32_t)((n - base) < (uint64_t)C::TILE ? (n - base) : (uint64_t)C::TILE);
  K *sk = reinterpret_cast<K *>(buf);
  V *sv = reinterpret_cast<V *>(buf + C::KEY_BYTES);
  const uint32_t bk = count & ~(KC - 1);
  for (uint32_t i = bk; i < count; ++i) sk[i] = keys[base + i];
  const uint32_t vbytes = (uint32_t)align_up(count * sizeof(V), 16);  // within the slot
  mbar_arrive_expect_tx(bar, bk * (uint32_t)sizeof(K) + vbytes);
  if (bk) tma_load_1d_hint(sk, keys + base, bk * (uint32_t)sizeof(K), bar, policy);
  tma_load_1d_hint(sv, marks, vbytes, bar, policy);
  return true;
}

// Compute threads: plain copy of a tile's keys and tail marks for phase 2.
template <typename K, typename V>
__device__ __forceinline__ void rbk_sync_reload(const K *keys, const V *marks, uint64_t n, unsigned int tile,
                                                unsigned char *buf) {
  using C = RbkCfg<K, V>;
  const uint64_t base = (uint64_t)tile * C::TILE;
  const uint32_t count = (uint32_t)((n - base) < (uint64_t)C::TILE ? (n - base) : (uint64_t)C::TILE);
  K *sk = reinterpret_cast<K *>(buf);
  V *sv = reinterpret_cast<V *>(buf + C::KEY_BYTES);
  for (uint32_t i = threadIdx.x; i < count; i += kRbkWarps * 32) {
    sk[i] = keys[base + i];
    sv[i] = marks[i];
  }
}

// Loads a lane's B bytes (B = 32 or 64: C = B/16 chunks of 16 bytes) starting
// at byte offset lane_off of `base` into dst, conflict-free: eight lanes share
// one 128-byte bank period, so lane l fetches its chunks starting at chunk
// r = (l / (8 / C)) mod C, which gives the eight lanes of every access phase
// distinct banks; two select stages then rotate the chunks back into order.
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

// A lane's M consecutive elements of a staged tile, with head / tail flags.
template <typename K, typename V, int M>
struct LaneRun {
  K key[M];
  V val[M];
  uint32_t head;  // bit j: element j starts a run
  uint32_t tail;  // bit j: element j ends a run
  int nvalid;     // elements of this lane inside the tile
};

// Loads a lane's M consecutive keys and values of a staged tile (element
// index of its first: e0 = (warp * 32 + lane) * M); elements past the tile's
// end read as key K() and value 0.
// FULL: the tile holds TILE elements, so every lane's are all inside it.
template <typename K, typename V, bool FULL>
__device__ __forceinline__ void rbk_load_lane(const unsigned char *buf, uint32_t count, int warp, int lane,
                                              LaneRun<K, V, RbkCfg<K, V>::M> &lr) {
  using C = RbkCfg<K, V>;
  constexpr int M = C::M;
  const uint32_t e0 = (uint32_t)(warp * 32 + lane) * M;
  load_lane_rotated<M * sizeof(K)>(lr.key, buf, e0 * (uint32_t)sizeof(K), lane);
  load_lane_rotated<M * sizeof(V)>(lr.val, buf + C::KEY_BYTES, e0 * (uint32_t)sizeof(V), lane);
  const int nvalid = FULL ? M : (int)min(max((int)count - (int)e0, 0), M);
  lr.nvalid = nvalid;
  if (!FULL && nvalid < M) {
#pragma unroll
    for (int j = 0; j < M; ++j)
      if (j >= nvalid) {
        lr.key[j] = K();
        lr.val[j] = V(0);
      }
  }
}

// Head and tail flags of a lane's loaded elements.  A head's key differs
// from its predecessor's, so an element before a head is a tail; the lane's
// last element compares with the next lane's first key, read by a shuffle
// (lane 31: from shared memory, or the halo hb[1][0] after the tile).  Lane 0
// reads the key before the warp's range from shared memory, or the halo
// hb[0][KC-1] before the tile.  first_tile: the tile starts the input;
// last_tile: it ends it.
template <typename K, typename V, bool FULL>
__device__ __forceinline__ void rbk_flags(const unsigned char *buf, const K (*hb)[16 / sizeof(K)], uint32_t count,
                                          bool first_tile, bool last_tile, int warp, int lane,
                                          LaneRun<K, V, RbkCfg<K, V>::M> &lr) {
  using C = RbkCfg<K, V>;
  constexpr int M = C::M;
  constexpr int KC = 16 / sizeof(K);
  const K *sk = reinterpret_cast<const K *>(buf);
  const uint32_t e0 = (uint32_t)(warp * 32 + lane) * M;
  const int nvalid = FULL ? M : lr.nvalid;
  K prev = shfl_up(lr.key[M - 1], 1);
  K next = shfl_down_any(lr.key[0], 1);
  if (lane == 0) prev = e0 == 0 ? hb[0][KC - 1] : sk[e0 - 1];
  if (lane == 31) next = e0 + M < count ? sk[e0 + M] : hb[1][0];
  uint32_t head = 0;
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const K pk = j == 0 ? prev : lr.key[j - 1];
    head |= (uint32_t)((j < nvalid) && !(lr.key[j] == pk)) << j;
  }
  if (first_tile && e0 == 0 && nvalid > 0) head |= 1u;  // the input's first element
  // element j < nvalid - 1 ends a run exactly when j + 1 starts one
  uint32_t tail = nvalid > 0 ? (head >> 1) & ((1u << (nvalid - 1)) - 1u) : 0u;
  if (nvalid == M) {
    const bool tile_end = e0 + M == count;
    const bool tl = tile_end ? (last_tile || !(hb[1][0] == lr.key[M - 1])) : !(next == lr.key[M - 1]);
    tail |= (uint32_t)tl << (M - 1);
  } else if (nvalid > 0) {  // the lane holding the tile's last element
    K kl = lr.key[0];
#pragma unroll
    for (int j = 1; j < M; ++j)
      if (j == nvalid - 1) kl = lr.key[j];
    tail |= (uint32_t)(last_tile || !(hb[1][0] == kl)) << (nvalid - 1);
  }
  lr.head = head;
  lr.tail = tail;
}

// (c, v) of a lane's elements folded in order.  At every tail the run's value
// so far -- from the run's head, or from the lane's first element when the
// run began before the lane -- goes to the lane's tail-mark slot (marks[j]
// for element j), where the re-read for phase 2 picks it up.
template <typename K, typename V, int M>
__device__ __forceinline__ Seg<V> lane_fold_mark(const LaneRun<K, V, M> &lr, V *marks) {
  uint32_t c = __popc(lr.head);
  V v = V(0);
#pragma unroll
  for (int j = 0; j < M; ++j) {
    if (lr.head & (1u << j)) v = lr.val[j];
    else v = (V)(v + lr.val[j]);
    if (lr.tail & (1u << j)) marks[j] = v;
  }
  return Seg<V>{c, v};
}

// Persistent two-phase reduce_by_key; the roles, buffer rotation and
// hand-over protocol are scan_kernel's (scan.cu), with these differences: a
// buffer holds a tile's keys, values and halo keys; phase 1 also writes each
// tail's value so far to the CTA's tail-mark slot for the tile (ring slot
// blockIdx.x * 3 + iteration mod 3), and the re-read for phase 2 brings back
// the tile's keys with those marks in place of its values, so phase 2 costs
// one step per run, not per element; phase 2 only reads its buffer (the runs
// go straight to out_keys / out_vals), so the loader reuses a buffer once the
// compute warps are done reading it, with no store to drain; and without TMA
// (pointers not 16-byte aligned) the compute warps stage both tiles
// themselves between two compute-only barriers.
template <typename K, typename V, typename Src>
__global__ void __launch_bounds__(kRbkThreads, 2) rbk_kernel(const __grid_constant__ Src src,
                                                             typename RbkCfg<K, V>::Status st, WsHeader *hdr,
                                                             V *ring, unsigned long long spin_limit_ns,
                                                             long long skip_publish_tile, unsigned int num_tiles) {
  using C = RbkCfg<K, V>;
  using P = typename C::P;
  constexpr int M = C::M, TILE = C::TILE, NB = kRbkBufs, Q = kRbkQueue;
  V *const cta_ring = ring + (size_t)blockIdx.x * 3 * TILE;  // this CTA's three tail-mark slots
  constexpr unsigned int NONE = 0xffffffffu;
  OpSeg<V> op;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(16) K s_halo[NB][2][16 / sizeof(K)];
  __shared__ __align__(8) uint64_t s_full[NB];
  __shared__ __align__(8) uint64_t s_p1[NB];
  __shared__ __align__(8) uint64_t s_p2[NB];
  __shared__ __align__(8) uint64_t s_qbar[Q];
  __shared__ unsigned int s_ticket[NB];
  __shared__ P s_wagg[4][kRbkWarps];  // per-warp (c, v) of t_i, by iteration mod 4
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

  uint64_t keep = 0, stream = 0;
  uint32_t armed[NB];  // loader: phases armed on s_full[b]
#pragma unroll
  for (int b = 0; b < NB; ++b) armed[b] = 0u;
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
    if (t_first != NONE) {
      const RbkTile<K, V> tl = src.tile(t_first);
      tx = rbk_issue_load<K, V>(tl.keys, tl.vals, tl.n, tl.local, buf(0), s_halo[0], &s_full[0], keep, tl.tma);
    }
    if (!tx) mbar_arrive(&s_full[0]);
    armed[0] = 1u;
    mbar_arrive(&s_full[NB - 1]);  // iteration 0's phase 2 reads buffer NB - 1: an empty phase
    armed[NB - 1] = 1u;
    if (t_first != NONE) next_raw = atomicAdd(&hdr->tile_ticket, 1u);
  }
  __syncthreads();

  if (warp == kRbkWarps) {
    // ================= the loader (lane 0) =================
    if (lane != 0) return;
    uint32_t p1par[NB], p2par[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) p1par[b] = p2par[b] = 0u;
    unsigned int t = t_first, p_tile = NONE, q_tile = NONE;
    for (int it = 0;; ++it) {
      const int bt = it % NB, bp = (it + NB - 1) % NB, bn = (it + 1) % NB;
      // prefetch t_{i+1} into bn (the compute warps finished reading it last iteration)
      const unsigned int tn = (t != NONE && next_raw < num_tiles) ? next_raw : NONE;
      s_ticket[bn] = tn;
      bool tx = false;
      if (tn != NONE) {
        const RbkTile<K, V> tl = src.tile(tn);
        tx = rbk_issue_load<K, V>(tl.keys, tl.vals, tl.n, tl.local, buf(bn), s_halo[bn], &s_full[bn], keep, tl.tma);
      }
      if (!tx) mbar_arrive(&s_full[bn]);
      ++armed[bn];
      next_raw = (tn != NONE) ? atomicAdd(&hdr->tile_ticket, 1u) : NONE;
      // re-read t_{i-1} into t's buffer once phase 1 of t is done with it
      if (!mbar_wait_or_abort(&s_p1[bt], p1par[bt], spin_limit_ns, &s_abort)) {
        record_error(hdr, BK_ERR_SPIN_TIMEOUT, t);
        abort_now();
        break;
      }
      p1par[bt] ^= 1u;
      tx = false;
      if (q_tile != NONE) {  // t_{it-1}: its phase 1 ran in iteration it-1
        const RbkTile<K, V> tl = src.tile(q_tile);
        tx = rbk_issue_reload<K, V>(tl.keys, cta_ring + (size_t)((it + 2) % 3) * TILE, tl.n, tl.local, buf(bt),
                                    &s_full[bt], stream, tl.tma);
      }
      if (!tx) mbar_arrive(&s_full[bt]);
      ++armed[bt];
      // buffer bp is free once phase 2 of p has read it
      if (!mbar_wait_or_abort(&s_p2[bp], p2par[bp], spin_limit_ns, &s_abort)) {
        record_error(hdr, BK_ERR_SPIN_TIMEOUT, p_tile);
        abort_now();
        break;
      }
      p2par[bp] ^= 1u;
      p_tile = q_tile;
      q_tile = t;
      t = tn;
      if (t == NONE && p_tile == NONE && q_tile == NONE) break;
    }
    // every load must land before the CTA's shared memory goes away
    for (int b = 0; b < NB; ++b)
      if (armed[b] != 0u) (void)mbar_wait(&s_full[b], (armed[b] - 1u) & 1u, spin_limit_ns);
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
  uint32_t fpar[NB];
#pragma unroll
  for (int b = 0; b < NB; ++b) fpar[b] = 0u;
  unsigned int p_tile = NONE, q_tile = NONE;
  bool bad = false;

  for (int it = 0;; ++it) {
    const int bt = it % NB, bp = (it + NB - 1) % NB;
    const unsigned int p = p_tile;

    // ---- phase 1 of t
    unsigned int t = NONE;
    if (!mbar_wait_or_abort(&s_full[bt], fpar[bt], spin_limit_ns, &s_abort)) bad = true;
    fpar[bt] ^= 1u;
    bad = __any_sync(0xffffffffu, bad);
    if (!bad) t = s_ticket[bt];
    if (src.any_unaligned) {
      // stage the tiles that have no TMA copy here (previous iteration's
      // readers are past the first barrier)
      named_barrier_sync(2, 32 * kRbkWarps);
      if (t != NONE) {
        const RbkTile<K, V> tl = src.tile(t);
        if (!tl.tma) rbk_sync_load<K, V>(tl.keys, tl.vals, tl.n, tl.local, buf(bt));
      }
      if (p != NONE) {  // t_{it-2}: its phase 1 ran in iteration it-2
        const RbkTile<K, V> tl = src.tile(p);
        if (!tl.tma) rbk_sync_reload<K, V>(tl.keys, cta_ring + (size_t)((it + 1) % 3) * TILE, tl.n, tl.local, buf(bp));
      }
      named_barrier_sync(2, 32 * kRbkWarps);
    }
    if (t != NONE) {
      const RbkTile<K, V> tl = src.tile(t);
      const uint32_t count = tl.count();
      LaneRun<K, V, M> lr;
      if (count == (uint32_t)TILE) {  // every tile but an array's last: no bounds checks
        rbk_load_lane<K, V, true>(buf(bt), count, warp, lane, lr);
        rbk_flags<K, V, true>(buf(bt), s_halo[bt], count, tl.first(), tl.last(), warp, lane, lr);
      } else {
        rbk_load_lane<K, V, false>(buf(bt), count, warp, lane, lr);
        rbk_flags<K, V, false>(buf(bt), s_halo[bt], count, tl.first(), tl.last(), warp, lane, lr);
      }
      V *marks = cta_ring + (size_t)(it % 3) * TILE + (warp * 32 + lane) * M;
      const P incl = warp_inclusive_scan(lane_fold_mark(lr, marks), op, lane);
      fence_proxy_async_global();  // the marks are read back by a TMA copy
      if (lane == 31) s_wagg[it & 3][warp] = incl;
      P lex = shfl_up(incl, 1);
      if (lane == 0) lex = OpSeg<V>::identity();
      const int sl = it % 3, li = warp * 32 + lane;
      s_lflags[sl][li] = lr.head | (lr.tail << 16);
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
    if (!mbar_wait_or_abort(&s_full[bp], fpar[bp], spin_limit_ns, &s_abort)) bad = true;
    fpar[bp] ^= 1u;
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
      const uint32_t e0 = (uint32_t)li * M;
      const bool holds_last = tl.last() && e0 < count && count <= e0 + M;  // the input's last element
      if (tail != 0u || holds_last) {
        P carry = op(s_q_prefix[e % Q], s_wexcl[(it + 2) & 3][warp]);
        carry = op(carry, P{s_lc[sl][li], s_lv[sl][li]});
        // each tail: its key, and its mark (the run's value from its head, or
        // from the lane's first element when the run began before the lane)
        const K *sk = reinterpret_cast<const K *>(buf(bp)) + e0;
        const V *sv = reinterpret_cast<const V *>(buf(bp) + C::KEY_BYTES) + e0;
        for (uint32_t tb = tail; tb != 0u; tb &= tb - 1u) {
          const int j = __ffs(tb) - 1;
          const uint32_t upto = head & ((2u << j) - 1u);  // heads at or before j
          const uint32_t c = carry.c + (uint32_t)__popc(upto);
          V v = sv[j];
          if (upto == 0u) v = (V)(carry.v + v);
          tl.out_keys[c - 1] = sk[j];
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
  const size_t smem = (size_t)kRbkBufs * C::BUF_BYTES;
  struct Site {};
  host::KernelSetup ks;
  if ((st = host::kernel_setup<Site>(rbk_kernel<K, V, Src>, kRbkThreads, smem, &ks)) != BK_OK) return st;
  const unsigned grid = (unsigned)std::min<size_t>(tiles, std::min<size_t>((size_t)di.sm_count * 2, kRbkMaxGrid));
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
  const int tma = ((reinterpret_cast<uintptr_t>(keys) | reinterpret_cast<uintptr_t>(vals)) & 15) == 0;
  const RbkOne<K, V> src{keys, vals, n, out_keys, out_vals, d_num_out, tma, !tma};
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
  b.any_unaligned = 0;
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
    if (((reinterpret_cast<uintptr_t>(it.keys) | reinterpret_cast<uintptr_t>(it.vals)) & 15) != 0) b.any_unaligned = 1;
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
