// scan.cu -- single-pass inclusive scan with decoupled look-back, sm_100a.
//
// Replaces the reference's three-pass ::inclusive_scan (scan.cu:87-148):
// upsweep accumulate_tiles (:57-84) -> spine exclusive_scan_n (:24-31) ->
// downsweep inclusive_downsweep (:34-54), each calling the group scan of
// bulk/algorithm/scan.hpp:222-384.  That design moves 3*N*s bytes; this one
// moves the minimum 2*N*s (read once, write once).
//
// Per tile (32 KB): an atomic ticket names the tile (launch order, so every
// predecessor is already running); a TMA bulk copy brings it into shared
// memory, where the compute warps reduce it and the tile publishes its
// aggregate; a dedicated look-back warp later finds its exclusive prefix
// over the predecessors' published statuses (bk_lookback.cuh) and publishes
// its inclusive prefix; the tile is then re-read from L2, scanned, and
// written with one TMA bulk store.  A tiny init kernel clears the tile
// status words before each scan.
//
// Semantics follow scan.cu:166-169 and bulk/algorithm/scan.hpp:455-486:
// out[i] = init (+) in[0] (+) ... (+) in[i].
#include "bk_common.cuh"
#include "bk_tune.hpp"
#include "bk_lookback.cuh"
#include "bk_tma.cuh"

namespace bk {

constexpr int kScanWarps = 8;                        // compute warps (0-7)
constexpr int kScanThreads = 32 * (kScanWarps + 2);  // + the loader warp (8; one lane works) + the look-back warp (9)
constexpr int kScanRowsPerWarp = 8;
constexpr int kScanBufs = 3;   // tile buffers in rotation (see scan_kernel)
constexpr int kScanQueue = 4;  // look-back queue entries (more than the 2-iteration lag)

template <typename T>
struct ScanCfg {
  static constexpr int V = 16 / sizeof(T);                              // elements per 16-byte chunk
  static constexpr int ROW = 32 * V;                                    // elements per warp row
  static constexpr int TILE = kScanWarps * kScanRowsPerWarp * ROW;     // 8192 (4 B) / 4096 (8 B)
  static constexpr int TILE_BYTES = TILE * (int)sizeof(T);              // 32 KB
  using Status = TileStatus<T>;
};

template <typename T>
size_t scan_num_tiles(uint64_t n) {
  return (size_t)((n + ScanCfg<T>::TILE - 1) / ScanCfg<T>::TILE);
}

template <typename T>
size_t scan_ws_bytes(uint64_t n) {
  return kHeaderBytes + ScanCfg<T>::Status::bytes(scan_num_tiles<T>(n));
}

template <typename Status>
__host__ __device__ inline Status scan_status_at(void *ws, size_t tiles) {
  return Status::at(reinterpret_cast<char *>(ws) + kHeaderBytes, tiles);
}

// Clears the status words of `tiles` tiles and resets the tile ticket.
template <typename Status>
__global__ void lookback_init_kernel(Status st, size_t tiles, WsHeader *hdr) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t padded = align_up(tiles, (size_t)kLbPerLane);  // whole look-back groups
  for (size_t t = i; t < padded; t += stride) st.clear(t);
  if (i == 0) hdr->tile_ticket = 0u;
}

// Where one tile lives.
template <typename T>
struct ScanTile {
  const T *in;     // the tile's first input element
  T *out;          // its first output element
  uint32_t count;  // elements in the tile
  bool first;      // first tile of its array: publishes its inclusive prefix at once
  bool tma;        // moved by TMA copies (in and out 16-byte aligned; in the
                   // blocked layout also inside whole rows of both row views)
  T init;          // its array's init
  uint32_t index;  // tile index within its array
};

// Tile source: one array.  For 8-byte elements (kSwz) tiles move by tiled
// tensor copies of 128-byte rows with the 128-byte swizzle, and each lane
// owns 16 consecutive elements (the "blocked" layout: one lane-local scan and
// one warp scan per 16 elements, where the row layout needs a warp scan for
// every 2), read and written conflict-free; tiles past `covered` (the ragged
// end) are read and written by the compute warps directly.  4-byte elements
// keep the row layout (rows of 32 lanes x 16 bytes) and untiled bulk copies.
template <typename T>
struct ScanOne {
  static constexpr bool kSwz = sizeof(T) == 8;
  CUtensorMap imap;  // input as rows of 128 bytes (kSwz)
  CUtensorMap omap;  // output as rows of 128 bytes (kSwz)
  const T *in;
  T *out;
  uint64_t n;
  T init;
  const T *init_ptr;  // init read from device memory instead (the _dinit entry points), else null
  int tma;            // in and out 16-byte aligned
  uint64_t covered;   // kSwz: leading elements inside whole rows of both views
  __device__ __forceinline__ ScanTile<T> tile(unsigned int t) const {
    const uint64_t base = (uint64_t)t * ScanCfg<T>::TILE;
    const uint64_t rem = n - base;
    const uint32_t cnt = (uint32_t)(rem < (uint64_t)ScanCfg<T>::TILE ? rem : (uint64_t)ScanCfg<T>::TILE);
    const bool t_tma = kSwz ? (base + cnt <= covered) : (tma != 0);
    // only the first tile uses init; a device-resident one was written before
    // this launch (stream order) and is read-only during it
    const T iv = (t == 0u && init_ptr != nullptr) ? __ldg(init_ptr) : init;
    return ScanTile<T>{in + base, out + base, cnt, t == 0u, t_tma, iv, t};
  }
  __device__ __forceinline__ const CUtensorMap *in_map() const { return &imap; }
  __device__ __forceinline__ const CUtensorMap *out_map() const { return &omap; }
};

// Tile source: a batch of independent arrays scanned by one launch.  Array
// i owns global tiles [start[i], start[i + 1]); its first tile publishes an
// inclusive prefix at once, so no look-back crosses into another array.  The
// descriptors travel in the kernel's parameters.
constexpr int kScanBatchMax = 256;
template <typename T>
struct ScanBatch {
  static constexpr bool kSwz = false;
  const T *in[kScanBatchMax];
  T *out[kScanBatchMax];
  uint64_t n[kScanBatchMax];
  T init[kScanBatchMax];
  uint32_t start[kScanBatchMax + 1];
  uint32_t count;
  __device__ __forceinline__ ScanTile<T> tile(unsigned int t) const {
    int lo = 0, hi = (int)count - 1;  // the last array whose first tile is <= t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (start[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    const uint32_t local = t - start[lo];
    const uint64_t base = (uint64_t)local * ScanCfg<T>::TILE;
    const uint64_t rem = n[lo] - base;
    const bool tma = ((reinterpret_cast<uintptr_t>(in[lo]) | reinterpret_cast<uintptr_t>(out[lo])) & 15) == 0;
    return ScanTile<T>{in[lo] + base, out[lo] + base,
                       (uint32_t)(rem < (uint64_t)ScanCfg<T>::TILE ? rem : (uint64_t)ScanCfg<T>::TILE),
                       local == 0u, tma, init[lo], local};
  }
  __device__ __forceinline__ const CUtensorMap *in_map() const { return nullptr; }
  __device__ __forceinline__ const CUtensorMap *out_map() const { return nullptr; }
};

// Copies a tile into shared memory `buf`: the 16-byte-aligned body with one
// TMA bulk copy completing on `bar` (returns whether one was issued), the
// ragged tail (fewer than V elements) with plain loads by the calling thread.
// Called by one thread, only for tiles whose pointers are 16-byte aligned.
template <typename T, typename Src>
__device__ __forceinline__ bool scan_issue_tile_load(const Src &src, const ScanTile<T> &tl, T *buf, uint64_t *bar,
                                                     uint64_t policy) {
  using C = ScanCfg<T>;
  if constexpr (Src::kSwz) {  // blocked layout: the tile's rows, swizzled (a TMA tile is whole rows)
    mbar_arrive_expect_tx(bar, (uint32_t)C::TILE_BYTES);
    tma_load_rows(buf, src.in_map(), tl.index * (uint32_t)(C::TILE_BYTES / 128), bar, policy);
    return true;
  }
  const uint32_t bulk = tl.count & ~(uint32_t)(C::V - 1);
  for (uint32_t i = bulk; i < tl.count; ++i) buf[i] = tl.in[i];
  if (bulk == 0) return false;
  mbar_arrive_expect_tx(bar, bulk * (uint32_t)sizeof(T));
  tma_load_1d_hint(buf, tl.in, bulk * (uint32_t)sizeof(T), bar, policy);
  return true;
}

// Blocked layout (8-byte elements): compute lane li = warp * 32 + lane owns
// elements [li * M, li * M + M) of its tile, M = 16 (one 128-byte row); in a
// swizzled buffer its 16-byte chunk c sits at swz128(li * 128 + 16 c).
// Loads a lane's elements (elements past the tile's end read as identity);
// tiles without a TMA copy are read from global memory directly.
template <typename T, typename Op>
__device__ __forceinline__ void scan_blk_load(const ScanTile<T> &tl, const T *buf, uint32_t li,
                                              T (&x)[ScanCfg<T>::TILE / (32 * kScanWarps)]) {
  constexpr int M = ScanCfg<T>::TILE / (32 * kScanWarps), VC = 16 / sizeof(T);
  const uint32_t e0 = li * M;
  if (tl.tma) {
    const unsigned char *b = reinterpret_cast<const unsigned char *>(buf);
#pragma unroll
    for (int c = 0; c < M / VC; ++c) {
      const uint4 q = *reinterpret_cast<const uint4 *>(b + swz128(e0 * (uint32_t)sizeof(T) + 16u * c));
      memcpy(&x[c * VC], &q, 16);
    }
    if (tl.count < (uint32_t)ScanCfg<T>::TILE) {
#pragma unroll
      for (int j = 0; j < M; ++j)
        if (e0 + j >= tl.count) x[j] = Op::identity();
    }
  } else {
#pragma unroll
    for (int j = 0; j < M; ++j) x[j] = (e0 + j < tl.count) ? tl.in[e0 + j] : Op::identity();
  }
}

// Persistent two-phase scan.  Warps 0-7 compute, warp 8 (lane 0) loads and
// stores, warp 9 looks back.  Each CTA loops over tiles taken from an atomic
// ticket (fetched one iteration ahead; the atomic's result is read only an
// iteration later, so its latency is hidden).  Tile t_i, ticketed for
// iteration i, lives in buffer i mod 3 and goes through:
//   iteration i-1  loader: TMA prefetch from HBM (L2 evict-last);
//   iteration i    compute: phase 1, the tile's reduction from shared
//                  memory; then compute thread 0 publishes its aggregate and
//                  queues it for the look-back warp; the loader re-reads
//                  t_{i-1}, whose phase 1 ended an iteration ago, from L2 into
//                  this buffer (its phase-1 data is no longer needed);
//   iteration i+1  compute: phase 2 of t_{i-1} from this buffer -- scan,
//                  add the prefix, write back; loader: TMA bulk store
//                  (evict-first), after which the buffer takes the prefetch
//                  of t_{i+2}.
// So every TMA load is issued about an iteration before it is needed, and a
// tile's data waits in L2, not shared memory, between its two phases.
//
// The three roles never share a barrier: they hand over through mbarriers.
// full[b]: the loader completes one phase per use of buffer b (a TMA copy,
// or a plain arrival when there is nothing to copy), after writing the
// buffer's ticket, so the compute warps learn the ticket by waiting on it;
// p1[b] / p2[b]: each compute warp arrives when it has finished reading
// (phase 1) or writing (phase 2) buffer b, which is when the loader may reuse
// it; qbar[e]: the look-back warp hands over queue entry e's exclusive
// prefix.  Consecutive phases of one barrier are three iterations apart and
// each waits on the previous one's data, so they cannot alias.  The compute
// warps meet only each other, once per iteration (the warp totals), in a
// barrier that also ORs their failure flags, so they all stop together.
// The look-back warp takes queued tiles in order, each once the next one is
// queued (its predecessors have then had an iteration to publish), so its L2
// round trips are off everyone's critical path.  Every look-back wait points
// at a lower tile whose ticket a running CTA already took and whose aggregate
// depends only on its load and on a look-back for a still lower tile, so the
// waits always end; every wait is still bounded by spin_limit_ns and gives up
// at once when anyone in the CTA has failed.
template <typename T, typename Op, typename Src>
__global__ void __launch_bounds__(kScanThreads, 2) scan_kernel(const __grid_constant__ Src src,
                                                               typename ScanCfg<T>::Status st, WsHeader *hdr,
                                                               unsigned long long spin_limit_ns,
                                                               long long skip_publish_tile, unsigned int num_tiles) {
  using C = ScanCfg<T>;
  constexpr int V = C::V, TILE = C::TILE, R = kScanRowsPerWarp, NB = kScanBufs, Q = kScanQueue;
  constexpr unsigned int NONE = 0xffffffffu;
  Op op;
  constexpr bool BLK = Src::kSwz;
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  // NB tile buffers from the first 1024-byte boundary (the swizzle's period)
  T *const buf0 = reinterpret_cast<T *>(smem_dyn + ((1024u - (smem_addr(smem_dyn) & 1023u)) & 1023u));
  __shared__ __align__(8) uint64_t s_full[NB];
  __shared__ __align__(8) uint64_t s_p1[NB];
  __shared__ __align__(8) uint64_t s_p2[NB];
  __shared__ __align__(8) uint64_t s_qbar[Q];
  __shared__ unsigned int s_ticket[NB];  // ticket of the tile prefetched into buffer b
  __shared__ T s_wtot[4][kScanWarps];    // per-warp totals of t_i, by iteration mod 4
  __shared__ T s_wexcl[4][kScanWarps];   // the warps before each warp, folded (thread 0)
  __shared__ unsigned int s_q_tile[Q];   // look-back queue: entry j = t_j
  __shared__ T s_q_agg[Q];
  __shared__ T s_q_prefix[Q];
  __shared__ unsigned int s_q_in;        // entries queued
  __shared__ int s_abort;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  auto abort_now = [&]() { *reinterpret_cast<volatile int *>(&s_abort) = 1; };
  auto aborted = [&]() -> bool { return *reinterpret_cast<volatile int *>(&s_abort) != 0; };
  auto buf = [&](int b) { return buf0 + b * TILE; };

  uint64_t keep = 0, stream = 0;
  uint32_t armpar = 0u, armany = 0u;  // loader: parity of the phases armed on s_full[b] / any armed
  unsigned int next_raw = NONE;  // loader: next ticket, not yet range-checked
  unsigned int t_first = NONE;   // loader: t_0
  if (tid == 32 * kScanWarps) {
    keep = l2_policy_evict_last();
    stream = l2_policy_evict_first();
    for (int b = 0; b < NB; ++b) {
      mbar_init(&s_full[b], 1);
      mbar_init(&s_p1[b], kScanWarps);
      mbar_init(&s_p2[b], kScanWarps);
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
      const ScanTile<T> tl = src.tile(t_first);
      if (tl.tma) tx = scan_issue_tile_load(src, tl, buf(0), &s_full[0], keep);
    }
    if (!tx) mbar_arrive(&s_full[0]);
    armpar |= 1u;
    // iteration 0's phase 2 reads buffer NB - 1, which no re-read filled:
    // give it an empty phase
    mbar_arrive(&s_full[NB - 1]);
    armpar |= 1u << (NB - 1);
    armany = armpar;
    if (t_first != NONE) next_raw = atomicAdd(&hdr->tile_ticket, 1u);
  }
  __syncthreads();

  if (warp == kScanWarps) {
    // ================= the loader (lane 0) =================
    if (lane != 0) return;
    uint32_t p1par = 0u, p2par = 0u;  // bit b: parity of the next phase of s_p1[b] / s_p2[b]
    bool issued_store = false;
    unsigned int t = t_first, p_tile = NONE, q_tile = NONE;
    for (int it = 0;; ++it) {
      const int bt = it % NB, bp = (it + NB - 1) % NB, bn = (it + 1) % NB;
      const unsigned int p = p_tile;
      // prefetch t_{i+1} into bn (stored last iteration), take the ticket after that
      const unsigned int tn = (t != NONE && next_raw < num_tiles) ? next_raw : NONE;
      s_ticket[bn] = tn;
      bool tx = false;
      if (tn != NONE) {
        const ScanTile<T> tl = src.tile(tn);
        if (tl.tma) {
          if (issued_store) tma_store_wait_read();
          tx = scan_issue_tile_load(src, tl, buf(bn), &s_full[bn], keep);
        }
      }
      if (!tx) mbar_arrive(&s_full[bn]);
      armpar ^= 1u << bn;
      armany |= 1u << bn;
      next_raw = (tn != NONE) ? atomicAdd(&hdr->tile_ticket, 1u) : NONE;
      // tiles are ticketed about in order, gridDim.x per iteration: ask L2
      // now for the one some CTA will load an iteration from now
      if (tn != NONE && tn + gridDim.x < num_tiles) {
        const ScanTile<T> f = src.tile(tn + gridDim.x);
        prefetch_l2_range(f.in, (uint64_t)f.count * sizeof(T));
      }
      // once the compute warps are done with buffer bt (phase 1 of t, or
      // just its empty phase), re-read t_{i-1} from L2 into it
      if (!mbar_wait_or_abort(&s_p1[bt], (p1par >> bt) & 1u, spin_limit_ns, &s_abort)) {
        record_error(hdr, BK_ERR_SPIN_TIMEOUT, t);
        abort_now();
        break;
      }
      p1par ^= 1u << bt;
      tx = false;
      if (q_tile != NONE) {
        const ScanTile<T> tl = src.tile(q_tile);
        if (tl.tma) tx = scan_issue_tile_load(src, tl, buf(bt), &s_full[bt], stream);
      }
      if (!tx) mbar_arrive(&s_full[bt]);
      armpar ^= 1u << bt;
      armany |= 1u << bt;
      // once the compute warps are done with buffer bp (phase 2 of p, or just
      // its empty phase), store p; the buffer then takes the next prefetch
      if (!mbar_wait_or_abort(&s_p2[bp], (p2par >> bp) & 1u, spin_limit_ns, &s_abort)) {
        record_error(hdr, BK_ERR_SPIN_TIMEOUT, p);
        abort_now();
        break;
      }
      p2par ^= 1u << bp;
      if (p != NONE) {
        const ScanTile<T> tl = src.tile(p);
        if (BLK && tl.tma) {  // whole rows: the tensor store undoes the swizzle
          tma_store_rows(src.out_map(), tl.index * (uint32_t)(C::TILE_BYTES / 128), buf(bp), stream);
          tma_store_commit();
          issued_store = true;
        } else if (tl.tma) {
          const T *bP = buf(bp);
          const uint32_t bulk = tl.count & ~(uint32_t)(V - 1);
          if (bulk > 0) {
            tma_store_1d_hint(tl.out, bP, bulk * (uint32_t)sizeof(T), stream);
            tma_store_commit();
            issued_store = true;
          }
          for (uint32_t i = bulk; i < tl.count; ++i) tl.out[i] = bP[i];
        }
      }
      p_tile = q_tile;
      q_tile = t;
      t = tn;
      if (t == NONE && p_tile == NONE && q_tile == NONE) break;  // tickets only grow: nothing left
    }
    // Drain: stores must finish reading shared memory and every load must
    // land before the CTA's shared memory goes away.  Phases of a barrier
    // complete in order, so waiting for the last one armed covers them all;
    // a phase that already completed returns at once.
    if (issued_store) tma_store_wait_all();
    for (int b = 0; b < NB; ++b)
      if ((armany >> b) & 1u) (void)mbar_wait(&s_full[b], ((armpar >> b) & 1u) ^ 1u, spin_limit_ns);
    return;
  }

  if (warp == kScanWarps + 1) {
    // ================= the look-back warp =================
    // Waits (bounded) until `count` entries are queued; false on an abort or
    // a timeout.
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
      if (q == NONE) break;  // tickets only grow: nothing after this
      // a real tile is always followed by another entry; taking the tile
      // once that entry is queued gives its predecessors an iteration to
      // publish their aggregates
      if (!wait_queued(j + 2u)) break;
      const T agg = s_q_agg[j % Q];
      const ScanTile<T> tl = src.tile(q);
      T excl = tl.init;
      bool ok = true;
      if (!tl.first) ok = lookback_exclusive<T>(st, q, op, excl, hdr, spin_limit_ns);
      if (lane == 0) {
        if (ok) {
          if (!tl.first && (long long)q != skip_publish_tile) st.publish(q, kStPrefix, op(excl, agg));
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
  uint32_t fpar = 0u;  // bit b: parity of the next phase of s_full[b]
  unsigned int p_tile = NONE, q_tile = NONE;  // t_{i-2}, t_{i-1}
  bool bad = false;                           // this thread saw a failure

  for (int it = 0;; ++it) {
    const int bt = it % NB, bp = (it + NB - 1) % NB;
    const unsigned int p = p_tile;

    // ---- phase 1 of t: wait for buffer bt, learn t
    unsigned int t = NONE;
    if (!mbar_wait_or_abort(&s_full[bt], (fpar >> bt) & 1u, spin_limit_ns, &s_abort)) bad = true;
    fpar ^= 1u << bt;
    bad = __any_sync(0xffffffffu, bad);  // warp-uniform, so the shuffles below never diverge
    if (!bad) t = s_ticket[bt];
    if (t != NONE) {
      const ScanTile<T> tl = src.tile(t);
      const uint32_t count = tl.count;
      const T *bT = buf(bt);
      T a = Op::identity();
      if constexpr (BLK) {
        constexpr int M = C::TILE / (32 * kScanWarps);
        T x[M];
        scan_blk_load<T, Op>(tl, bT, (uint32_t)(warp * 32 + lane), x);
#pragma unroll
        for (int j = 0; j < M; ++j) a = op(a, x[j]);
      } else if (tl.tma && count == (uint32_t)C::TILE) {
        // a full tile in shared memory: no element is past its end
#pragma unroll
        for (int k = 0; k < R; ++k) {
          const uint32_t elem = (uint32_t)(((warp * R + k) * 32 + lane) * V);
          T x[V];
          const uint4 c = reinterpret_cast<const uint4 *>(bT)[elem / V];
          memcpy(&x[0], &c, 16);
#pragma unroll
          for (int j = 0; j < V; ++j) a = op(a, x[j]);
        }
      } else {
#pragma unroll
        for (int k = 0; k < R; ++k) {
          const uint32_t elem = (uint32_t)(((warp * R + k) * 32 + lane) * V);
          T x[V];
          if (tl.tma) {
            const uint4 c = reinterpret_cast<const uint4 *>(bT)[elem / V];
            memcpy(&x[0], &c, 16);
          } else {
#pragma unroll
            for (int j = 0; j < V; ++j) x[j] = (elem + j < count) ? tl.in[elem + j] : Op::identity();
          }
#pragma unroll
          for (int j = 0; j < V; ++j)
            if (elem + j < count) a = op(a, x[j]);
        }
      }
      a = warp_reduce(a, op);
      if (lane == 0) s_wtot[it & 3][warp] = a;
    }
    // done with buffer bt (also when it held nothing); after a failure the
    // loader is told nothing more -- it gives up on the abort flag instead
    __syncwarp();
    if (!bad && lane == 0) mbar_arrive(&s_p1[bt]);
    if (named_barrier_or(1, 32 * kScanWarps, bad || aborted())) break;
    // no thread failed before this barrier, so t is the same everywhere

    // ---- thread 0: publish t's aggregate and queue t for the look-back
    if (tid == 0) {
      T agg = Op::identity();
      if (t != NONE) {
        agg = s_wtot[it & 3][0];
        s_wexcl[it & 3][0] = Op::identity();
#pragma unroll
        for (int i = 1; i < kScanWarps; ++i) {
          s_wexcl[it & 3][i] = agg;
          agg = op(agg, s_wtot[it & 3][i]);
        }
        if ((long long)t != skip_publish_tile) {
          const ScanTile<T> tl = src.tile(t);
          if (tl.first) st.publish(t, kStPrefix, op(tl.init, agg));
          else st.publish(t, kStAggregate, agg);
        }
      }
      s_q_tile[it % Q] = t;
      s_q_agg[it % Q] = agg;
      st_release_cta_u32(&s_q_in, (unsigned int)it + 1u);
    }

    // ---- phase 2 of p: buffer bp (re-read last iteration), prefix = queue entry it - 2
    if (!mbar_wait_or_abort(&s_full[bp], (fpar >> bp) & 1u, spin_limit_ns, &s_abort)) bad = true;
    fpar ^= 1u << bp;
    if (p != NONE && !bad) {
      const unsigned int e = (unsigned int)it - 2u;
      if (!mbar_wait_or_abort(&s_qbar[e % Q], (e / Q) & 1u, spin_limit_ns, &s_abort)) bad = true;
    }
    bad = __any_sync(0xffffffffu, bad);
    if (p != NONE && !bad) {
      const ScanTile<T> tl = src.tile(p);
      const uint32_t count = tl.count;
      T *const bP = buf(bp);
      const unsigned int e = (unsigned int)it - 2u;
      // everything before this warp's first element
      T before = warp == 0 ? s_q_prefix[e % Q] : op(s_q_prefix[e % Q], s_wexcl[(it + 2) & 3][warp]);
      if constexpr (BLK) {
        constexpr int M = C::TILE / (32 * kScanWarps), VC = 16 / sizeof(T);
        const uint32_t li = (uint32_t)(warp * 32 + lane), e0 = li * M;
        T y[M];
        scan_blk_load<T, Op>(tl, bP, li, y);
#pragma unroll
        for (int j = 1; j < M; ++j) y[j] = op(y[j - 1], y[j]);
        const T incl = warp_inclusive_scan(y[M - 1], op, lane);
        const T ex = shfl_up(incl, 1);
        const T b = lane != 0 ? op(before, ex) : before;
#pragma unroll
        for (int j = 0; j < M; ++j) y[j] = op(b, y[j]);
        if (tl.tma) {
          unsigned char *bb = reinterpret_cast<unsigned char *>(bP);
#pragma unroll
          for (int c = 0; c < M / VC; ++c) {
            uint4 q;
            memcpy(&q, &y[c * VC], 16);
            *reinterpret_cast<uint4 *>(bb + swz128(e0 * (uint32_t)sizeof(T) + 16u * c)) = q;
          }
          fence_proxy_async_smem();  // the tensor store reads what this thread wrote
        } else {
#pragma unroll
          for (int j = 0; j < M; ++j)
            if (e0 + j < count) tl.out[e0 + j] = y[j];
        }
      } else {
        T y[R][V], incl[R];
  #pragma unroll
        for (int k = 0; k < R; ++k) {
          const uint32_t elem = (uint32_t)(((warp * R + k) * 32 + lane) * V);
          if (tl.tma) {
            const uint4 c = reinterpret_cast<const uint4 *>(bP)[elem / V];
            memcpy(&y[k][0], &c, 16);
          } else {
  #pragma unroll
            for (int j = 0; j < V; ++j) y[k][j] = (elem + j < count) ? tl.in[elem + j] : Op::identity();
          }
        }
  #pragma unroll
        for (int k = 0; k < R; ++k) {
          const uint32_t elem = (uint32_t)(((warp * R + k) * 32 + lane) * V);
          if (elem + V > count) {
  #pragma unroll
            for (int j = 0; j < V; ++j)
              if (elem + j >= count) y[k][j] = Op::identity();
          }
  #pragma unroll
          for (int j = 1; j < V; ++j) y[k][j] = op(y[k][j - 1], y[k][j]);
          incl[k] = y[k][V - 1];
        }
        // the rows' warp scans, interleaved so their shuffle chains overlap
  #pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
  #pragma unroll
          for (int k = 0; k < R; ++k) {
            const T o = shfl_up(incl[k], d);
            if (lane >= d) incl[k] = op(o, incl[k]);
          }
        }
  #pragma unroll
        for (int k = 0; k < R; ++k) {
          const T ex = shfl_up(incl[k], 1);
          const T tot = shfl_idx_any(incl[k], 31);
          const T b = lane != 0 ? op(before, ex) : before;
  #pragma unroll
          for (int j = 0; j < V; ++j) y[k][j] = op(b, y[k][j]);
          before = op(before, tot);
          const uint32_t elem = (uint32_t)(((warp * R + k) * 32 + lane) * V);
          if (tl.tma) {
            uint4 c;
            memcpy(&c, &y[k][0], 16);
            reinterpret_cast<uint4 *>(bP)[elem / V] = c;
          } else {
  #pragma unroll
            for (int j = 0; j < V; ++j)
              if (elem + j < count) tl.out[elem + j] = y[k][j];
          }
        }
        if (tl.tma) fence_proxy_async_smem();
      }
    }
    __syncwarp();
    if (!bad && lane == 0) mbar_arrive(&s_p2[bp]);

    p_tile = q_tile;
    q_tile = t;
    if (t == NONE && p_tile == NONE && q_tile == NONE) break;  // tickets only grow: nothing left
  }
}

// Clears the status words, then runs the persistent scan over `tiles` tiles
// of `src` (one array or a batch).
template <typename T, typename Op, typename Src>
int scan_run(const Src &src, size_t tiles, void *d_ws, size_t ws_bytes, cudaStream_t stream) {
  using C = ScanCfg<T>;
  host::DeviceInfo di;
  int st = host::device_info(&di);
  if (st != BK_OK) return st;
  if (tiles >= 0x7fffffffull) return BK_ERR_TOO_LARGE;
  st = host::check_ws(d_ws, ws_bytes, kHeaderBytes + C::Status::bytes(tiles));
  if (st != BK_OK) return st;
  WsHeader *hdr = reinterpret_cast<WsHeader *>(d_ws);
  auto status = scan_status_at<typename C::Status>(d_ws, tiles);
  const unsigned init_grid = (unsigned)std::min<size_t>((tiles + 255) / 256, (size_t)di.sm_count * 8);
  lookback_init_kernel<<<init_grid, 256, 0, stream>>>(status, tiles, hdr);
  st = host::launch_status();
  if (st != BK_OK) return st;
  const host::DebugFault dbg = host::debug_fault();
  const unsigned long long limit = dbg.spin_limit_ns ? dbg.spin_limit_ns : host::kDefaultSpinLimitNs;
  const size_t smem = (size_t)kScanBufs * C::TILE_BYTES + 1024;  // + room to align the buffers to 1024 bytes
  struct Site {};
  host::KernelSetup ks;
  if ((st = host::kernel_setup<Site>(scan_kernel<T, Op, Src>, kScanThreads, smem, &ks)) != BK_OK) return st;
  const tune::Knobs kn = tune::knobs_for(tune::kScan, (int)sizeof(T), (uint64_t)tiles * C::TILE);
  const unsigned grid =
      (unsigned)std::min<size_t>(tiles, (size_t)di.sm_count * (size_t)std::min(std::max(kn.ctas_per_sm, 1), 2));
  scan_kernel<T, Op, Src><<<grid, kScanThreads, smem, stream>>>(src, status, hdr, limit, dbg.skip_publish_tile,
                                                                (unsigned)tiles);
  return host::launch_status();
}

// init_ptr: when not null, init is read from device memory at run time (so a
// scan can continue from a value still on the device: the last output of the
// previous chunk of a stream, say) and `init` is ignored.
template <typename T, typename Op>
int scan_launch(const T *d_in, uint64_t n, T init, T *d_out, void *d_ws, size_t ws_bytes, cudaStream_t stream,
                const T *init_ptr = nullptr) {
  if (n == 0) {
    host::DeviceInfo di;
    return host::device_info(&di);
  }
  if (d_in == nullptr || d_out == nullptr) return BK_ERR_INVALID_ARGUMENT;
  if (!host::aligned_to<T>(d_in) || !host::aligned_to<T>(d_out)) return BK_ERR_MISALIGNED;
  const int tma = ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) & 15) == 0;
  ScanOne<T> src;
  memset(&src, 0, sizeof(src));
  src.in = d_in;
  src.out = d_out;
  src.n = n;
  src.init = init;
  src.init_ptr = init_ptr;
  if (init_ptr != nullptr && !host::aligned_to<T>(init_ptr)) return BK_ERR_MISALIGNED;
  src.tma = tma;
  if constexpr (ScanOne<T>::kSwz) {
    // row views of the input and output: the tiles inside whole 128-byte rows
    // of both move by tensor copies, the ragged end by plain loads and stores
    constexpr uint32_t box_rows = (uint32_t)(ScanCfg<T>::TILE_BYTES / 128);
    const uint64_t rows = n * sizeof(T) / 128;
    if (tma && rows > 0 && host::encode_rows_128b(&src.imap, d_in, rows, box_rows) == BK_OK &&
        host::encode_rows_128b(&src.omap, d_out, rows, box_rows) == BK_OK)
      src.covered = rows * (128 / sizeof(T));
  }
  return scan_run<T, Op>(src, scan_num_tiles<T>(n), d_ws, ws_bytes, stream);
}

// A batch item as the C-ABI passes it (bk_scan_item_<type>).
template <typename T>
struct ScanItem {
  const T *d_in;
  T *d_out;
  uint64_t n;
  T init;
};

template <typename T>
size_t scan_batch_tiles(const uint64_t *sizes, uint32_t count) {
  size_t tiles = 0;
  for (uint32_t i = 0; i < count; ++i) tiles += scan_num_tiles<T>(sizes[i]);
  return tiles;
}

template <typename T, typename Op>
int scan_batch_launch(const ScanItem<T> *items, uint32_t count, void *d_ws, size_t ws_bytes, cudaStream_t stream) {
  if (count > 0 && items == nullptr) return BK_ERR_INVALID_ARGUMENT;
  if (count > (uint32_t)kScanBatchMax) return BK_ERR_TOO_LARGE;
  ScanBatch<T> b;
  b.count = 0;
  size_t tiles = 0;
  for (uint32_t i = 0; i < count; ++i) {
    const ScanItem<T> &it = items[i];
    if (it.n == 0) continue;  // nothing to do; takes no tile
    if (it.d_in == nullptr || it.d_out == nullptr) return BK_ERR_INVALID_ARGUMENT;
    if (!host::aligned_to<T>(it.d_in) || !host::aligned_to<T>(it.d_out)) return BK_ERR_MISALIGNED;
    const uint32_t k = b.count++;
    b.in[k] = it.d_in;
    b.out[k] = it.d_out;
    b.n[k] = it.n;
    b.init[k] = it.init;
    b.start[k] = (uint32_t)tiles;
    tiles += scan_num_tiles<T>(it.n);
    if (tiles >= 0x7fffffffull) return BK_ERR_TOO_LARGE;
  }
  b.start[b.count] = (uint32_t)tiles;
  if (b.count == 0) {
    host::DeviceInfo di;
    return host::device_info(&di);
  }
  return scan_run<T, Op>(b, tiles, d_ws, ws_bytes, stream);
}

size_t scan_batch_workspace_bytes(int dtype, const uint64_t *sizes, uint32_t count) {
  if (count > 0 && sizes == nullptr) return 0;
  switch (dtype) {
    case BK_DTYPE_I32: case BK_DTYPE_U32: case BK_DTYPE_F32:
      return kHeaderBytes + ScanCfg<float>::Status::bytes(scan_batch_tiles<float>(sizes, count));
    case BK_DTYPE_I64: case BK_DTYPE_U64: case BK_DTYPE_F64:
      return kHeaderBytes + ScanCfg<double>::Status::bytes(scan_batch_tiles<double>(sizes, count));
    default: return 0;
  }
}

size_t scan_workspace_bytes(int dtype, uint64_t n) {
  switch (dtype) {
    case BK_DTYPE_I32: case BK_DTYPE_U32: case BK_DTYPE_F32: return scan_ws_bytes<float>(n);
    case BK_DTYPE_I64: case BK_DTYPE_U64: case BK_DTYPE_F64: return scan_ws_bytes<double>(n);
    default: return 0;
  }
}

}  // namespace bk

#define BK_DEFINE_SCAN(OPNAME, OPT, TN, T)                                                                   \
  extern "C" int bk_inclusive_scan_##OPNAME##_##TN(const T *d_in, uint64_t n, T init, T *d_out, void *d_ws, \
                                                   size_t ws_bytes, bk_stream_t stream) {                   \
    return bk::scan_launch<T, bk::OPT<T>>(d_in, n, init, d_out, d_ws, ws_bytes, (cudaStream_t)stream);      \
  }                                                                                                          \
  extern "C" int bk_inclusive_scan_##OPNAME##_##TN##_dinit(const T *d_in, uint64_t n, const T *d_init,       \
                                                           T *d_out, void *d_ws, size_t ws_bytes,            \
                                                           bk_stream_t stream) {                             \
    if (d_init == nullptr) return BK_ERR_INVALID_ARGUMENT;                                                   \
    return bk::scan_launch<T, bk::OPT<T>>(d_in, n, bk::OPT<T>::identity(), d_out, d_ws, ws_bytes,            \
                                          (cudaStream_t)stream, d_init);                                     \
  }

#define BK_DEFINE_SCAN_ALL_T(OPNAME, OPT)      \
  BK_DEFINE_SCAN(OPNAME, OPT, i32, int32_t)    \
  BK_DEFINE_SCAN(OPNAME, OPT, u32, uint32_t)   \
  BK_DEFINE_SCAN(OPNAME, OPT, i64, int64_t)    \
  BK_DEFINE_SCAN(OPNAME, OPT, u64, uint64_t)   \
  BK_DEFINE_SCAN(OPNAME, OPT, f32, float)      \
  BK_DEFINE_SCAN(OPNAME, OPT, f64, double)

BK_DEFINE_SCAN_ALL_T(sum, OpSum)

#define BK_DEFINE_SCAN_BATCH(TN, T)                                                                            \
  static_assert(sizeof(bk_scan_item_##TN) == sizeof(bk::ScanItem<T>), "bk_scan_item layout");              \
  extern "C" int bk_inclusive_scan_sum_##TN##_batch(const bk_scan_item_##TN *items, uint32_t count,          \
                                                    void *d_ws, size_t ws_bytes, bk_stream_t stream) {       \
    return bk::scan_batch_launch<T, bk::OpSum<T>>(reinterpret_cast<const bk::ScanItem<T> *>(items), count,   \
                                                  d_ws, ws_bytes, (cudaStream_t)stream);                    \
  }

BK_DEFINE_SCAN_BATCH(i32, int32_t)
BK_DEFINE_SCAN_BATCH(u32, uint32_t)
BK_DEFINE_SCAN_BATCH(i64, int64_t)
BK_DEFINE_SCAN_BATCH(u64, uint64_t)
BK_DEFINE_SCAN_BATCH(f32, float)
BK_DEFINE_SCAN_BATCH(f64, double)
BK_DEFINE_SCAN_ALL_T(min, OpMin)
BK_DEFINE_SCAN_ALL_T(max, OpMax)
