// scan.cu -- single-pass inclusive scan with decoupled look-back, sm_100a.
//
// Replaces the reference's three-pass ::inclusive_scan (scan.cu:87-148):
// upsweep accumulate_tiles (:57-84) -> spine exclusive_scan_n (:24-31) ->
// downsweep inclusive_downsweep (:34-54), each calling the group scan of
// bulk/algorithm/scan.hpp:222-384.  That design moves 3*N*s bytes; this one
// moves the minimum 2*N*s (read once, write once).
//
// Per tile (32 KB): an atomic ticket names the tile (launch order, so every
// predecessor is already running); one TMA bulk copy brings the tile into
// shared memory; each warp scans its rows of 16-byte chunks with shuffles;
// the tile publishes its aggregate, warp 0 looks back over its predecessors
// for the exclusive prefix (bk_lookback.cuh) and publishes the inclusive
// prefix; the results leave with one TMA bulk store.  A tiny init kernel
// clears the tile status words before each scan.
//
// Semantics follow scan.cu:166-169 and bulk/algorithm/scan.hpp:455-486:
// out[i] = init (+) in[0] (+) ... (+) in[i].
#include "bk_common.cuh"
#include "bk_lookback.cuh"
#include "bk_tma.cuh"

namespace bk {

constexpr int kScanWarps = 8;                       // compute warps
constexpr int kScanThreads = 32 * (kScanWarps + 1);  // + one control warp
constexpr int kScanRowsPerWarp = 8;

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

// Copies tile `tile` of `src` into shared memory `buf`: the 16-byte-aligned
// body with one TMA bulk copy completing on `bar` (returns whether one was
// issued), the ragged tail (fewer than V elements) with plain loads by the
// calling thread.  Called by one thread.
template <typename T>
__device__ __forceinline__ bool scan_issue_tile_load(const T *src, uint64_t n, unsigned int tile, T *buf,
                                                     uint64_t *bar, uint64_t policy) {
  using C = ScanCfg<T>;
  const uint64_t base = (uint64_t)tile * C::TILE;
  const uint32_t count = (uint32_t)((n - base) < (uint64_t)C::TILE ? (n - base) : (uint64_t)C::TILE);
  const uint32_t bulk = count & ~(uint32_t)(C::V - 1);
  for (uint32_t i = bulk; i < count; ++i) buf[i] = src[base + i];
  if (bulk == 0) return false;
  mbar_arrive_expect_tx(bar, bulk * (uint32_t)sizeof(T));
  tma_load_1d_hint(buf, src + base, bulk * (uint32_t)sizeof(T), bar, policy);
  return true;
}

// All threads: plain coalesced copy of a tile into shared memory (used when
// the pointers are not 16-byte aligned).
template <typename T>
__device__ __forceinline__ void scan_sync_tile_load(const T *src, uint64_t n, unsigned int tile, T *buf) {
  using C = ScanCfg<T>;
  const uint64_t base = (uint64_t)tile * C::TILE;
  const uint32_t count = (uint32_t)((n - base) < (uint64_t)C::TILE ? (n - base) : (uint64_t)C::TILE);
  for (uint32_t i = threadIdx.x; i < count; i += kScanWarps * 32) buf[i] = src[base + i];
}

template <typename T>
__device__ __forceinline__ uint32_t scan_tile_count(uint64_t n, unsigned int tile) {
  const uint64_t base = (uint64_t)tile * ScanCfg<T>::TILE;
  return (uint32_t)((n - base) < (uint64_t)ScanCfg<T>::TILE ? (n - base) : (uint64_t)ScanCfg<T>::TILE);
}

// Persistent two-phase scan with a control warp.  Each CTA loops over tiles
// taken from an atomic ticket (the next ticket is always fetched one iteration
// ahead, so its latency is hidden).  Iteration i of a CTA:
//   * control warp: starts the TMA load of the next phase-1 tile (kept in L2
//     with an evict-last hint) and the re-read of the previous tile p from L2
//     (evict-first);
//   * compute warps: phase 1 of the current tile t -- reduce it (pass A);
//   * control warp: publishes t's aggregate (tile 0: its inclusive prefix),
//     then looks back for p's exclusive prefix -- every predecessor's
//     aggregate is an iteration old by now, so nothing waits on a slow load --
//     and publishes p's inclusive prefix;
//   * compute warps, meanwhile: scan p's rows in registers (pass B); once the
//     prefix is known they add it and write the tile back to shared memory;
//   * control warp: one TMA bulk store writes the tile out (evict-first).
// A tile waiting for its prefix holds no shared memory: its data waits in L2.
// Every wait points at a lower tile whose ticket a running CTA already took,
// so the waits always end; each is still bounded by spin_limit_ns.
template <typename T, typename Op>
__global__ void __launch_bounds__(kScanThreads, 2) scan_kernel(const T *in, T *out, uint64_t n, T init,
                                                               typename ScanCfg<T>::Status st, WsHeader *hdr,
                                                               unsigned long long spin_limit_ns,
                                                               long long skip_publish_tile, int tma_ok,
                                                               unsigned int num_tiles) {
  using C = ScanCfg<T>;
  constexpr int V = C::V, TILE = C::TILE, R = kScanRowsPerWarp;
  constexpr unsigned int NONE = 0xffffffffu;
  Op op;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T *const bufA0 = reinterpret_cast<T *>(smem_raw);
  T *const bufA1 = bufA0 + TILE;
  T *const bufB = bufA1 + TILE;
  __shared__ __align__(8) uint64_t s_bar[3];  // 0, 1: phase-1 slots; 2: phase-2 buffer
  __shared__ unsigned int s_ticket[2];
  __shared__ int s_has_tma[3];
  __shared__ T s_wtot[2][kScanWarps];
  __shared__ T s_prefix;
  __shared__ int s_abort;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool control = (warp == kScanWarps);
  const bool leader = control && lane == 0;

  unsigned int next_ticket = NONE;  // leader only: ticket for the next phase-1 load
  bool issued_store = false;        // leader only
  uint64_t keep = 0, stream = 0;
  if (leader) {
    keep = l2_policy_evict_last();
    stream = l2_policy_evict_first();
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    mbar_init(&s_bar[2], 1);
    fence_proxy_async_smem();
    s_abort = 0;
    s_has_tma[0] = s_has_tma[1] = s_has_tma[2] = 0;
    const unsigned int t0 = atomicAdd(&hdr->tile_ticket, 1u);
    s_ticket[0] = t0 < num_tiles ? t0 : NONE;
    if (t0 < num_tiles) {
      if (tma_ok) s_has_tma[0] = scan_issue_tile_load(in, n, t0, bufA0, &s_bar[0], keep);
      const unsigned int t1 = atomicAdd(&hdr->tile_ticket, 1u);
      next_ticket = t1 < num_tiles ? t1 : NONE;
    }
  }
  __syncthreads();

  uint32_t parity[3] = {0u, 0u, 0u};
  uint32_t inflight = s_has_tma[0] ? 1u : 0u;  // bit b: a TMA load on s_bar[b] not yet waited for
  unsigned int pending = NONE;                 // tile whose phase 2 is due this iteration
  T pending_agg = Op::identity();

  for (int it = 0;; ++it) {
    const int slot = it & 1;
    const unsigned int t = s_ticket[slot];
    T *const bA = slot ? bufA1 : bufA0;
    T *const bA_next = slot ? bufA0 : bufA1;

    // ---- control: start the loads (phase-2 re-read first), fetch a ticket
    if (leader) {
      s_has_tma[2] = 0;
      if (pending != NONE && tma_ok) {
        if (issued_store) tma_store_wait_read();  // bufB free again
        s_has_tma[2] = scan_issue_tile_load(in, n, pending, bufB, &s_bar[2], stream);
      }
      const unsigned int tn = (t != NONE) ? next_ticket : NONE;
      s_ticket[slot ^ 1] = tn;
      s_has_tma[slot ^ 1] = 0;
      if (tn != NONE && tma_ok) s_has_tma[slot ^ 1] = scan_issue_tile_load(in, n, tn, bA_next, &s_bar[slot ^ 1], keep);
      next_ticket = NONE;
      if (tn != NONE) {
        const unsigned int x = atomicAdd(&hdr->tile_ticket, 1u);  // used next iteration
        next_ticket = x < num_tiles ? x : NONE;
      }
    }
    if (!tma_ok && !control) {
      if (t != NONE) scan_sync_tile_load(in, n, t, bA);
      if (pending != NONE) scan_sync_tile_load(in, n, pending, bufB);
    }
    __syncthreads();
    if (s_has_tma[slot ^ 1]) inflight |= 1u << (slot ^ 1);
    if (s_has_tma[2]) inflight |= 4u;

    // ---- compute: phase 1 of t (pass A)
    if (t != NONE) {
      if (inflight & (1u << slot)) {
        if (!control && !mbar_wait(&s_bar[slot], parity[slot], spin_limit_ns)) {
          record_error(hdr, BK_ERR_SPIN_TIMEOUT, t);
          s_abort = 1;
        }
        parity[slot] ^= 1u;
        inflight &= ~(1u << slot);
      }
      if (!control) {
        const uint32_t count = scan_tile_count<T>(n, t);
        T a = Op::identity();
#pragma unroll
        for (int k = 0; k < R; ++k) {
          const uint32_t chunk = (uint32_t)((warp * R + k) * 32 + lane);
          T x[V];
          uint4 c = reinterpret_cast<const uint4 *>(bA)[chunk];
          memcpy(&x[0], &c, 16);
#pragma unroll
          for (int j = 0; j < V; ++j)
            if (chunk * V + j < count) a = op(a, x[j]);
        }
        a = warp_reduce(a, op);
        if (lane == 0) s_wtot[slot][warp] = a;
      }
    }
    __syncthreads();
    T agg_t = Op::identity();
    if (t != NONE) {
      agg_t = s_wtot[slot][0];
#pragma unroll
      for (int i = 1; i < kScanWarps; ++i) agg_t = op(agg_t, s_wtot[slot][i]);
    }

    T y[R][V];
    if (control) {
      // ---- publish t's aggregate, look back for p
      if (leader && t != NONE && !s_abort && (long long)t != skip_publish_tile) {
        if (t == 0) st.publish(0u, kStPrefix, op(init, agg_t));
        else st.publish(t, kStAggregate, agg_t);
      }
      if (pending != NONE) {
        const unsigned int p = pending;
        T excl = init;
        bool ok = true;
        if (p != 0) ok = lookback_exclusive<T>(st, p, op, excl, hdr, spin_limit_ns);
        if (leader) {
          if (ok) {
            if (p != 0 && (long long)p != skip_publish_tile) st.publish(p, kStPrefix, op(excl, pending_agg));
            s_prefix = excl;
          } else {
            s_abort = 1;
          }
        }
      }
      if (pending != NONE && (inflight & 4u)) {
        parity[2] ^= 1u;
        inflight &= ~4u;
      }
    } else if (pending != NONE) {
      // ---- pass B: p's rows in registers, offset by the earlier warps' totals
      const uint32_t count = scan_tile_count<T>(n, pending);
      if (inflight & 4u) {
        if (!mbar_wait(&s_bar[2], parity[2], spin_limit_ns)) {
          record_error(hdr, BK_ERR_SPIN_TIMEOUT, pending);
          s_abort = 1;
        }
        parity[2] ^= 1u;
        inflight &= ~4u;
      }
      T carry = Op::identity();
      bool have = false;
      for (int i = 0; i < warp; ++i) {
        carry = have ? op(carry, s_wtot[slot ^ 1][i]) : s_wtot[slot ^ 1][i];
        have = true;
      }
#pragma unroll
      for (int k = 0; k < R; ++k) {
        const uint32_t chunk = (uint32_t)((warp * R + k) * 32 + lane);
        uint4 c = reinterpret_cast<const uint4 *>(bufB)[chunk];
        memcpy(&y[k][0], &c, 16);
        if (chunk * V + V > count) {
#pragma unroll
          for (int j = 0; j < V; ++j)
            if (chunk * V + j >= count) y[k][j] = Op::identity();
        }
#pragma unroll
        for (int j = 1; j < V; ++j) y[k][j] = op(y[k][j - 1], y[k][j]);
        const T incl = warp_inclusive_scan(y[k][V - 1], op, lane);
        const T excl = shfl_up(incl, 1);
        const T row_total = shfl_idx_any(incl, 31);
        if (lane == 0) {
          if (have) {
#pragma unroll
            for (int j = 0; j < V; ++j) y[k][j] = op(carry, y[k][j]);
          }
        } else {
          const T pre = have ? op(carry, excl) : excl;
#pragma unroll
          for (int j = 0; j < V; ++j) y[k][j] = op(pre, y[k][j]);
        }
        carry = have ? op(carry, row_total) : row_total;
        have = true;
      }
    }
    __syncthreads();
    if (s_abort) break;

    if (pending != NONE) {
      const uint32_t count = scan_tile_count<T>(n, pending);
      const uint64_t base = (uint64_t)pending * TILE;
      if (!control) {
        // ---- add the tile's exclusive prefix, back to shared memory
        const T prefix = s_prefix;
#pragma unroll
        for (int k = 0; k < R; ++k) {
          const uint32_t chunk = (uint32_t)((warp * R + k) * 32 + lane);
#pragma unroll
          for (int j = 0; j < V; ++j) y[k][j] = op(prefix, y[k][j]);
          uint4 c;
          memcpy(&c, &y[k][0], 16);
          reinterpret_cast<uint4 *>(bufB)[chunk] = c;
        }
        if (tma_ok) fence_proxy_async_smem();
      }
      __syncthreads();
      if (tma_ok) {
        if (leader) {
          const uint32_t bulk = count & ~(uint32_t)(V - 1);
          if (bulk > 0) {
            tma_store_1d_hint(out + base, bufB, bulk * (uint32_t)sizeof(T), stream);
            tma_store_commit();
            issued_store = true;
          }
          for (uint32_t i = bulk; i < count; ++i) out[base + i] = bufB[i];
        }
      } else if (!control) {
        for (uint32_t i = tid; i < count; i += kScanWarps * 32) out[base + i] = bufB[i];
      }
    }

    if (t == NONE) break;  // nothing left: the pending tile was the last
    pending = t;
    pending_agg = agg_t;
    __syncthreads();  // the non-TMA path's plain stores read bufB
  }

  // Drain: every bulk store must finish reading shared memory, and on an
  // abort every prefetch must land, before the CTA's shared memory goes away.
  if (leader) {
    if (issued_store) tma_store_wait_all();
    for (int b = 0; b < 3; ++b)
      if (inflight & (1u << b)) (void)mbar_wait(&s_bar[b], parity[b], spin_limit_ns);
  }
}

template <typename T, typename Op>
int scan_launch(const T *d_in, uint64_t n, T init, T *d_out, void *d_ws, size_t ws_bytes, cudaStream_t stream) {
  using C = ScanCfg<T>;
  host::DeviceInfo di;
  int st = host::device_info(&di);
  if (st != BK_OK) return st;
  if (n == 0) return BK_OK;
  if (d_in == nullptr || d_out == nullptr) return BK_ERR_INVALID_ARGUMENT;
  if (!host::aligned_to<T>(d_in) || !host::aligned_to<T>(d_out)) return BK_ERR_MISALIGNED;
  const size_t tiles = scan_num_tiles<T>(n);
  if (tiles >= 0x7fffffffull) return BK_ERR_TOO_LARGE;
  st = host::check_ws(d_ws, ws_bytes, scan_ws_bytes<T>(n));
  if (st != BK_OK) return st;

  WsHeader *hdr = reinterpret_cast<WsHeader *>(d_ws);
  auto status = scan_status_at<typename C::Status>(d_ws, tiles);
  const unsigned init_grid = (unsigned)std::min<size_t>((tiles + 255) / 256, (size_t)di.sm_count * 8);
  lookback_init_kernel<<<init_grid, 256, 0, stream>>>(status, tiles, hdr);
  st = host::launch_status();
  if (st != BK_OK) return st;

  const host::DebugFault dbg = host::debug_fault();
  const unsigned long long limit = dbg.spin_limit_ns ? dbg.spin_limit_ns : host::kDefaultSpinLimitNs;
  const int tma_ok = ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) & 15) == 0;
  const size_t smem = 3 * (size_t)C::TILE_BYTES;
  static thread_local bool attr_set = false;  // per host thread; cheap and idempotent
  if (!attr_set) {
    if ((st = host::set_smem_attrs(scan_kernel<T, Op>, smem)) != BK_OK) return st;
    attr_set = true;
  }
  const unsigned grid = (unsigned)std::min<size_t>(tiles, (size_t)di.sm_count * 2);
  scan_kernel<T, Op><<<grid, kScanThreads, smem, stream>>>(d_in, d_out, n, init, status, hdr, limit,
                                                           dbg.skip_publish_tile, tma_ok, (unsigned)tiles);
  return host::launch_status();
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
  }

#define BK_DEFINE_SCAN_ALL_T(OPNAME, OPT)      \
  BK_DEFINE_SCAN(OPNAME, OPT, i32, int32_t)    \
  BK_DEFINE_SCAN(OPNAME, OPT, u32, uint32_t)   \
  BK_DEFINE_SCAN(OPNAME, OPT, i64, int64_t)    \
  BK_DEFINE_SCAN(OPNAME, OPT, u64, uint64_t)   \
  BK_DEFINE_SCAN(OPNAME, OPT, f32, float)      \
  BK_DEFINE_SCAN(OPNAME, OPT, f64, double)

BK_DEFINE_SCAN_ALL_T(sum, OpSum)
BK_DEFINE_SCAN_ALL_T(min, OpMin)
BK_DEFINE_SCAN_ALL_T(max, OpMax)
