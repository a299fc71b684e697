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
// is the scan's (scan.cu): persistent CTAs with a control warp, TMA bulk tile
// loads (keys and values) plus a one-key halo on each side, phase 1 publishes
// the tile aggregate, phase 2 looks back and emits the tile's runs.
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

constexpr int kRbkWarps = 8;
constexpr int kRbkThreads = 32 * (kRbkWarps + 1);  // + control warp

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
template <typename K, typename V>
size_t rbk_ws_bytes(uint64_t n) {
  return kHeaderBytes + RbkCfg<K, V>::Status::bytes(rbk_num_tiles<K, V>(n));
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

// Element index of the lane's first element: e0 = (warp * 32 + lane) * M.
// Neighbouring keys come from the adjacent lanes by shuffles; lane 0 / lane
// 31 read the key before / after the warp's range from shared memory, or the
// halo at the tile's edges (hb[0][KC-1] precedes the tile, hb[1][0] follows
// it).  first_tile: the tile starts the input; last_tile: it ends it.
template <typename K, typename V>
__device__ __forceinline__ void rbk_read_lane(const unsigned char *buf, const K (*hb)[16 / sizeof(K)], uint32_t count,
                                              bool first_tile, bool last_tile, int warp, int lane,
                                              LaneRun<K, V, RbkCfg<K, V>::M> &lr) {
  using C = RbkCfg<K, V>;
  constexpr int M = C::M;
  constexpr int KC = 16 / sizeof(K);
  const K *sk = reinterpret_cast<const K *>(buf);
  const uint32_t e0 = (uint32_t)(warp * 32 + lane) * M;
  load_lane_rotated<M * sizeof(K)>(lr.key, buf, e0 * (uint32_t)sizeof(K), lane);
  load_lane_rotated<M * sizeof(V)>(lr.val, buf + C::KEY_BYTES, e0 * (uint32_t)sizeof(V), lane);
  const int nvalid = (int)min(max((int)count - (int)e0, 0), M);
  lr.nvalid = nvalid;
#pragma unroll
  for (int j = 0; j < M; ++j)
    if (j >= nvalid) {
      lr.key[j] = K();
      lr.val[j] = V(0);
    }
  K prev = shfl_up(lr.key[M - 1], 1);
  K next = shfl_down_any(lr.key[0], 1);
  if (lane == 0) prev = e0 == 0 ? hb[0][KC - 1] : sk[e0 - 1];
  if (lane == 31) next = e0 + M < count ? sk[e0 + M] : hb[1][0];
  uint32_t head = 0, tail = 0;
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const K pk = j == 0 ? prev : lr.key[j - 1];
    const bool h = (j < nvalid) && !(lr.key[j] == pk);
    head |= (uint32_t)h << j;
    // successor inside the lane, in the next lane / warp, or after the tile
    const bool last_of_tile = (e0 + j + 1 == count);
    const K nk = j + 1 < M ? lr.key[j + 1] : next;
    const bool t = (j < nvalid) && (last_of_tile ? (last_tile || !(hb[1][0] == lr.key[j])) : !(nk == lr.key[j]));
    tail |= (uint32_t)t << j;
  }
  if (first_tile && e0 == 0 && nvalid > 0) head |= 1u;  // the input's first element
  lr.head = head;
  lr.tail = tail;
}

// (c, v) of a lane's elements folded in order.
template <typename K, typename V, int M>
__device__ __forceinline__ Seg<V> lane_fold(const LaneRun<K, V, M> &lr) {
  uint32_t c = __popc(lr.head);
  V v = V(0);
#pragma unroll
  for (int j = 0; j < M; ++j) {
    if (lr.head & (1u << j)) v = lr.val[j];
    else v = (V)(v + lr.val[j]);
  }
  return Seg<V>{c, v};
}

template <typename K, typename V>
__global__ void __launch_bounds__(kRbkThreads, 2) rbk_kernel(const K *keys, const V *vals, uint64_t n, K *out_keys,
                                                             V *out_vals, uint64_t *d_num_out,
                                                             typename RbkCfg<K, V>::Status st, WsHeader *hdr,
                                                             unsigned long long spin_limit_ns,
                                                             long long skip_publish_tile, int tma_ok,
                                                             unsigned int num_tiles) {
  using C = RbkCfg<K, V>;
  using P = typename C::P;
  constexpr int M = C::M, TILE = C::TILE;
  constexpr unsigned int NONE = 0xffffffffu;
  OpSeg<V> op;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *const buf[3] = {smem_raw, smem_raw + C::BUF_BYTES, smem_raw + 2 * C::BUF_BYTES};
  __shared__ __align__(8) uint64_t s_bar[3];
  __shared__ __align__(16) K s_halo[3][2][16 / sizeof(K)];
  __shared__ unsigned int s_ticket[2];
  __shared__ int s_has_tma[3];
  __shared__ P s_wagg[2][kRbkWarps];
  __shared__ P s_prefix;
  __shared__ int s_abort;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool control = (warp == kRbkWarps);
  const bool leader = control && lane == 0;

  unsigned int next_ticket = NONE;
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
      s_has_tma[0] = rbk_issue_load<K, V>(keys, vals, n, t0, buf[0], s_halo[0], &s_bar[0], keep, tma_ok);
      const unsigned int t1 = atomicAdd(&hdr->tile_ticket, 1u);
      next_ticket = t1 < num_tiles ? t1 : NONE;
    }
  }
  __syncthreads();

  uint32_t parity[3] = {0u, 0u, 0u};
  uint32_t inflight = s_has_tma[0] ? 1u : 0u;
  unsigned int pending = NONE;
  P pending_agg = OpSeg<V>::identity();

  for (int it = 0;; ++it) {
    const int slot = it & 1;
    const unsigned int t = s_ticket[slot];

    if (leader) {
      s_has_tma[2] = 0;
      if (pending != NONE)
        s_has_tma[2] = rbk_issue_load<K, V>(keys, vals, n, pending, buf[2], s_halo[2], &s_bar[2], stream, tma_ok);
      const unsigned int tn = (t != NONE) ? next_ticket : NONE;
      s_ticket[slot ^ 1] = tn;
      s_has_tma[slot ^ 1] = 0;
      if (tn != NONE)
        s_has_tma[slot ^ 1] =
            rbk_issue_load<K, V>(keys, vals, n, tn, buf[slot ^ 1], s_halo[slot ^ 1], &s_bar[slot ^ 1], keep, tma_ok);
      next_ticket = NONE;
      if (tn != NONE) {
        const unsigned int x = atomicAdd(&hdr->tile_ticket, 1u);
        next_ticket = x < num_tiles ? x : NONE;
      }
    }
    if (!tma_ok && !control) {
      if (t != NONE) rbk_sync_load<K, V>(keys, vals, n, t, buf[slot]);
      if (pending != NONE) rbk_sync_load<K, V>(keys, vals, n, pending, buf[2]);
    }
    __syncthreads();
    if (s_has_tma[slot ^ 1]) inflight |= 1u << (slot ^ 1);
    if (s_has_tma[2]) inflight |= 4u;

    // ---- phase 1 of t: tile aggregate
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
        const uint64_t base = (uint64_t)t * TILE;
        const uint32_t count = (uint32_t)((n - base) < (uint64_t)TILE ? (n - base) : (uint64_t)TILE);
        LaneRun<K, V, M> lr;
        rbk_read_lane<K, V>(buf[slot], s_halo[slot], count, t == 0, base + count == n, warp, lane, lr);
        const P incl = warp_inclusive_scan(lane_fold(lr), op, lane);
        if (lane == 31) s_wagg[slot][warp] = incl;
      }
    }
    __syncthreads();
    P agg_t = OpSeg<V>::identity();
    if (t != NONE) {
#pragma unroll
      for (int i = 0; i < kRbkWarps; ++i) agg_t = op(agg_t, s_wagg[slot][i]);
    }

    LaneRun<K, V, M> lr2;                // phase-2 lane data, kept across the barrier
    P lane_incl = OpSeg<V>::identity();  // its inclusive scan over the warp's lanes
    if (control) {
      if (leader && t != NONE && !s_abort && (long long)t != skip_publish_tile)
        st.publish(t, t == 0 ? kStPrefix : kStAggregate, agg_t);
      if (pending != NONE) {
        const unsigned int p = pending;
        P excl = OpSeg<V>::identity();
        bool ok = true;
        if (p != 0) ok = lookback_exclusive<P>(st, p, op, excl, hdr, spin_limit_ns);
        if (leader) {
          if (ok) {
            if (p != 0 && (long long)p != skip_publish_tile) st.publish(p, kStPrefix, op(excl, pending_agg));
            s_prefix = excl;
          } else {
            s_abort = 1;
          }
        }
        if (inflight & 4u) {
          parity[2] ^= 1u;
          inflight &= ~4u;
        }
      }
    } else if (pending != NONE) {
      // phase 2, the part that needs no prefix: overlaps the look-back
      if (inflight & 4u) {
        if (!mbar_wait(&s_bar[2], parity[2], spin_limit_ns)) {
          record_error(hdr, BK_ERR_SPIN_TIMEOUT, pending);
          s_abort = 1;
        }
        parity[2] ^= 1u;
        inflight &= ~4u;
      }
      const uint64_t base = (uint64_t)pending * TILE;
      const uint32_t count = (uint32_t)((n - base) < (uint64_t)TILE ? (n - base) : (uint64_t)TILE);
      rbk_read_lane<K, V>(buf[2], s_halo[2], count, pending == 0, base + count == n, warp, lane, lr2);
      lane_incl = warp_inclusive_scan(lane_fold(lr2), op, lane);
    }
    __syncthreads();  // the prefix is known
    if (s_abort) break;

    // ---- phase 2 of the pending tile: emit its runs
    if (pending != NONE && !control) {
      const uint64_t base = (uint64_t)pending * TILE;
      const uint32_t count = (uint32_t)((n - base) < (uint64_t)TILE ? (n - base) : (uint64_t)TILE);
      P carry = s_prefix;
      for (int i = 0; i < warp; ++i) carry = op(carry, s_wagg[slot ^ 1][i]);
      const bool last_tile = base + count == n;
      const LaneRun<K, V, M> &lr = lr2;
      const P excl = shfl_up(lane_incl, 1);
      if (lane > 0) carry = op(carry, excl);
      // walk the lane's elements with the running (c, v); each tail emits its run
      const uint32_t e0 = (uint32_t)(warp * 32 + lane) * M;
      uint32_t c = carry.c;
      V v = carry.v;
#pragma unroll
      for (int j = 0; j < M; ++j) {
        if (j < lr.nvalid) {
          if (lr.head & (1u << j)) {
            ++c;
            v = lr.val[j];
          } else {
            v = (V)(v + lr.val[j]);
          }
          if (lr.tail & (1u << j)) {
            out_keys[c - 1] = lr.key[j];
            out_vals[c - 1] = v;
            if (last_tile && e0 + j + 1 == count) *d_num_out = c;
          }
        }
      }
    }

    if (t == NONE) break;
    pending = t;
    pending_agg = agg_t;
    __syncthreads();  // buf[2], s_wagg[slot ^ 1] and the halo are reused next iteration
  }

  if (leader) {
    for (int b = 0; b < 3; ++b)
      if (inflight & (1u << b)) (void)mbar_wait(&s_bar[b], parity[b], spin_limit_ns);
  }
}

template <typename K, typename V>
int rbk_launch(const K *keys, const V *vals, uint64_t n, K *out_keys, V *out_vals, uint64_t *d_num_out, void *d_ws,
               size_t ws_bytes, cudaStream_t stream) {
  using C = RbkCfg<K, V>;
  host::DeviceInfo di;
  int st = host::device_info(&di);
  if (st != BK_OK) return st;
  if (d_num_out == nullptr) return BK_ERR_INVALID_ARGUMENT;
  if (n == 0) {
    write_count_kernel<V><<<1, 1, 0, stream>>>(d_num_out);
    return host::launch_status();
  }
  if (keys == nullptr || vals == nullptr || out_keys == nullptr || out_vals == nullptr) return BK_ERR_INVALID_ARGUMENT;
  if (!host::aligned_to<K>(keys) || !host::aligned_to<V>(vals) || !host::aligned_to<K>(out_keys) ||
      !host::aligned_to<V>(out_vals) || !host::aligned_to<uint64_t>(d_num_out))
    return BK_ERR_MISALIGNED;
  if (n >= 0xffffffffull) return BK_ERR_TOO_LARGE;  // run counts are 32-bit
  const size_t tiles = rbk_num_tiles<K, V>(n);
  st = host::check_ws(d_ws, ws_bytes, rbk_ws_bytes<K, V>(n));
  if (st != BK_OK) return st;
  WsHeader *hdr = reinterpret_cast<WsHeader *>(d_ws);
  auto status = C::Status::at(reinterpret_cast<char *>(d_ws) + kHeaderBytes, tiles);
  const unsigned init_grid = (unsigned)std::min<size_t>((tiles + 255) / 256 + 1, (size_t)di.sm_count * 8);
  rbk_init_kernel<<<init_grid, 256, 0, stream>>>(status, tiles, hdr);
  if ((st = host::launch_status()) != BK_OK) return st;
  const host::DebugFault dbg = host::debug_fault();
  const unsigned long long limit = dbg.spin_limit_ns ? dbg.spin_limit_ns : host::kDefaultSpinLimitNs;
  const int tma_ok = ((reinterpret_cast<uintptr_t>(keys) | reinterpret_cast<uintptr_t>(vals)) & 15) == 0;
  const size_t smem = 3 * C::BUF_BYTES;
  static thread_local bool attr_set = false;
  if (!attr_set) {
    if ((st = host::set_smem_attrs(rbk_kernel<K, V>, smem)) != BK_OK) return st;
    attr_set = true;
  }
  const unsigned grid = (unsigned)std::min<size_t>(tiles, (size_t)di.sm_count * 2);
  rbk_kernel<K, V><<<grid, kRbkThreads, smem, stream>>>(keys, vals, n, out_keys, out_vals, d_num_out, status, hdr,
                                                        limit, dbg.skip_publish_tile, tma_ok, (unsigned)tiles);
  return host::launch_status();
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
