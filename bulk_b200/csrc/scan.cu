// scan.cu -- single-pass inclusive scan with decoupled look-back, sm_100a.
//
// Replaces the reference's three-pass ::inclusive_scan (scan.cu:87-148):
// upsweep accumulate_tiles (:57-84) -> spine exclusive_scan_n (:24-31) ->
// downsweep inclusive_downsweep (:34-54), each calling the group scan of
// bulk/algorithm/scan.hpp:222-384.  That design moves 3*N*s bytes; this one
// moves the minimum 2*N*s (read once, write once).
//
// Per tile (THREADS x ITEMS elements, 16 KB): an atomic ticket names the tile
// (launch order, so every predecessor is already running); each thread loads
// ITEMS contiguous elements with 16-byte vector loads, scans them serially in
// registers, the CTA scans the per-thread totals with warp shuffles, the tile
// publishes its aggregate, warp 0 looks back over its predecessors for the
// exclusive prefix (bk_lookback.cuh), publishes the inclusive prefix, and the
// threads write their outputs with 16-byte streaming stores.  A tiny init
// kernel clears the tile status words before each scan.
//
// Semantics follow scan.cu:166-169 and bulk/algorithm/scan.hpp:455-486:
// out[i] = init (+) in[0] (+) ... (+) in[i].
#include "bk_common.cuh"
#include "bk_lookback.cuh"

namespace bk {

constexpr int kScanThreads = 256;

template <typename T>
struct ScanCfg {
  static constexpr int ITEMS = 64 / sizeof(T);  // 16 for 4-byte, 8 for 8-byte types
  static constexpr int TILE = kScanThreads * ITEMS;
  static constexpr int V = 16 / sizeof(T);
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
  for (size_t t = i; t < tiles; t += stride) st.clear(t);
  if (i == 0) hdr->tile_ticket = 0u;
}

template <typename T, typename Op>
__global__ void __launch_bounds__(kScanThreads, 5) scan_kernel(const T *in, T *out, uint64_t n, T init,
                                                            typename ScanCfg<T>::Status st, WsHeader *hdr,
                                                            unsigned long long spin_limit_ns,
                                                            long long skip_publish_tile, int vec_ok) {
  using C = ScanCfg<T>;
  constexpr int ITEMS = C::ITEMS, TILE = C::TILE, V = C::V;
  Op op;
  __shared__ unsigned int s_tile;
  __shared__ T s_warp[kScanThreads / 32 + 1];
  __shared__ T s_prefix;
  __shared__ int s_abort;
  const int tid = threadIdx.x;

  if (tid == 0) {
    s_tile = atomicAdd(&hdr->tile_ticket, 1u);
    s_abort = 0;
  }
  __syncthreads();
  const unsigned int tile = s_tile;
  const uint64_t base = (uint64_t)tile * TILE;
  const uint64_t my0 = base + (uint64_t)tid * ITEMS;
  const bool full = (base + TILE <= n);

  T x[ITEMS];
  if (full && vec_ok) {
#pragma unroll
    for (int k = 0; k < ITEMS / V; ++k) {
      uint4 r;
      asm("ld.global.nc.v4.u32 {%0,%1,%2,%3}, [%4];"
          : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
          : "l"(in + my0 + k * V));
      memcpy(&x[k * V], &r, 16);
    }
  } else {
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) x[i] = (my0 + i < n) ? in[my0 + i] : Op::identity();
  }

  // Thread-local inclusive scan.
#pragma unroll
  for (int i = 1; i < ITEMS; ++i) x[i] = op(x[i - 1], x[i]);

  T aggregate;
  const T thread_excl = block_exclusive_scan<kScanThreads>(x[ITEMS - 1], op, s_warp, aggregate);

  const bool publish = ((long long)tile != skip_publish_tile);
  if (tile == 0) {
    if (tid == 0) {
      if (publish) st.publish(0u, kStPrefix, op(init, aggregate));
      s_prefix = init;
    }
  } else if (tid < 32) {
    if (tid == 0 && publish) st.publish(tile, kStAggregate, aggregate);
    T excl;
    const bool ok = lookback_exclusive<T>(st, tile, op, excl, hdr, spin_limit_ns);
    if (tid == 0) {
      if (ok) {
        if (publish) st.publish(tile, kStPrefix, op(excl, aggregate));
        s_prefix = excl;
      } else {
        s_abort = 1;
      }
    }
  }
  __syncthreads();
  if (s_abort) return;

  const T tile_excl = s_prefix;
  const T carry = (tid == 0) ? tile_excl : op(tile_excl, thread_excl);
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) x[i] = op(carry, x[i]);

  if (full && vec_ok) {
#pragma unroll
    for (int k = 0; k < ITEMS / V; ++k) {
      uint4 r;
      memcpy(&r, &x[k * V], 16);
      st_stream_v4(out + my0 + k * V, r);
    }
  } else {
#pragma unroll
    for (int i = 0; i < ITEMS; ++i)
      if (my0 + i < n) out[my0 + i] = x[i];
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
  const int vec_ok = ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) & 15) == 0;
  scan_kernel<T, Op><<<(unsigned)tiles, kScanThreads, 0, stream>>>(d_in, d_out, n, init, status, hdr, limit,
                                                                   dbg.skip_publish_tile, vec_ok);
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
