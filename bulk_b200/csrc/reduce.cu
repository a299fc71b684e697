// reduce.cu -- single-launch device-wide reduction for sm_100a.
//
// Replaces the reference's two-kernel my_reduce (reduce.cu:58-97): a
// partition kernel that calls bulk::reduce(group, ...) per aligned partition
// (bulk/algorithm/reduce.hpp:110-219, decomposition.hpp:142-210), a second
// single-group launch over the partial sums, and a synchronous D2H read.
//
// Here one launch does it all: a grid of (SMs x CTAs-per-SM) CTAs streams the
// input with 16-byte non-coherent loads (UNROLL independent loads in flight
// per thread), each thread keeps 4*V independent accumulators, the CTA
// folds them with warp shuffles, writes one partial to the workspace, and the
// last CTA to finish (atomic counter) folds the partials in index order and
// writes init (+) total to d_out.  The partition of the input depends only on
// n and the SM count, so floating-point results repeat exactly run to run.
#include <algorithm>

#include "bk_common.cuh"
#include "bk_tune.hpp"

namespace bk {

constexpr int kReduceThreads = 256;
constexpr int kReduceUnroll = 8;
constexpr int kReduceMaxCtasPerSm = 8;  // the largest grid the launch-shape table may pick

template <typename T>
struct ReduceLayout {
  static constexpr int V = 16 / sizeof(T);  // elements per 16-byte vector
};

__host__ inline size_t reduce_partials_offset() { return kHeaderBytes; }

template <typename T>
size_t reduce_ws_bytes(int sm_count) {
  return kHeaderBytes + align_up(sizeof(T) * (size_t)sm_count * kReduceMaxCtasPerSm, 256);
}

template <typename T, typename Op>
__global__ void __launch_bounds__(kReduceThreads, 4) reduce_kernel(const T *__restrict__ in, uint64_t head, uint64_t nvec,
                                                                 uint64_t tail, T init, T *__restrict__ out,
                                                                 T *__restrict__ partials, WsHeader *hdr) {
  constexpr int V = ReduceLayout<T>::V;
  constexpr int U = kReduceUnroll;
  constexpr int A = 4;  // accumulator vectors: load u folds into acc[u % A]
  Op op;
  T acc[A][V];
#pragma unroll
  for (int a = 0; a < A; ++a)
#pragma unroll
    for (int j = 0; j < V; ++j) acc[a][j] = Op::identity();

  const int tid = threadIdx.x;
  const uint4 *vin = reinterpret_cast<const uint4 *>(in + head);
  const uint64_t stride = (uint64_t)gridDim.x * kReduceThreads;
  uint64_t v = (uint64_t)blockIdx.x * kReduceThreads + tid;

  // Main body: U independent 16-byte loads per thread per iteration.
  for (; v + (U - 1) * stride < nvec; v += U * stride) {
    uint4 r[U];
#pragma unroll
    for (int u = 0; u < U; ++u) r[u] = ld_stream_v4(vin + v + u * stride);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      T e[V];
      memcpy(e, &r[u], 16);
#pragma unroll
      for (int j = 0; j < V; ++j) acc[u % A][j] = op(acc[u % A][j], e[j]);
    }
  }
  // Fewer than U strides left: one more batch with each load predicated, so
  // the last loads are in flight together instead of one DRAM round trip
  // apiece.
  {
    uint4 r[U];
#pragma unroll
    for (int u = 0; u < U - 1; ++u)
      if (v + u * stride < nvec) r[u] = ld_stream_v4(vin + v + u * stride);
#pragma unroll
    for (int u = 0; u < U - 1; ++u) {
      if (v + u * stride < nvec) {
        T e[V];
        memcpy(e, &r[u], 16);
#pragma unroll
        for (int j = 0; j < V; ++j) acc[u % A][j] = op(acc[u % A][j], e[j]);
      }
    }
  }
  // Unaligned head and ragged tail (fewer than V elements each): CTA 0.
  if (blockIdx.x == 0) {
    if ((uint64_t)tid < head) acc[1][0] = op(acc[1][0], in[tid]);
    if ((uint64_t)tid < tail) acc[2][0] = op(acc[2][0], in[head + nvec * V + tid]);
  }

  // Fold the thread's accumulators pairwise (fixed order).
#pragma unroll
  for (int w = 1; w < A * V; w <<= 1) {
#pragma unroll
    for (int i = 0; i + w < A * V; i += 2 * w) {
      acc[i / V][i % V] = op(acc[i / V][i % V], acc[(i + w) / V][(i + w) % V]);
    }
  }
  __shared__ T s_warp[kReduceThreads / 32];
  __shared__ bool s_last;
  T cta = block_reduce<kReduceThreads>(acc[0][0], op, s_warp);

  if (tid == 0) {
    partials[blockIdx.x] = cta;
    __threadfence();
    const unsigned int prev = atomicAdd(&hdr->done_count, 1u);
    s_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;

  // Last CTA: fold the partials in index order.
  __threadfence();
  T x = Op::identity();
  for (unsigned int i = tid; i < gridDim.x; i += kReduceThreads) x = op(x, __ldcg(partials + i));
  T total = block_reduce<kReduceThreads>(x, op, s_warp);
  if (tid == 0) {
    out[0] = op(init, total);
    hdr->done_count = 0u;  // leave the workspace as found
  }
}

template <typename T>
__global__ void write_scalar_kernel(T *out, T v) {
  out[0] = v;
}

template <typename T, typename Op>
int reduce_launch(const T *d_in, uint64_t n, T init, T *d_out, void *d_ws, size_t ws_bytes, cudaStream_t stream) {
  host::DeviceInfo di;
  int st = host::device_info(&di);
  if (st != BK_OK) return st;
  if (d_out == nullptr || (n > 0 && d_in == nullptr)) return BK_ERR_INVALID_ARGUMENT;
  if (!host::aligned_to<T>(d_in) || !host::aligned_to<T>(d_out)) return BK_ERR_MISALIGNED;
  if (n == 0) {
    write_scalar_kernel<T><<<1, 1, 0, stream>>>(d_out, init);
    return host::launch_status();
  }
  st = host::check_ws(d_ws, ws_bytes, reduce_ws_bytes<T>(di.sm_count));
  if (st != BK_OK) return st;

  constexpr int V = ReduceLayout<T>::V;
  const uintptr_t addr = reinterpret_cast<uintptr_t>(d_in);
  uint64_t head = ((16 - (addr & 15)) & 15) / sizeof(T);
  if (head > n) head = n;
  const uint64_t nvec = (n - head) / V;
  const uint64_t tail = (n - head) - nvec * V;
  const uint64_t per_cta = (uint64_t)kReduceThreads * kReduceUnroll;
  uint64_t grid = (nvec + per_cta - 1) / per_cta;
  const tune::Knobs kn = tune::knobs_for(tune::kReduce, (int)sizeof(T), n);
  const uint64_t max_grid = (uint64_t)di.sm_count * (uint64_t)std::min(kn.ctas_per_sm, kReduceMaxCtasPerSm);
  if (grid > max_grid) grid = max_grid;
  if (grid < 1) grid = 1;

  WsHeader *hdr = reinterpret_cast<WsHeader *>(d_ws);
  T *partials = reinterpret_cast<T *>(reinterpret_cast<char *>(d_ws) + reduce_partials_offset());
  reduce_kernel<T, Op><<<(unsigned)grid, kReduceThreads, 0, stream>>>(d_in, head, nvec, tail, init, d_out, partials, hdr);
  return host::launch_status();
}

size_t reduce_workspace_bytes(int dtype, uint64_t /*n*/) {
  host::DeviceInfo di;
  if (host::device_info(&di) != BK_OK) di.sm_count = 160;  // upper bound when no device is visible
  switch (dtype) {
    case BK_DTYPE_I32: case BK_DTYPE_U32: case BK_DTYPE_F32: return reduce_ws_bytes<float>(di.sm_count);
    case BK_DTYPE_I64: case BK_DTYPE_U64: case BK_DTYPE_F64: return reduce_ws_bytes<double>(di.sm_count);
    default: return 0;
  }
}

}  // namespace bk

#define BK_DEFINE_REDUCE(OPNAME, OPT, TN, T)                                                             \
  extern "C" int bk_reduce_##OPNAME##_##TN(const T *d_in, uint64_t n, T init, T *d_out, void *d_ws,    \
                                           size_t ws_bytes, bk_stream_t stream) {                      \
    return bk::reduce_launch<T, bk::OPT<T>>(d_in, n, init, d_out, d_ws, ws_bytes, (cudaStream_t)stream); \
  }

#define BK_DEFINE_REDUCE_ALL_T(OPNAME, OPT)        \
  BK_DEFINE_REDUCE(OPNAME, OPT, i32, int32_t)      \
  BK_DEFINE_REDUCE(OPNAME, OPT, u32, uint32_t)     \
  BK_DEFINE_REDUCE(OPNAME, OPT, i64, int64_t)      \
  BK_DEFINE_REDUCE(OPNAME, OPT, u64, uint64_t)     \
  BK_DEFINE_REDUCE(OPNAME, OPT, f32, float)        \
  BK_DEFINE_REDUCE(OPNAME, OPT, f64, double)

BK_DEFINE_REDUCE_ALL_T(sum, OpSum)
BK_DEFINE_REDUCE_ALL_T(min, OpMin)
BK_DEFINE_REDUCE_ALL_T(max, OpMax)
