// merge.cu -- device-wide merge and merge_by_key (merge path), sm_100a.
//
// Replaces the reference's my_merge (merge.cu:127-162): a thrust::tabulate of
// merge_path at every tile diagonal (locate_merge_path, merge.cu:100-124)
// followed by one staged merge per tile (merge_kernel / staged_merge,
// merge.cu:12-97), which is keys-only; the by-key form follows the bounded
// group merge_by_key (bulk/algorithm/merge.hpp:507-607).  Here: a partition
// kernel computes the A/B split at every tile boundary, then each CTA merges
// one 4096-output tile through shared memory (bk_merge.cuh) and writes it with
// 16-byte coalesced stores.
#include "bk_common.cuh"
#include "bk_merge.cuh"

namespace bk {

constexpr int kMergeThreads = 256;

template <typename K>
struct MergeCfg {
  static constexpr int ITEMS = sizeof(K) == 4 ? 16 : 8;
  static constexpr int TILE = kMergeThreads * ITEMS;
};

template <typename K, typename P>
constexpr size_t merge_smem_bytes() {
  return align_up(sizeof(K) * padded_len(MergeCfg<K>::TILE), 16) +
         (size_t)payload_bytes<P>() * padded_len(MergeCfg<K>::TILE);
}

// parts[k] = number of A elements among the first min(k*TILE, na+nb) outputs.
template <typename K>
__global__ void merge_partition_kernel(const K *a, uint64_t na, const K *b, uint64_t nb, uint64_t tile,
                                       uint64_t num_parts, uint64_t *parts) {
  const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= num_parts) return;
  const uint64_t total = na + nb;
  const uint64_t diag = k * tile < total ? k * tile : total;
  parts[k] = merge_path<K, uint64_t>(a, na, b, nb, diag);
}

// One CTA per output tile.  Thread 0 first asks L2 for the inputs of tile
// k + ahead (the CTA that will start about when every CTA now resident has
// finished), so that CTA's loads hit L2 instead of waiting on memory.
template <typename K, typename P>
__global__ void __launch_bounds__(kMergeThreads, 4) merge_kernel(const K *a, const P *av, uint64_t na, const K *b,
                                                              const P *bv, uint64_t nb, K *out, P *outv,
                                                              const uint64_t *parts, uint64_t ahead) {
  constexpr int TILE = MergeCfg<K>::TILE;
  extern __shared__ __align__(16) unsigned char smem[];
  const uint64_t k = blockIdx.x;
  const uint64_t total = na + nb;
  if (threadIdx.x == 0 && k + ahead < gridDim.x) {
    const uint64_t f = k + ahead;
    const uint64_t e0 = f * TILE, e1 = e0 + TILE < total ? e0 + TILE : total;
    const uint64_t fa0 = parts[f], fa1 = parts[f + 1], fb0 = e0 - fa0, fb1 = e1 - fa1;
    prefetch_l2_range(a + fa0, (fa1 - fa0) * sizeof(K));
    prefetch_l2_range(b + fb0, (fb1 - fb0) * sizeof(K));
    if constexpr (has_payload<P>()) {
      prefetch_l2_range(av + fa0, (fa1 - fa0) * sizeof(P));
      prefetch_l2_range(bv + fb0, (fb1 - fb0) * sizeof(P));
    }
  }
  const uint64_t d0 = k * TILE;
  const uint64_t d1 = d0 + TILE < total ? d0 + TILE : total;
  const uint64_t a0 = parts[k], a1 = parts[k + 1];
  const uint64_t b0 = d0 - a0, b1 = d1 - a1;
  merge_tile<kMergeThreads, MergeCfg<K>::ITEMS, K, P>(
      a + a0, has_payload<P>() ? av + a0 : nullptr, (int)(a1 - a0), b + b0, has_payload<P>() ? bv + b0 : nullptr,
      (int)(b1 - b0), out + d0, has_payload<P>() ? outv + d0 : nullptr, smem);
}

template <typename K>
size_t merge_ws_bytes(uint64_t n) {
  const uint64_t tiles = (n + MergeCfg<K>::TILE - 1) / MergeCfg<K>::TILE;
  return kHeaderBytes + align_up((tiles + 1) * sizeof(uint64_t), 256);
}

template <typename K, typename P>
int merge_launch(const K *a, const P *av, uint64_t na, const K *b, const P *bv, uint64_t nb, K *out, P *outv,
                 void *d_ws, size_t ws_bytes, cudaStream_t stream) {
  host::DeviceInfo di;
  int st = host::device_info(&di);
  if (st != BK_OK) return st;
  const uint64_t n = na + nb;
  if (n == 0) return BK_OK;
  if ((na && a == nullptr) || (nb && b == nullptr) || out == nullptr) return BK_ERR_INVALID_ARGUMENT;
  if (has_payload<P>() && ((na && av == nullptr) || (nb && bv == nullptr) || outv == nullptr))
    return BK_ERR_INVALID_ARGUMENT;
  if (!host::aligned_to<K>(a) || !host::aligned_to<K>(b) || !host::aligned_to<K>(out)) return BK_ERR_MISALIGNED;
  if constexpr (has_payload<P>()) {
    if (!host::aligned_to<P>(av) || !host::aligned_to<P>(bv) || !host::aligned_to<P>(outv)) return BK_ERR_MISALIGNED;
  }
  const uint64_t tiles = (n + MergeCfg<K>::TILE - 1) / MergeCfg<K>::TILE;
  if (tiles >= 0x7fffffffull) return BK_ERR_TOO_LARGE;
  st = host::check_ws(d_ws, ws_bytes, merge_ws_bytes<K>(n));
  if (st != BK_OK) return st;
  uint64_t *parts = reinterpret_cast<uint64_t *>(reinterpret_cast<char *>(d_ws) + kHeaderBytes);
  const uint64_t np = tiles + 1;
  merge_partition_kernel<K><<<(unsigned)((np + 255) / 256), 256, 0, stream>>>(a, na, b, nb, MergeCfg<K>::TILE, np,
                                                                              parts);
  st = host::launch_status();
  if (st != BK_OK) return st;
  constexpr size_t smem = merge_smem_bytes<K, P>();
  struct Site {};
  host::KernelSetup ks;
  if ((st = host::kernel_setup<Site>(merge_kernel<K, P>, kMergeThreads, smem, &ks)) != BK_OK) return st;
  merge_kernel<K, P><<<(unsigned)tiles, kMergeThreads, smem, stream>>>(a, av, na, b, bv, nb, out, outv, parts,
                                                                       ks.resident_ctas);
  return host::launch_status();
}

size_t merge_workspace_bytes(int key_dtype, int value_dtype, uint64_t n) {
  if (value_dtype != BK_DTYPE_NONE && value_dtype != BK_DTYPE_U32 && value_dtype != BK_DTYPE_U64 &&
      value_dtype != BK_DTYPE_I32 && value_dtype != BK_DTYPE_I64 && value_dtype != BK_DTYPE_F32 &&
      value_dtype != BK_DTYPE_F64)
    return 0;
  switch (key_dtype) {
    case BK_DTYPE_I32: case BK_DTYPE_U32: case BK_DTYPE_F32: return merge_ws_bytes<float>(n);
    case BK_DTYPE_I64: case BK_DTYPE_U64: case BK_DTYPE_F64: return merge_ws_bytes<double>(n);
    default: return 0;
  }
}

}  // namespace bk

#define BK_DEFINE_MERGE(KN, K)                                                                               \
  extern "C" int bk_merge_##KN(const K *a, uint64_t na, const K *b, uint64_t nb, K *out, void *d_ws,         \
                               size_t ws_bytes, bk_stream_t stream) {                                       \
    return bk::merge_launch<K, bk::NoPayload>(a, nullptr, na, b, nullptr, nb, out, nullptr, d_ws, ws_bytes,  \
                                              (cudaStream_t)stream);                                        \
  }                                                                                                          \
  extern "C" int bk_merge_by_key_##KN##_u32(const K *a_keys, const uint32_t *a_vals, uint64_t na,            \
                                            const K *b_keys, const uint32_t *b_vals, uint64_t nb,            \
                                            K *out_keys, uint32_t *out_vals, void *d_ws, size_t ws_bytes,    \
                                            bk_stream_t stream) {                                           \
    return bk::merge_launch<K, uint32_t>(a_keys, a_vals, na, b_keys, b_vals, nb, out_keys, out_vals, d_ws,   \
                                         ws_bytes, (cudaStream_t)stream);                                   \
  }                                                                                                          \
  extern "C" int bk_merge_by_key_##KN##_u64(const K *a_keys, const uint64_t *a_vals, uint64_t na,            \
                                            const K *b_keys, const uint64_t *b_vals, uint64_t nb,            \
                                            K *out_keys, uint64_t *out_vals, void *d_ws, size_t ws_bytes,    \
                                            bk_stream_t stream) {                                           \
    return bk::merge_launch<K, unsigned long long>(                                                          \
        a_keys, reinterpret_cast<const unsigned long long *>(a_vals), na, b_keys,                            \
        reinterpret_cast<const unsigned long long *>(b_vals), nb, out_keys,                                  \
        reinterpret_cast<unsigned long long *>(out_vals), d_ws, ws_bytes, (cudaStream_t)stream);             \
  }

BK_DEFINE_MERGE(i32, int32_t)
BK_DEFINE_MERGE(u32, uint32_t)
BK_DEFINE_MERGE(i64, int64_t)
BK_DEFINE_MERGE(u64, uint64_t)
BK_DEFINE_MERGE(f32, float)
BK_DEFINE_MERGE(f64, double)
