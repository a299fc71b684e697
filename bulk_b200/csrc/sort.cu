// sort.cu -- device-wide stable merge sort by key, sm_100a.
//
// Replaces the reference's stable_merge_sort_by_key (merge_sort_by_key.cu:
// 150-209): a block sort of every 896-element tile (stable_sort_each_kernel,
// :12-25, through bulk/algorithm/detail/stable_merge_sort.hpp:125-206) and
// ceil(log2 tiles) merge passes, each a thrust::tabulate of merge paths
// (locate_merge_path, :90-131) plus merge_by_key_kernel (:61-87), ping-ponging
// with temporaries and copying back at the end.  Here the block sort covers
// 8192 (4-byte keys) or 4096 (8-byte keys) elements per CTA -- a stable
// odd-even transposition sort of 16 / 8 register items per thread, then
// log2(threads) merge-path rounds in shared memory, with the barriers the
// reference's block sort lacks (each round reads the stage only after every
// thread has written it) -- so a 2^26-element sort needs 13-14 global passes
// instead of 17.  The passes use the merge tile of bk_merge.cuh; the pass
// parity is chosen so the last pass lands in the caller's buffers (no copy
// back).
#include "bk_common.cuh"
#include "bk_merge.cuh"

namespace bk {

constexpr int kBsThreads = 512;  // block sort
constexpr int kMpThreads = 256;  // merge passes

template <typename K>
struct SortCfg {
  static constexpr int BS_ITEMS = sizeof(K) == 4 ? 16 : 8;
  static constexpr int BS_TILE = kBsThreads * BS_ITEMS;  // 8192 / 4096
  static constexpr int MP_ITEMS = sizeof(K) == 4 ? 16 : 8;
  static constexpr int MP_TILE = kMpThreads * MP_ITEMS;  // 4096 / 2048 (divides BS_TILE)
};

template <typename K, typename P>
constexpr size_t bs_smem_bytes() {
  return align_up(sizeof(K) * padded_len(SortCfg<K>::BS_TILE), 16) +
         (size_t)payload_bytes<P>() * padded_len(SortCfg<K>::BS_TILE);
}
template <typename K, typename P>
constexpr size_t mp_smem_bytes() {
  return align_up(sizeof(K) * padded_len(SortCfg<K>::MP_TILE), 16) +
         (size_t)payload_bytes<P>() * padded_len(SortCfg<K>::MP_TILE);
}

// Stable sort of one tile: in -> out (may alias).
template <typename K, typename P>
__global__ void __launch_bounds__(kBsThreads) block_sort_kernel(const K *in_k, const P *in_v, K *out_k, P *out_v,
                                                                uint64_t n) {
  constexpr int ITEMS = SortCfg<K>::BS_ITEMS, TILE = SortCfg<K>::BS_TILE;
  extern __shared__ __align__(16) unsigned char smem[];
  K *sk = reinterpret_cast<K *>(smem);
  P *sv = reinterpret_cast<P *>(smem + align_up(sizeof(K) * padded_len(TILE), 16));  // padded layout
  const uint64_t base = (uint64_t)blockIdx.x * TILE;
  const int count = (int)((n - base) < (uint64_t)TILE ? (n - base) : (uint64_t)TILE);
  const int tid = threadIdx.x;

  // stage in (all loads in flight before the first store); pad a partial
  // tile with the largest key (kept after real keys)
  {
    K tk[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const int i = j * kBsThreads + tid;
      tk[j] = i < count ? __ldg(in_k + base + i) : key_max<K>();
    }
    if constexpr (has_payload<P>()) {
      P tv[ITEMS];
#pragma unroll
      for (int j = 0; j < ITEMS; ++j) {
        const int i = j * kBsThreads + tid;
        tv[j] = i < count ? __ldg(in_v + base + i) : P();
      }
#pragma unroll
      for (int j = 0; j < ITEMS; ++j) sv[pad32(j * kBsThreads + tid)] = tv[j];
    }
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) sk[pad32(j * kBsThreads + tid)] = tk[j];
  }
  __syncthreads();

  // per-thread stable odd-even transposition sort of ITEMS consecutive items
  K k[ITEMS];
  P v[ITEMS];
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    k[i] = sk[pad32(tid * ITEMS + i)];
    if constexpr (has_payload<P>()) v[i] = sv[pad32(tid * ITEMS + i)];
  }
#pragma unroll
  for (int r = 0; r < ITEMS; ++r) {
#pragma unroll
    for (int i = r & 1; i + 1 < ITEMS; i += 2) {
      if (k[i + 1] < k[i]) {  // swap only on strict order: stable
        const K tk = k[i]; k[i] = k[i + 1]; k[i + 1] = tk;
        if constexpr (has_payload<P>()) { const P tv = v[i]; v[i] = v[i + 1]; v[i + 1] = tv; }
      }
    }
  }

  // merge rounds: runs of width w -> 2w
  for (int w = ITEMS; w < TILE; w *= 2) {
    __syncthreads();  // everyone has read the previous stage
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      sk[pad32(tid * ITEMS + i)] = k[i];
      if constexpr (has_payload<P>()) sv[pad32(tid * ITEMS + i)] = v[i];
    }
    __syncthreads();  // the stage is complete before anyone merges from it
    const int d = tid * ITEMS;
    const int p0 = d & ~(2 * w - 1);
    const int diag = d - p0;
    const PView<K> pa{sk, p0}, pb{sk, p0 + w};
    const int ia = merge_path<K, int>(pa, w, pb, w, diag);
    int src[ITEMS];
    serial_merge<ITEMS, K>(pa, w, w, ia, diag - ia, k, src, ITEMS);
    if constexpr (has_payload<P>()) {
#pragma unroll
      for (int i = 0; i < ITEMS; ++i) v[i] = sv[pad32(p0 + src[i])];
    }
  }

  // stage out through shared memory (coalesced stores)
  __syncthreads();
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    sk[pad32(tid * ITEMS + i)] = k[i];
    if constexpr (has_payload<P>()) sv[pad32(tid * ITEMS + i)] = v[i];
  }
  __syncthreads();
  stage_out_padded<kBsThreads>(out_k + base, sk, count);
  if constexpr (has_payload<P>()) stage_out_padded<kBsThreads>(out_v + base, sv, count);
}

// Merge pass: runs of width w in `src` -> runs of 2w in `dst`.
// parts[t] = A-split of output tile t at its diagonal inside its pair.
template <typename K>
__global__ void sort_partition_kernel(const K *keys, uint64_t n, uint64_t w, uint64_t num_tiles, uint64_t *parts) {
  constexpr uint64_t T = SortCfg<K>::MP_TILE;
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= num_tiles) return;
  const uint64_t d = t * T;
  const uint64_t p0 = d / (2 * w) * (2 * w);
  const uint64_t a_end = p0 + w < n ? p0 + w : n;
  const uint64_t b_end = p0 + 2 * w < n ? p0 + 2 * w : n;
  parts[t] = merge_path<K, uint64_t>(keys + p0, a_end - p0, keys + a_end, b_end - a_end, d - p0);
}

template <typename K, typename P>
__global__ void __launch_bounds__(kMpThreads, 4) sort_merge_kernel(const K *sk, const P *sv, K *dk, P *dv, uint64_t n,
                                                                uint64_t w, const uint64_t *parts,
                                                                uint64_t num_tiles) {
  constexpr uint64_t T = SortCfg<K>::MP_TILE;
  extern __shared__ __align__(16) unsigned char smem[];
  const uint64_t t = blockIdx.x;
  const uint64_t d = t * T;
  const uint64_t p0 = d / (2 * w) * (2 * w);
  const uint64_t a_end = p0 + w < n ? p0 + w : n;
  const uint64_t b_end = p0 + 2 * w < n ? p0 + 2 * w : n;
  const uint64_t la_all = a_end - p0, lb_all = b_end - a_end;
  const uint64_t diag0 = d - p0;
  const uint64_t diag1 = (diag0 + T < la_all + lb_all) ? diag0 + T : la_all + lb_all;
  const uint64_t a0 = parts[t];
  // the next tile's split belongs to this pair only if it starts inside it
  const uint64_t a1 = (t + 1 < num_tiles && d + T < b_end) ? parts[t + 1] : la_all;
  const uint64_t b0 = diag0 - a0, b1 = diag1 - a1;
  merge_tile<kMpThreads, SortCfg<K>::MP_ITEMS, K, P>(
      sk + p0 + a0, has_payload<P>() ? sv + p0 + a0 : nullptr, (int)(a1 - a0), sk + a_end + b0,
      has_payload<P>() ? sv + a_end + b0 : nullptr, (int)(b1 - b0), dk + d, has_payload<P>() ? dv + d : nullptr,
      smem);
}

template <typename K, typename P>
size_t sort_ws_bytes_t(uint64_t n) {
  const uint64_t mp_tiles = (n + SortCfg<K>::MP_TILE - 1) / SortCfg<K>::MP_TILE;
  return kHeaderBytes + align_up(n * sizeof(K), 256) + align_up(n * (size_t)payload_bytes<P>(), 256) +
         align_up((mp_tiles + 1) * sizeof(uint64_t), 256);
}

template <typename Kern>
static int set_smem(Kern kern, size_t bytes) {
  return host::set_smem_attrs(kern, bytes);
}

template <typename K, typename P>
int sort_launch(K *keys, P *vals, uint64_t n, void *d_ws, size_t ws_bytes, cudaStream_t stream) {
  using C = SortCfg<K>;
  host::DeviceInfo di;
  int st = host::device_info(&di);
  if (st != BK_OK) return st;
  if (n <= 1) return BK_OK;
  if (keys == nullptr || (has_payload<P>() && vals == nullptr)) return BK_ERR_INVALID_ARGUMENT;
  if (!host::aligned_to<K>(keys)) return BK_ERR_MISALIGNED;
  if constexpr (has_payload<P>()) {
    if (!host::aligned_to<P>(vals)) return BK_ERR_MISALIGNED;
  }
  const uint64_t bs_tiles = (n + C::BS_TILE - 1) / C::BS_TILE;
  const uint64_t mp_tiles = (n + C::MP_TILE - 1) / C::MP_TILE;
  if (mp_tiles >= 0x7fffffffull) return BK_ERR_TOO_LARGE;
  st = host::check_ws(d_ws, ws_bytes, sort_ws_bytes_t<K, P>(n));
  if (st != BK_OK) return st;
  char *ws = reinterpret_cast<char *>(d_ws) + kHeaderBytes;
  K *tk = reinterpret_cast<K *>(ws);
  ws += align_up(n * sizeof(K), 256);
  P *tv = reinterpret_cast<P *>(ws);
  ws += align_up(n * (size_t)payload_bytes<P>(), 256);
  uint64_t *parts = reinterpret_cast<uint64_t *>(ws);

  int passes = 0;
  for (uint64_t w = C::BS_TILE; w < n; w *= 2) ++passes;

  static thread_local bool attr_set = false;
  if (!attr_set) {
    if ((st = set_smem(block_sort_kernel<K, P>, bs_smem_bytes<K, P>())) != BK_OK) return st;
    if ((st = set_smem(sort_merge_kernel<K, P>, mp_smem_bytes<K, P>())) != BK_OK) return st;
    attr_set = true;
  }
  // an odd number of passes starts in the temporaries so the last lands in place
  K *ck = (passes & 1) ? tk : keys;
  P *cv = (passes & 1) ? tv : vals;
  block_sort_kernel<K, P><<<(unsigned)bs_tiles, kBsThreads, bs_smem_bytes<K, P>(), stream>>>(keys, vals, ck, cv, n);
  if ((st = host::launch_status()) != BK_OK) return st;
  for (uint64_t w = C::BS_TILE; w < n; w *= 2) {
    K *nk = (ck == keys) ? tk : keys;
    P *nv = (ck == keys) ? tv : vals;
    sort_partition_kernel<K><<<(unsigned)((mp_tiles + 255) / 256), 256, 0, stream>>>(ck, n, w, mp_tiles, parts);
    if ((st = host::launch_status()) != BK_OK) return st;
    sort_merge_kernel<K, P><<<(unsigned)mp_tiles, kMpThreads, mp_smem_bytes<K, P>(), stream>>>(ck, cv, nk, nv, n, w,
                                                                                             parts, mp_tiles);
    if ((st = host::launch_status()) != BK_OK) return st;
    ck = nk;
    cv = nv;
  }
  return BK_OK;
}

size_t sort_workspace_bytes(int key_dtype, int value_dtype, uint64_t n) {
  const bool k4 = key_dtype == BK_DTYPE_I32 || key_dtype == BK_DTYPE_U32 || key_dtype == BK_DTYPE_F32;
  const bool k8 = key_dtype == BK_DTYPE_I64 || key_dtype == BK_DTYPE_U64 || key_dtype == BK_DTYPE_F64;
  const bool v0 = value_dtype == BK_DTYPE_NONE;
  const bool v4 = value_dtype == BK_DTYPE_I32 || value_dtype == BK_DTYPE_U32 || value_dtype == BK_DTYPE_F32;
  const bool v8 = value_dtype == BK_DTYPE_I64 || value_dtype == BK_DTYPE_U64 || value_dtype == BK_DTYPE_F64;
  if (k4) return v0 ? sort_ws_bytes_t<float, NoPayload>(n) : v4 ? sort_ws_bytes_t<float, uint32_t>(n)
                 : v8 ? sort_ws_bytes_t<float, unsigned long long>(n) : 0;
  if (k8) return v0 ? sort_ws_bytes_t<double, NoPayload>(n) : v4 ? sort_ws_bytes_t<double, uint32_t>(n)
                 : v8 ? sort_ws_bytes_t<double, unsigned long long>(n) : 0;
  return 0;
}

}  // namespace bk

#define BK_DEFINE_SORT(KN, K)                                                                                  \
  extern "C" int bk_sort_keys_##KN(K *keys, uint64_t n, void *d_ws, size_t ws_bytes, bk_stream_t stream) {    \
    return bk::sort_launch<K, bk::NoPayload>(keys, nullptr, n, d_ws, ws_bytes, (cudaStream_t)stream);          \
  }                                                                                                            \
  extern "C" int bk_sort_by_key_##KN##_u32(K *keys, uint32_t *vals, uint64_t n, void *d_ws, size_t ws_bytes,   \
                                           bk_stream_t stream) {                                              \
    return bk::sort_launch<K, uint32_t>(keys, vals, n, d_ws, ws_bytes, (cudaStream_t)stream);                  \
  }                                                                                                            \
  extern "C" int bk_sort_by_key_##KN##_u64(K *keys, uint64_t *vals, uint64_t n, void *d_ws, size_t ws_bytes,   \
                                           bk_stream_t stream) {                                              \
    return bk::sort_launch<K, unsigned long long>(keys, reinterpret_cast<unsigned long long *>(vals), n, d_ws, \
                                                  ws_bytes, (cudaStream_t)stream);                            \
  }

BK_DEFINE_SORT(i32, int32_t)
BK_DEFINE_SORT(u32, uint32_t)
BK_DEFINE_SORT(i64, int64_t)
BK_DEFINE_SORT(u64, uint64_t)
BK_DEFINE_SORT(f32, float)
BK_DEFINE_SORT(f64, double)
