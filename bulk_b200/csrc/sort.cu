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

// radix_sort.cu: the stable radix sort used below kRadixMaxN elements
template <typename K, typename P>
int radix_sort_launch(K *keys, P *vals, uint64_t n, void *d_ws, size_t ws_bytes, cudaStream_t stream);
template <typename K, typename P>
size_t radix_sort_ws_bytes(uint64_t n);
template <typename K, typename P>
struct RsItem {  // as radix_sort.cu defines it: in_* sorted into keys / vals
  const K *in_keys;
  const P *in_vals;
  K *keys;
  P *vals;
  uint64_t n;
};
template <typename K, typename P>
int radix_sort_batch_launch(const RsItem<K, P> *items, uint32_t count, void *d_ws, size_t ws_bytes,
                            cudaStream_t stream);
template <typename K, typename P>
size_t radix_sort_batch_ws_bytes(const uint64_t *sizes, uint32_t count);
constexpr uint64_t kRadixMaxN = 1ull << 30;

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

// A block-sort tile: `count` elements from in_* to out_* (may alias), both
// already offset to the tile.
template <typename K, typename P>
struct BsTile {
  const K *in_k;
  const P *in_v;
  K *out_k;
  P *out_v;
  int count;
};

// Block-sort tiles of one array.
template <typename K, typename P>
struct BsOne {
  const K *in_k;
  const P *in_v;
  K *out_k;
  P *out_v;
  uint64_t n;
  __device__ __forceinline__ BsTile<K, P> tile(unsigned int t) const {
    const uint64_t base = (uint64_t)t * SortCfg<K>::BS_TILE;
    const int count = (int)((n - base) < (uint64_t)SortCfg<K>::BS_TILE ? (n - base) : (uint64_t)SortCfg<K>::BS_TILE);
    return BsTile<K, P>{in_k + base, has_payload<P>() ? in_v + base : nullptr, out_k + base,
                        has_payload<P>() ? out_v + base : nullptr, count};
  }
};

// Finds the batch item owning global tile t: the last i with start[i] <= t.
__device__ __forceinline__ int batch_item_of(const uint32_t *start, uint32_t count, unsigned int t) {
  int lo = 0, hi = (int)count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

constexpr int kSortBatchMax = 256;

// Block-sort tiles of a batch of arrays (array i owns global tiles
// [start[i], start[i + 1])); the descriptors travel in the kernel parameters.
template <typename K, typename P>
struct BsBatch {
  const K *in_k[kSortBatchMax];
  const P *in_v[kSortBatchMax];
  K *out_k[kSortBatchMax];
  P *out_v[kSortBatchMax];
  uint64_t n[kSortBatchMax];
  uint32_t start[kSortBatchMax + 1];
  uint32_t count;
  __device__ __forceinline__ BsTile<K, P> tile(unsigned int t) const {
    const int i = batch_item_of(start, count, t);
    const uint64_t base = (uint64_t)(t - start[i]) * SortCfg<K>::BS_TILE;
    const int cnt = (int)((n[i] - base) < (uint64_t)SortCfg<K>::BS_TILE ? (n[i] - base) : (uint64_t)SortCfg<K>::BS_TILE);
    return BsTile<K, P>{in_k[i] + base, has_payload<P>() ? in_v[i] + base : nullptr, out_k[i] + base,
                        has_payload<P>() ? out_v[i] + base : nullptr, cnt};
  }
};

// Stable sort of one tile: in -> out (may alias).
template <typename K, typename P, typename Src>
__global__ void __launch_bounds__(kBsThreads) block_sort_kernel(const __grid_constant__ Src src) {
  constexpr int ITEMS = SortCfg<K>::BS_ITEMS, TILE = SortCfg<K>::BS_TILE;
  extern __shared__ __align__(16) unsigned char smem[];
  K *sk = reinterpret_cast<K *>(smem);
  P *sv = reinterpret_cast<P *>(smem + align_up(sizeof(K) * padded_len(TILE), 16));  // padded layout
  const BsTile<K, P> tl = src.tile(blockIdx.x);
  const K *in_k = tl.in_k;
  const P *in_v = tl.in_v;
  const int count = tl.count;
  const int tid = threadIdx.x;

  // stage in (all loads in flight before the first store); pad a partial
  // tile with the largest key (kept after real keys)
  {
    K tk[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const int i = j * kBsThreads + tid;
      tk[j] = i < count ? __ldg(in_k + i) : key_max<K>();
    }
    if constexpr (has_payload<P>()) {
      P tv[ITEMS];
#pragma unroll
      for (int j = 0; j < ITEMS; ++j) {
        const int i = j * kBsThreads + tid;
        tv[j] = i < count ? __ldg(in_v + i) : P();
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
  stage_out_padded<kBsThreads>(tl.out_k, sk, count);
  if constexpr (has_payload<P>()) stage_out_padded<kBsThreads>(tl.out_v, sv, count);
}

// A merge-pass tile: output tile `local` of a pass over one array that
// merges runs of width w in src_* into runs of 2w in dst_*; parts[t] is the
// A-split of the array's output tile t at its diagonal inside its pair.
template <typename K, typename P>
struct MpTile {
  const K *src_k;
  const P *src_v;
  K *dst_k;
  P *dst_v;
  uint64_t n;
  uint64_t w;
  uint64_t *parts;
  uint64_t local;
  uint64_t num_tiles;
};

template <typename K, typename P>
struct MpOne {
  const K *src_k;
  const P *src_v;
  K *dst_k;
  P *dst_v;
  uint64_t n;
  uint64_t w;
  uint64_t *parts;
  uint64_t num_tiles;
  __device__ __forceinline__ MpTile<K, P> tile(uint64_t t) const {
    return MpTile<K, P>{src_k, src_v, dst_k, dst_v, n, w, parts, t, num_tiles};
  }
};

// One merge pass over a batch of arrays (only those that still need it).
template <typename K, typename P>
struct MpBatch {
  const K *src_k[kSortBatchMax];
  const P *src_v[kSortBatchMax];
  K *dst_k[kSortBatchMax];
  P *dst_v[kSortBatchMax];
  uint64_t n[kSortBatchMax];
  uint64_t *parts[kSortBatchMax];
  uint32_t start[kSortBatchMax + 1];
  uint64_t w;
  uint32_t count;
  __device__ __forceinline__ MpTile<K, P> tile(uint64_t t) const {
    const int i = batch_item_of(start, count, (unsigned int)t);
    return MpTile<K, P>{src_k[i], src_v[i], dst_k[i], dst_v[i], n[i], w, parts[i], t - start[i],
                        (uint64_t)(start[i + 1] - start[i])};
  }
};

template <typename K, typename P, typename Src>
__global__ void sort_partition_kernel(const __grid_constant__ Src src, uint64_t total_tiles) {
  constexpr uint64_t T = SortCfg<K>::MP_TILE;
  const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total_tiles) return;
  const MpTile<K, P> m = src.tile(g);
  const uint64_t d = m.local * T;
  const uint64_t p0 = d / (2 * m.w) * (2 * m.w);
  const uint64_t a_end = p0 + m.w < m.n ? p0 + m.w : m.n;
  const uint64_t b_end = p0 + 2 * m.w < m.n ? p0 + 2 * m.w : m.n;
  m.parts[m.local] = merge_path<K, uint64_t>(m.src_k + p0, a_end - p0, m.src_k + a_end, b_end - a_end, d - p0);
}

// A merge-pass tile's inputs: elements [a_lo, a_lo + la) and [b_lo, b_lo + lb)
// of the source array, and its first output element.
struct MpRanges {
  uint64_t a_lo, b_lo, out;
  int la, lb;
};
template <typename K, typename P>
__device__ __forceinline__ MpRanges mp_ranges(const MpTile<K, P> &m) {
  constexpr uint64_t T = SortCfg<K>::MP_TILE;
  const uint64_t t = m.local, n = m.n, w = m.w;
  const uint64_t d = t * T;
  const uint64_t p0 = d / (2 * w) * (2 * w);
  const uint64_t a_end = p0 + w < n ? p0 + w : n;
  const uint64_t b_end = p0 + 2 * w < n ? p0 + 2 * w : n;
  const uint64_t la_all = a_end - p0, lb_all = b_end - a_end;
  const uint64_t diag0 = d - p0;
  const uint64_t diag1 = (diag0 + T < la_all + lb_all) ? diag0 + T : la_all + lb_all;
  const uint64_t a0 = m.parts[t];
  // the next tile's split belongs to this pair only if it starts inside it
  const uint64_t a1 = (t + 1 < m.num_tiles && d + T < b_end) ? m.parts[t + 1] : la_all;
  const uint64_t b0 = diag0 - a0, b1 = diag1 - a1;
  return MpRanges{p0 + a0, a_end + b0, d, (int)(a1 - a0), (int)(b1 - b0)};
}

// One merge-pass tile per CTA.  Thread 0 first asks L2 for the inputs of
// global tile blockIdx.x + ahead (the CTA that will start about when every CTA
// now resident has finished).
template <typename K, typename P, typename Src>
__global__ void __launch_bounds__(kMpThreads, 4) sort_merge_kernel(const __grid_constant__ Src src, uint64_t ahead) {
  extern __shared__ __align__(16) unsigned char smem[];
  if (threadIdx.x == 0 && blockIdx.x + ahead < gridDim.x) {
    const MpTile<K, P> f = src.tile(blockIdx.x + ahead);
    const MpRanges r = mp_ranges<K, P>(f);
    prefetch_l2_range(f.src_k + r.a_lo, (uint64_t)r.la * sizeof(K));
    prefetch_l2_range(f.src_k + r.b_lo, (uint64_t)r.lb * sizeof(K));
    if constexpr (has_payload<P>()) {
      prefetch_l2_range(f.src_v + r.a_lo, (uint64_t)r.la * sizeof(P));
      prefetch_l2_range(f.src_v + r.b_lo, (uint64_t)r.lb * sizeof(P));
    }
  }
  const MpTile<K, P> m = src.tile(blockIdx.x);
  const MpRanges r = mp_ranges<K, P>(m);
  const K *sk = m.src_k;
  const P *sv = m.src_v;
  merge_tile<kMpThreads, SortCfg<K>::MP_ITEMS, K, P>(
      sk + r.a_lo, has_payload<P>() ? sv + r.a_lo : nullptr, r.la, sk + r.b_lo,
      has_payload<P>() ? sv + r.b_lo : nullptr, r.lb, m.dst_k + r.out, has_payload<P>() ? m.dst_v + r.out : nullptr,
      smem);
}

template <typename K, typename P>
size_t merge_sort_ws_bytes_t(uint64_t n) {
  const uint64_t mp_tiles = (n + SortCfg<K>::MP_TILE - 1) / SortCfg<K>::MP_TILE;
  return kHeaderBytes + align_up(n * sizeof(K), 256) + align_up(n * (size_t)payload_bytes<P>(), 256) +
         align_up((mp_tiles + 1) * sizeof(uint64_t), 256);
}

// Which sort an array gets: one block-sort launch when it fits one block
// tile (the radix sort's passes are 4 or 8 times three launches), the radix
// sort up to 2^30 elements, the merge sort above.
template <typename K>
bool use_radix(uint64_t n) {
  return n > (uint64_t)SortCfg<K>::BS_TILE && n < kRadixMaxN;
}

template <typename K, typename P>
size_t sort_ws_bytes_t(uint64_t n) {
  return use_radix<K>(n) ? radix_sort_ws_bytes<K, P>(n) : merge_sort_ws_bytes_t<K, P>(n);
}

template <typename Kern>
static int set_smem(Kern kern, size_t bytes) {
  return host::set_smem_attrs(kern, bytes);
}

template <typename K>
int sort_passes(uint64_t n) {
  int passes = 0;
  for (uint64_t w = SortCfg<K>::BS_TILE; w < n; w *= 2) ++passes;
  return passes;
}

// Sets the kernels' shared-memory attributes once per device and returns (in *ahead)
// how many merge-pass CTAs are resident at once.
template <typename K, typename P, typename BsSrc, typename MpSrc>
int sort_set_attrs(uint64_t *ahead) {
  struct Site {};
  return host::once_per_device<Site>(ahead, [](uint64_t *mp_resident) -> int {
    int st;
    if ((st = set_smem(block_sort_kernel<K, P, BsSrc>, bs_smem_bytes<K, P>())) != BK_OK) return st;
    if ((st = set_smem(sort_merge_kernel<K, P, MpSrc>, mp_smem_bytes<K, P>())) != BK_OK) return st;
    host::DeviceInfo di;
    if ((st = host::device_info(&di)) != BK_OK) return st;
    *mp_resident =
        host::resident_ctas(sort_merge_kernel<K, P, MpSrc>, kMpThreads, mp_smem_bytes<K, P>(), di.sm_count);
    return BK_OK;
  });
}

template <typename K, typename P>
int sort_check_array(K *keys, P *vals, uint64_t n) {
  if (n > 0 && (keys == nullptr || (has_payload<P>() && vals == nullptr))) return BK_ERR_INVALID_ARGUMENT;
  if (!host::aligned_to<K>(keys)) return BK_ERR_MISALIGNED;
  if constexpr (has_payload<P>()) {
    if (!host::aligned_to<P>(vals)) return BK_ERR_MISALIGNED;
  }
  if ((n + SortCfg<K>::MP_TILE - 1) / SortCfg<K>::MP_TILE >= 0x7fffffffull) return BK_ERR_TOO_LARGE;
  return BK_OK;
}

template <typename K, typename P>
int sort_launch(K *keys, P *vals, uint64_t n, void *d_ws, size_t ws_bytes, cudaStream_t stream) {
  using C = SortCfg<K>;
  host::DeviceInfo di;
  int st = host::device_info(&di);
  if (st != BK_OK) return st;
  if (n <= 1) return BK_OK;
  if ((st = sort_check_array(keys, vals, n)) != BK_OK) return st;
  if (use_radix<K>(n)) return radix_sort_launch<K, P>(keys, vals, n, d_ws, ws_bytes, stream);
  const uint64_t bs_tiles = (n + C::BS_TILE - 1) / C::BS_TILE;
  const uint64_t mp_tiles = (n + C::MP_TILE - 1) / C::MP_TILE;
  st = host::check_ws(d_ws, ws_bytes, sort_ws_bytes_t<K, P>(n));
  if (st != BK_OK) return st;
  char *ws = reinterpret_cast<char *>(d_ws) + kHeaderBytes;
  K *tk = reinterpret_cast<K *>(ws);
  ws += align_up(n * sizeof(K), 256);
  P *tv = reinterpret_cast<P *>(ws);
  ws += align_up(n * (size_t)payload_bytes<P>(), 256);
  uint64_t *parts = reinterpret_cast<uint64_t *>(ws);
  const int passes = sort_passes<K>(n);
  uint64_t ahead = 0;
  if ((st = sort_set_attrs<K, P, BsOne<K, P>, MpOne<K, P>>(&ahead)) != BK_OK) return st;
  // an odd number of passes starts in the temporaries so the last lands in place
  K *ck = (passes & 1) ? tk : keys;
  P *cv = (passes & 1) ? tv : vals;
  block_sort_kernel<K, P, BsOne<K, P>><<<(unsigned)bs_tiles, kBsThreads, bs_smem_bytes<K, P>(), stream>>>(
      BsOne<K, P>{keys, vals, ck, cv, n});
  if ((st = host::launch_status()) != BK_OK) return st;
  for (uint64_t w = C::BS_TILE; w < n; w *= 2) {
    K *nk = (ck == keys) ? tk : keys;
    P *nv = (ck == keys) ? tv : vals;
    const MpOne<K, P> src{ck, cv, nk, nv, n, w, parts, mp_tiles};
    sort_partition_kernel<K, P, MpOne<K, P>><<<(unsigned)((mp_tiles + 255) / 256), 256, 0, stream>>>(src, mp_tiles);
    if ((st = host::launch_status()) != BK_OK) return st;
    sort_merge_kernel<K, P, MpOne<K, P>><<<(unsigned)mp_tiles, kMpThreads, mp_smem_bytes<K, P>(), stream>>>(src, ahead);
    if ((st = host::launch_status()) != BK_OK) return st;
    ck = nk;
    cv = nv;
  }
  return BK_OK;
}

// A batch item as the C-ABI passes it (bk_sort_item_<key>_<payload>).
template <typename K, typename P>
struct SortItem {
  K *keys;
  P *vals;
  uint64_t n;
};
// Out of place: in_keys / in_vals (left unchanged) sorted into keys / vals.
template <typename K, typename P>
struct SortCopyItem {
  const K *in_keys;
  const P *in_vals;
  K *keys;
  P *vals;
  uint64_t n;
};

// Workspace of a batch: per array (n > 1), its key and payload temporaries
// and its merge-pass splits, one after another.
template <typename K, typename P>
size_t merge_sort_batch_ws_bytes_t(const uint64_t *sizes, uint32_t count) {
  size_t b = kHeaderBytes;
  for (uint32_t i = 0; i < count; ++i) {
    const uint64_t n = sizes[i];
    if (n <= 1) continue;
    const uint64_t mp_tiles = (n + SortCfg<K>::MP_TILE - 1) / SortCfg<K>::MP_TILE;
    b += align_up(n * sizeof(K), 256) + align_up(n * (size_t)payload_bytes<P>(), 256) +
         align_up((mp_tiles + 1) * sizeof(uint64_t), 256);
  }
  return b;
}

// A batch uses the radix sort when all its arrays are below 2^30 elements
// and one needs more than a block tile; otherwise the merge sort (a single
// block-sort launch when every array fits one tile).
template <typename K, typename P>
bool sort_batch_radix(const uint64_t *sizes, uint32_t count) {
  bool any_large = false;
  for (uint32_t i = 0; i < count; ++i) {
    if (sizes[i] >= kRadixMaxN) return false;
    any_large = any_large || use_radix<K>(sizes[i]);
  }
  return any_large;
}

template <typename K, typename P>
size_t sort_batch_ws_bytes_t(const uint64_t *sizes, uint32_t count) {
  return sort_batch_radix<K, P>(sizes, count) ? radix_sort_batch_ws_bytes<K, P>(sizes, count)
                                              : merge_sort_batch_ws_bytes_t<K, P>(sizes, count);
}

template <typename K, typename P>
int sort_batch_copy_launch(const SortCopyItem<K, P> *items, uint32_t count, void *d_ws, size_t ws_bytes,
                           cudaStream_t stream);

// In place: the copy form with each array as its own source.
template <typename K, typename P>
int sort_batch_launch(const SortItem<K, P> *items, uint32_t count, void *d_ws, size_t ws_bytes, cudaStream_t stream) {
  if (count > 0 && items == nullptr) return BK_ERR_INVALID_ARGUMENT;
  if (count > (uint32_t)kSortBatchMax) return BK_ERR_TOO_LARGE;
  SortCopyItem<K, P> c[kSortBatchMax];
  for (uint32_t i = 0; i < count; ++i) c[i] = SortCopyItem<K, P>{items[i].keys, items[i].vals, items[i].keys, items[i].vals, items[i].n};
  return sort_batch_copy_launch<K, P>(c, count, d_ws, ws_bytes, stream);
}

template <typename K, typename P>
int sort_batch_copy_launch(const SortCopyItem<K, P> *items, uint32_t count, void *d_ws, size_t ws_bytes,
                           cudaStream_t stream) {
  using C = SortCfg<K>;
  if (count > 0 && items == nullptr) return BK_ERR_INVALID_ARGUMENT;
  if (count > (uint32_t)kSortBatchMax) return BK_ERR_TOO_LARGE;
  {
    uint64_t sizes[kSortBatchMax];
    for (uint32_t i = 0; i < count; ++i) sizes[i] = items[i].n;
    static_assert(sizeof(SortCopyItem<K, P>) == sizeof(RsItem<K, P>), "same item layout");
    if (sort_batch_radix<K, P>(sizes, count))
      return radix_sort_batch_launch<K, P>(reinterpret_cast<const RsItem<K, P> *>(items), count, d_ws, ws_bytes,
                                           stream);
  }
  host::DeviceInfo di;
  int st = host::device_info(&di);
  if (st != BK_OK) return st;
  // the arrays that need sorting, with their temporaries
  struct Arr {
    K *keys;
    P *vals;
    uint64_t n;
    K *tk;
    P *tv;
    uint64_t *parts;
    int passes;
  };
  Arr arr[kSortBatchMax];
  uint32_t na = 0;
  uint64_t sizes[kSortBatchMax];
  for (uint32_t i = 0; i < count; ++i) {
    if ((st = sort_check_array(items[i].keys, items[i].vals, items[i].n)) != BK_OK) return st;
    if ((st = sort_check_array(const_cast<K *>(items[i].in_keys), const_cast<P *>(items[i].in_vals), items[i].n)) !=
        BK_OK)
      return st;
    sizes[i] = items[i].n;
  }
  st = host::check_ws(d_ws, ws_bytes, merge_sort_batch_ws_bytes_t<K, P>(sizes, count));
  if (st != BK_OK) return st;
  char *ws = reinterpret_cast<char *>(d_ws) + kHeaderBytes;
  int max_passes = 0;
  size_t bs_total = 0;
  BsBatch<K, P> bs;
  bs.count = 0;
  for (uint32_t i = 0; i < count; ++i) {
    const uint64_t n = items[i].n;
    if (n == 1 && items[i].in_keys != items[i].keys) {  // a single element out of place: copied
      if ((st = host::from_cuda(cudaMemcpyAsync(items[i].keys, items[i].in_keys, sizeof(K), cudaMemcpyDeviceToDevice,
                                                stream))) != BK_OK)
        return st;
      if constexpr (has_payload<P>()) {
        if ((st = host::from_cuda(cudaMemcpyAsync(items[i].vals, items[i].in_vals, sizeof(P),
                                                  cudaMemcpyDeviceToDevice, stream))) != BK_OK)
          return st;
      }
    }
    if (n <= 1) continue;  // already sorted
    Arr &a = arr[na++];
    a.keys = items[i].keys;
    a.vals = items[i].vals;
    a.n = n;
    a.tk = reinterpret_cast<K *>(ws);
    ws += align_up(n * sizeof(K), 256);
    a.tv = reinterpret_cast<P *>(ws);
    ws += align_up(n * (size_t)payload_bytes<P>(), 256);
    a.parts = reinterpret_cast<uint64_t *>(ws);
    ws += align_up(((n + C::MP_TILE - 1) / C::MP_TILE + 1) * sizeof(uint64_t), 256);
    a.passes = sort_passes<K>(n);
    max_passes = a.passes > max_passes ? a.passes : max_passes;
    // an odd number of passes starts in the temporaries so the last lands in place
    const uint32_t k = bs.count++;
    bs.in_k[k] = items[i].in_keys;  // the block sort reads the source (the array itself in place)
    bs.in_v[k] = items[i].in_vals;
    bs.out_k[k] = (a.passes & 1) ? a.tk : a.keys;
    bs.out_v[k] = (a.passes & 1) ? a.tv : a.vals;
    bs.n[k] = n;
    bs.start[k] = (uint32_t)bs_total;
    bs_total += (n + C::BS_TILE - 1) / C::BS_TILE;
  }
  if (na == 0) return BK_OK;
  bs.start[bs.count] = (uint32_t)bs_total;
  if (bs_total >= 0x7fffffffull) return BK_ERR_TOO_LARGE;
  uint64_t ahead = 0;
  if ((st = sort_set_attrs<K, P, BsBatch<K, P>, MpBatch<K, P>>(&ahead)) != BK_OK) return st;
  block_sort_kernel<K, P, BsBatch<K, P>><<<(unsigned)bs_total, kBsThreads, bs_smem_bytes<K, P>(), stream>>>(bs);
  if ((st = host::launch_status()) != BK_OK) return st;
  // pass p merges runs of width BS_TILE << p for every array with more than p passes
  for (int p = 0; p < max_passes; ++p) {
    MpBatch<K, P> mp;
    mp.count = 0;
    mp.w = (uint64_t)C::BS_TILE << p;
    size_t mp_total = 0;
    for (uint32_t j = 0; j < na; ++j) {
      const Arr &a = arr[j];
      if (a.passes <= p) continue;
      // after the block sort the data is in the temporaries iff passes is odd;
      // each pass moves it to the other buffer
      const bool from_tmp = ((a.passes - p) & 1) != 0;
      const uint32_t k = mp.count++;
      mp.src_k[k] = from_tmp ? a.tk : a.keys;
      mp.src_v[k] = from_tmp ? a.tv : a.vals;
      mp.dst_k[k] = from_tmp ? a.keys : a.tk;
      mp.dst_v[k] = from_tmp ? a.vals : a.tv;
      mp.n[k] = a.n;
      mp.parts[k] = a.parts;
      mp.start[k] = (uint32_t)mp_total;
      mp_total += (a.n + C::MP_TILE - 1) / C::MP_TILE;
    }
    mp.start[mp.count] = (uint32_t)mp_total;
    if (mp_total >= 0x7fffffffull) return BK_ERR_TOO_LARGE;
    sort_partition_kernel<K, P, MpBatch<K, P>><<<(unsigned)((mp_total + 255) / 256), 256, 0, stream>>>(mp, mp_total);
    if ((st = host::launch_status()) != BK_OK) return st;
    sort_merge_kernel<K, P, MpBatch<K, P>><<<(unsigned)mp_total, kMpThreads, mp_smem_bytes<K, P>(), stream>>>(mp, ahead);
    if ((st = host::launch_status()) != BK_OK) return st;
  }
  return BK_OK;
}

size_t sort_batch_workspace_bytes(int key_dtype, int value_dtype, const uint64_t *sizes, uint32_t count) {
  if (count > 0 && sizes == nullptr) return 0;
  const bool k4 = key_dtype == BK_DTYPE_I32 || key_dtype == BK_DTYPE_U32 || key_dtype == BK_DTYPE_F32;
  const bool k8 = key_dtype == BK_DTYPE_I64 || key_dtype == BK_DTYPE_U64 || key_dtype == BK_DTYPE_F64;
  const bool v4 = value_dtype == BK_DTYPE_I32 || value_dtype == BK_DTYPE_U32 || value_dtype == BK_DTYPE_F32;
  const bool v8 = value_dtype == BK_DTYPE_I64 || value_dtype == BK_DTYPE_U64 || value_dtype == BK_DTYPE_F64;
  if (k4) return v4 ? sort_batch_ws_bytes_t<float, uint32_t>(sizes, count)
                 : v8 ? sort_batch_ws_bytes_t<float, unsigned long long>(sizes, count) : 0;
  if (k8) return v4 ? sort_batch_ws_bytes_t<double, uint32_t>(sizes, count)
                 : v8 ? sort_batch_ws_bytes_t<double, unsigned long long>(sizes, count) : 0;
  return 0;
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

#define BK_DEFINE_SORT_BATCH(KN, K, VN, V, VI)                                                                  \
  static_assert(sizeof(bk_sort_item_##KN##_##VN) == sizeof(bk::SortItem<K, VI>), "bk_sort_item layout");     \
  extern "C" int bk_sort_by_key_##KN##_##VN##_batch(const bk_sort_item_##KN##_##VN *items, uint32_t count,    \
                                                    void *d_ws, size_t ws_bytes, bk_stream_t stream) {       \
    return bk::sort_batch_launch<K, VI>(reinterpret_cast<const bk::SortItem<K, VI> *>(items), count, d_ws,    \
                                        ws_bytes, (cudaStream_t)stream);                                      \
  }
#define BK_DEFINE_SORT_COPY_BATCH(KN, K, VN, V, VI)                                                             \
  static_assert(sizeof(bk_sort_copy_item_##KN##_##VN) == sizeof(bk::SortCopyItem<K, VI>), "bk_sort_copy_item");  \
  extern "C" int bk_sort_by_key_##KN##_##VN##_copy_batch(const bk_sort_copy_item_##KN##_##VN *items,          \
                                                         uint32_t count, void *d_ws, size_t ws_bytes,          \
                                                         bk_stream_t stream) {                                 \
    return bk::sort_batch_copy_launch<K, VI>(reinterpret_cast<const bk::SortCopyItem<K, VI> *>(items), count,   \
                                             d_ws, ws_bytes, (cudaStream_t)stream);                             \
  }
#define BK_DEFINE_SORT_BATCH_K(KN, K)                                 \
  BK_DEFINE_SORT_BATCH(KN, K, u32, uint32_t, uint32_t)                \
  BK_DEFINE_SORT_BATCH(KN, K, u64, uint64_t, unsigned long long)      \
  BK_DEFINE_SORT_COPY_BATCH(KN, K, u32, uint32_t, uint32_t)           \
  BK_DEFINE_SORT_COPY_BATCH(KN, K, u64, uint64_t, unsigned long long)

BK_DEFINE_SORT_BATCH_K(i32, int32_t)
BK_DEFINE_SORT_BATCH_K(u32, uint32_t)
BK_DEFINE_SORT_BATCH_K(i64, int64_t)
BK_DEFINE_SORT_BATCH_K(u64, uint64_t)
BK_DEFINE_SORT_BATCH_K(f32, float)
BK_DEFINE_SORT_BATCH_K(f64, double)
