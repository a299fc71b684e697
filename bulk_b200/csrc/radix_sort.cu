// radix_sort.cu -- stable LSD radix sort by key (the sort_by_key entry
// points below 2^30 elements), sm_100a.
//
// The reference sorts by merging (stable_merge_sort_by_key,
// merge_sort_by_key.cu:150-209): ceil(log2(n / 896)) global passes, 17 at
// 2^26.  A stable sort's output is unique -- equal keys keep their input
// order -- so a stable least-significant-digit radix sort gives exactly the
// same keys and payloads, in sizeof(K) passes of 8 bits instead: 4 for 32-bit
// keys, 8 for 64-bit ones.  Keys are mapped to unsigned integers with the same
// order (signed: flip the sign bit; floating point: flip all bits of
// negatives and the sign bit of the rest, with -0.0 read as +0.0 so that the
// two zeros tie as they do under operator<).  Keys must not be NaN.
//
// One pass over tiles of 4096 keys is three steps with no serial dependency
// between tiles:
//   upsweep    each tile counts its keys per digit; the counts are stored
//              digit-major (count of digit d in tile t at d * tiles + t);
//   scan       one inclusive sum scan of all counts (the library's own u32
//              scan): in digit-major order the scanned value of (d, t) minus
//              the count itself is exactly where tile t's keys of digit d
//              start in the output;
//   downsweep  each tile ranks its keys by digit (the lanes of a warp that
//              share a digit are found with eight ballots; per-warp counters
//              keep input order inside a digit), stages them in shared memory
//              in digit order and writes each digit's run contiguously to its
//              position.
// A batch lays its arrays' count regions one after another, so the one scan
// serves all of them: an array's positions are the scanned values minus the
// number of elements of the arrays before it.
//
// A single array of up to 131,072 keys is sorted instead by one launch of one
// thread-block cluster whose CTAs exchange their digit counts through
// distributed shared memory (rs_cluster_kernel below).
#include <type_traits>

#include "bk_common.cuh"
#include "bk_tune.hpp"
#include "bk_merge.cuh"  // NoPayload, has_payload, payload_bytes
#include "bk_tma.cuh"    // smem_addr
#include "bulk_b200.h"

namespace bk {

constexpr int kRsThreads = 256;
constexpr int kRsItems = 16;
constexpr int kRsTile = kRsThreads * kRsItems;  // 4096 keys
constexpr int kRsBins = 256;                    // 8-bit digits
constexpr int kRsWarps = kRsThreads / 32;
constexpr uint64_t kRsMaxN = 1ull << 30;
constexpr int kRsBatchMax = 256;

// Order-preserving map of a key to an unsigned integer.
template <typename K>
struct RadixKey;
template <>
struct RadixKey<uint32_t> {
  using U = uint32_t;
  static __device__ __forceinline__ U to(uint32_t k) { return k; }
};
template <>
struct RadixKey<int32_t> {
  using U = uint32_t;
  static __device__ __forceinline__ U to(int32_t k) { return (uint32_t)k ^ 0x80000000u; }
};
template <>
struct RadixKey<float> {
  using U = uint32_t;
  static __device__ __forceinline__ U to(float k) {
    uint32_t b = __float_as_uint(k);
    if (b == 0x80000000u) b = 0u;  // -0.0 ties with +0.0
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
  }
};
template <>
struct RadixKey<uint64_t> {
  using U = uint64_t;
  static __device__ __forceinline__ U to(uint64_t k) { return k; }
};
template <>
struct RadixKey<int64_t> {
  using U = uint64_t;
  static __device__ __forceinline__ U to(int64_t k) { return (uint64_t)k ^ 0x8000000000000000ull; }
};
template <>
struct RadixKey<double> {
  using U = uint64_t;
  static __device__ __forceinline__ U to(double k) {
    uint64_t b = (uint64_t)__double_as_longlong(k);
    if (b == 0x8000000000000000ull) b = 0ull;
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
  }
};

template <typename K>
constexpr int rs_passes() {
  return (int)sizeof(K);  // 8-bit digits
}

template <typename K>
__device__ __forceinline__ int rs_digit(K k, int shift) {
  return (int)((RadixKey<K>::to(k) >> shift) & (kRsBins - 1));
}

// Lanes of the warp whose 8-bit digit equals this lane's, from eight
// ballots (__match_any_sync gives the same mask, but on a unit that
// saturated at one match a key here).
__device__ __forceinline__ unsigned int rs_peers(unsigned int d) {
  unsigned int peers = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const bool set = (d >> b) & 1u;
    const unsigned int m = __ballot_sync(0xffffffffu, set);
    peers &= set ? m : ~m;
  }
  return peers;
}

// A tile of one pass: its array (keys and temporaries: even passes read the
// keys, odd passes the temporaries), length, local index, and where the
// array's digit counts and elements start in the batch.
template <typename K, typename P>
struct RsTile {
  K *keys;
  P *vals;
  K *tk;
  P *tv;
  const K *src_k;       // what the first pass reads (keys, or a separate source)
  const P *src_v;
  uint64_t n;
  uint32_t local;
  uint32_t tiles;       // the array's tiles
  uint64_t count_base;  // first count of the array (its digit-major region)
  uint32_t elem_base;   // elements of the arrays before it (mod 2^32)
};

template <typename K, typename P>
struct RsOne {
  K *keys;
  P *vals;
  K *tk;
  P *tv;
  uint64_t n;
  uint32_t tiles;
  __device__ __forceinline__ RsTile<K, P> tile(unsigned int g) const {
    return RsTile<K, P>{keys, vals, tk, tv, keys, vals, n, g, tiles, 0ull, 0u};
  }
};

// A batch: array i owns global tiles [start[i], start[i + 1]).
template <typename K, typename P>
struct RsBatch {
  K *keys[kRsBatchMax];
  P *vals[kRsBatchMax];
  const K *src_k[kRsBatchMax];  // what the first pass reads
  const P *src_v[kRsBatchMax];
  K *tk[kRsBatchMax];
  P *tv[kRsBatchMax];
  uint64_t n[kRsBatchMax];
  uint32_t elem_base[kRsBatchMax];
  uint32_t start[kRsBatchMax + 1];
  uint32_t count;
  __device__ __forceinline__ RsTile<K, P> tile(unsigned int g) const {
    int lo = 0, hi = (int)count - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (start[mid] <= g) lo = mid;
      else hi = mid - 1;
    }
    return RsTile<K, P>{keys[lo], vals[lo], tk[lo], tv[lo], src_k[lo], src_v[lo], n[lo], g - start[lo],
                        start[lo + 1] - start[lo],
                        (uint64_t)start[lo] * kRsBins, elem_base[lo]};
  }
};

// Upsweep: the tile's count of every digit, stored digit-major.  Keys are
// read warp-striped (element w*512 + j*32 + lane: coalesced) and counted with
// shared-memory atomics into one histogram per warp; a warp whose 32 keys
// share one digit adds 32 with one atomic (constant high digits are common).
// Tile g's keys (and payloads) of this pass into L2, for the CTA that will
// start about when every CTA now resident has finished.
template <typename K, typename P, typename Src>
__device__ __forceinline__ void rs_prefetch_tile(const Src &src, unsigned int g, int pass, bool payload) {
  if (g >= gridDim.x) return;
  const RsTile<K, P> f = src.tile(g);
  const uint64_t base = (uint64_t)f.local * kRsTile;
  const uint64_t cnt = (f.n - base) < (uint64_t)kRsTile ? (f.n - base) : (uint64_t)kRsTile;
  prefetch_l2_range(((pass & 1) ? f.tk : (pass == 0 ? f.src_k : f.keys)) + base, cnt * sizeof(K));
  if constexpr (has_payload<P>()) {
    if (payload) prefetch_l2_range(((pass & 1) ? f.tv : (pass == 0 ? f.src_v : f.vals)) + base, cnt * sizeof(P));
  }
}

// Six CTAs per SM (40 registers) for 4-byte keys on one array: the u32/u32
// sort at 2^26 ran 1.1 % faster than with five (48 registers) on a B200;
// 8-byte keys and a batch's tile lookup would spill there and keep five.
template <typename K, typename P, typename Src>
constexpr int rs_up_min_blocks() {
  return sizeof(K) == 4 && std::is_same<Src, RsOne<K, P>>::value ? 6 : 5;
}
template <typename K, typename P, typename Src>
__global__ void __launch_bounds__(kRsThreads, rs_up_min_blocks<K, P, Src>()) rs_upsweep_kernel(const __grid_constant__ Src src, int pass,
                                                                unsigned int *counts, unsigned int ahead) {
  __shared__ unsigned int s_wcnt[kRsWarps][kRsBins];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int shift = 8 * pass;
  if (tid == 0 && ahead != 0) rs_prefetch_tile<K, P>(src, blockIdx.x + ahead, pass, false);
  const RsTile<K, P> tl = src.tile(blockIdx.x);
  const K *in_k = (pass & 1) ? tl.tk : (pass == 0 ? tl.src_k : tl.keys);
  const uint64_t tbase = (uint64_t)tl.local * kRsTile;
  const int count = (int)((tl.n - tbase) < (uint64_t)kRsTile ? (tl.n - tbase) : (uint64_t)kRsTile);
#pragma unroll
  for (int w = 0; w < kRsWarps; ++w) s_wcnt[w][tid] = 0u;
  __syncthreads();
  K k[kRsItems];
#pragma unroll
  for (int j = 0; j < kRsItems; ++j) {
    const int e = warp * 32 * kRsItems + j * 32 + lane;
    k[j] = e < count ? in_k[tbase + e] : K();
  }
#pragma unroll
  for (int j = 0; j < kRsItems; ++j) {
    const bool valid = warp * 32 * kRsItems + j * 32 + lane < count;
    const unsigned int d = (unsigned int)rs_digit(k[j], shift);
    const unsigned int d0 = __shfl_sync(0xffffffffu, d, 0);
    if (__all_sync(0xffffffffu, valid && d == d0)) {
      if (lane == 0) atomicAdd(&s_wcnt[warp][d0], 32u);
    } else if (valid) {
      atomicAdd(&s_wcnt[warp][d], 1u);
    }
  }
  __syncthreads();
  unsigned int c = 0;
#pragma unroll
  for (int w = 0; w < kRsWarps; ++w) c += s_wcnt[w][tid];
  counts[tl.count_base + (uint64_t)tid * tl.tiles + tl.local] = c;
}

// Downsweep: stable scatter by digit (keys -> temporaries on even passes,
// back on odd ones) to the positions the scan gave.  If the count scan
// reported an error its positions are not trusted: the pass writes nothing
// and the error is copied into the sort's own workspace header.
template <int TH, typename K, typename P>
constexpr int rs_down_min_blocks() {
  return TH == 512 ? 2 : (sizeof(K) == 4 && payload_bytes<P>() <= 4 ? 3 : 2);
}
// TH threads; V = 1 finds every item's peers before the ranking chain
// (more registers, more independent ballots), V = 0 item by item.
template <typename K, typename P, typename Src, int V, int TH>
__global__ void __launch_bounds__(TH, rs_down_min_blocks<TH, K, P>()) rs_downsweep_kernel(
    const __grid_constant__ Src src, int pass, const unsigned int *scanned, const WsHeader *scan_hdr,
    WsHeader *hdr, unsigned int ahead) {
  constexpr int ITEMS = kRsTile / TH, WARPS = TH / 32;
  extern __shared__ __align__(16) unsigned char smem[];
  K *sk = reinterpret_cast<K *>(smem);  // the tile in digit order
  P *sv = reinterpret_cast<P *>(smem + align_up(sizeof(K) * kRsTile, 16));
  __shared__ unsigned int s_whist[WARPS][kRsBins];  // per-warp digit counters
  __shared__ unsigned int s_dst[kRsBins];  // output position of tile position 0 for digit d (mod 2^32)
  __shared__ unsigned int s_scan[TH / 32 + 1];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int scan_status = scan_hdr->status;
  if (scan_status != 0) {
    if (tid == 0) record_error(hdr, scan_status, blockIdx.x);
    return;
  }
  const int shift = 8 * pass;
  if (tid == 0 && ahead != 0) rs_prefetch_tile<K, P>(src, blockIdx.x + ahead, pass, true);
  const RsTile<K, P> tl = src.tile(blockIdx.x);
  const K *in_k = (pass & 1) ? tl.tk : (pass == 0 ? tl.src_k : tl.keys);
  const P *in_v = (pass & 1) ? tl.tv : (pass == 0 ? tl.src_v : tl.vals);
  K *out_k = (pass & 1) ? tl.keys : tl.tk;
  P *out_v = (pass & 1) ? tl.vals : tl.tv;
  const uint64_t tbase = (uint64_t)tl.local * kRsTile;
  const int count = (int)((tl.n - tbase) < (uint64_t)kRsTile ? (tl.n - tbase) : (uint64_t)kRsTile);
  for (int i = tid; i < WARPS * kRsBins; i += TH) (&s_whist[0][0])[i] = 0u;
  __syncthreads();

  // The tile body, compiled twice: for full tiles (no bounds checks) and for
  // an array's last, partial tile.
  auto body = [&](auto full_tag) {
    constexpr bool FULL = decltype(full_tag)::value;
    K k[ITEMS];
    P v[ITEMS];
    auto elem = [&](int j) { return warp * 32 * ITEMS + j * 32 + lane; };
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const bool ok = FULL || elem(j) < count;
      k[j] = ok ? in_k[tbase + elem(j)] : K();
      if constexpr (has_payload<P>()) v[j] = ok ? in_v[tbase + elem(j)] : P();
    }
    // the items' digits, four to a register.  Past the tile's end the digit
    // is 255: those items come after every real one in (warp, item, lane)
    // order, so they rank last in the tile and are never written out.
    uint32_t dig4[ITEMS / 4];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const uint32_t dj = (FULL || elem(j) < count) ? (uint32_t)rs_digit(k[j], shift) : kRsBins - 1u;
      if (j & 3) dig4[j >> 2] |= dj << (8 * (j & 3));
      else dig4[j >> 2] = dj;
    }
    auto digit_of = [&](int j) { return (int)((dig4[j >> 2] >> (8 * (j & 3))) & 0xffu); };
    // rank within the warp: keys of one digit in input order (a rank is
    // below 512, so two share a register).  The lowest lane of each digit
    // reserves the digit's keys in the warp's counter; the shuffle that hands
    // the old count to the other lanes also orders item j's atomic before
    // item j+1's.
    unsigned int rank2[ITEMS / 2];
    const unsigned int lt = (1u << lane) - 1u;
    unsigned int pm[V == 1 ? ITEMS : 1];
    if constexpr (V == 1) {
#pragma unroll
      for (int j = 0; j < ITEMS; ++j) pm[j] = rs_peers((unsigned int)digit_of(j));
    }
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const int dj = digit_of(j);
      unsigned int peers;
      if constexpr (V == 1) peers = pm[j];
      else peers = rs_peers((unsigned int)dj);
      const int leader = __ffs(peers) - 1;
      unsigned int before = 0;
      if (lane == leader) before = atomicAdd(&s_whist[warp][dj], (unsigned int)__popc(peers));
      before = __shfl_sync(0xffffffffu, before, leader);
      const unsigned int r = before + __popc(peers & lt);
      if (j & 1) rank2[j >> 1] |= r << 16;
      else rank2[j >> 1] = r;
    }
    __syncthreads();

    // thread d < 256: the digit's tile count, then its start in the staged
    // tile for each warp (the tile's exclusive count plus the warps before)
    const int d = tid;
    unsigned int cnt = 0;
    if (d < kRsBins) {
#pragma unroll
      for (int w = 0; w < WARPS; ++w) cnt += s_whist[w][d];
    }
    unsigned int tile_total;
    const unsigned int tile_excl = block_exclusive_scan<TH>(cnt, OpSum<unsigned int>(), s_scan, tile_total);
    if (d < kRsBins) {
      unsigned int run = tile_excl;
#pragma unroll
      for (int w = 0; w < WARPS; ++w) {
        const unsigned int c = s_whist[w][d];
        s_whist[w][d] = run;
        run += c;
      }
      if (!FULL && d == kRsBins - 1) cnt -= (unsigned int)(kRsTile - count);  // real keys of digit 255
      const unsigned int incl = scanned[tl.count_base + (uint64_t)d * tl.tiles + tl.local];
      s_dst[d] = incl - cnt - tl.elem_base - tile_excl;
    }
    __syncthreads();

    // stage in digit order
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const int dj = digit_of(j);
      const unsigned int rank = (rank2[j >> 1] >> (16 * (j & 1))) & 0xffffu;
      const unsigned int pos = s_whist[warp][dj] + rank;
      sk[pos] = k[j];
      if constexpr (has_payload<P>()) sv[pos] = v[j];
    }
    __syncthreads();
    // write out: position p of the staged tile goes to s_dst[digit] + p
#pragma unroll 4
    for (int p = tid; p < (FULL ? kRsTile : count); p += TH) {
      const K key = sk[p];
      const uint64_t g = (uint64_t)(s_dst[rs_digit(key, shift)] + (unsigned int)p);
      if (g < tl.n) {  // always true when the counts are consistent
        out_k[g] = key;
        if constexpr (has_payload<P>()) out_v[g] = sv[p];
      }
    }
  };
  if (count == kRsTile) body(std::true_type{});
  else body(std::false_type{});
}

// ---------------------------------------------------------------------------
// Small arrays (up to 16 tiles of 4096 or 8192 keys): every pass in one launch
// of one thread-block cluster, one CTA per tile.  The CTAs exchange their digit counts through
// distributed shared memory (each reads every other CTA's 256 counts across
// the cluster) instead of a count scan in global memory, and a cluster barrier
// takes the place of each kernel boundary: two barriers a pass replace the
// three launches a pass of the global-memory path takes.  The keys move
// between passes through the workspace temporaries, which stay in L2 at these
// sizes (storing each key straight into the owning CTA's shared memory was
// measured slower: 42.9 against 32.8 us for 2^16 u32/u32 keys on a B200).
constexpr int kRsClusterMax = 16;  // CTAs (non-portable above 8)
constexpr int kRsClThreads = 1024;  // four or eight items a thread: short ranking chains, 32 warps an SM

__device__ __forceinline__ uint32_t rs_cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t rs_cluster_size() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
// Barrier over every thread of the cluster; earlier shared-memory writes
// (local and remote) are visible to every thread after it.
__device__ __forceinline__ void rs_cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// Address of `local` (this CTA's shared memory) in CTA `rank`'s window.
__device__ __forceinline__ uint32_t rs_peer_addr(const void *local, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_addr(local)), "r"(rank));
  return r;
}
// Load from another CTA's shared memory.  The cluster barriers around its
// uses order it, so it has no memory clobber and one thread's loads may all
// be in flight at once.
__device__ __forceinline__ uint32_t rs_peer_ld_u32(uint32_t a) {
  uint32_t v;
  asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(a));
  return v;
}
// Exclusive sum scan of v over threads 0-255 of the CTA (the digit threads;
// the other warps do not take part), with the total; s_w holds 8 words.
__device__ __forceinline__ unsigned int rs_scan_digits(unsigned int v, unsigned int *s_w, unsigned int &total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned int incl = warp_inclusive_scan(v, OpSum<unsigned int>(), lane);
  if (lane == 31) s_w[warp] = incl;
  named_barrier_sync(1, kRsBins);
  unsigned int pre = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < kRsBins / 32; ++w) {
    const unsigned int x = s_w[w];
    tot += x;
    if (w < warp) pre += x;
  }
  total = tot;
  return pre + incl - v;
}
// Shared memory of a cluster-sort CTA of ITEMS items a thread: one tile
// (1024 * ITEMS keys and payloads).
template <typename K, typename P, int ITEMS>
constexpr size_t rs_cluster_smem_bytes() {
  return align_up(sizeof(K) * kRsClThreads * ITEMS, 16) + (size_t)payload_bytes<P>() * kRsClThreads * ITEMS;
}

// The cluster sort: CTA r of the cluster owns tile r.  Each pass reads the
// tile from the pass's input (the array on even passes, the workspace
// temporaries on odd ones; all L2-resident at these sizes), ranks its keys as
// the scatter above does (ITEMS items a thread), exchanges its 256 digit
// counts with the other CTAs through distributed shared memory, stages the
// tile in digit order and writes each digit's run to the pass's output.  The
// cluster barrier after the writes (release / acquire at cluster scope) makes
// them visible to the CTA that reads that tile next.  Even passes end in the
// array, so the last one leaves the result in place.
template <typename K, typename P, int ITEMS>
__global__ void __launch_bounds__(kRsClThreads, 1) rs_cluster_kernel(K *keys, P *vals, K *tk, P *tv, uint32_t n) {
  constexpr int WARPS = kRsClThreads / 32, TILE = kRsClThreads * ITEMS;
  constexpr size_t VOFF = align_up(sizeof(K) * TILE, 16);
  extern __shared__ __align__(16) unsigned char rs_cl_smem[];
  K *sk = reinterpret_cast<K *>(rs_cl_smem);  // the tile in digit order
  P *sv = reinterpret_cast<P *>(rs_cl_smem + VOFF);
  __shared__ unsigned int s_whist[WARPS][kRsBins];  // per-warp digit counters, then staging starts
  __shared__ unsigned int s_cnt[kRsBins];           // this tile's count of each digit (read by the peers)
  __shared__ unsigned int s_dst[kRsBins];           // output position of staged position 0 for digit d
  __shared__ unsigned int s_scan[2 * (kRsBins / 32)];  // the two digit scans' warp totals
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t me = rs_cluster_rank(), csize = rs_cluster_size();
  const uint32_t base = me * (uint32_t)TILE;
  const int count = (int)((n - base) < (uint32_t)TILE ? (n - base) : (uint32_t)TILE);
  for (int i = tid; i < WARPS * kRsBins; i += kRsClThreads) (&s_whist[0][0])[i] = 0u;
  __syncthreads();
  const unsigned int lt = (1u << lane) - 1u;
  for (int pass = 0; pass < rs_passes<K>(); ++pass) {
    const int shift = 8 * pass;
    const K *in_k = (pass & 1) ? tk : keys;
    const P *in_v = (pass & 1) ? tv : vals;
    K *out_k = (pass & 1) ? keys : tk;
    P *out_v = (pass & 1) ? vals : tv;
    K k[ITEMS];
    P v[ITEMS];
    auto elem = [&](int j) { return warp * 32 * ITEMS + j * 32 + lane; };
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const bool ok = elem(j) < count;
      k[j] = ok ? __ldcg(in_k + base + elem(j)) : K();
      if constexpr (has_payload<P>()) v[j] = ok ? __ldcg(in_v + base + elem(j)) : P();
    }
    uint32_t dig4[ITEMS / 4];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const uint32_t dj = elem(j) < count ? (uint32_t)rs_digit(k[j], shift) : kRsBins - 1u;
      if (j & 3) dig4[j >> 2] |= dj << (8 * (j & 3));
      else dig4[j >> 2] = dj;
    }
    auto digit_of = [&](int j) { return (int)((dig4[j >> 2] >> (8 * (j & 3))) & 0xffu); };
    unsigned int rank2[ITEMS / 2];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const int dj = digit_of(j);
      const unsigned int peers = rs_peers((unsigned int)dj);
      const int leader = __ffs(peers) - 1;
      unsigned int before = 0;
      if (lane == leader) before = atomicAdd(&s_whist[warp][dj], (unsigned int)__popc(peers));
      before = __shfl_sync(0xffffffffu, before, leader);
      const unsigned int r = before + __popc(peers & lt);
      if (j & 1) rank2[j >> 1] |= r << 16;
      else rank2[j >> 1] = r;
    }
    __syncthreads();
    const int d = tid;
    unsigned int tile_excl = 0;
    if (d < kRsBins) {
      unsigned int cnt = 0;
#pragma unroll
      for (int w = 0; w < WARPS; ++w) cnt += s_whist[w][d];
      unsigned int tile_total;
      tile_excl = rs_scan_digits(cnt, s_scan, tile_total);
      unsigned int run = tile_excl;
#pragma unroll
      for (int w = 0; w < WARPS; ++w) {
        const unsigned int c = s_whist[w][d];
        s_whist[w][d] = run;
        run += c;
      }
      s_cnt[d] = d == kRsBins - 1 ? cnt - (unsigned int)(TILE - count) : cnt;
    }
    rs_cluster_sync();
    if (d < kRsBins) {
      unsigned int c[kRsClusterMax];
#pragma unroll
      for (int q = 0; q < kRsClusterMax; ++q)
        c[q] = (uint32_t)q < csize ? rs_peer_ld_u32(rs_peer_addr(&s_cnt[d], (uint32_t)q)) : 0u;
      unsigned int before = 0, total = 0;
#pragma unroll
      for (int q = 0; q < kRsClusterMax; ++q) {
        total += c[q];
        if ((uint32_t)q < me) before += c[q];
      }
      unsigned int all;
      const unsigned int start = rs_scan_digits(total, s_scan + kRsBins / 32, all);
      s_dst[d] = start + before - tile_excl;
    }
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const int dj = digit_of(j);
      const unsigned int pos = s_whist[warp][dj] + ((rank2[j >> 1] >> (16 * (j & 1))) & 0xffffu);
      sk[pos] = k[j];
      if constexpr (has_payload<P>()) sv[pos] = v[j];
    }
    __syncthreads();
    for (int i = tid; i < WARPS * kRsBins; i += kRsClThreads) (&s_whist[0][0])[i] = 0u;
    for (int p = tid; p < count; p += kRsClThreads) {
      const K key = sk[p];
      const uint32_t g = s_dst[rs_digit(key, shift)] + (uint32_t)p;
      if (g < n) {
        out_k[g] = key;
        if constexpr (has_payload<P>()) out_v[g] = sv[p];
      }
    }
    rs_cluster_sync();
  }
}

// Once per device: the largest cluster (16 or 8 CTAs, 0 for none) that the
// cluster sort can be launched with, for tiles of 1024 * ITEMS keys.
template <typename K, typename P, int ITEMS>
int rs_cluster_setup(int *max_ctas) {
  struct Site {};
  return host::once_per_device<Site>(max_ctas, [](int *mx) -> int {
    auto kern = rs_cluster_kernel<K, P, ITEMS>;
    constexpr size_t smem = rs_cluster_smem_bytes<K, P, ITEMS>();
    int st;
    if ((st = host::set_smem_attrs(kern, smem)) != BK_OK) return st;
    *mx = 0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
      (void)cudaGetLastError();
    for (int c : {kRsClusterMax, 8}) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)c);
      cfg.blockDim = dim3(kRsClThreads);
      cfg.dynamicSmemBytes = smem;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = (unsigned)c;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int clusters = 0;
      if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess) {
        (void)cudaGetLastError();
        continue;
      }
      if (clusters > 0) {
        *mx = c;
        break;
      }
    }
    return BK_OK;
  });
}

// The cluster sort of n elements (n <= 1024 * ITEMS * max_ctas), one launch;
// tk / tv are the workspace temporaries of n elements.
template <typename K, typename P, int ITEMS>
int rs_cluster_launch(K *keys, P *vals, K *tk, P *tv, uint64_t n, cudaStream_t stream) {
  constexpr uint64_t TILE = (uint64_t)kRsClThreads * ITEMS;
  const unsigned c = (unsigned)((n + TILE - 1) / TILE);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(c);
  cfg.blockDim = dim3(kRsClThreads);
  cfg.dynamicSmemBytes = rs_cluster_smem_bytes<K, P, ITEMS>();
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = c;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return host::from_cuda(cudaLaunchKernelEx(&cfg, rs_cluster_kernel<K, P, ITEMS>, keys, vals, tk, tv, (uint32_t)n));
}

template <typename K, typename P>
constexpr size_t rs_smem_bytes() {
  return align_up(sizeof(K) * kRsTile, 16) + (size_t)payload_bytes<P>() * kRsTile;
}

// Workspace (after the 256-byte header): every array's key and payload
// temporaries, the digit counts of all tiles, and the count scan's workspace.
template <typename K, typename P>
struct RsLayout {
  size_t tmp, counts, scan_ws, scan_ws_bytes, total;
  uint64_t tiles;
  RsLayout(const uint64_t *sizes, uint32_t count) {
    size_t o = kHeaderBytes;
    tmp = o;
    tiles = 0;
    for (uint32_t i = 0; i < count; ++i) {
      o += align_up(sizes[i] * sizeof(K), 256) + align_up(sizes[i] * (size_t)payload_bytes<P>(), 256);
      tiles += (sizes[i] + kRsTile - 1) / kRsTile;
    }
    counts = o;
    o += align_up(tiles * kRsBins * 4, 256);
    scan_ws = o;
    scan_ws_bytes = bk_workspace_bytes(BK_ALGO_INCLUSIVE_SCAN, BK_DTYPE_U32, BK_DTYPE_NONE, tiles * kRsBins);
    o += align_up(scan_ws_bytes, 256);
    total = o;
  }
};

template <typename K, typename P>
size_t radix_sort_ws_bytes(uint64_t n) {
  return RsLayout<K, P>(&n, 1).total;
}

template <typename K, typename P>
size_t radix_sort_batch_ws_bytes(const uint64_t *sizes, uint32_t count) {
  uint64_t sz[kRsBatchMax];
  uint32_t m = 0;
  for (uint32_t i = 0; i < count && m < (uint32_t)kRsBatchMax; ++i)
    if (sizes[i] > 1) sz[m++] = sizes[i];  // arrays of 0 or 1 element need nothing
  return RsLayout<K, P>(sz, m).total;
}

// The passes over `src` (one array or a batch): upsweep, scan, downsweep each.
template <typename K, typename P, typename Src>
int radix_sort_run(const Src &src, const RsLayout<K, P> &L, char *ws, cudaStream_t stream) {
  // measured on 2^26 keys with a 4-byte payload: 256 threads ranking item
  // by item for 4-byte keys, 512 threads with every item's peers found
  // first for 8-byte keys
  constexpr int kDownTh = sizeof(K) == 8 ? 512 : 256;
  constexpr int kDownV = sizeof(K) == 8 ? 1 : 0;
  int st;
  auto *counts = reinterpret_cast<unsigned int *>(ws + L.counts);
  void *scan_ws = ws + L.scan_ws;
  auto *hdr = reinterpret_cast<WsHeader *>(ws);
  const auto *scan_hdr = reinterpret_cast<const WsHeader *>(scan_ws);
  struct UpSite {};
  struct DownSite {};
  host::KernelSetup up, down;
  if ((st = host::kernel_setup<UpSite>(rs_upsweep_kernel<K, P, Src>, kRsThreads, 0, &up)) != BK_OK) return st;
  if ((st = host::kernel_setup<DownSite>(rs_downsweep_kernel<K, P, Src, kDownV, kDownTh>, kDownTh,
                                         rs_smem_bytes<K, P>(), &down)) != BK_OK)
    return st;
  // L2 prefetch distance: the table's number of residencies ahead (0: none)
  const tune::Knobs kn = tune::knobs_for(tune::kSort, (int)(sizeof(K) + payload_bytes<P>()), L.tiles * kRsTile);
  const unsigned int up_ahead = (unsigned)up.resident_ctas * (unsigned)kn.prefetch;
  const unsigned int down_ahead = (unsigned)down.resident_ctas * (unsigned)kn.prefetch;
  // the scan's workspace must start zeroed, like any workspace
  if ((st = host::from_cuda(cudaMemsetAsync(scan_ws, 0, kHeaderBytes, stream))) != BK_OK) return st;
  for (int p = 0; p < rs_passes<K>(); ++p) {
    rs_upsweep_kernel<K, P, Src><<<(unsigned)L.tiles, kRsThreads, 0, stream>>>(src, p, counts, up_ahead);
    if ((st = host::launch_status()) != BK_OK) return st;
    st = bk_inclusive_scan_sum_u32(counts, L.tiles * kRsBins, 0u, counts, scan_ws, L.scan_ws_bytes,
                                   (bk_stream_t)stream);
    if (st != BK_OK) return st;
    rs_downsweep_kernel<K, P, Src, kDownV, kDownTh><<<(unsigned)L.tiles, kDownTh, rs_smem_bytes<K, P>(), stream>>>(
        src, p, counts, scan_hdr, hdr, down_ahead);
    if ((st = host::launch_status()) != BK_OK) return st;
  }
  return BK_OK;
}

template <typename K, typename P>
int radix_sort_launch(K *keys, P *vals, uint64_t n, void *d_ws, size_t ws_bytes, cudaStream_t stream) {
  host::DeviceInfo di;
  int st = host::device_info(&di);
  if (st != BK_OK) return st;
  if (n <= 1) return BK_OK;
  if (keys == nullptr || (has_payload<P>() && vals == nullptr)) return BK_ERR_INVALID_ARGUMENT;
  if (!host::aligned_to<K>(keys)) return BK_ERR_MISALIGNED;
  if constexpr (has_payload<P>()) {
    if (!host::aligned_to<P>(vals)) return BK_ERR_MISALIGNED;
  }
  if (n >= kRsMaxN) return BK_ERR_TOO_LARGE;  // the caller sorts these by merging
  const RsLayout<K, P> L(&n, 1);
  if ((st = host::check_ws(d_ws, ws_bytes, L.total)) != BK_OK) return st;
  char *ws = reinterpret_cast<char *>(d_ws);
  K *tk = reinterpret_cast<K *>(ws + L.tmp);
  P *tv = reinterpret_cast<P *>(ws + L.tmp + align_up(n * sizeof(K), 256));
  // one cluster launch: four items a thread up to 16 tiles of 4096 keys (more
  // CTAs, a shorter pass), eight up to 16 tiles of 8192
  int cl4 = 0, cl8 = 0;
  if ((st = rs_cluster_setup<K, P, 4>(&cl4)) != BK_OK) return st;
  if (n <= (uint64_t)kRsClThreads * 4 * (uint64_t)cl4) return rs_cluster_launch<K, P, 4>(keys, vals, tk, tv, n, stream);
  if ((st = rs_cluster_setup<K, P, 8>(&cl8)) != BK_OK) return st;
  if (n <= (uint64_t)kRsClThreads * 8 * (uint64_t)cl8) return rs_cluster_launch<K, P, 8>(keys, vals, tk, tv, n, stream);
  return radix_sort_run<K, P>(RsOne<K, P>{keys, vals, tk, tv, n, (uint32_t)L.tiles}, L, ws, stream);
}

// A batch item: sort in_keys / in_vals (left unchanged) into keys / vals;
// in place when they are the same arrays.
template <typename K, typename P>
struct RsItem {
  const K *in_keys;
  const P *in_vals;
  K *keys;
  P *vals;
  uint64_t n;
};

template <typename K, typename P>
int radix_sort_batch_launch(const RsItem<K, P> *items, uint32_t count, void *d_ws, size_t ws_bytes,
                            cudaStream_t stream) {
  if (count > 0 && items == nullptr) return BK_ERR_INVALID_ARGUMENT;
  if (count > (uint32_t)kRsBatchMax) return BK_ERR_TOO_LARGE;
  host::DeviceInfo di;
  int st = host::device_info(&di);
  if (st != BK_OK) return st;
  uint64_t sz[kRsBatchMax];
  uint32_t m = 0;
  for (uint32_t i = 0; i < count; ++i) {
    const RsItem<K, P> &it = items[i];
    if (it.n > 0 && (it.keys == nullptr || it.in_keys == nullptr ||
                     (has_payload<P>() && (it.vals == nullptr || it.in_vals == nullptr))))
      return BK_ERR_INVALID_ARGUMENT;
    if (!host::aligned_to<K>(it.keys) || !host::aligned_to<K>(it.in_keys)) return BK_ERR_MISALIGNED;
    if constexpr (has_payload<P>()) {
      if (!host::aligned_to<P>(it.vals) || !host::aligned_to<P>(it.in_vals)) return BK_ERR_MISALIGNED;
    }
    if (it.n == 1 && it.in_keys != it.keys) {  // a single element out of place: copied, not sorted
      if ((st = host::from_cuda(cudaMemcpyAsync(it.keys, it.in_keys, sizeof(K), cudaMemcpyDeviceToDevice,
                                                stream))) != BK_OK)
        return st;
      if constexpr (has_payload<P>()) {
        if ((st = host::from_cuda(cudaMemcpyAsync(it.vals, it.in_vals, sizeof(P), cudaMemcpyDeviceToDevice,
                                                  stream))) != BK_OK)
          return st;
      }
    }
    if (it.n >= kRsMaxN) return BK_ERR_TOO_LARGE;
    if (it.n > 1) sz[m++] = it.n;
  }
  if (m == 0) return BK_OK;
  const RsLayout<K, P> L(sz, m);
  if (L.tiles >= 0x7fffffffull || L.tiles * kRsBins >= 0xffffffffull) return BK_ERR_TOO_LARGE;
  if ((st = host::check_ws(d_ws, ws_bytes, L.total)) != BK_OK) return st;
  char *ws = reinterpret_cast<char *>(d_ws);
  RsBatch<K, P> b;
  b.count = 0;
  size_t off = L.tmp;
  uint64_t tiles = 0, elems = 0;
  for (uint32_t i = 0; i < count; ++i) {
    const RsItem<K, P> &it = items[i];
    if (it.n <= 1) continue;
    const uint32_t k = b.count++;
    b.keys[k] = it.keys;
    b.vals[k] = it.vals;
    b.src_k[k] = it.in_keys;
    b.src_v[k] = it.in_vals;
    b.tk[k] = reinterpret_cast<K *>(ws + off);
    off += align_up(it.n * sizeof(K), 256);
    b.tv[k] = reinterpret_cast<P *>(ws + off);
    off += align_up(it.n * (size_t)payload_bytes<P>(), 256);
    b.n[k] = it.n;
    b.elem_base[k] = (uint32_t)elems;  // the scan runs in u32: positions are taken mod 2^32
    b.start[k] = (uint32_t)tiles;
    tiles += (it.n + kRsTile - 1) / kRsTile;
    elems += it.n;
  }
  b.start[b.count] = (uint32_t)tiles;
  return radix_sort_run<K, P>(b, L, ws, stream);
}

// explicit instantiations used by sort.cu
#define BK_RS_INST_P(K, P)                                                                                  \
  template int radix_sort_launch<K, P>(K *, P *, uint64_t, void *, size_t, cudaStream_t);                  \
  template size_t radix_sort_ws_bytes<K, P>(uint64_t);                                                      \
  template int radix_sort_batch_launch<K, P>(const RsItem<K, P> *, uint32_t, void *, size_t, cudaStream_t); \
  template size_t radix_sort_batch_ws_bytes<K, P>(const uint64_t *, uint32_t);
#define BK_RS_INST(K)        \
  BK_RS_INST_P(K, NoPayload) \
  BK_RS_INST_P(K, uint32_t)  \
  BK_RS_INST_P(K, unsigned long long)
BK_RS_INST(int32_t)
BK_RS_INST(uint32_t)
BK_RS_INST(int64_t)
BK_RS_INST(uint64_t)
BK_RS_INST(float)
BK_RS_INST(double)

}  // namespace bk
