// merge.cu -- device-wide merge and merge_by_key (merge path), sm_100a.
//
// Replaces the reference's my_merge (merge.cu:127-162): a thrust::tabulate of
// merge_path at every tile diagonal (locate_merge_path, merge.cu:100-124)
// followed by one staged merge per tile (merge_kernel / staged_merge,
// merge.cu:12-97), which is keys-only; the by-key form follows the bounded
// group merge_by_key (bulk/algorithm/merge.hpp:507-607).
//
// Here: a partition kernel computes the A/B split at every tile boundary;
// then persistent CTAs merge 4096-output tiles (2048 for 8-byte keys) in a
// two-buffer pipeline.  A loader lane brings a tile's A and B key and
// payload ranges into shared memory with untiled bulk (TMA) copies -- each
// range widened to whole 16-byte chunks, the ragged ends by plain loads --
// while the compute warps merge the previous tile: each thread finds its
// diagonal with a merge-path search in shared memory, merges its outputs
// serially (branch-free: keys plus the shared-memory index of each output's
// source, which gathers the payload), and, once every thread has read its
// inputs, writes them back in place in the 128-byte-swizzled layout; the
// loader then stores the tile with tiled tensor copies, which undo the
// swizzle.  No thread loads or stores a tile element itself on this path.
#include <algorithm>

#include "bk_common.cuh"
#include "bk_merge.cuh"
#include "bk_tma.cuh"
#include "bk_tune.hpp"

namespace bk {

constexpr int kMergeWarps = 8;                       // compute warps
constexpr int kMergeCompute = 32 * kMergeWarps;      // compute threads
constexpr int kMergeThreads = kMergeCompute + 32;    // + the loader warp (one lane works)
constexpr int kMergeBufs = 2;

template <typename K, typename P>
struct MergeCfg {
  static constexpr int ITEMS = sizeof(K) == 4 ? 16 : 8;         // outputs per thread (64 bytes of keys)
  static constexpr int TILE = kMergeCompute * ITEMS;            // 4096 / 2048 outputs
  static constexpr int PB = payload_bytes<P>();                 // 0, 4 or 8
  static constexpr int KV = 16 / (int)sizeof(K);                // keys per 16-byte chunk
  static constexpr int PV = PB ? 16 / PB : 1;                   // payloads per 16-byte chunk
  static constexpr int L = KV > PV ? KV : PV;                   // the ranges are widened to multiples of L
  // the keys area holds A's range then B's (each widened by < L on either
  // side, B starting at a multiple of L) plus one element read past either
  // end; it takes the tile's outputs afterwards (1024-byte swizzle period).
  // The payloads area is laid out the same way: index i there belongs to the
  // key at index i.
  static constexpr size_t KEY_AREA = align_up(sizeof(K) * (TILE + 4 * L + 1), 1024);
  static constexpr size_t PAY_AREA = PB ? align_up((size_t)PB * (TILE + 4 * L + 1), 1024) : 0;
  static constexpr size_t BUF = KEY_AREA + PAY_AREA;
  static constexpr uint32_t KROWS = sizeof(K) * TILE / 128;     // 128-byte rows of output keys per tile
  static constexpr uint32_t PROWS = PB * TILE / 128;
};

template <typename K, typename P>
constexpr size_t merge_smem_bytes() {
  return (size_t)kMergeBufs * MergeCfg<K, P>::BUF + 1024;  // + room to align the buffers to 1024 bytes
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

// What the compute warps need to know of a tile in a buffer (written by the
// loader before it arms the buffer's barrier).
struct MergeDesc {
  uint32_t la, lb;    // A and B elements of the tile
  uint32_t ia, ib;    // index of A's / B's first element in the keys (and payloads) area
  uint32_t count;     // outputs (la + lb)
  uint32_t tile;      // tile index
};

// The kernel's parameters.
template <typename K, typename P>
struct MergeArgs {
  CUtensorMap okmap;  // output keys as rows of 128 bytes (boxes of KROWS rows)
  CUtensorMap opmap;  // output payloads (boxes of PROWS rows)
  const K *a;
  const P *av;
  uint64_t na;
  const K *b;
  const P *bv;
  uint64_t nb;
  K *out;
  P *outv;
  const uint64_t *parts;
  uint64_t tiles;
  uint64_t covered_out;  // leading outputs inside whole rows of both output views (0: none)
  int tma_in;            // a, b, av, bv 16-byte aligned: inputs arrive by bulk copies
};

// Bytes of the bulk copy that merge_load_range issues for [lo, hi).
template <typename T>
__device__ __forceinline__ uint32_t merge_bulk_bytes(uint64_t lo, uint64_t hi) {
  constexpr uint64_t V = 16 / sizeof(T);
  const uint64_t bulk_hi = hi & ~(V - 1);
  return bulk_hi > lo ? (uint32_t)((bulk_hi - lo) * sizeof(T)) : 0u;
}

// Loader: one input range [lo, hi) of `src` (T elements, 16-byte aligned
// array) into shared memory at `dst` (16-byte aligned): the whole 16-byte
// chunks by one bulk copy completing on bar (its bytes already expected),
// the ragged end by plain loads.  lo is a multiple of 16 / sizeof(T).
template <typename T>
__device__ __forceinline__ void merge_load_range(T *dst, const T *src, uint64_t lo, uint64_t hi, uint64_t *bar,
                                                 uint64_t policy) {
  constexpr uint64_t V = 16 / sizeof(T);
  const uint64_t bulk_hi = hi & ~(V - 1);
  if (bulk_hi > lo) tma_load_1d_hint(dst, src + lo, (uint32_t)((bulk_hi - lo) * sizeof(T)), bar, policy);
  for (uint64_t i = bulk_hi > lo ? bulk_hi : lo; i < hi; ++i) dst[i - lo] = src[i];
}

// Persistent merge.  Warps 0-7 merge; warp 8's lane 0 loads and stores.
// CTA c takes tiles c, c + G, c + 2G, ... (G = gridDim.x); tile i of the CTA
// uses buffer i mod 2 and goes through:
//   loader: (once the compute warps have written tile i-2's outputs to the
//           buffer and that tile's stores have read them) write the tile's
//           descriptor, bulk-copy its ranges in; full[b] completes;
//   compute: merge-path search and serial merge into registers; a barrier
//           among the compute warps (every input read); outputs written in
//           place, swizzled; each warp arrives on out[b];
//   loader: tensor stores of the keys and payloads (rows past the output
//           view are clipped; a last tile's ragged end is stored by the
//           compute threads directly).
// All waits are bounded; after a timeout the kernel records
// BK_ERR_SPIN_TIMEOUT in the header and every role stops.
template <typename K, typename P>
__global__ void __launch_bounds__(kMergeThreads, (sizeof(K) == 4 && payload_bytes<P>() == 8) ? 2 : 3)
merge_kernel(const __grid_constant__ MergeArgs<K, P> args,
                                                                 WsHeader *hdr, unsigned long long spin_limit_ns) {
  using C = MergeCfg<K, P>;
  constexpr int ITEMS = C::ITEMS, TILE = C::TILE, NB = kMergeBufs;
  constexpr bool HP = has_payload<P>();
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char *const smem_raw = smem_dyn + ((1024u - (smem_addr(smem_dyn) & 1023u)) & 1023u);
  __shared__ __align__(8) uint64_t s_full[NB];
  __shared__ __align__(8) uint64_t s_out[NB];
  __shared__ MergeDesc s_desc[NB];
  __shared__ int s_abort;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  auto buf = [&](int b) { return smem_raw + (size_t)b * C::BUF; };
  auto aborted = [&]() -> bool { return *reinterpret_cast<volatile int *>(&s_abort) != 0; };
  const uint64_t total = args.na + args.nb;
  const uint64_t G = gridDim.x;

  if (tid == kMergeCompute) {
    for (int b = 0; b < NB; ++b) {
      mbar_init(&s_full[b], 1);
      mbar_init(&s_out[b], kMergeWarps);
    }
    fence_proxy_async_smem();
    s_abort = 0;
  }
  __syncthreads();

  // tiles of this CTA: blockIdx.x + i * G for i < mine (the grid is no larger than the tile count)
  const uint64_t mine = (args.tiles - blockIdx.x + G - 1) / G;

  if (warp == kMergeWarps) {
    // ================= the loader (lane 0) =================
    if (lane != 0) return;
    const uint64_t policy = l2_policy_evict_first();  // inputs and outputs are read / written once
    uint32_t outpar = 0u, armpar = 0u, armany = 0u;
    bool stored = false, failed = false;
    uint64_t fail_tile = 0;
    for (uint64_t i = 0; i < mine + 2; ++i) {
      const int b = (int)(i & 1);
      if (i >= 2) {
        // tile i-2's outputs are in buffer b: store them
        if (!mbar_wait_or_abort(&s_out[b], (outpar >> b) & 1u, spin_limit_ns, &s_abort)) {
          failed = true;
          fail_tile = blockIdx.x + (i - 2) * G;
          break;
        }
        outpar ^= 1u << b;
        const uint32_t tile = s_desc[b].tile;
        if (args.covered_out > (uint64_t)tile * TILE) {
          tma_store_rows(&args.okmap, tile * C::KROWS, buf(b), policy);
          if constexpr (HP) tma_store_rows(&args.opmap, tile * C::PROWS, buf(b) + C::KEY_AREA, policy);
          tma_store_commit();
          stored = true;
        }
      }
      if (i >= mine) continue;
      if (stored) tma_store_wait_read();  // the stores have read the buffer
      // ---- tile k: its A range [a0, a1) and B range [b0, b1)
      const uint64_t k = blockIdx.x + i * G;
      const uint64_t d0 = k * TILE, d1 = d0 + TILE < total ? d0 + TILE : total;
      const uint64_t a0 = args.parts[k], a1 = args.parts[k + 1];
      const uint64_t b0 = d0 - a0, b1 = d1 - a1;
      MergeDesc d;
      d.la = (uint32_t)(a1 - a0);
      d.lb = (uint32_t)(b1 - b0);
      d.count = (uint32_t)(d1 - d0);
      d.tile = (uint32_t)k;
      if (args.tma_in) {
        const uint64_t alo = a0 & ~(uint64_t)(C::L - 1), blo = b0 & ~(uint64_t)(C::L - 1);
        const uint32_t bstart = (uint32_t)align_up(a1 - alo, (size_t)C::L);  // B's copy: a multiple of L
        d.ia = (uint32_t)(a0 - alo);
        d.ib = bstart + (uint32_t)(b0 - blo);
        uint32_t bytes = (a1 > a0 ? merge_bulk_bytes<K>(alo, a1) : 0u) + (b1 > b0 ? merge_bulk_bytes<K>(blo, b1) : 0u);
        if constexpr (HP)
          bytes += (a1 > a0 ? merge_bulk_bytes<P>(alo, a1) : 0u) + (b1 > b0 ? merge_bulk_bytes<P>(blo, b1) : 0u);
        if (bytes) mbar_expect_tx(&s_full[b], bytes);
        K *sk = reinterpret_cast<K *>(buf(b));
        P *sp = reinterpret_cast<P *>(buf(b) + C::KEY_AREA);
        if (a1 > a0) merge_load_range<K>(sk, args.a, alo, a1, &s_full[b], policy);
        if (b1 > b0) merge_load_range<K>(sk + bstart, args.b, blo, b1, &s_full[b], policy);
        if constexpr (HP) {
          if (a1 > a0) merge_load_range<P>(sp, args.av, alo, a1, &s_full[b], policy);
          if (b1 > b0) merge_load_range<P>(sp + bstart, args.bv, blo, b1, &s_full[b], policy);
        }
      } else {  // the compute warps copy the ranges themselves
        d.ia = 0;
        d.ib = d.la;
      }
      s_desc[b] = d;
      // the loader's one arrival, after its plain stores (descriptor, ragged
      // ends): the phase completes once the bulk copies' bytes have landed
      mbar_arrive(&s_full[b]);
      armpar ^= 1u << b;
      armany |= 1u << b;
    }
    if (failed) {
      record_error(hdr, BK_ERR_SPIN_TIMEOUT, (unsigned int)fail_tile);
      *reinterpret_cast<volatile int *>(&s_abort) = 1;
    }
    if (stored) tma_store_wait_all();
    // every load must land before the CTA's shared memory goes away
    for (int b = 0; b < NB; ++b)
      if ((armany >> b) & 1u) (void)mbar_wait(&s_full[b], ((armpar >> b) & 1u) ^ 1u, spin_limit_ns);
    return;
  }

  // ================= the compute warps =================
  uint32_t fullpar = 0u;
  bool bad = false;
  for (uint64_t i = 0; i < mine; ++i) {
    const int b = (int)(i & 1);
    const uint64_t k = blockIdx.x + i * G;
    if (!mbar_wait_or_abort(&s_full[b], (fullpar >> b) & 1u, spin_limit_ns, &s_abort)) bad = true;
    fullpar ^= 1u << b;
    if (named_barrier_or(1, kMergeCompute, bad || aborted())) {
      if (tid == 0) record_error(hdr, BK_ERR_SPIN_TIMEOUT, (unsigned int)k);
      *reinterpret_cast<volatile int *>(&s_abort) = 1;
      break;
    }
    const MergeDesc d = s_desc[b];
    K *const sk = reinterpret_cast<K *>(buf(b));
    P *const sp = reinterpret_cast<P *>(buf(b) + C::KEY_AREA);
    if (!args.tma_in) {  // a launch-wide flag: every compute warp takes this branch or none
      const uint64_t d0 = k * TILE, a0 = args.parts[k], b0 = d0 - a0;
      for (uint32_t j = tid; j < d.la; j += kMergeCompute) {
        sk[j] = args.a[a0 + j];
        if constexpr (HP) sp[j] = args.av[a0 + j];
      }
      for (uint32_t j = tid; j < d.lb; j += kMergeCompute) {
        sk[d.la + j] = args.b[b0 + j];
        if constexpr (HP) sp[d.la + j] = args.bv[b0 + j];
      }
      named_barrier_sync(2, kMergeCompute);
    }
    // ---- merge-path search for this thread's first output, then its outputs
    const uint32_t diag = (uint32_t)tid * ITEMS;
    K okey[ITEMS];
    uint32_t osrc[ITEMS];
    const int valid = (int)min((int)d.count - (int)diag, ITEMS);
    if (valid > 0) {
      uint32_t lo = diag > d.lb ? diag - d.lb : 0u;
      uint32_t hi = diag < d.la ? diag : d.la;
      while (lo < hi) {  // ties go to A: move left while b[diag-1-mid] < a[mid]
        const uint32_t mid = (lo + hi) >> 1;
        if (sk[d.ib + diag - 1 - mid] < sk[d.ia + mid]) hi = mid;
        else lo = mid + 1;
      }
      uint32_t ia = d.ia + lo, ib = d.ib + (diag - lo);
      const uint32_t ea = d.ia + d.la, eb = d.ib + d.lb;
      // reads reach at most one element past either range (a neighbour
      // inside the buffer, never used): the loop stops at `valid`
      K ka = sk[ia], kb = sk[ib];
#pragma unroll
      for (int j = 0; j < ITEMS; ++j) {
        if (valid == ITEMS || j < valid) {
          // take A while B is exhausted or !(b < a): equal keys keep A first
          const bool take_a = ia < ea && (ib >= eb || !(kb < ka));
          okey[j] = take_a ? ka : kb;
          osrc[j] = take_a ? ia : ib;
          ia += take_a ? 1u : 0u;
          ib += take_a ? 0u : 1u;
          if (j + 1 < ITEMS) {
            const K nk = sk[take_a ? ia : ib];
            ka = take_a ? nk : ka;
            kb = take_a ? kb : nk;
          }
        }
      }
    }
    P opay[ITEMS];
    if constexpr (HP) {
#pragma unroll
      for (int j = 0; j < ITEMS; ++j)
        if (j < valid) opay[j] = sp[osrc[j]];
    }
    named_barrier_sync(2, kMergeCompute);  // every thread has read its inputs
    // ---- outputs: in place, swizzled for the tensor stores (which write
    // the rows inside the output views); outputs past covered_out (a last
    // tile's ragged end, or every output when the views could not be made)
    // are also stored directly
    const uint64_t o0 = k * TILE + diag;
    if (valid == ITEMS) {
      constexpr int KCH = ITEMS * (int)sizeof(K) / 16;
#pragma unroll
      for (int c = 0; c < KCH; ++c) {
        uint4 q;
        memcpy(&q, &okey[c * (16 / sizeof(K))], 16);
        *reinterpret_cast<uint4 *>(buf(b) + swz128(diag * (uint32_t)sizeof(K) + 16u * c)) = q;
      }
      if constexpr (HP) {
        constexpr int PCH = ITEMS * C::PB / 16;
#pragma unroll
        for (int c = 0; c < PCH; ++c) {
          uint4 q;
          memcpy(&q, &opay[c * (16 / C::PB)], 16);
          *reinterpret_cast<uint4 *>(buf(b) + C::KEY_AREA + swz128(diag * (uint32_t)C::PB + 16u * c)) = q;
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < ITEMS; ++j) {
        if (j < valid) {
          *reinterpret_cast<K *>(buf(b) + swz128((diag + j) * (uint32_t)sizeof(K))) = okey[j];
          if constexpr (HP)
            *reinterpret_cast<P *>(buf(b) + C::KEY_AREA + swz128((diag + j) * (uint32_t)C::PB)) = opay[j];
        }
      }
    }
    if (valid > 0 && o0 + (uint64_t)valid > args.covered_out) {
#pragma unroll
      for (int j = 0; j < ITEMS; ++j) {
        if (j < valid && o0 + j >= args.covered_out) {
          args.out[o0 + j] = okey[j];
          if constexpr (HP) args.outv[o0 + j] = opay[j];
        }
      }
    }
    fence_proxy_async_smem();  // the tensor stores read what this thread wrote
    __syncwarp();
    if (lane == 0) mbar_arrive(&s_out[b]);
  }
}

template <typename K>
size_t merge_ws_bytes(uint64_t n) {
  const uint64_t tiles = (n + MergeCfg<K, NoPayload>::TILE - 1) / MergeCfg<K, NoPayload>::TILE;
  return kHeaderBytes + align_up((tiles + 1) * sizeof(uint64_t), 256);
}

template <typename K, typename P>
int merge_launch(const K *a, const P *av, uint64_t na, const K *b, const P *bv, uint64_t nb, K *out, P *outv,
                 void *d_ws, size_t ws_bytes, cudaStream_t stream) {
  using C = MergeCfg<K, P>;
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
  const uint64_t tiles = (n + C::TILE - 1) / C::TILE;
  if (tiles >= 0x7fffffffull) return BK_ERR_TOO_LARGE;
  st = host::check_ws(d_ws, ws_bytes, merge_ws_bytes<K>(n));
  if (st != BK_OK) return st;
  WsHeader *hdr = reinterpret_cast<WsHeader *>(d_ws);
  uint64_t *parts = reinterpret_cast<uint64_t *>(reinterpret_cast<char *>(d_ws) + kHeaderBytes);
  const uint64_t np = tiles + 1;
  merge_partition_kernel<K><<<(unsigned)((np + 255) / 256), 256, 0, stream>>>(a, na, b, nb, C::TILE, np, parts);
  if ((st = host::launch_status()) != BK_OK) return st;

  MergeArgs<K, P> args;
  memset(&args, 0, sizeof(args));
  args.a = a;
  args.av = av;
  args.na = na;
  args.b = b;
  args.bv = bv;
  args.nb = nb;
  args.out = out;
  args.outv = outv;
  args.parts = parts;
  args.tiles = tiles;
  auto a16 = [](const void *p) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  args.tma_in = a16(a) && a16(b) && a16(av) && a16(bv);
  // output row views: the outputs inside whole 128-byte rows of both leave by
  // tensor stores, the rest by plain stores
  const uint64_t krows = n * sizeof(K) / 128, prows = n * (uint64_t)C::PB / 128;
  if (a16(out) && a16(outv) && krows > 0 && host::encode_rows_128b(&args.okmap, out, krows, C::KROWS) == BK_OK) {
    args.covered_out = krows * (128 / sizeof(K));
    if constexpr (has_payload<P>()) {
      if (prows > 0 && host::encode_rows_128b(&args.opmap, outv, prows, C::PROWS) == BK_OK)
        args.covered_out = std::min<uint64_t>(args.covered_out, prows * (128 / C::PB));
      else
        args.covered_out = 0;
    }
  }
  const size_t smem = merge_smem_bytes<K, P>();
  struct Site {};
  host::KernelSetup ks;
  if ((st = host::kernel_setup<Site>(merge_kernel<K, P>, kMergeThreads, smem, &ks)) != BK_OK) return st;
  const tune::Knobs kn = tune::knobs_for(tune::kMerge, (int)(sizeof(K) + C::PB), n);
  const uint64_t per_sm = ks.resident_ctas / (uint64_t)di.sm_count;  // what fits (shared memory, registers)
  const uint64_t want = (uint64_t)di.sm_count * (uint64_t)std::max(kn.ctas_per_sm, 1);
  const unsigned grid = (unsigned)std::min<uint64_t>(tiles, std::min<uint64_t>(want, std::max<uint64_t>(per_sm, 1) * di.sm_count));
  const host::DebugFault dbg = host::debug_fault();
  const unsigned long long limit = dbg.spin_limit_ns ? dbg.spin_limit_ns : host::kDefaultSpinLimitNs;
  merge_kernel<K, P><<<grid, kMergeThreads, smem, stream>>>(args, hdr, limit);
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
