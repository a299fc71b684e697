// noalloc.cu -- an inclusive-scan entry point that allocates nothing.
//
// Some callers cannot allocate device memory for a workspace: a plugin that
// runs inside a host application which owns all GPU memory and hands out none,
// code on a latency-critical path where cudaMalloc's implicit device-wide
// synchronisation is not acceptable, or a C/FFI caller with no allocator of
// its own.  For them this file keeps the scan's scratch (the look-back status
// slots and the header with the tile ticket) in a fixed-size array in the
// library's own device memory.  The caller passes only the input and output.
//
// The array is a file-scope __device__ variable, so every GPU that loads the
// library holds it (1 MiB + 256 bytes) until the process exits.  Host code
// cannot use the array's name as a device address (it names a host-side
// shadow), so the device address is looked up with cudaGetSymbolAddress once
// per device, with that device current, on the first call made on it (make
// that first call before any stream capture).  Only a successful lookup is
// kept: a failed one is tried again on the next call.  The kept address
// belongs to the device's current context, so the entry point must not be
// called on a device after cudaDeviceReset has destroyed that context.
#include "bk_common.cuh"

namespace {

// Largest input accepted: 2^30 elements (4 GiB of float32).
constexpr uint64_t kNoAllocMaxN = 1ull << 30;
// 256-byte header + one 8-byte look-back slot per 8192-element tile.
constexpr size_t kNoAllocScratchBytes = 256 + (kNoAllocMaxN / 8192) * 8;

static __device__ __align__(256) unsigned char g_noalloc_scan_scratch[kNoAllocScratchBytes];

struct NoAllocSite {};

}  // namespace

extern "C" int bk_inclusive_scan_sum_f32_noalloc(const float *d_in, uint64_t n, float init, float *d_out,
                                                 bk_stream_t stream) {
  if (n > kNoAllocMaxN) return BK_ERR_TOO_LARGE;
  // First call on this device (which is current): find the array's device address.
  void *scratch = nullptr;
  int st = bk::host::once_per_device<NoAllocSite>(&scratch, [](void **p) -> int {
    return bk::host::from_cuda(cudaGetSymbolAddress(p, g_noalloc_scan_scratch));
  });
  if (st != BK_OK) return st;
  cudaError_t e;

  const size_t need = bk_workspace_bytes(BK_ALGO_INCLUSIVE_SCAN, BK_DTYPE_F32, BK_DTYPE_NONE, n);
  if (need > kNoAllocScratchBytes) return BK_ERR_TOO_LARGE;
  // The array keeps the previous call's contents.  The header (tile ticket and
  // error word) must start at zero; the look-back slots are cleared by the
  // scan's own init kernel on every call.
  e = cudaMemsetAsync(scratch, 0, bk::kHeaderBytes, (cudaStream_t)stream);
  if (e != cudaSuccess) return (int)e;
  return bk_inclusive_scan_sum_f32(d_in, n, init, d_out, scratch, kNoAllocScratchBytes, stream);
}
