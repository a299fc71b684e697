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
// per device, with that device current, on the first call made on it.
#include <mutex>

#include "bk_common.cuh"

namespace {

// Largest input accepted: 2^30 elements (4 GiB of float32).
constexpr uint64_t kNoAllocMaxN = 1ull << 30;
// 256-byte header + one 8-byte look-back slot per 8192-element tile.
constexpr size_t kNoAllocScratchBytes = 256 + (kNoAllocMaxN / 8192) * 8;

static __device__ __align__(256) unsigned char g_noalloc_scan_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::once_flag g_once[kMaxDevices];
void *g_scratch[kMaxDevices];
int g_setup_status[kMaxDevices];

}  // namespace

extern "C" int bk_inclusive_scan_sum_f32_noalloc(const float *d_in, uint64_t n, float init, float *d_out,
                                                 bk_stream_t stream) {
  if (n > kNoAllocMaxN) return BK_ERR_TOO_LARGE;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= kMaxDevices) return BK_ERR_UNSUPPORTED;
  // First call on this device (which is current): find the array's device address.
  std::call_once(g_once[dev], [dev]() {
    void *p = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scan_scratch);
    g_scratch[dev] = p;
    g_setup_status[dev] = (err == cudaSuccess) ? BK_OK : (int)err;
  });
  if (g_setup_status[dev] != BK_OK) return g_setup_status[dev];
  void *scratch = g_scratch[dev];

  const size_t need = bk_workspace_bytes(BK_ALGO_INCLUSIVE_SCAN, BK_DTYPE_F32, BK_DTYPE_NONE, n);
  if (need > kNoAllocScratchBytes) return BK_ERR_TOO_LARGE;
  // The array keeps the previous call's contents.  The header (tile ticket and
  // error word) must start at zero; the look-back slots are cleared by the
  // scan's own init kernel on every call.
  e = cudaMemsetAsync(scratch, 0, bk::kHeaderBytes, (cudaStream_t)stream);
  if (e != cudaSuccess) return (int)e;
  return bk_inclusive_scan_sum_f32(d_in, n, init, d_out, scratch, kNoAllocScratchBytes, stream);
}
