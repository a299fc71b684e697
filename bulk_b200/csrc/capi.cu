// capi.cu -- library-wide C-ABI entry points: version, status strings,
// workspace sizing / initialisation / status readback, device property cache,
// the tensor-map encoder and the process-wide test hook.
#include <atomic>
#include <mutex>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "bk_common.cuh"

namespace bk {
size_t reduce_workspace_bytes(int dtype, uint64_t n);
size_t scan_workspace_bytes(int dtype, uint64_t n);
size_t merge_workspace_bytes(int key_dtype, int value_dtype, uint64_t n);
size_t sort_workspace_bytes(int key_dtype, int value_dtype, uint64_t n);
size_t rbk_workspace_bytes(int key_dtype, int value_dtype, uint64_t n);
size_t scan_batch_workspace_bytes(int dtype, const uint64_t *sizes, uint32_t count);
size_t rbk_batch_workspace_bytes(int key_dtype, int value_dtype, const uint64_t *sizes, uint32_t count);
size_t sort_batch_workspace_bytes(int key_dtype, int value_dtype, const uint64_t *sizes, uint32_t count);

namespace host {

namespace {
constexpr int kMaxDevices = 64;
std::once_flag g_once[kMaxDevices];
DeviceInfo g_info[kMaxDevices];
int g_info_status[kMaxDevices];

std::atomic<long long> g_skip_tile{-1};
std::atomic<unsigned long long> g_spin_limit{0};
}  // namespace

int device_info(DeviceInfo *out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= kMaxDevices) return BK_ERR_UNSUPPORTED;
  std::call_once(g_once[dev], [dev]() {
    DeviceInfo d{};
    cudaError_t e1 = cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e2 = cudaDeviceGetAttribute(&d.cc_major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaError_t e3 = cudaDeviceGetAttribute(&d.cc_minor, cudaDevAttrComputeCapabilityMinor, dev);
    cudaError_t e4 = cudaDeviceGetAttribute(&d.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    int st = BK_OK;
    if (e1 != cudaSuccess) st = (int)e1;
    else if (e2 != cudaSuccess) st = (int)e2;
    else if (e3 != cudaSuccess) st = (int)e3;
    else if (e4 != cudaSuccess) st = (int)e4;
    else if (d.cc_major != 10) st = BK_ERR_UNSUPPORTED;  // built for sm_100a only
    g_info[dev] = d;
    g_info_status[dev] = st;
  });
  *out = g_info[dev];
  return g_info_status[dev];
}

DebugFault debug_fault() { return DebugFault{g_skip_tile.load(), g_spin_limit.load()}; }

namespace {
std::once_flag g_encode_once;
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
}  // namespace

int encode_rows_128b(void *map, const void *base, uint64_t rows, uint32_t box_rows) {
  std::call_once(g_encode_once, []() {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    else
      (void)cudaGetLastError();
  });
  if (g_encode == nullptr) return BK_ERR_UNSUPPORTED;
  if (rows == 0 || box_rows == 0 || box_rows > 256 || (reinterpret_cast<uintptr_t>(base) & 15) != 0)
    return BK_ERR_INVALID_ARGUMENT;
  const cuuint64_t dims[2] = {128, rows};
  const cuuint64_t strides[1] = {128};
  const cuuint32_t box[2] = {128, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = g_encode(reinterpret_cast<CUtensorMap *>(map), CU_TENSOR_MAP_DATA_TYPE_UINT8, 2,
                              const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? BK_OK : BK_ERR_INVALID_ARGUMENT;
}

}  // namespace host
}  // namespace bk

extern "C" int bk_version(void) { return 1 * 10000 + 0 * 100 + 0; }

extern "C" const char *bk_status_string(int status) {
  switch (status) {
    case BK_OK: return "success";
    case BK_ERR_INVALID_ARGUMENT: return "invalid argument";
    case BK_ERR_WORKSPACE_TOO_SMALL: return "workspace too small";
    case BK_ERR_SPIN_TIMEOUT: return "device-side wait timed out";
    case BK_ERR_MISALIGNED: return "pointer misaligned";
    case BK_ERR_TOO_LARGE: return "input too large";
    case BK_ERR_UNSUPPORTED: return "unsupported device or type combination";
    default: return status > 0 ? cudaGetErrorString((cudaError_t)status) : "unknown library status";
  }
}

extern "C" size_t bk_workspace_bytes(int algo, int key_dtype, int value_dtype, uint64_t n) {
  switch (algo) {
    case BK_ALGO_REDUCE: return value_dtype == BK_DTYPE_NONE ? bk::reduce_workspace_bytes(key_dtype, n) : 0;
    case BK_ALGO_INCLUSIVE_SCAN: return value_dtype == BK_DTYPE_NONE ? bk::scan_workspace_bytes(key_dtype, n) : 0;
    case BK_ALGO_MERGE: return bk::merge_workspace_bytes(key_dtype, value_dtype, n);
    case BK_ALGO_SORT_BY_KEY: return bk::sort_workspace_bytes(key_dtype, value_dtype, n);
    case BK_ALGO_REDUCE_BY_KEY: return bk::rbk_workspace_bytes(key_dtype, value_dtype, n);
    default: return 0;
  }
}

extern "C" size_t bk_batch_workspace_bytes(int algo, int key_dtype, int value_dtype, const uint64_t *sizes,
                                           uint32_t count) {
  switch (algo) {
    case BK_ALGO_INCLUSIVE_SCAN:
      return value_dtype == BK_DTYPE_NONE ? bk::scan_batch_workspace_bytes(key_dtype, sizes, count) : 0;
    case BK_ALGO_REDUCE_BY_KEY: return bk::rbk_batch_workspace_bytes(key_dtype, value_dtype, sizes, count);
    case BK_ALGO_SORT_BY_KEY: return bk::sort_batch_workspace_bytes(key_dtype, value_dtype, sizes, count);
    default: return 0;
  }
}

extern "C" int bk_workspace_init(void *d_ws, size_t ws_bytes, bk_stream_t stream) {
  if (d_ws == nullptr || ws_bytes < bk::kHeaderBytes) return BK_ERR_INVALID_ARGUMENT;
  return bk::host::from_cuda(cudaMemsetAsync(d_ws, 0, ws_bytes, (cudaStream_t)stream));
}

extern "C" int bk_workspace_status(void *d_ws, size_t ws_bytes, bk_stream_t stream) {
  if (d_ws == nullptr || ws_bytes < bk::kHeaderBytes) return BK_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return (int)e;
  bk::WsHeader h;
  e = cudaMemcpy(&h, d_ws, sizeof(h), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return (int)e;
  if (h.status != BK_OK) {
    // Clear the error and every counter a failed kernel may have left behind.
    e = cudaMemset(d_ws, 0, sizeof(h));
    if (e != cudaSuccess) return (int)e;
  }
  return h.status;
}

extern "C" int bk_debug_set_fault(int64_t skip_publish_tile, uint64_t spin_limit_ns) {
  bk::host::g_skip_tile.store(skip_publish_tile);
  bk::host::g_spin_limit.store(spin_limit_ns);
  return BK_OK;
}
