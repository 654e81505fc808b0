// ghb_noalloc.cu — fused filter + group-by that allocates no device memory.
//
// Some callers of this library cannot call cudaMalloc: a Hive/Tez task whose
// device memory was handed in full to another allocator (a pooled executor
// that reserves all of HBM up front, so cudaMalloc fails), or code that must
// not risk the device-wide synchronisation cudaMalloc/cudaFree may imply
// (a serving thread with a latency budget).  ghb_filter_groupby allocates
// through its context (the context itself, its scratch and its hash table);
// this entry point instead keeps the group-by hash table and the device
// status word in one file-scope __device__ array of fixed size, so the
// caller passes only its input and output buffers.
//
// The array is GHB_NOALLOC_SCRATCH_BYTES (8 MiB) and every GPU that loads the
// library holds it until the process exits.  Its device address is looked up
// once per device with cudaGetSymbolAddress (in host code the array's name is
// only a host-side stand-in, not a device address).  The first call on a
// device does that set-up, and with it loads this file's module (which
// creates the array) and every kernel the call can launch: CUDA loads code
// lazily, and loading may allocate device memory.  After that first call no
// call loads code or allocates.  The cached address assumes the device's
// primary context lives as long as the process (no cudaDeviceReset).
#include <mutex>

#include "ghb_ctx.hpp"

namespace ghb {

int32_t filter_groupby_impl(ghb_ctx*, const ghb_predicate*, const ghb_column*, int32_t,
                            const int32_t*, int32_t, const ghb_agg_desc*, int32_t, ghb_out_column*,
                            int64_t, int64_t*, const ghb_groupby_cfg*, cudaStream_t, void*, size_t);
int32_t preload_fixed_table_kernels(ghb_ctx* ctx);

namespace {

constexpr size_t kScratchBytes = GHB_NOALLOC_SCRATCH_BYTES;
constexpr size_t kStatusBytes = 256;   // device status word, then the hash table
constexpr int kMaxDevices = 64;

// The scratch: status word in the first 256 bytes, group-by table after it.
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch on the current device (looked up once, with
// the kernels the call launches loaded at the same time).
int32_t scratch_address(ghb_ctx* local, int device, void** out) {
  if (device < 0 || device >= kMaxDevices) return GHB_ERR_INVALID;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[device]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      cudaGetLastError();
      return GHB_ERR_CUDA;
    }
    if (int32_t st = preload_fixed_table_kernels(local)) return st;
    g_scratch_ptr[device] = ptr;
  }
  *out = g_scratch_ptr[device];
  return GHB_OK;
}

}  // namespace
}  // namespace ghb

using namespace ghb;

extern "C" int32_t ghb_filter_groupby_noalloc(const ghb_predicate* pred, const ghb_column* cols,
                                              int32_t ncols, const int32_t* key_cols, int32_t nkeys,
                                              const ghb_agg_desc* aggs, int32_t naggs,
                                              ghb_out_column* out, int64_t out_capacity,
                                              int64_t* d_out_groups, const ghb_groupby_cfg* cfg,
                                              void* stream) {
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return GHB_ERR_CUDA;
  }
  cudaStream_t s = (cudaStream_t)stream;
  // a host-side context object only: its device pointers stay empty except
  // the status word, which lives in the scratch
  ghb_ctx local;
  local.device = device;
  cudaDeviceGetAttribute(&local.num_sms, cudaDevAttrMultiProcessorCount, device);
  void* base = nullptr;
  int32_t st = scratch_address(&local, device, &base);
  if (st) return st;
  local.d_status = (int32_t*)base;
  if (cudaMemsetAsync(base, 0, kStatusBytes, s) != cudaSuccess) {
    cudaGetLastError();
    return GHB_ERR_CUDA;
  }
  st = filter_groupby_impl(&local, pred, cols, ncols, key_cols, nkeys, aggs, naggs, out, out_capacity,
                           d_out_groups, cfg, s, (char*)base + kStatusBytes,
                           kScratchBytes - kStatusBytes);
  if (st) return st;
  // wait, then report what the kernels raised (a full table, a short output)
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return GHB_ERR_CUDA;
  }
  int32_t dev_status = 0;
  if (cudaMemcpy(&dev_status, base, sizeof(dev_status), cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return GHB_ERR_CUDA;
  }
  return dev_status;
}
