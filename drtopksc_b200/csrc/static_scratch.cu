// static_scratch.cu -- a select that allocates no device memory.
//
// Some callers cannot allocate device memory when they want a top-k: their
// framework's caching allocator already owns the whole device memory and
// hands none out, or cudaMalloc's implicit device synchronisation is not
// acceptable on their latency-critical path, or they run as a plugin whose
// host application forbids allocation from inside it.  For them,
// drtopk_select_noalloc runs the same select as drtopk_select, but its
// scratch lives in one fixed array compiled into this library instead of
// in memory allocated per handle or per call.
//
// The array below is a file-scope __device__ variable: every GPU that loads
// this library's device code holds its 32 MiB until the process exits.  With
// CUDA's lazy module loading (the default) that memory is taken when the
// module is first used on a device, which for this array is the first call
// on that device; make that call at initialisation, before the framework's
// allocator reserves the device memory and before capturing any stream work
// (or set CUDA_MODULE_LOADING=EAGER to take it when the context is created).
// Its name is only a host-side stand-in in host code, so the device address
// is looked up once per device with cudaGetSymbolAddress (by that first
// call) and passed to the kernels.  All calls share the one array and it
// keeps the contents of the last call; the select clears the part that must
// start at zero (its control block, which holds the device error word) at
// the start of every call.  Two calls whose GPU work overlaps (different
// streams, or different host threads) race on the array and give wrong
// results: serialise them.
//
// Device-side failures (a bounded wait that gave up, an internal check) are
// recorded in the control block's error word, as for the handle-based
// select; drtopk_noalloc_sync_check synchronises the caller's stream and
// turns that word into a status.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/drtopk.h"
#include "plan.h"

namespace {

constexpr size_t kStaticScratchBytes = size_t(32) << 20;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_static_mu;
void* g_static_ptr[64] = {};
size_t g_static_ctrl[64] = {};  // offset of the last plan's control block in the array

// device address of g_static_scratch on `device` (that device must be current)
drtopk_status_t static_scratch_ptr(int device, char** out) {
  if (device < 0 || device >= 64) return DRTOPK_EINVAL;
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (!g_static_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return DRTOPK_ECUDA;
    }
    g_static_ptr[device] = p;
  }
  *out = static_cast<char*>(g_static_ptr[device]);
  return DRTOPK_OK;
}

}  // namespace

extern "C" drtopk_status_t drtopk_select_noalloc(const void* d_keys, drtopk_dtype_t dtype, uint64_t n, uint64_t k,
                                                 const drtopk_params_t* p, void* d_kth, void* d_vals,
                                                 int64_t* d_idx, void* stream) {
  if (!d_keys) return DRTOPK_EINVAL;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return DRTOPK_ECUDA;
  drtopk::Plan P;
  drtopk_status_t s = drtopk::plan_select(device, n, k, dtype, p, d_idx != nullptr, &P);
  if (s != DRTOPK_OK) return s;
  // the whole workspace of this (n, k, params) must fit the fixed array
  if (P.ws_bytes > kStaticScratchBytes) return DRTOPK_EUNSUPPORTED;
  char* ws = nullptr;
  s = static_scratch_ptr(device, &ws);
  if (s != DRTOPK_OK) return s;
  {
    std::lock_guard<std::mutex> lk(g_static_mu);
    g_static_ctrl[device] = P.off_ctrl;
  }
  return drtopk::enqueue_select(P, device, d_keys, d_kth, d_vals, d_idx, ws, static_cast<cudaStream_t>(stream),
                                nullptr);
}

extern "C" drtopk_status_t drtopk_noalloc_sync_check(void* stream) {
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return DRTOPK_ECUDA;
  if (device < 0 || device >= 64) return DRTOPK_EINVAL;
  if (cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess) return DRTOPK_ECUDA;
  char* ws = nullptr;
  size_t off = 0;
  {
    std::lock_guard<std::mutex> lk(g_static_mu);
    ws = static_cast<char*>(g_static_ptr[device]);
    off = g_static_ctrl[device];
  }
  if (!ws) return DRTOPK_OK;  // no no-allocation select has run on this device
  uint32_t err = 0;
  if (cudaMemcpy(&err, ws + off + 4 * drtopk::CW_ERR, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return DRTOPK_ECUDA;
  return drtopk::device_error_status(err);
}
