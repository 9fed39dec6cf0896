// batch.cu -- host side of the batched form: per-segment planning
// (autotuned mode and subrange size), the ticket-ordered task table, the
// resident workspace, launch and CUDA-graph capture/replay.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/drtopk.h"
#define DRTOPK_DEFINE_SEGMENTED_KERNEL
#include "segmented.cuh"

using namespace drtopk;

namespace drtopk {
cudaError_t launch_segmented(const SegArgs& a, int grid, size_t smem, cudaStream_t st) {
  k_segmented<<<grid, SEG_THREADS, smem, st>>>(a);
  return cudaGetLastError();
}
cudaError_t segmented_shape(int device, int* grid, size_t* smem) {
  *smem = (size_t)(256 + 3 * SEG_MAX_K) * 4;
  int occ = 0, sms = 0;
  cudaError_t e = cudaFuncSetAttribute(k_segmented, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_segmented, SEG_THREADS, *smem);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  *grid = (occ > 0 ? occ : 1) * sms;
  return e;
}
}  // namespace drtopk

struct drtopk_batch {
  int device = 0;
  int nseg = 0;
  int sorted = 0;
  std::vector<SegDesc> seg;
  std::vector<uint2> tasks;
  char* ws = nullptr;  // one allocation: descriptors, tasks, pools, control
  size_t ws_bytes = 0;
  size_t off_seg = 0, off_tasks = 0, off_del = 0, off_cand = 0, off_ctrl = 0, ctrl_bytes = 0;
  int grid = 0;
  size_t smem = 0;
  cudaGraphExec_t gexec = nullptr;
  cudaGraph_t graph = nullptr;
  cudaStream_t cap_stream = nullptr;
  const void* g_keys = nullptr;
  void *g_kth = nullptr, *g_vals = nullptr;
  int64_t* g_idx = nullptr;
  std::mutex mu;
};

namespace {

inline size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

// Per-segment choice: plain block select for short segments, else the
// delegate path with S ~ sqrt(5 len / k) (delegates are written once and
// read ~4x from L2 by the block select; the k kept subranges are re-read).
void choose(uint32_t len, uint32_t k, int& mode, int& alpha) {
  if (len <= 32768) {
    mode = SEG_PLAIN;
    alpha = 0;
    return;
  }
  double s = std::sqrt(5.0 * (double)len / (double)k);
  int a = (int)std::lround(std::log2(std::max(2.0, s)));
  a = std::max(5, std::min(a, 15));
  while (a > 5 && ((((uint64_t)len + (1ull << a) - 1) >> a) < k)) a--;
  if ((((uint64_t)len + (1ull << a) - 1) >> a) < k) {
    mode = SEG_PLAIN;
    alpha = 0;
    return;
  }
  mode = SEG_DELEGATE;
  alpha = a;
}

cudaError_t free_graph(drtopk_batch* b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->gexec = nullptr;
  b->graph = nullptr;
  return cudaSuccess;
}

drtopk_status_t enqueue_batch(drtopk_batch* b, const void* d_keys, void* d_kth, void* d_vals, int64_t* d_idx,
                              cudaStream_t st) {
  if (cudaMemsetAsync(b->ws + b->off_ctrl, 0, b->ctrl_bytes, st) != cudaSuccess) return DRTOPK_ECUDA;
  uint32_t* ctrl = reinterpret_cast<uint32_t*>(b->ws + b->off_ctrl);
  SegArgs a;
  std::memset(&a, 0, sizeof(a));
  a.keys = static_cast<const uint32_t*>(d_keys);
  a.seg = reinterpret_cast<const SegDesc*>(b->ws + b->off_seg);
  a.tasks = reinterpret_cast<const uint2*>(b->ws + b->off_tasks);
  a.n_sampler_tasks = (uint32_t)b->tasks.size();
  a.nseg = (uint32_t)b->nseg;
  a.del_pool = reinterpret_cast<uint32_t*>(b->ws + b->off_del);
  a.cand_pool = reinterpret_cast<uint2*>(b->ws + b->off_cand);
  a.ticket = ctrl + 0;
  a.err = ctrl + 1;
  a.done = ctrl + 8;
  a.seg_err = ctrl + 8 + b->nseg;
  a.out_kth = static_cast<uint32_t*>(d_kth);
  a.out_vals = static_cast<uint32_t*>(d_vals);
  a.out_idx = d_idx;
  return launch_segmented(a, b->grid, b->smem, st) == cudaSuccess ? DRTOPK_OK : DRTOPK_ECUDA;
}

}  // namespace

extern "C" drtopk_status_t drtopk_batch_create(drtopk_batch_t* out, int device) {
  if (!out) return DRTOPK_EINVAL;
  *out = nullptr;
  drtopk_batch* b = new (std::nothrow) drtopk_batch();
  if (!b) return DRTOPK_ENOMEM;
  b->device = device;
  *out = b;
  return DRTOPK_OK;
}

extern "C" drtopk_status_t drtopk_batch_destroy(drtopk_batch_t b) {
  if (!b) return DRTOPK_OK;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(b->device);
  free_graph(b);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  if (b->ws) cudaFree(b->ws);
  cudaSetDevice(cur);
  delete b;
  return DRTOPK_OK;
}

extern "C" drtopk_status_t drtopk_batch_plan(drtopk_batch_t b, int nseg, const uint64_t* h_offsets,
                                             const uint32_t* h_ks, const int* h_dtypes, int sorted) {
  if (!b || nseg <= 0 || !h_offsets || !h_ks) return DRTOPK_EINVAL;
  std::lock_guard<std::mutex> lk(b->mu);
  std::vector<SegDesc> seg(nseg);
  std::vector<uint2> tasks;
  uint64_t del_total = 0, cand_total = 0, out_total = 0;
  for (int s = 0; s < nseg; ++s) {
    if (h_offsets[s + 1] < h_offsets[s]) return DRTOPK_EINVAL;
    const uint64_t len = h_offsets[s + 1] - h_offsets[s];
    const uint32_t k = h_ks[s];
    if (len == 0 || len > 0xffffffffull || k < 1 || k > len) return DRTOPK_EINVAL;
    if (k > (uint32_t)SEG_MAX_K) return DRTOPK_EUNSUPPORTED;
    const int dt = h_dtypes ? h_dtypes[s] : 0;
    if (dt != DRTOPK_U32 && dt != DRTOPK_F32) return DRTOPK_EINVAL;
    SegDesc& d = seg[s];
    d.key_off = h_offsets[s];
    d.len = (uint32_t)len;
    d.k = k;
    d.sorted = sorted;
    d.km = dt == DRTOPK_F32 ? KM_F32 : KM_U32;
    choose(d.len, k, d.mode, d.alpha);
    d.out_off = out_total;
    out_total += k;
    if (d.mode == SEG_DELEGATE) {
      const uint64_t S = 1ull << d.alpha, M = (len + S - 1) >> d.alpha;
      d.del_off = del_total;
      del_total += M;
      d.cand_off = cand_total;
      cand_total += (uint64_t)k * S;
      d.ntasks = (int)((len + SEG_CH - 1) / SEG_CH);
      for (int c = 0; c < d.ntasks; ++c) tasks.push_back(make_uint2((uint32_t)s, (uint32_t)c));
    } else {
      d.ntasks = 0;
    }
  }
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(b->device);
  drtopk_status_t st = DRTOPK_OK;
  size_t off = 0;
  const size_t off_seg = off;
  off += al256(sizeof(SegDesc) * nseg);
  const size_t off_tasks = off;
  off += al256(sizeof(uint2) * std::max<size_t>(1, tasks.size()));
  const size_t off_del = off;
  off += al256(4 * std::max<uint64_t>(1, del_total));
  const size_t off_cand = off;
  off += al256(8 * std::max<uint64_t>(1, cand_total));
  const size_t off_ctrl = off;
  const size_t ctrl_bytes = 4 * (8 + 2 * (size_t)nseg);
  off += al256(ctrl_bytes);
  free_graph(b);
  if (off > b->ws_bytes) {
    if (b->ws) cudaFree(b->ws);
    b->ws = nullptr;
    b->ws_bytes = 0;
    if (cudaMalloc(&b->ws, off) != cudaSuccess) {
      cudaGetLastError();
      st = DRTOPK_ENOMEM;
    } else {
      b->ws_bytes = off;
    }
  }
  if (st == DRTOPK_OK) {
    if (cudaMemcpy(b->ws + off_seg, seg.data(), sizeof(SegDesc) * nseg, cudaMemcpyHostToDevice) != cudaSuccess ||
        (!tasks.empty() && cudaMemcpy(b->ws + off_tasks, tasks.data(), sizeof(uint2) * tasks.size(),
                                      cudaMemcpyHostToDevice) != cudaSuccess))
      st = DRTOPK_ECUDA;
  }
  if (st == DRTOPK_OK) {
    if (segmented_shape(b->device, &b->grid, &b->smem) != cudaSuccess) st = DRTOPK_ECUDA;
  }
  if (st == DRTOPK_OK) {
    b->nseg = nseg;
    b->sorted = sorted;
    b->seg.swap(seg);
    b->tasks.swap(tasks);
    b->off_seg = off_seg;
    b->off_tasks = off_tasks;
    b->off_del = off_del;
    b->off_cand = off_cand;
    b->off_ctrl = off_ctrl;
    b->ctrl_bytes = ctrl_bytes;
  }
  cudaSetDevice(cur);
  return st;
}

extern "C" drtopk_status_t drtopk_batch_run(drtopk_batch_t b, const void* d_keys, void* d_kth, void* d_vals,
                                            int64_t* d_idx, void* stream) {
  if (!b || !d_keys || !d_kth || b->nseg == 0) return DRTOPK_EINVAL;
  std::lock_guard<std::mutex> lk(b->mu);
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(b->device);
  drtopk_status_t s = enqueue_batch(b, d_keys, d_kth, d_vals, d_idx, static_cast<cudaStream_t>(stream));
  cudaSetDevice(cur);
  return s;
}

extern "C" drtopk_status_t drtopk_batch_run_graph(drtopk_batch_t b, const void* d_keys, void* d_kth, void* d_vals,
                                                  int64_t* d_idx, void* stream) {
  if (!b || !d_keys || !d_kth || b->nseg == 0) return DRTOPK_EINVAL;
  std::lock_guard<std::mutex> lk(b->mu);
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(b->device);
  drtopk_status_t s = DRTOPK_OK;
  if (b->gexec && (b->g_keys != d_keys || b->g_kth != d_kth || b->g_vals != d_vals || b->g_idx != d_idx))
    free_graph(b);
  if (!b->gexec) {
    if (!b->cap_stream && cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking) != cudaSuccess)
      s = DRTOPK_ECUDA;
    if (s == DRTOPK_OK && cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      s = DRTOPK_ECUDA;
    if (s == DRTOPK_OK) {
      drtopk_status_t e = enqueue_batch(b, d_keys, d_kth, d_vals, d_idx, b->cap_stream);
      cudaError_t ce = cudaStreamEndCapture(b->cap_stream, &b->graph);
      if (e != DRTOPK_OK || ce != cudaSuccess) s = DRTOPK_ECUDA;
    }
    if (s == DRTOPK_OK && cudaGraphInstantiate(&b->gexec, b->graph, 0) != cudaSuccess) s = DRTOPK_ECUDA;
    if (s == DRTOPK_OK) {
      b->g_keys = d_keys;
      b->g_kth = d_kth;
      b->g_vals = d_vals;
      b->g_idx = d_idx;
    } else {
      free_graph(b);
      cudaGetLastError();
    }
  }
  if (s == DRTOPK_OK && cudaGraphLaunch(b->gexec, static_cast<cudaStream_t>(stream)) != cudaSuccess) s = DRTOPK_ECUDA;
  cudaSetDevice(cur);
  return s;
}

extern "C" drtopk_status_t drtopk_batch_sync_check(drtopk_batch_t b, void* stream) {
  if (!b || b->nseg == 0) return DRTOPK_EINVAL;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(b->device);
  drtopk_status_t s = DRTOPK_OK;
  uint32_t err = 0;
  if (cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess) s = DRTOPK_ECUDA;
  if (s == DRTOPK_OK &&
      cudaMemcpy(&err, b->ws + b->off_ctrl + 4, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    s = DRTOPK_ECUDA;
  if (s == DRTOPK_OK && err) s = (err & DE_BARRIER_TIMEOUT) ? DRTOPK_ETIMEOUT : DRTOPK_EDEVICE;
  cudaSetDevice(cur);
  return s;
}

extern "C" drtopk_status_t drtopk_batch_describe(drtopk_batch_t b, int* h_algo, int* h_alpha, int* h_beta) {
  if (!b || b->nseg == 0) return DRTOPK_EINVAL;
  for (int s = 0; s < b->nseg; ++s) {
    const SegDesc& d = b->seg[s];
    if (h_algo) h_algo[s] = d.mode == SEG_DELEGATE ? DRTOPK_ALGO_RADIX : DRTOPK_ALGO_PLAIN_RADIX;
    if (h_alpha) h_alpha[s] = d.alpha;
    if (h_beta) h_beta[s] = d.mode == SEG_DELEGATE ? 1 : 0;
  }
  return DRTOPK_OK;
}
