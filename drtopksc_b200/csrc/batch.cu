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

// ------------------------------------------------------------ autotuner
// Per segment, the configuration with the lowest modelled cost: HBM bytes at
// the copy bandwidth plus the select task's CTA time shared by the resident
// CTAs.  A block pass over n entries costs SEG_T_PASS (histogram clear,
// barriers, the pick) plus n * SEG_T_ELEM of one CTA.  The model prices every
// knob of drtopk_seg_params_t; it has no view of the keys, so it prices
// bucket levels as radix ones plus the min/max pass (the bucket select pays
// off on keys of a narrow range, which a caller can ask for) and 4-bit
// digits as twice the passes.
// Calibrated on B200 against forced-knob runs of the 4096-segment batch
// (lengths 2^10..2^22): a block pass is latency-bound (~2K entries per us
// and a few us of barriers and picks); a delegate entry costs about six
// times a candidate entry (the fastest alpha sat near 2^alpha ~
// sqrt(5 len / k)) and a raw key of a plain segment about 2.5 (plain
// segments were fastest up to ~16K keys); the bitonic network of a whole
// segment lost to the radix passes from ~1K keys up; and the beta-2
// sampler's top-two bookkeeping costs about as much as the keys' HBM time.
constexpr double SEG_BW = 6.0e6;        // HBM bytes per us (whole GPU)
constexpr double SEG_T_PASS = 4.0;      // us per block pass (one CTA)
constexpr double SEG_T_ELEM = 0.0005;   // us per entry per pass (one CTA)
constexpr double SEG_DEL_WEIGHT = 6.0;  // a delegate entry against a candidate entry
constexpr double SEG_KEY_WEIGHT = 2.5;  // a raw key of a plain segment against a candidate entry
constexpr double SEG_T_TASK = 1.0;      // us per sampler task (ticket, barriers)
constexpr double SEG_T_SAMP = 0.0006;   // us per key sampled (one CTA)
constexpr double SEG_T_SAMP2 = 8.6e-7;  // us of batch time per key: beta 2's top-two sampler
constexpr double SEG_T_STAGE = 1.0;     // us per bitonic stage (one CTA, up to 4096 entries)

struct SegChoice {
  int mode, alpha, beta, nbits, sel, chunk_log2;
  double cost;
};

double passes_of(int nbits, int sel) { return sel == SEG_BUCKET ? 1.0 + 32.0 / 8.0 : 32.0 / nbits; }

// one block select (passes) + the ordered take over n entries
double block_cost(double n, int nbits, int sel, double ctas) {
  const double p = passes_of(nbits, sel) + 1.0;
  return p * (SEG_T_PASS + n * SEG_T_ELEM) / ctas;
}

double sort_cost(uint32_t k, int sorted, double ctas) {
  if (!sorted) return 0.0;
  const double L = std::ceil(std::log2(std::max(2.0, (double)k)));
  return L * (L + 1.0) / 2.0 * SEG_T_STAGE / ctas;
}

SegChoice cost_plain(uint32_t len, uint32_t k, int sorted, int nbits, int sel, double ctas) {
  const double c = SEG_KEY_WEIGHT * block_cost(len, nbits, sel, ctas) + sort_cost(k, sorted, ctas);
  return {SEG_PLAIN, 0, 0, nbits, sel, 0, c + 4.0 * len / SEG_BW};
}

SegChoice cost_bitonic(uint32_t len, double ctas) {
  const double L = std::ceil(std::log2(std::max(2.0, (double)len)));
  const double c = (SEG_T_PASS + len * SEG_T_ELEM + L * (L + 1.0) / 2.0 * SEG_T_STAGE) / ctas;
  return {SEG_BITONIC, 0, 0, 8, SEG_RADIX, 0, c + 4.0 * len / SEG_BW};
}

SegChoice cost_delegate(uint32_t len, uint32_t k, int sorted, int alpha, int beta, int nbits, int sel, int chunk_log2,
                        double ctas) {
  const double S = std::ldexp(1.0, alpha), M = std::ceil(len / S);
  const double tasks = std::ceil(len / std::ldexp(1.0, chunk_log2));
  double hbm = 4.0 * len + 4.0 * M * (beta == 2 ? 3 : 1);
  double c = (tasks * SEG_T_TASK + len * SEG_T_SAMP) / ctas + (beta == 2 ? len * SEG_T_SAMP2 : 0.0);
  double cand;
  if (beta == 1) {
    c += SEG_DEL_WEIGHT * block_cost(M, nbits, sel, ctas);
    cand = k * S;  // the k kept subranges, read whole
    hbm += 4.0 * cand;
  } else {
    c += SEG_DEL_WEIGHT * block_cost(2.0 * M, nbits, sel, ctas);
    c += (SEG_T_PASS * 3.0 + M * SEG_T_ELEM * 2.0) / ctas;  // the ordered list of kept subranges
    // subranges holding >= 2 of the top keys are read whole, the others
    // give their Max (keys i.i.d.: lam top keys per subrange)
    const double lam = k * S / len;
    const double whole = M * (1.0 - std::exp(-lam) * (1.0 + lam));
    cand = whole * S + k;
    hbm += 4.0 * whole * S;
    c += cand * SEG_T_ELEM * 2.0 / ctas;  // virtual positions found by binary search
  }
  c += (SEG_T_PASS + cand * SEG_T_ELEM) / ctas;  // concatenation
  c += block_cost(cand, nbits, sel, ctas) + sort_cost(k, sorted, ctas);
  return {SEG_DELEGATE, alpha, beta, nbits, sel, chunk_log2, c + hbm / SEG_BW};
}

// keys per sampler task: about 16 tasks per segment (load balance), 8K..128K
// keys (ticket overhead), a whole number of subranges
int tuned_chunk(uint32_t len, int alpha) {
  const int c = (int)std::ceil(std::log2(std::max(1.0, len / 16.0)));
  return std::max(alpha, std::max(13, std::min(c, 17)));
}

// The tuner: every field of `want` that is -1 is chosen; the others are
// taken as given (checked).  Returns false for an impossible request.
bool choose(uint32_t len, uint32_t k, int sorted, const drtopk_seg_params_t& want, double ctas, SegDesc& d) {
  const int wa = want.algo, wal = want.alpha, wb = want.beta, wn = want.nbits, ws = want.bucket, wc = want.chunk_log2;
  if (wn != -1 && wn != 4 && wn != 8) return false;
  if (ws != -1 && ws != 0 && ws != 1) return false;
  if (wb != -1 && wb != 1 && wb != 2) return false;
  if (wc != -1 && (wc < 13 || wc > 20)) return false;
  SegChoice best = {SEG_PLAIN, 0, 0, 8, SEG_RADIX, 0, 1e300};
  auto consider = [&](const SegChoice& c) {
    if (c.cost < best.cost) best = c;
  };
  for (int nbits : {8, 4}) {
    if (wn != -1 && nbits != wn) continue;
    for (int sel : {SEG_RADIX, SEG_BUCKET}) {
      if (ws != -1 && sel != ws) continue;
      if ((wa == -1 || wa == DRTOPK_ALGO_PLAIN_RADIX) && wal <= 0 && wb == -1 && wc == -1)
        consider(cost_plain(len, k, sorted, nbits, sel, ctas));
      if (wa == -1 || wa == DRTOPK_ALGO_RADIX) {
        for (int alpha = 2; alpha <= 16; ++alpha) {
          if (wal != -1 && alpha != wal) continue;
          const uint64_t M = ((uint64_t)len + (1ull << alpha) - 1) >> alpha;
          for (int beta : {1, 2}) {
            if (wb != -1 && beta != wb) continue;
            if (beta == 1 && M < k) continue;
            if (beta == 2 && (2 * M < k || k > (uint32_t)SEG_B2_MAX_K)) continue;
            const int ch = wc != -1 ? wc : tuned_chunk(len, alpha);
            if (ch < alpha) continue;
            consider(cost_delegate(len, k, sorted, alpha, beta, nbits, sel, ch, ctas));
          }
        }
      }
    }
  }
  if ((wa == -1 || wa == DRTOPK_ALGO_BITONIC) && len <= (uint32_t)SEG_SORT_MAX && wal <= 0 && wb == -1 &&
      (wn == -1 || wn == 8) && ws <= 0 && wc == -1)
    consider(cost_bitonic(len, ctas));
  if (best.cost >= 1e300) return false;
  d.mode = best.mode;
  d.alpha = best.alpha;
  d.beta = best.mode == SEG_DELEGATE ? best.beta : 0;
  d.nbits = best.nbits;
  d.sel = best.sel;
  d.chunk_log2 = best.mode == SEG_DELEGATE ? best.chunk_log2 : 0;
  return true;
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
  return drtopk_batch_plan_params(b, nseg, h_offsets, h_ks, h_dtypes, sorted, nullptr);
}

extern "C" drtopk_status_t drtopk_batch_plan_params(drtopk_batch_t b, int nseg, const uint64_t* h_offsets,
                                                    const uint32_t* h_ks, const int* h_dtypes, int sorted,
                                                    const drtopk_seg_params_t* h_params) {
  if (!b || nseg <= 0 || !h_offsets || !h_ks) return DRTOPK_EINVAL;
  std::lock_guard<std::mutex> lk(b->mu);
  int grid = 0;
  size_t smem = 0;
  {
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(b->device);
    const cudaError_t e = segmented_shape(b->device, &grid, &smem);
    cudaSetDevice(cur);
    if (e != cudaSuccess) return DRTOPK_ECUDA;
  }
  const drtopk_seg_params_t tuned = {-1, -1, -1, -1, -1, -1};
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
    if (!choose(d.len, k, sorted, h_params ? h_params[s] : tuned, (double)grid, d)) return DRTOPK_EINVAL;
    d.out_off = out_total;
    out_total += k;
    if (d.mode == SEG_DELEGATE) {
      const uint64_t S = 1ull << d.alpha, M = (len + S - 1) >> d.alpha;
      d.del_off = del_total;
      del_total += M * (d.beta == 2 ? 3 : 1);
      d.cand_off = cand_total;
      // beta 1: the k kept subranges; beta 2: fewer than 2k read whole and
      // fewer than k single Maxes
      cand_total += d.beta == 2 ? 2 * (uint64_t)k * S + k : (uint64_t)k * S;
      const uint64_t CH = 1ull << d.chunk_log2;
      d.ntasks = (int)((len + CH - 1) / CH);
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

static int seg_algo(const SegDesc& d) {
  return d.mode == SEG_DELEGATE ? DRTOPK_ALGO_RADIX
                                : (d.mode == SEG_BITONIC ? DRTOPK_ALGO_BITONIC : DRTOPK_ALGO_PLAIN_RADIX);
}

extern "C" drtopk_status_t drtopk_batch_describe(drtopk_batch_t b, int* h_algo, int* h_alpha, int* h_beta) {
  if (!b || b->nseg == 0) return DRTOPK_EINVAL;
  for (int s = 0; s < b->nseg; ++s) {
    const SegDesc& d = b->seg[s];
    if (h_algo) h_algo[s] = seg_algo(d);
    if (h_alpha) h_alpha[s] = d.alpha;
    if (h_beta) h_beta[s] = d.beta;
  }
  return DRTOPK_OK;
}

extern "C" drtopk_status_t drtopk_batch_describe_params(drtopk_batch_t b, drtopk_seg_params_t* h_params) {
  if (!b || b->nseg == 0 || !h_params) return DRTOPK_EINVAL;
  for (int s = 0; s < b->nseg; ++s) {
    const SegDesc& d = b->seg[s];
    h_params[s] = {seg_algo(d), d.alpha, d.beta, d.nbits, d.sel, d.chunk_log2};
  }
  return DRTOPK_OK;
}
