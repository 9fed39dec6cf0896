// api.cu -- host orchestration and the C ABI of libdrtopk.so.
//
// One select = memset of a small control block + the delegate sampler + one
// cooperative "fused" kernel (first select, filter/concatenation, second
// select, output).  Stream-ordered, no host synchronisation, graph-capturable.
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <new>
#include <vector>

#include "../../include/drtopk.h"
#include "bitonic.cuh"
#include "fused.cuh"
#include "kernels.h"
#include "plan.h"
#include "tail.cuh"
#include "sampler.cuh"

using namespace drtopk;

namespace drtopk {

// ------------------------------------------------------------ device info
struct DevInfo {
  int device = -1;
  int sms = 0;
  int occ_fused[4] = {0, 0, 0, 0};
  size_t occ_fused_smem[4] = {0, 0, 0, 0};
};

static std::mutex g_dev_mu;
static DevInfo g_dev[64];

static cudaError_t dev_info(int device, DevInfo** out) {
  std::lock_guard<std::mutex> lk(g_dev_mu);
  if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
  DevInfo& d = g_dev[device];
  if (d.device < 0) {
    cudaError_t e = cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    d.device = device;
  }
  *out = &d;
  return cudaSuccess;
}

static void* fused_ptr(int km) { return const_cast<void*>(kernels(km).fused); }

// the sampler kernel for (key mode, beta, positions, subrange size)
static const void* sampler_fn(int km, int beta, bool pos, int alpha) {
  const KernelSet& ks = kernels(km);
  if (alpha >= 9) return beta == 2 ? (pos ? ks.sample2posw : ks.sample2w) : ks.sample1w;
  return beta == 2 ? (pos ? ks.sample2pos : ks.sample2) : ks.sample1;
}

// resident CTAs per SM of a sampler kernel (cached per device)
static int sampler_occ(int device, const void* fn) {
  static std::map<std::pair<int, const void*>, int> cache;
  std::lock_guard<std::mutex> lk(g_dev_mu);
  int& o = cache[std::make_pair(device, fn)];
  if (o == 0) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, SAMPLE_THREADS, 0) != cudaSuccess) {
      cudaGetLastError();
      occ = 1;
    }
    o = std::max(1, occ);
  }
  return o;
}

static void* fused_cl_ptr(int km) { return const_cast<void*>(kernels(km).fused_cl); }

static void* fused_one_ptr(int km) { return const_cast<void*>(kernels(km).fused_one); }

// dynamic shared memory limit of the grouped one-CTA last levels
static bool fused_one_group_ready(int device, int km, size_t smem) {
  static size_t set[64][4];
  std::lock_guard<std::mutex> lk(g_dev_mu);
  if (device < 0 || device >= 64) return false;
  if (set[device][km] >= smem) return true;
  if (cudaFuncSetAttribute(kernels(km).fused_one_g, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  set[device][km] = smem;
  return true;
}

// dynamic shared memory limit of the one-CTA last-levels kernel (set once
// per device and key mode; the largest plan's need)
static bool fused_one_ready(int device, int km, size_t smem) {
  static size_t set[64][4];
  std::lock_guard<std::mutex> lk(g_dev_mu);
  if (device < 0 || device >= 64) return false;
  if (set[device][km] >= smem) return true;
  if (cudaFuncSetAttribute(fused_one_ptr(km), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  set[device][km] = smem;
  return true;
}

// Largest cluster (16, else 8, else 4) of k_fused_cl CTAs that the device
// can co-schedule with the largest dynamic shared memory a plan uses
// (FUSED_CL_SMEM_MAX, set once as the kernel's limit); 0 if none.
constexpr size_t FUSED_CL_SMEM_MAX = 100 * 1024;
static int cluster_size(DevInfo* d, int km, size_t smem) {
  static int cache[64][4];
  if (smem > FUSED_CL_SMEM_MAX) return 0;
  std::lock_guard<std::mutex> lk(g_dev_mu);
  int& c = cache[d->device][km];
  if (c != 0) return c > 0 ? c : 0;
  void* fn = fused_cl_ptr(km);
  c = -1;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FUSED_CL_SMEM_MAX) != cudaSuccess ||
      cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  for (int want : {16, 8, 4}) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(want);
    cfg.blockDim = dim3(FUSED_THREADS);
    cfg.dynamicSmemBytes = FUSED_CL_SMEM_MAX;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = want;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int ncl = 0;
    if (cudaOccupancyMaxActiveClusters(&ncl, fn, &cfg) == cudaSuccess && ncl > 0) {
      c = want;
      break;
    }
    cudaGetLastError();
  }
  return c > 0 ? c : 0;
}

static void* tail_ptr(int km) { return const_cast<void*>(kernels(km).tail); }
static cudaLaunchConfig_t tail_config(cudaStream_t st, cudaLaunchAttribute* at) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(TAIL_CLUSTER);
  cfg.blockDim = dim3(TAIL_THREADS);
  cfg.dynamicSmemBytes = TAIL_SMEM;
  cfg.stream = st;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = TAIL_CLUSTER;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cfg;
}
// whether the shared-memory tail cluster can run on this device (its
// shared-memory limit is set once per device and key mode)
static bool tail_ready(int device, int km) {
  static int state[64][4];  // 0 unknown, 1 ready, -1 unavailable
  std::lock_guard<std::mutex> lk(g_dev_mu);
  if (device < 0 || device >= 64) return false;
  int& s = state[device][km];
  if (s == 0) {
    s = -1;
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t cfg = tail_config(nullptr, at);
    int ncl = 0;
    if (cudaFuncSetAttribute(tail_ptr(km), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TAIL_SMEM) ==
            cudaSuccess &&
        cudaOccupancyMaxActiveClusters(&ncl, tail_ptr(km), &cfg) == cudaSuccess && ncl > 0)
      s = 1;
    else
      cudaGetLastError();
  }
  return s > 0;
}

// the ordinary (non-cooperative) kernels of split mode
enum SplitKernel : int {
  SK_GATHER = 0, SK_FILTER = 1, SK_LEVEL_HIST = 2, SK_SPLIT0 = 3, SK_EMIT = 4, SK_PRESAMPLE = 5, SK_PREREFINE = 6,
  SK_CAND_HIST = 7
};
static void* split_ptr(int km, int which) {
  const KernelSet& ks = kernels(km);
  switch (which) {
    case SK_FILTER: return const_cast<void*>(ks.filter);
    case SK_LEVEL_HIST: return const_cast<void*>(ks.level_hist);
    case SK_SPLIT0: return const_cast<void*>(ks.split0);
    case SK_EMIT: return const_cast<void*>(ks.emit);
    case SK_PRESAMPLE: return const_cast<void*>(ks.presample);
    case SK_PREREFINE: return const_cast<void*>(ks.prerefine);
    case SK_CAND_HIST: return const_cast<void*>(ks.cand_hist);
    default: return const_cast<void*>(ks.gather);
  }
}

// Candidates the sampled-threshold path expects: k, the six-sigma margin of
// the key sample (in keys), and one 16-bit prefix bin of uniform keys.
static double emit_cand_estimate(uint64_t n, uint64_t k, uint32_t stride) {
  const double s = stride ? (double)stride : (double)PRE_STRIDE_MIN;
  const double ks = (double)k / s;
  return (double)k + s * (6.0 * std::sqrt(ks) + 16.0) + (double)n / 65536.0;
}

// dynamic shared memory of a split-mode kernel: histogram words + warp stages
static size_t split_smem(int nb, int which) {
  if (which == SK_PRESAMPLE || which == SK_PREREFINE) return 0;
  const size_t h = (size_t)std::max(nb, 256) * 4;
  if (which == SK_FILTER) return h + SPLIT_FILTER_SMEM;
  if (which == SK_GATHER) return h + SPLIT_GATHER_SMEM;
  if (which == SK_EMIT) return SPLIT_GATHER_SMEM;
  return h;
}

static cudaError_t split_grid(DevInfo* d, int km, int which, size_t smem, int* grid) {
  static std::map<std::tuple<int, int, int, size_t>, int> occ_cache;
  std::lock_guard<std::mutex> lk(g_dev_mu);
  int& occ = occ_cache[std::make_tuple(d->device, km, which, smem)];
  if (occ == 0) {
    cudaError_t e = cudaFuncSetAttribute(split_ptr(km, which), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int o = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, split_ptr(km, which), FUSED_THREADS, smem);
    if (e != cudaSuccess) return e;
    occ = std::max(1, o);
  }
  *grid = occ * d->sms;
  return cudaSuccess;
}

static cudaError_t fused_max_grid(DevInfo* d, int km, size_t smem, int* grid) {
  std::lock_guard<std::mutex> lk(g_dev_mu);
  if (d->occ_fused[km] == 0 || d->occ_fused_smem[km] != smem) {
    int occ = 0;
    cudaError_t e = cudaFuncSetAttribute(fused_ptr(km), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fused_ptr(km), FUSED_THREADS, smem);
    if (e != cudaSuccess) return e;
    d->occ_fused[km] = std::max(1, occ);
    d->occ_fused_smem[km] = smem;
  }
  *grid = d->occ_fused[km] * d->sms;
  return cudaSuccess;
}

static void* bitonic_ptr(int km) { return const_cast<void*>(kernels(km).bitonic); }

static cudaError_t bitonic_max_grid(DevInfo* d, int km, size_t smem, int* grid) {
  static int occ_cache[64][4];
  std::lock_guard<std::mutex> lk(g_dev_mu);
  int& occ = occ_cache[d->device][km];
  if (occ == 0) {
    cudaError_t e = cudaFuncSetAttribute(bitonic_ptr(km), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int o = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, bitonic_ptr(km), FUSED_THREADS, smem);
    if (e != cudaSuccess) return e;
    occ = std::max(1, o);
  }
  *grid = occ * d->sms;
  return cudaSuccess;
}

// ------------------------------------------------------------ planning
static inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

drtopk_status_t device_error_status(uint32_t err) {
  if (!err) return DRTOPK_OK;
  return (err & DE_BARRIER_TIMEOUT) ? DRTOPK_ETIMEOUT : DRTOPK_EDEVICE;
}

int ref_alpha(double log2n, double k) {
  // baseline+filter+beta+shuffle/main.cu:83, evaluated as the reference does
  return (int)(0.5 * (log2n - std::log(k) / std::log(2.0) + 3));
}

drtopk_status_t make_plan(uint64_t n, uint64_t k, drtopk_dtype_t dtype, const drtopk_params_t* pin, int sms,
                          int fused_grid, Plan* P) {
  drtopk_params_t p;
  if (pin) p = *pin;
  else drtopk_params_default(&p);
  std::memset(P, 0, sizeof(*P));
  if (n == 0 || k < 1 || k > n) return DRTOPK_EINVAL;
  if (n > 0xffffffffull) return DRTOPK_EUNSUPPORTED;
  if (dtype != DRTOPK_U32 && dtype != DRTOPK_F32) return DRTOPK_EINVAL;
  if (!(p.nbits == 1 || p.nbits == 2 || p.nbits == 4 || p.nbits == 8)) return DRTOPK_EINVAL;
  if (p.algo == DRTOPK_ALGO_AUTO || p.alpha == -2) {
    drtopk_status_t s = drtopk_autotune(n, k, dtype, &p);
    if (s != DRTOPK_OK) return s;
  }
  if (p.algo != DRTOPK_ALGO_RADIX && p.algo != DRTOPK_ALGO_BUCKET && p.algo != DRTOPK_ALGO_PLAIN_RADIX &&
      p.algo != DRTOPK_ALGO_BITONIC)
    return DRTOPK_EINVAL;
  P->n = n;
  P->k = k;
  P->km = (dtype == DRTOPK_F32 ? 1 : 0) + (p.largest ? 0 : 2);
  P->algo = p.algo;
  P->bucket = p.algo == DRTOPK_ALGO_BUCKET;
  P->nbits = p.nbits;
  if (P->bucket) {
    if (p.num_bucket < 2 || p.num_bucket > 4096) return DRTOPK_EINVAL;
    P->nb = p.num_bucket;
  } else {
    P->nb = 1 << p.nbits;
  }
  P->sorted = p.sorted;
  const double log2n = std::log2((double)n);
  if (p.algo == DRTOPK_ALGO_BITONIC) {
    // bitonic/sampleBitonic.cu:198-221: k a power of two, NSubranges >= k;
    // the shared-memory network bounds k (bitonic_com.cuh:619-637)
    if ((k & (k - 1)) != 0 || k > (uint64_t)BITONIC_MAX_K) return DRTOPK_EINVAL;
    P->path = PATH_BITONIC;
    P->sorted = 1;
    int alpha = p.alpha;
    if (alpha < 0) {
      alpha = ref_alpha(log2n, (double)k);
      while (alpha > 2 && ((n + (1ull << alpha) - 1) >> alpha) < k) alpha--;
    }
    if (alpha == 0 || p.path == 3) {
      P->normal = 1;
      P->alpha = 0;
    } else {
      if (alpha < 2 || alpha > 24) return DRTOPK_EINVAL;
      P->alpha = alpha;
      P->S = 1ull << alpha;
      P->M = (n + P->S - 1) >> alpha;
      if (P->M < k) return DRTOPK_EINVAL;
    }
    P->fused_grid = fused_grid;
    return DRTOPK_OK;
  }
  if (p.path == 4 && p.algo == DRTOPK_ALGO_RADIX) {
    // sampled-threshold concatenation: no delegate vector (alpha unused)
    P->path = PATH_EMIT;
    P->alpha = 0;
    // sampled keys: one 512-key chunk in pre_stride, the sparsest stride in
    // [PRE_STRIDE_MIN, PRE_STRIDE_MAX] that keeps PRE_SAMPLE_CHUNKS chunks
    // (the sample passes' cost falls with the stride; the six-sigma margin
    // and the candidates it admits grow only with its square root); the
    // predicted threshold must keep k scaled to the sample plus a six-sigma
    // margin above it
    P->pre_stride = pre_stride_for(n);
    const uint64_t ns_keys = ((n >> 9) / P->pre_stride) * 512;
    const double ks = ns_keys ? (double)k * (double)ns_keys / (double)n : 0.0;
    const double t = std::ceil(ks + 6.0 * std::sqrt(ks) + 16.0);
    P->pre_target = (uint32_t)std::min(t, 4294967295.0);
    P->fused_grid = fused_grid;
    return DRTOPK_OK;
  }
  int alpha = p.alpha;
  const bool auto_alpha = alpha < 0;
  if (auto_alpha) {
    alpha = ref_alpha(log2n, (double)k);
    if (P->bucket && alpha < 5) alpha++;  // bucket_select/main.cu:67
  }
  if (alpha > 24) return DRTOPK_EINVAL;
  if (p.algo == DRTOPK_ALGO_PLAIN_RADIX || alpha <= 0) {
    P->path = PATH_PLAIN;
    P->alpha = 0;
  } else {
    int path;
    if (p.path == 0) path = alpha > 5 ? PATH_DEFAULT : PATH_BETA;  // main.cu:87-89
    else if (p.path == 1) path = PATH_DEFAULT;
    else if (p.path == 2) path = PATH_BETA;
    else return DRTOPK_EINVAL;

    if (path == PATH_BETA && p.beta != 2) return DRTOPK_EINVAL;  // beta 3/4 paths are broken in the reference
    uint64_t S = 1ull << alpha;
    uint64_t M = (n + S - 1) >> alpha;
    if (path == PATH_DEFAULT) {
      if (M < k || alpha < 2) {
        if (!auto_alpha || p.path == 1) return DRTOPK_EINVAL;
        // non-power-of-two n: shrink the subranges until k fit, else beta path
        while (alpha > 5 && ((n + (1ull << alpha) - 1) >> alpha) < k) alpha--;
        if (alpha <= 5) path = PATH_BETA;
        S = 1ull << alpha;
        M = (n + S - 1) >> alpha;
      }
    }
    if (path == PATH_BETA && alpha > 16) return DRTOPK_EINVAL;
    P->path = path;
    P->alpha = alpha;
    P->S = S;
    P->M = M;
  }
  const int D = 32 / P->nbits;
  if (P->path == PATH_BETA) {
    if (P->bucket) P->first_levels = 2;  // bucketselect_combined.cuh:972-1095 (two bucket levels)
    else if (p.first_digits == 0) P->first_levels = std::max(0, D - 3);
    else P->first_levels = std::min(p.first_digits > 0 ? p.first_digits : -p.first_digits, D);
    // first_digits < 0 (the autotuner's choice): at least that many digits,
    // refined while the chosen bin still holds more than max(2k, 256)
    // delegates.  The tuned digit count assumes keys spread like independent
    // uniform draws; where the delegates crowd into one bin (few distinct
    // values, float exponents) every subrange would otherwise qualify (uniform
    // [0,1) floats at n = 2^22, alpha 12: all 2048 delegate values share
    // their top 16 bits).  The reference's digit rule (0) and explicit counts
    // keep their digits, and the reference's counters.
    if (p.first_digits < 0 && !P->bucket) P->adapt_first = (uint32_t)std::max<uint64_t>(2 * k, 256);
  }
  P->fused_grid = fused_grid;
  return DRTOPK_OK;
}

// workspace layout; want_idx decides whether the beta sampler records positions
void layout(Plan* P, bool want_idx) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += align256(bytes);
    return o;
  };
  const uint64_t k = P->k;
  P->has_pos = (P->path == PATH_BETA && want_idx) ? 1 : 0;
  // control block (zeroed each call)
  // each run's histograms hold max(nb, 256) bins: the tie-fill sub-run
  // always uses 8-bit digits even when the bucket variant has fewer buckets
  P->hist_words = std::max(P->nb, 256);
  P->run_words = 3 * P->hist_words + (MAX_LEVELS + 2) + 1 + 4;
  size_t ctrl_words = CTRL_HDR_WORDS + 4 * (size_t)P->run_words + 8 * 256 + 8;  // large-k sort: totals + flag
  P->pre_hist_word = ctrl_words;
  ctrl_words += PRE_STATE + PRE_STATE_WORDS;  // sampled-threshold path: one 256-bin histogram per byte level
                                               // of the key sample, then the walk's state
  P->off_ctrl = take(ctrl_words * 4);
  P->ctrl_bytes = ctrl_words * 4;
  uint64_t ncand_cap = 0;
  if (P->path == PATH_BITONIC) {
    const uint64_t T = BITONIC_TILE;
    uint64_t cap;
    if (P->normal) cap = (P->n + T - 1) / T * k;
    else cap = std::max<uint64_t>((P->M + T - 1) / T * k, k * P->S);
    cap = std::max<uint64_t>(cap, T);
    P->bbuf_cap = cap;
    if (!P->normal) P->off_del = take(P->M * 4);
    P->off_bbuf0 = take(cap * 8);
    P->off_bbuf1 = take(cap * 8);
    P->ws_bytes = off;
    return;
  }
  if (P->path == PATH_DEFAULT) {
    P->off_del = take(P->M * 4);
    P->off_Atop = take(k * 8);
    P->off_Acbuf0 = take(P->M * 8);
    P->off_Acbuf1 = take(P->M * 8);
    ncand_cap = std::min<uint64_t>(P->n, k * P->S);
  } else if (P->path == PATH_BETA) {
    P->off_del = take(P->M * 8);
    if (P->has_pos) P->off_pos = take(P->M * 2);
    P->off_sel = take(P->M * 4);
    ncand_cap = P->n;
  } else {
    ncand_cap = (P->bounded && P->cap_bound) ? std::min<uint64_t>(P->n, P->cap_bound) : P->n;
  }
  P->cand_cap = ncand_cap;
  P->off_cand = take(ncand_cap * 8);
  P->off_Ccbuf0 = take(ncand_cap * 8);
  P->off_Ctop = take(k * 8);
  if (P->sorted && k > (uint64_t)SMALL_SORT) {
    P->off_sort0 = take(k * 8);
    P->off_sort1 = take(k * 8);
    P->off_sortcnt = take((size_t)P->fused_grid * 256 * 4);
  }
  P->ws_bytes = off;
}

}  // namespace drtopk

// ------------------------------------------------------------ handle
struct drtopk_handle {
  int device = 0;
  size_t budget = 0;
  void* ws = nullptr;
  size_t ws_bytes = 0;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  void* last_ctrl = nullptr;  // control block of the last call (for stats)
  Plan last_plan;
  bool have_last = false;
  std::vector<cudaEvent_t> prof;  // 3 events per recorded call
  int prof_max = 0, prof_used = 0;
  bool prof_on = false;
  std::mutex mu;
};

extern "C" void drtopk_params_default(drtopk_params_t* p) {
  p->team = 0;
  p->nbits = 8;
  p->alpha = -1;
  p->beta = 2;
  p->path = 0;
  p->algo = DRTOPK_ALGO_RADIX;
  p->num_bucket = 256;
  p->largest = 1;
  p->sorted = 0;
  p->first_digits = 0;
}

extern "C" const char* drtopk_status_str(drtopk_status_t s) {
  switch (s) {
    case DRTOPK_OK: return "ok";
    case DRTOPK_EINVAL: return "invalid argument";
    case DRTOPK_ENOMEM: return "out of device memory / workspace too small";
    case DRTOPK_ECUDA: return "CUDA error";
    case DRTOPK_EDEVICE: return "device-side check failed";
    case DRTOPK_EBUDGET: return "HBM budget exceeded";
    case DRTOPK_EUNSUPPORTED: return "unsupported";
    case DRTOPK_ETIMEOUT: return "device wait timed out";
    case DRTOPK_EAGAIN: return "try again";
    case DRTOPK_ECANCELLED: return "cancelled";
  }
  return "unknown";
}

extern "C" drtopk_status_t drtopk_create(drtopk_handle_t* h, int device, size_t hbm_budget_bytes) {
  if (!h) return DRTOPK_EINVAL;
  *h = nullptr;
  int cur = 0;
  if (cudaGetDevice(&cur) != cudaSuccess) return DRTOPK_ECUDA;
  if (cudaSetDevice(device) != cudaSuccess) return DRTOPK_EINVAL;
  DevInfo* di = nullptr;
  if (dev_info(device, &di) != cudaSuccess) { cudaSetDevice(cur); return DRTOPK_ECUDA; }
  drtopk_handle* hh = new (std::nothrow) drtopk_handle();
  if (!hh) { cudaSetDevice(cur); return DRTOPK_ENOMEM; }
  hh->device = device;
  hh->budget = hbm_budget_bytes;
  for (auto& e : hh->ev)
    if (cudaEventCreate(&e) != cudaSuccess) { cudaSetDevice(cur); delete hh; return DRTOPK_ECUDA; }
  cudaSetDevice(cur);
  *h = hh;
  return DRTOPK_OK;
}

extern "C" drtopk_status_t drtopk_destroy(drtopk_handle_t h) {
  if (!h) return DRTOPK_OK;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(h->device);
  if (h->ws) cudaFree(h->ws);
  for (auto& e : h->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : h->prof)
    if (e) cudaEventDestroy(e);
  cudaSetDevice(cur);
  delete h;
  return DRTOPK_OK;
}

namespace drtopk {
drtopk_status_t plan_select(int device, uint64_t n, uint64_t k, drtopk_dtype_t dtype, const drtopk_params_t* p,
                            bool want_idx, Plan* P);
}
static drtopk_status_t plan_for(int device, uint64_t n, uint64_t k, drtopk_dtype_t dtype, const drtopk_params_t* p,
                                bool want_idx, Plan* P, DevInfo** dout) {
  DevInfo* di = nullptr;
  if (dev_info(device, &di) != cudaSuccess) return DRTOPK_ECUDA;
  drtopk_status_t s = make_plan(n, k, dtype, p, di->sms, 0, P);
  if (s != DRTOPK_OK) return s;
  // dynamic shared memory of the fused kernel: histogram + two SMALL_SET
  // buffers for runs finished in one CTA (or the small top-k sort)
  size_t smem = (size_t)((std::max(P->nb, 256) + 3) & ~3) * 4 + 2 * (size_t)SMALL_SET * 8;
  if (P->sorted && k <= (uint64_t)SMALL_SORT) {
    size_t np2 = 1;
    while (np2 < k) np2 <<= 1;
    smem = std::max(smem, np2 * 8);
  }
  if (P->path == PATH_BITONIC) smem = (size_t)BITONIC_TILE * 8;
  P->fused_smem = smem;
  int maxgrid = 0;
  if ((P->path == PATH_BITONIC ? bitonic_max_grid(di, P->km, smem, &maxgrid)
                                : fused_max_grid(di, P->km, smem, &maxgrid)) != cudaSuccess)
    return DRTOPK_ECUDA;
  // grid: the whole GPU for large inputs, fewer CTAs for small ones (fewer
  // barrier participants)
  uint64_t want = std::max<uint64_t>((uint64_t)di->sms / 2, n >> 15);
  P->fused_grid = (int)std::min<uint64_t>((uint64_t)maxgrid, std::max<uint64_t>(1, want));
  // split mode: the concatenation reads >= 16 MB (beta filter over >= 2^21
  // subranges, or >= 2^22 keys re-read): run it as high-occupancy kernels
  if (P->path == PATH_BETA || P->path == PATH_DEFAULT) {
    const uint64_t concat = P->path == PATH_BETA ? P->M * 8 : k * P->S * 4;
    P->split = concat >= (16ull << 20) ? 1 : 0;
    if (P->split && (split_grid(di, P->km, SK_FILTER, split_smem(P->nb, SK_FILTER), &P->filter_grid) != cudaSuccess ||
                     split_grid(di, P->km, SK_GATHER, split_smem(P->nb, SK_GATHER), &P->split_grid) != cudaSuccess ||
                     split_grid(di, P->km, SK_LEVEL_HIST, split_smem(P->nb, SK_LEVEL_HIST), &P->hist_grid) !=
                         cudaSuccess ||
                     split_grid(di, P->km, SK_SPLIT0, split_smem(P->nb, SK_SPLIT0), &P->split0_grid) != cudaSuccess))
      return DRTOPK_ECUDA;
    // the beta path's threshold-only first select (radix, <= 2 levels) needs
    // no cooperative launch: its one histogram pass is k_level_hist and the
    // picks are made by every k_filter CTA
    P->first_pre = (P->split && P->path == PATH_BETA && !P->bucket && P->first_levels <= 2) ? 1 : 0;
  }
  if (P->path == PATH_EMIT) {
    // the streaming pass appends the candidates; the second select runs as
    // in split mode
    P->split = 1;
    if (split_grid(di, P->km, SK_EMIT, split_smem(P->nb, SK_EMIT), &P->emit_grid) != cudaSuccess ||
        split_grid(di, P->km, SK_SPLIT0, split_smem(P->nb, SK_SPLIT0), &P->split0_grid) != cudaSuccess ||
        split_grid(di, P->km, SK_PRESAMPLE, 0, &P->presample_grid) != cudaSuccess ||
        split_grid(di, P->km, SK_CAND_HIST, split_smem(P->nb, SK_CAND_HIST), &P->hist_grid) != cudaSuccess)
      return DRTOPK_ECUDA;
    // persistent grid over the sampled chunks, PRE_ROUND per warp and round
    const uint64_t nsw = ((n >> 9) / P->pre_stride + PRE_ROUND * SPLIT_WARPS - 1) / (PRE_ROUND * SPLIT_WARPS);
    P->presample_grid =
        (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)di->sms * PRE_CTAS_PER_SM, nsw));
    const uint64_t nct = ((n + 511) / 512 + SPLIT_WARPS - 1) / SPLIT_WARPS;
    P->emit_grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)P->emit_grid, nct));
    // team 5: every launch an ordinary one, the last levels in one CTA.  The
    // automatic team takes it too for unsorted outputs with k <= n/2048: the
    // bin left after level 0 is then small, and one CTA finishes it sooner
    // than the cooperative kernel's grid barriers (measured on B200 over the
    // n = 2^30 sweep: 1-2 % faster at k = 2^17..2^19, even at 2^20, slower
    // from 2^21)
    const int team_req = p ? p->team : 0;
    const bool one = team_req == 5 || (team_req == 0 && !P->sorted && k <= (n >> 11));
    P->one_cta = (one && fused_one_ready(di->device, P->km, smem)) ? 1 : 0;
  }
  // team of the phases after the sampler: one CTA with the sets in shared
  // memory when they are small (their cost is then round trips, not
  // bandwidth), else the whole GPU; a thread-block cluster on request
  P->cluster = 0;
  P->tail = 0;
  if (P->path != PATH_BITONIC && P->path != PATH_EMIT) {
    const int team = p ? p->team : 0;
    const double dn = (double)n, dk = (double)k, S = (double)P->S;
    // delegates, kept list and candidates must fit TAIL_CAP entries, and the
    // concatenation must be short enough for one CTA to stream
    const uint64_t Md = P->path == PATH_DEFAULT ? P->M : (P->path == PATH_BETA ? 2 * P->M : n);
    const bool fits = !P->bucket && P->nb <= 256 && Md <= (uint64_t)TAIL_CAP && k <= (uint64_t)TAIL_CAP &&
                      (!P->sorted || k <= (uint64_t)SMALL_SORT);
    double gather = 0.0, cand = 0.0;
    if (P->path == PATH_DEFAULT) {
      gather = dk * S;
      cand = dk;
    } else if (P->path == PATH_BETA) {
      const double q = dk / dn + std::ldexp(1.0, -8 * std::max(1, P->first_levels));
      const double lam = q * S, e = std::exp(-lam), M = dn / S;
      const double p_sel = 1.0 - e * (1.0 + lam);
      gather = M * p_sel * S;
      cand = M * lam * e + M * p_sel * (lam + 1.0);
    } else {
      cand = dn;
    }
    if (team == 3) {
      if (!fits || !tail_ready(di->device, P->km)) return DRTOPK_EUNSUPPORTED;
      P->tail = 1;
    } else if ((team == 0 || team == 4) && fits && gather <= TAIL_GATHER_AUTO && cand <= TAIL_CAP / 2 &&
               tail_ready(di->device, P->km)) {
      P->tail = 1;
    } else if (team == 2) {
      P->cluster = cluster_size(di, P->km, smem);
      if (P->cluster <= 0) return DRTOPK_EUNSUPPORTED;
    } else if (team == 4) {
      // shared GPU: a portable-size cluster finds room beside other kernels
      P->cluster = std::min(8, cluster_size(di, P->km, smem));
      if (P->cluster <= 0) P->cluster = 0;  // no cluster fits: the cooperative grid
    }
    if (P->tail || P->cluster) P->split = P->first_pre = 0;
  }
  // sampler grid: persistent, capped by the work items
  if (P->path != PATH_PLAIN && P->path != PATH_EMIT && !(P->path == PATH_BITONIC && P->normal)) {
    uint64_t items = P->alpha >= 9 ? P->M : ((n + 511) >> 9);
    uint64_t ctas = (items + SAMPLE_WARPS - 1) / SAMPLE_WARPS;
    const int beta = P->path == PATH_BETA ? 2 : 1;
    const bool pos = P->path == PATH_BETA && want_idx;
    // the warp-per-subrange pass streams best with 4 CTAs per SM (more
    // resident warps measured ~3 % slower at alpha 12-13)
    int occ = sampler_occ(di->device, sampler_fn(P->km, beta, pos, P->alpha));
    if (P->alpha >= 9) occ = std::min(occ, 4);
    P->sample_grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(ctas, (uint64_t)di->sms * occ));
  }
  layout(P, want_idx);
  if (dout) *dout = di;
  return DRTOPK_OK;
}

// plan (grid, shared memory, workspace layout) of a select on `device`
drtopk_status_t drtopk::plan_select(int device, uint64_t n, uint64_t k, drtopk_dtype_t dtype,
                                    const drtopk_params_t* p, bool want_idx, Plan* P) {
  return plan_for(device, n, k, dtype, p, want_idx, P, nullptr);
}

drtopk_status_t drtopk::plan_select_bounded(int device, uint64_t n, uint64_t k, drtopk_dtype_t dtype,
                                            const drtopk_params_t* p, bool want_idx, Plan* P) {
  drtopk_status_t s = plan_for(device, n, k, dtype, p, want_idx, P, nullptr);
  if (s != DRTOPK_OK || P->path != PATH_EMIT || !P->one_cta) return s;
  // twice the expected candidates (k, the six-sigma margin, one 16-bit
  // prefix bin) plus 64K
  const double est = emit_cand_estimate(n, k, P->pre_stride);
  P->bounded = 1;
  P->cap_bound = (uint64_t)(2.0 * est) + 65536;
  layout(P, want_idx);
  return DRTOPK_OK;
}

extern "C" drtopk_status_t drtopk_workspace_size(uint64_t n, uint64_t k, drtopk_dtype_t dtype,
                                                 const drtopk_params_t* p, size_t* bytes) {
  if (!bytes) return DRTOPK_EINVAL;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    // no device: plan with a nominal B200 shape (148 SMs, 4 CTAs/SM)
    Plan P;
    drtopk_status_t s = make_plan(n, k, dtype, p, 148, 592, &P);
    if (s != DRTOPK_OK) return s;
    layout(&P, true);
    *bytes = P.ws_bytes;
    return DRTOPK_OK;
  }
  Plan P;
  drtopk_status_t s = plan_for(dev, n, k, dtype, p, true, &P, nullptr);
  if (s != DRTOPK_OK) {
    // CPU-only process or unusable device: fall back to the nominal shape
    if (s != DRTOPK_ECUDA) return s;
    s = make_plan(n, k, dtype, p, 148, 592, &P);
    if (s != DRTOPK_OK) return s;
    layout(&P, true);
  }
  *bytes = P.ws_bytes;
  return DRTOPK_OK;
}

// ------------------------------------------------------------ launch
namespace drtopk {

static cudaError_t launch_sample(int km, SampleArgs sa, int beta, bool pos, int grid, cudaStream_t st) {
  const void* fn = sampler_fn(km, beta, pos, sa.alpha);
  void* args[] = {&sa};
  return cudaLaunchKernel(fn, dim3(grid), dim3(SAMPLE_THREADS), args, 0, st);
}

static RunBufs run_bufs(char* ctrl, const Plan& P, int which) {
  uint32_t* base = reinterpret_cast<uint32_t*>(ctrl) + CTRL_HDR_WORDS + (size_t)which * P.run_words;
  RunBufs r;
  r.H[0] = base;
  r.H[1] = base + P.hist_words;
  r.H[2] = base + 2 * P.hist_words;
  r.set_count = base + 3 * P.hist_words;
  r.top_count = base + 3 * P.hist_words + MAX_LEVELS + 2;
  r.res = base + 3 * P.hist_words + MAX_LEVELS + 2 + 1;
  r.cbuf[0] = r.cbuf[1] = nullptr;
  r.top = nullptr;
  r.top_cap = 0;
  r.cbuf_cap = 0;
  r.err = reinterpret_cast<uint32_t*>(ctrl) + CW_ERR;
  r.out_km = 0;
  r.out_vals = nullptr;
  r.out_idx = nullptr;
  return r;
}

static cudaError_t launch_sampler_km(const Plan& P, const SampleArgs& sa, int beta, cudaStream_t st) {
  return launch_sample(P.km, sa, beta, P.has_pos, P.sample_grid, st);
}

constexpr int PHASE3_GRID = 64;  // CTAs of the split-mode phase-3 launch (unsorted output)

static drtopk_status_t launch_coop(void* fn, const Plan& P, void* argp, cudaStream_t st, int grid = 0) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid > 0 ? grid : P.fused_grid);
  cfg.blockDim = dim3(FUSED_THREADS);
  cfg.dynamicSmemBytes = P.fused_smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* args[] = {argp};
  return cudaLaunchKernelExC(&cfg, fn, args) == cudaSuccess ? DRTOPK_OK : DRTOPK_ECUDA;
}

static drtopk_status_t launch_cluster(const Plan& P, const FusedArgs* a, cudaStream_t st) {
  const int csize = P.cluster;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(csize);
  cfg.blockDim = dim3(FUSED_THREADS);
  cfg.dynamicSmemBytes = P.fused_smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const FusedArgs* list = nullptr;
  void* args[] = {const_cast<FusedArgs*>(a), &list};
  return cudaLaunchKernelExC(&cfg, fused_cl_ptr(P.km), args) == cudaSuccess ? DRTOPK_OK : DRTOPK_ECUDA;
}

static drtopk_status_t enqueue_bitonic(const Plan& P, const void* d_keys, void* d_kth, void* d_vals, int64_t* d_idx,
                                       char* ws, cudaStream_t st, cudaEvent_t* ev) {
  char* ctrl = ws + P.off_ctrl;
  uint32_t* cw = reinterpret_cast<uint32_t*>(ctrl);
  const bool vec_ok = (reinterpret_cast<uintptr_t>(d_keys) & 15u) == 0;
  BitonicArgs b;
  std::memset(&b, 0, sizeof(b));
  b.keys = static_cast<const uint32_t*>(d_keys);
  b.n = P.n;
  b.k = (uint32_t)P.k;
  b.km = P.km;
  b.alpha = P.alpha;
  b.M = P.M;
  b.normal = P.normal;
  b.vec_ok = vec_ok;
  b.del = P.normal ? nullptr : reinterpret_cast<const uint32_t*>(ws + P.off_del);
  b.buf[0] = reinterpret_cast<uint64_t*>(ws + P.off_bbuf0);
  b.buf[1] = reinterpret_cast<uint64_t*>(ws + P.off_bbuf1);
  b.buf_cap = P.bbuf_cap;
  b.cand_count = cw + CW_CAND_COUNT;
  b.out_kth = static_cast<uint32_t*>(d_kth);
  b.out_vals = static_cast<uint32_t*>(d_vals);
  b.out_idx = d_idx;
  b.stats = cw + CW_STATS;
  b.gb.count = cw + CW_BAR_COUNT;
  b.gb.err = cw + CW_ERR;
  b.gb.nblocks = (uint32_t)P.fused_grid;
  if (!P.normal) {
    SampleArgs sa;
    std::memset(&sa, 0, sizeof(sa));
    sa.keys = b.keys;
    sa.n = P.n;
    sa.alpha = P.alpha;
    sa.nbits = 8;
    sa.hmode = 0;
    sa.vec_ok = vec_ok;
    sa.del = const_cast<uint32_t*>(b.del);
    sa.err = cw + CW_ERR;
    if (launch_sampler_km(P, sa, 1, st) != cudaSuccess) return DRTOPK_ECUDA;
  }
  if (ev) cudaEventRecord(ev[1], st);
  drtopk_status_t s = launch_coop(bitonic_ptr(P.km), P, &b, st);
  if (ev) cudaEventRecord(ev[2], st);
  return s;
}

// the kernels' arguments of one select: plan P over d_keys with the
// workspace at ws and the control block at ctrl (normally ws + P.off_ctrl)
static void fill_args(const Plan& P, const void* d_keys, void* d_kth, void* d_vals, int64_t* d_idx, char* ws,
                      char* ctrl, FusedArgs* out) {
  uint32_t* cw = reinterpret_cast<uint32_t*>(ctrl);
  const bool vec_ok = (reinterpret_cast<uintptr_t>(d_keys) & 15u) == 0;
  FusedArgs& a = *out;
  std::memset(&a, 0, sizeof(a));
  a.keys = static_cast<const uint32_t*>(d_keys);
  a.n = P.n;
  a.k = (uint32_t)P.k;
  a.km = P.km;
  a.path = P.path;
  a.bucket = P.bucket;
  a.nbits = P.nbits;
  a.nb = P.nb;
  a.alpha = P.alpha;
  a.M = P.M;
  a.first_levels = P.first_levels;
  a.adapt_first = P.adapt_first;
  a.vec_ok = vec_ok;
  a.del_minmax = cw + CW_DEL_MINMAX;
  a.A = run_bufs(ctrl, P, 0);
  a.AF = run_bufs(ctrl, P, 1);
  a.C = run_bufs(ctrl, P, 2);
  a.CF = run_bufs(ctrl, P, 3);
  a.cand_count = cw + CW_CAND_COUNT;
  a.sel_count = cw + CW_SEL_COUNT;
  a.cand_minmax = cw + CW_CAND_MINMAX;
  a.stats = cw + CW_STATS;
  a.sort_tot = cw + CTRL_HDR_WORDS + 4 * (size_t)P.run_words;
  a.gb.count = cw + CW_BAR_COUNT;
  a.gb.err = cw + CW_ERR;
  a.gb.nblocks = (uint32_t)P.fused_grid;
  a.thr_word = cw + CW_THR;
  a.tail_flag = cw + CW_TAIL;
  a.tie_cut = cw + CW_TIE_CUT;
  a.pre_hist = cw + P.pre_hist_word;
  a.pre_target = P.pre_target;
  a.pre_stride = P.pre_stride ? P.pre_stride : PRE_STRIDE_MIN;
  a.bounded = P.bounded;
  a.phase_lo = 1;
  a.phase_hi = 3;
  a.out_kth = static_cast<uint32_t*>(d_kth);
  a.out_vals = static_cast<uint32_t*>(d_vals);
  a.out_idx = d_idx;
  a.sorted = P.sorted;
  a.cand = reinterpret_cast<uint2*>(ws + P.off_cand);
  a.cand_cap = P.cand_cap;
  a.C.top_cap = a.CF.top_cap = P.k;
  a.C.cbuf_cap = a.CF.cbuf_cap = P.cand_cap;
  if (P.path == PATH_DEFAULT) {
    a.A.top_cap = a.AF.top_cap = P.k;
    a.A.cbuf_cap = a.AF.cbuf_cap = P.M;
  }
  a.C.top = reinterpret_cast<uint2*>(ws + P.off_Ctop);
  a.C.out_km = P.km;
  a.C.out_vals = a.out_vals;
  a.C.out_idx = d_idx;
  a.C.cbuf[0] = reinterpret_cast<uint2*>(ws + P.off_Ccbuf0);
  a.C.cbuf[1] = a.cand;  // level >= 1 may overwrite the candidates
  if (P.path == PATH_DEFAULT) {
    a.del = reinterpret_cast<const uint32_t*>(ws + P.off_del);
    a.A.top = reinterpret_cast<uint2*>(ws + P.off_Atop);
    a.A.cbuf[0] = reinterpret_cast<uint2*>(ws + P.off_Acbuf0);
    a.A.cbuf[1] = reinterpret_cast<uint2*>(ws + P.off_Acbuf1);
  } else if (P.path == PATH_BETA) {
    a.del = reinterpret_cast<const uint32_t*>(ws + P.off_del);
    a.has_pos = P.has_pos;
    if (P.has_pos) a.pos = reinterpret_cast<const uint16_t*>(ws + P.off_pos);
    a.sel = reinterpret_cast<uint32_t*>(ws + P.off_sel);
  }
  if (P.sorted && P.k > (uint64_t)SMALL_SORT) {
    a.sort_buf[0] = reinterpret_cast<uint64_t*>(ws + P.off_sort0);
    a.sort_buf[1] = reinterpret_cast<uint64_t*>(ws + P.off_sort1);
    a.sort_cnt = reinterpret_cast<uint32_t*>(ws + P.off_sortcnt);
  }
}

drtopk_status_t enqueue_select(const Plan& P, int device, const void* d_keys, void* d_kth, void* d_vals,
                               int64_t* d_idx, char* ws, cudaStream_t st, cudaEvent_t* ev) {
  char* ctrl = ws + P.off_ctrl;
  uint32_t* cw = reinterpret_cast<uint32_t*>(ctrl);
  if (cudaMemsetAsync(ctrl, 0, P.ctrl_bytes, st) != cudaSuccess) return DRTOPK_ECUDA;
  if (ev) cudaEventRecord(ev[0], st);
  if (P.path == PATH_BITONIC) return enqueue_bitonic(P, d_keys, d_kth, d_vals, d_idx, ws, st, ev);
  const bool vec_ok = (reinterpret_cast<uintptr_t>(d_keys) & 15u) == 0;
  FusedArgs a;
  fill_args(P, d_keys, d_kth, d_vals, d_idx, ws, ctrl, &a);
  // ---- sampled-threshold path: sample, predict, emit, then the second select
  if (P.path == PATH_EMIT) {
    // the streaming interval (ev[0] -> ev[1]) is the sample passes and the
    // appending pass, the counterpart of the delegate paths' sampler
    void* args[] = {&a};
    drtopk_status_t s = DRTOPK_OK;
    if (cudaLaunchKernel(split_ptr(P.km, SK_PRESAMPLE), dim3(P.presample_grid), dim3(FUSED_THREADS), args, 0, st) !=
        cudaSuccess)
      s = DRTOPK_ECUDA;
    for (int level = 1; level < PRE_LEVELS && s == DRTOPK_OK; ++level) {
      void* rargs[] = {&a, &level};
      if (cudaLaunchKernel(split_ptr(P.km, SK_PREREFINE), dim3(P.presample_grid), dim3(FUSED_THREADS), rargs, 0,
                           st) != cudaSuccess)
        s = DRTOPK_ECUDA;
    }
    if (s == DRTOPK_OK && cudaLaunchKernel(split_ptr(P.km, SK_EMIT), dim3(P.emit_grid), dim3(FUSED_THREADS), args,
                                           split_smem(P.nb, SK_EMIT), st) != cudaSuccess)
      s = DRTOPK_ECUDA;
    if (ev) cudaEventRecord(ev[1], st);
    if (s == DRTOPK_OK &&
        cudaLaunchKernel(split_ptr(P.km, SK_CAND_HIST), dim3(P.hist_grid), dim3(FUSED_THREADS), args,
                         split_smem(P.nb, SK_CAND_HIST), st) != cudaSuccess)
      s = DRTOPK_ECUDA;
    if (s == DRTOPK_OK) {
      a.split0 = 1;
      a.direct0 = P.sorted ? 0 : 1;
      if (cudaLaunchKernel(split_ptr(P.km, SK_SPLIT0), dim3(P.split0_grid), dim3(FUSED_THREADS), args,
                           split_smem(P.nb, SK_SPLIT0), st) != cudaSuccess)
        s = DRTOPK_ECUDA;
    }
    if (s == DRTOPK_OK) {
      a.phase_lo = 3;
      a.phase_hi = 3;
      if (P.one_cta) {
        void* args1[] = {&a};
        a.gb.nblocks = 1;
        if (cudaLaunchKernel(fused_one_ptr(P.km), dim3(1), dim3(FUSED_THREADS), args1, P.fused_smem, st) !=
            cudaSuccess)
          s = DRTOPK_ECUDA;
      } else {
        const int g3 = !P.sorted ? std::min(P.fused_grid, PHASE3_GRID) : P.fused_grid;
        a.gb.nblocks = (uint32_t)g3;
        s = launch_coop(fused_ptr(P.km), P, &a, st, g3);
      }
    }
    if (ev) cudaEventRecord(ev[2], st);
    return s;
  }
  // ---- sampler
  if (P.path != PATH_PLAIN) {
    SampleArgs sa;
    sa.keys = a.keys;
    sa.n = P.n;
    sa.alpha = P.alpha;
    sa.nbits = P.nbits;
    sa.hmode = P.bucket ? 2 : 1;
    sa.vec_ok = vec_ok;
    sa.del = const_cast<uint32_t*>(a.del);
    sa.pos = const_cast<uint16_t*>(a.pos);
    sa.hist = a.A.H[0];
    sa.minmax = cw + CW_DEL_MINMAX;
    sa.err = cw + CW_ERR;
    const int beta = P.path == PATH_BETA ? 2 : 1;
    if (launch_sampler_km(P, sa, beta, st) != cudaSuccess) return DRTOPK_ECUDA;
  }
  if (ev) cudaEventRecord(ev[1], st);
  // ---- fused cooperative kernel (split mode: phase 1, concatenation kernels, phase 3)
  drtopk_status_t s;
  if (P.tail) {
    a.gb.nblocks = TAIL_CLUSTER;
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t cfg = tail_config(st, at);
    void* args[] = {&a};
    s = cudaLaunchKernelExC(&cfg, tail_ptr(P.km), args) == cudaSuccess ? DRTOPK_OK : DRTOPK_ECUDA;
  } else if (P.cluster > 0) {
    a.gb.nblocks = (uint32_t)P.cluster;
    s = launch_cluster(P, &a, st);
  } else if (!P.split) {
    s = launch_coop(fused_ptr(P.km), P, &a, st);
  } else {
    a.phase_hi = 1;
    if (P.first_pre) {
      a.first_pre = 1;
      s = DRTOPK_OK;
      if (P.first_levels >= 2) {
        void* args[] = {&a};
        if (cudaLaunchKernel(split_ptr(P.km, SK_LEVEL_HIST), dim3(P.hist_grid), dim3(FUSED_THREADS), args,
                             split_smem(P.nb, SK_LEVEL_HIST), st) != cudaSuccess)
          s = DRTOPK_ECUDA;
      }
    } else {
      s = launch_coop(fused_ptr(P.km), P, &a, st);
    }
    if (s == DRTOPK_OK && P.path == PATH_BETA) {
      void* args[] = {&a};
      if (cudaLaunchKernel(split_ptr(P.km, SK_FILTER), dim3(P.filter_grid), dim3(FUSED_THREADS), args,
                           split_smem(P.nb, SK_FILTER), st) != cudaSuccess)
        s = DRTOPK_ECUDA;
    }
    if (s == DRTOPK_OK) {
      void* args[] = {&a};
      if (cudaLaunchKernel(split_ptr(P.km, SK_GATHER), dim3(P.split_grid), dim3(FUSED_THREADS), args,
                           split_smem(P.nb, SK_GATHER), st) != cudaSuccess)
        s = DRTOPK_ECUDA;
    }
    if (s == DRTOPK_OK && !P.bucket) {
      // level 0 of the second select as an ordinary kernel; unsorted
      // output is written by it directly
      a.split0 = 1;
      a.direct0 = P.sorted ? 0 : 1;
      void* args[] = {&a};
      if (cudaLaunchKernel(split_ptr(P.km, SK_SPLIT0), dim3(P.split0_grid), dim3(FUSED_THREADS), args,
                           split_smem(P.nb, SK_SPLIT0), st) != cudaSuccess)
        s = DRTOPK_ECUDA;
    }
    if (s == DRTOPK_OK) {
      a.phase_lo = 3;
      a.phase_hi = 3;
      // after k_split0 the unsorted second select goes on with one bin's
      // members and copies the few later entries: round trips, not bytes,
      // so a smaller team (cheaper grid barriers and histogram flushes)
      const int g3 = (a.split0 && !P.sorted) ? std::min(P.fused_grid, PHASE3_GRID) : P.fused_grid;
      a.gb.nblocks = (uint32_t)g3;
      s = launch_coop(fused_ptr(P.km), P, &a, st, g3);
    }
  }
  if (ev) cudaEventRecord(ev[2], st);
  return s;
}

// ------------------------------------------------------------ grouped selects
// Stages of a grouped sampled-threshold chain, in launch order.
enum GroupStage : int {
  GS_PRESAMPLE = 0, GS_REFINE1, GS_REFINE2, GS_REFINE3, GS_EMIT, GS_CAND_HIST, GS_SPLIT0, GS_LAST, GS_COUNT
};

size_t group_desc_bytes(int nprob) {
  return align256(sizeof(FusedArgs) * (size_t)nprob) + align256(4 * (size_t)GS_COUNT * (nprob + 1));
}

// CTAs of one select at each stage of a grouped chain, sized to its work
// (each grouped launch covers every problem of the group)
static uint32_t group_ctas(const Plan& P, int stage) {
  const uint64_t n = P.n, k = P.k;
  const double cand = emit_cand_estimate(n, k, P.pre_stride);
  auto clampc = [](uint64_t v, uint64_t cap) { return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(v, cap)); };
  switch (stage) {
    case GS_PRESAMPLE:
    case GS_REFINE1:
    case GS_REFINE2:
    case GS_REFINE3: {
      const uint64_t ns = (n >> 9) / P.pre_stride;
      return clampc((ns + PRE_ROUND * SPLIT_WARPS - 1) / (PRE_ROUND * SPLIT_WARPS), (uint64_t)P.presample_grid);
    }
    case GS_EMIT:  // at least eight 512-key chunks per warp
      return clampc((((n + 511) >> 9) + 8 * SPLIT_WARPS - 1) / (8 * SPLIT_WARPS), (uint64_t)P.emit_grid);
    case GS_CAND_HIST:
      return clampc((uint64_t)(1.5 * cand / (FUSED_THREADS * 8)) + 1, (uint64_t)P.hist_grid);
    case GS_SPLIT0:
      return clampc((uint64_t)(1.5 * cand / (FUSED_THREADS * 8)) + 1, (uint64_t)P.split0_grid);
    default:
      return 1;
  }
}

drtopk_status_t enqueue_group(int device, int km, const GroupItem* items, int nprob, char* h_stage, char* d_desc,
                              uint32_t* d_err_out, cudaStream_t st) {
  (void)device;
  if (nprob <= 0) return DRTOPK_OK;
  FusedArgs* hargs = reinterpret_cast<FusedArgs*>(h_stage);
  uint32_t* hpre = reinterpret_cast<uint32_t*>(h_stage + align256(sizeof(FusedArgs) * (size_t)nprob));
  uint32_t tot[GS_COUNT] = {};
  size_t smem_last = 0;
  for (int i = 0; i < nprob; ++i) {
    const Plan& P = *items[i].P;
    if (P.path != PATH_EMIT || !P.one_cta || P.km != km) return DRTOPK_EINVAL;
    FusedArgs& a = hargs[i];
    fill_args(P, items[i].keys, items[i].d_kth, items[i].d_vals, items[i].d_idx, items[i].ws, items[i].ctrl, &a);
    a.split0 = 1;
    a.direct0 = P.sorted ? 0 : 1;
    a.phase_lo = 3;
    a.phase_hi = 3;
    a.gb.nblocks = 1;
    smem_last = std::max(smem_last, P.fused_smem);
    for (int s = 0; s < GS_COUNT; ++s) {
      hpre[s * (nprob + 1) + i] = tot[s];
      tot[s] += group_ctas(P, s);
    }
  }
  for (int s = 0; s < GS_COUNT; ++s) hpre[s * (nprob + 1) + nprob] = tot[s];
  if (cudaMemcpyAsync(d_desc, h_stage, group_desc_bytes(nprob), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return DRTOPK_ECUDA;
  const KernelSet& ks = kernels(km);
  const void* fns[GS_COUNT] = {ks.presample_g, ks.prerefine_g,  ks.prerefine_g, ks.prerefine_g,
                               ks.emit_g,      ks.cand_hist_g, ks.split0_g,    ks.fused_one_g};
  const int nb = items[0].P->nb;
  const size_t smem[GS_COUNT] = {0, 0, 0, 0, split_smem(nb, SK_EMIT), split_smem(nb, SK_CAND_HIST),
                                 split_smem(nb, SK_SPLIT0), smem_last};
  if (!fused_one_group_ready(device, km, smem_last)) return DRTOPK_ECUDA;
  const uint32_t* dpre = reinterpret_cast<const uint32_t*>(d_desc + align256(sizeof(FusedArgs) * (size_t)nprob));
  for (int s = 0; s < GS_COUNT; ++s) {
    GroupArgs g;
    g.probs = reinterpret_cast<const FusedArgs*>(d_desc);
    g.prefix = dpre + s * (nprob + 1);
    g.nprob = (uint32_t)nprob;
    int level = s - GS_PRESAMPLE;  // byte level of the refine stages (k_prerefine_g's second argument)
    void* args[] = {&g, &level};
    if (cudaLaunchKernel(fns[s], dim3(tot[s]), dim3(FUSED_THREADS), args, smem[s], st) != cudaSuccess)
      return DRTOPK_ECUDA;
  }
  k_group_errors<<<1, 256, 0, st>>>(reinterpret_cast<const FusedArgs*>(d_desc), (uint32_t)nprob, d_err_out);
  return cudaGetLastError() == cudaSuccess ? DRTOPK_OK : DRTOPK_ECUDA;
}

}  // namespace drtopk

static drtopk_status_t ensure_ws(drtopk_handle_t h, size_t bytes) {
  if (h->ws_bytes >= bytes) return DRTOPK_OK;
  if (h->budget && bytes > h->budget) return DRTOPK_EBUDGET;
  if (h->ws) {
    cudaFree(h->ws);
    h->ws = nullptr;
    h->ws_bytes = 0;
  }
  size_t want = std::max(bytes, (size_t)(1 << 20));
  if (cudaMalloc(&h->ws, want) != cudaSuccess) {
    cudaGetLastError();
    return DRTOPK_ENOMEM;
  }
  h->ws_bytes = want;
  return DRTOPK_OK;
}

static drtopk_status_t select_impl(drtopk_handle_t h, const void* d_keys, drtopk_dtype_t dtype, uint64_t n,
                                   uint64_t k, const drtopk_params_t* p, void* d_kth, void* d_vals, int64_t* d_idx,
                                   void* d_ws, size_t ws_bytes, void* stream) {
  if (!h || !d_keys) return DRTOPK_EINVAL;
  std::lock_guard<std::mutex> lk(h->mu);
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != h->device) cudaSetDevice(h->device);
  Plan P;
  drtopk_status_t s = plan_for(h->device, n, k, dtype, p, d_idx != nullptr, &P, nullptr);
  char* ws = nullptr;
  if (s == DRTOPK_OK) {
    if (d_ws) {
      if (ws_bytes < P.ws_bytes || (reinterpret_cast<uintptr_t>(d_ws) & 255u)) s = DRTOPK_ENOMEM;
      ws = static_cast<char*>(d_ws);
    } else {
      s = ensure_ws(h, P.ws_bytes);
      ws = static_cast<char*>(h->ws);
    }
  }
  if (s == DRTOPK_OK) {
    cudaEvent_t* ev = h->ev;
    if (h->prof_on && h->prof_used < h->prof_max) ev = &h->prof[3 * (size_t)h->prof_used++];
    s = enqueue_select(P, h->device, d_keys, d_kth, d_vals, d_idx, ws, static_cast<cudaStream_t>(stream), ev);
    if (s == DRTOPK_OK) {
      h->last_ctrl = ws + P.off_ctrl;
      h->last_plan = P;
      h->have_last = true;
    }
  }
  if (cur != h->device) cudaSetDevice(cur);
  return s;
}

extern "C" drtopk_status_t drtopk_select(drtopk_handle_t h, const void* d_keys, drtopk_dtype_t dtype, uint64_t n,
                                         uint64_t k, const drtopk_params_t* p, void* d_kth, void* d_vals,
                                         int64_t* d_idx, void* stream) {
  return select_impl(h, d_keys, dtype, n, k, p, d_kth, d_vals, d_idx, nullptr, 0, stream);
}

extern "C" drtopk_status_t drtopk_select_ws(drtopk_handle_t h, const void* d_keys, drtopk_dtype_t dtype, uint64_t n,
                                            uint64_t k, const drtopk_params_t* p, void* d_kth, void* d_vals,
                                            int64_t* d_idx, void* d_workspace, size_t workspace_bytes,
                                            void* stream) {
  if (!d_workspace) return DRTOPK_EINVAL;
  return select_impl(h, d_keys, dtype, n, k, p, d_kth, d_vals, d_idx, d_workspace, workspace_bytes, stream);
}

static drtopk_status_t read_ctrl(drtopk_handle_t h, uint32_t* hdr) {
  if (!h->have_last) return DRTOPK_EINVAL;
  if (cudaMemcpy(hdr, h->last_ctrl, CTRL_HDR_WORDS * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return DRTOPK_ECUDA;
  return DRTOPK_OK;
}

extern "C" drtopk_status_t drtopk_sync_check(drtopk_handle_t h, void* stream) {
  if (!h) return DRTOPK_EINVAL;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(h->device);
  drtopk_status_t s = DRTOPK_OK;
  if (cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess) s = DRTOPK_ECUDA;
  if (s == DRTOPK_OK && h->have_last) {
    uint32_t hdr[CTRL_HDR_WORDS];
    s = read_ctrl(h, hdr);
    if (s == DRTOPK_OK) s = device_error_status(hdr[CW_ERR]);
  }
  cudaSetDevice(cur);
  return s;
}

// BMW: device delegates, then the host heap scan that skips subranges whose
// Max is below the heap's minimum once the heap holds k keys (the
// reference's threshold applies from the first push on, which can drop keys
// the answer needs while the heap is not yet full; here it applies once the
// heap is full, so the k-th is exact)
extern "C" drtopk_status_t drtopk_bmw_select(drtopk_handle_t h, const void* d_keys, const uint32_t* h_keys, uint64_t n,
                                             uint64_t k, int alpha, uint32_t* kth, uint64_t* n_skipped,
                                             double* ms_sample, double* ms_scan) {
  if (!h || !d_keys || !h_keys || !kth || n == 0 || k < 1 || k > n || alpha < 1 || alpha > 24)
    return DRTOPK_EINVAL;
  std::lock_guard<std::mutex> lk(h->mu);
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != h->device) cudaSetDevice(h->device);
  drtopk_params_t p;
  drtopk_params_default(&p);
  p.alpha = alpha;
  p.path = 1;
  Plan P;
  const uint64_t M = (n + (1ull << alpha) - 1) >> alpha;
  drtopk_status_t s = M < k ? DRTOPK_EINVAL : plan_for(h->device, n, k, DRTOPK_U32, &p, false, &P, nullptr);
  if (s == DRTOPK_OK) s = ensure_ws(h, P.ws_bytes);
  std::vector<uint32_t> del;
  const auto t0 = std::chrono::steady_clock::now();
  if (s == DRTOPK_OK) {
    char* ws = static_cast<char*>(h->ws);
    uint32_t* cw = reinterpret_cast<uint32_t*>(ws + P.off_ctrl);
    SampleArgs sa;
    std::memset(&sa, 0, sizeof(sa));
    sa.keys = static_cast<const uint32_t*>(d_keys);
    sa.n = n;
    sa.alpha = alpha;
    sa.nbits = 8;
    sa.hmode = 0;
    sa.vec_ok = (reinterpret_cast<uintptr_t>(d_keys) & 15u) == 0;
    sa.del = reinterpret_cast<uint32_t*>(ws + P.off_del);
    sa.err = cw + CW_ERR;
    del.resize(M);
    if (cudaMemsetAsync(cw, 0, P.ctrl_bytes, nullptr) != cudaSuccess ||
        launch_sampler_km(P, sa, 1, nullptr) != cudaSuccess ||
        cudaMemcpy(del.data(), sa.del, M * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
      s = DRTOPK_ECUDA;
  }
  const auto t1 = std::chrono::steady_clock::now();
  if (s == DRTOPK_OK) {
    const uint64_t S = 1ull << alpha;
    std::vector<uint32_t> heap;  // min-heap of the k largest keys seen
    heap.reserve((size_t)k + 1);
    const auto gt = std::greater<uint32_t>();
    uint64_t skip = 0;
    for (uint64_t j = 0; j < M; ++j) {
      const uint64_t b = j * S, e = std::min(n, b + S);
      if (heap.size() == (size_t)k && del[j] < heap.front()) {
        skip += e - b;
        continue;
      }
      uint64_t i = b;
      for (; i < e && heap.size() < (size_t)k; ++i) {
        heap.push_back(h_keys[i]);
        std::push_heap(heap.begin(), heap.end(), gt);
      }
      for (; i < e; ++i) {
        if (h_keys[i] > heap.front()) {
          std::pop_heap(heap.begin(), heap.end(), gt);
          heap.back() = h_keys[i];
          std::push_heap(heap.begin(), heap.end(), gt);
        }
      }
    }
    *kth = heap.front();
    if (n_skipped) *n_skipped = skip;
  }
  const auto t2 = std::chrono::steady_clock::now();
  if (ms_sample) *ms_sample = std::chrono::duration<double, std::milli>(t1 - t0).count();
  if (ms_scan) *ms_scan = std::chrono::duration<double, std::milli>(t2 - t1).count();
  if (cur != h->device) cudaSetDevice(cur);
  return s;
}

// kernels one select of plan P launches (enqueue_select's launch sequence)
static int plan_launches(const Plan& P) {
  // k_presample, k_prerefine x 3, k_emit, k_cand_hist, k_split0, k_fused
  if (P.path == PATH_EMIT) return PRE_LEVELS + 4;
  const bool sampler = P.path != PATH_PLAIN && !(P.path == PATH_BITONIC && P.normal);
  int n = sampler ? 1 : 0;
  if (P.path == PATH_BITONIC || P.tail || P.cluster > 0 || !P.split) return n + 1;
  n += P.first_pre ? (P.first_levels >= 2 ? 1 : 0) : 1;  // k_level_hist, or the cooperative first select
  if (P.path == PATH_BETA) n += 1;                       // k_filter
  n += 1;                                                // k_gather
  if (!P.bucket) n += 1;                                 // k_split0
  return n + 1;                                          // the cooperative last levels
}

extern "C" drtopk_status_t drtopk_last_stats(drtopk_handle_t h, drtopk_stats_t* st) {
  if (!h || !st) return DRTOPK_EINVAL;
  std::memset(st, 0, sizeof(*st));
  if (!h->have_last) return DRTOPK_EINVAL;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(h->device);
  cudaEventSynchronize(h->ev[2]);
  uint32_t hdr[CTRL_HDR_WORDS];
  drtopk_status_t s = read_ctrl(h, hdr);
  if (s == DRTOPK_OK) {
    const Plan& P = h->last_plan;
    const uint32_t* S = hdr + CW_STATS;
    st->alpha = P.alpha;
    st->beta = P.path == PATH_BETA ? 2 : (P.path == PATH_DEFAULT ? 1 : 0);
    st->algo = P.algo;
    st->first_threshold = S[ST_THR1];
    st->n_subranges = P.M;
    st->n_selected = S[ST_NSEL];
    st->n_lonely = S[ST_NLONELY];
    st->n_candidates = S[ST_NCAND];
    st->levels_first = (int)S[ST_LVA];
    st->levels_second = (int)S[ST_LVC];
    st->device_error = hdr[CW_ERR];
    auto t64 = [&](int slot) { return (uint64_t)S[slot] | ((uint64_t)S[slot + 1] << 32); };
    const uint64_t t0 = t64(ST_T0), t1 = t64(ST_T1), t2 = t64(ST_T2), t3 = t64(ST_T3);
    float ms_s = 0, ms_all = 0;
    cudaEventElapsedTime(&ms_s, h->ev[0], h->ev[1]);
    cudaEventElapsedTime(&ms_all, h->ev[0], h->ev[2]);
    st->ms_sample = ms_s;
    st->ms_first = t1 > t0 ? (t1 - t0) * 1e-6 : 0.0;
    st->ms_concat = t2 > t1 ? (t2 - t1) * 1e-6 : 0.0;
    st->ms_second = t3 > t2 ? (t3 - t2) * 1e-6 : 0.0;
    st->ms_total = ms_all;
    st->team_ctas = P.tail ? TAIL_CLUSTER : (P.cluster > 0 ? P.cluster : (P.one_cta ? 1 : P.fused_grid));
    st->team_cluster = P.tail ? 3 : (P.cluster > 0 ? 1 : (P.one_cta ? 5 : 0));
    st->kernel_launches = plan_launches(P);
    st->sample_stride = P.path == PATH_EMIT ? (int)P.pre_stride : 0;
  }
  cudaSetDevice(cur);
  return s;
}

extern "C" drtopk_status_t drtopk_profile_begin(drtopk_handle_t h, int max_calls) {
  if (!h || max_calls < 1) return DRTOPK_EINVAL;
  std::lock_guard<std::mutex> lk(h->mu);
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(h->device);
  drtopk_status_t s = DRTOPK_OK;
  while ((int)h->prof.size() < 3 * max_calls) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) { s = DRTOPK_ECUDA; break; }
    h->prof.push_back(e);
  }
  cudaSetDevice(cur);
  if (s != DRTOPK_OK) return s;
  h->prof_max = max_calls;
  h->prof_used = 0;
  h->prof_on = true;
  return DRTOPK_OK;
}

extern "C" drtopk_status_t drtopk_profile_end(drtopk_handle_t h, double* ms_sample, double* ms_fused, int* ncalls) {
  if (!h) return DRTOPK_EINVAL;
  std::lock_guard<std::mutex> lk(h->mu);
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(h->device);
  double a = 0, b = 0;
  drtopk_status_t s = DRTOPK_OK;
  for (int i = 0; i < h->prof_used; ++i) {
    cudaEvent_t* e = &h->prof[3 * (size_t)i];
    float x = 0, y = 0;
    if (cudaEventSynchronize(e[2]) != cudaSuccess) { s = DRTOPK_ECUDA; break; }
    cudaEventElapsedTime(&x, e[0], e[1]);
    cudaEventElapsedTime(&y, e[1], e[2]);
    a += x;
    b += y;
  }
  cudaSetDevice(cur);
  if (ms_sample) *ms_sample = a;
  if (ms_fused) *ms_fused = b;
  if (ncalls) *ncalls = h->prof_used;
  h->prof_on = false;
  h->prof_used = 0;
  return s;
}

// Traffic model of the delegate paths (bytes beyond the 4n streaming read),
// for n keys, k wanted, subranges of S = 2^alpha keys (M = n/S), assuming
// keys i.i.d. in rank (q = k/n is the fraction of top keys):
//   one delegate (default path):  4M (write) + 4M (first select read)
//                                 + 4kS (the k kept subranges re-read)
//   two delegates (beta path):    8M (write) + 8M per extra threshold digit
//                                 + 8M (filter read) + 4S per subrange with
//                                 >= 2 keys above the threshold (scattered
//                                 subrange reads, weighted x2 against
//                                 streaming bytes as measured) + 8 per
//                                 candidate; a threshold of d digits admits
//                                 an extra ~2^-8d of the keys (truncation).
// Subrange counts per bucket follow Poisson(lambda = q' S).
// Measured delegate-sampler throughput as a fraction of the HBM copy
// bandwidth on B200 (n = 2^30, no index output), by log2 subrange size alpha
// (entries 0..16; alpha < 4 is not run on the one-delegate path).  Small
// subranges cost more instructions per key (lane-owned reductions, and the
// (Max, Second) pair for beta = 2) and more delegate bytes; float keys pay
// their order-preserving mapping.  A pass that mostly reads runs above the
// copy bandwidth (which counts a write per byte read).  Below ~4096
// subranges the warp-per-subrange pass does not fill the GPU, which the
// occupancy factor models.
static double sampler_eff(int alpha, bool beta2, bool f32, double M) {
  static const double u32_b1[17] = {.6, .6, .6, .6, .93, .93, 1., 1., 1.05, 1.06, 1.09, 1.1, 1.09, 1.1, 1.07, 1.07, 1.05};
  static const double u32_b2[17] = {.45, .45, .57, .76, .85, .9, .97, 1., .97, 1.05, 1.12, 1.13, 1.1, 1.1, 1.06, 1.05, 1.07};
  static const double f32_b1[17] = {.6, .6, .6, .6, .92, .91, 1., 1., 1.05, 1.1, 1.1, 1.1, 1.09, 1.09, 1.06, 1.04, 1.07};
  static const double f32_b2[17] = {.45, .45, .53, .7, .84, .89, .88, .85, .82, .94, 1.09, 1.12, 1.1, 1.1, 1.03, 1.04, 1.06};
  const int a = std::max(0, std::min(alpha, 16));
  double e = beta2 ? (f32 ? f32_b2[a] : u32_b2[a]) : (f32 ? f32_b1[a] : u32_b1[a]);
  if (alpha >= 9) e *= 0.7 + 0.3 * std::min(1.0, M / 4096.0);
  return e;
}

// Tail calibration (bytes at the HBM roofline): the phases after the sampler
// run at roughly a third of the copy bandwidth (appends, level barriers), and
// each path has a fixed part -- the one-delegate path's exact first select
// over the delegates costs ~20 us, growing to ~70 us once it must keep
// >= ~1K subranges, the beta path's threshold-only first select ~20 us
// (measured on B200 at n = 2^27 and 2^30).
constexpr double TAIL_BYTES_PER_US = 6.55e6;
static double tail_default(double n, double k, double S);
static double tail_beta(double n, double k, double S, int digits);

static double cost_default(double n, double k, double S) {
  const double M = n / S;
  return 8.0 * M + 4.0 * k * S + 24.0 * k;
}
static double cost_beta(double n, double k, double S, int digits) {
  const double M = n / S;
  const double q = k / n + std::ldexp(1.0, -8 * digits);
  const double lam = q * S;
  const double e = std::exp(-lam);
  const double p_sel = 1.0 - e * (1.0 + lam);
  const double p_lone = lam * e;
  const double cand = M * p_lone + M * p_sel * (lam + 1.0);
  return 16.0 * M + 8.0 * M * (digits - 1) + 2.0 * M * p_sel * 4.0 * S + 24.0 * cand;
}

static double tail_default(double n, double k, double S) {
  return 3.3 * cost_default(n, k, S) + (20.0 + 50.0 * std::min(1.0, k / 1024.0)) * TAIL_BYTES_PER_US;
}
static double tail_beta(double n, double k, double S, int digits) {
  return 2.8 * cost_beta(n, k, S, digits) + 20.0 * TAIL_BYTES_PER_US;
}

// Small k is latency, not bytes.  When the delegates, the kept subranges and
// the candidates fit one CTA's shared memory, the phases after the sampler run
// in one CTA (the tail eligibility rule of plan_for, mirrored here); its chain
// of dependent levels costs ~1.8 us per 1K delegates plus ~0.33 us per 1K
// gathered keys on the one-delegate path, ~2 us per 1K delegate values plus
// ~0.08 us per wanted key on the beta path, where the multi-CTA phases that
// the tail terms above were calibrated on cost ~40 us (measured on B200 at
// n = 2^16..2^22, k = 1..128, where the bandwidth terms are flat).  Returned
// as a correction to those terms, in bytes at the HBM roofline; 0 for k above
// SMALL_K_TUNE, where the bandwidth model alone was measured to choose well.
constexpr uint64_t SMALL_K_TUNE = 256;
static double small_k_latency(double n, double k, double S, int path, int digits, const drtopk_params_t* p) {
  if (k > (double)SMALL_K_TUNE) return 0.0;
  const double M = std::ceil(n / S), Md = path == 1 ? M : 2.0 * M;
  bool fits = p->algo == DRTOPK_ALGO_RADIX && p->nbits <= 8 && Md <= (double)TAIL_CAP &&
              k <= (double)TAIL_CAP && (!p->sorted || k <= (double)SMALL_SORT);
  double gather = 0.0, cand = 0.0;
  if (path == 1) {
    gather = k * S;
    cand = k;
  } else {
    const double q = k / n + std::ldexp(1.0, -8 * std::max(1, digits));
    const double lam = q * S, e = std::exp(-lam), Mf = n / S;
    const double p_sel = 1.0 - e * (1.0 + lam);
    gather = Mf * p_sel * S;
    cand = Mf * lam * e + Mf * p_sel * (lam + 1.0);
  }
  fits = fits && gather <= TAIL_GATHER_AUTO && cand <= TAIL_CAP / 2;
  if (!fits) return 0.0;
  const double us = path == 1 ? 1.8 * M / 1024.0 + 0.33 * gather / 1024.0 : 2.0 * Md / 1024.0 + 0.08 * k;
  return (us - 40.0) * TAIL_BYTES_PER_US;
}

// The sampler's pass: all keys at the sampler's measured share of the copy
// bandwidth, but no faster than one warp streams its own subrange (~4 GB/s
// per warp), which binds when few large subranges cover a small input.
static double sampler_bytes(double n, int alpha, bool beta2, bool f32, double M) {
  const double floor_us = std::ldexp(4.0, alpha) / 4000.0;
  return std::max(4.0 * n / sampler_eff(alpha, beta2, f32, M), floor_us * TAIL_BYTES_PER_US);
}

extern "C" drtopk_status_t drtopk_autotune(uint64_t n, uint64_t k, drtopk_dtype_t dtype, drtopk_params_t* p) {
  if (!p || n == 0 || k < 1 || k > n) return DRTOPK_EINVAL;
  if (p->algo == DRTOPK_ALGO_AUTO) p->algo = DRTOPK_ALGO_RADIX;
  if (p->algo == DRTOPK_ALGO_BITONIC) {
    if (p->alpha < 0) {
      int alpha = (int)std::lround(std::log2(std::sqrt(2.0 * (double)n / (double)k)));
      alpha = std::max(2, std::min(alpha, 16));
      while (alpha > 2 && (n >> alpha) < k) alpha--;
      p->alpha = alpha;
    }
    return DRTOPK_OK;
  }
  // small inputs: the delegate pass does not pay for itself (for k <= 64 it
  // does from 2^13 keys, where the plain select no longer fits one CTA:
  // 29 us against 36-40 us at n = 2^14..2^16 on B200)
  if (n <= (1ull << 16) && p->algo == DRTOPK_ALGO_RADIX && (n <= (uint64_t)TAIL_CAP || k > 64)) {
    p->algo = DRTOPK_ALGO_PLAIN_RADIX;
    p->alpha = 0;
    return DRTOPK_OK;
  }
  const double dn = (double)n, dk = (double)k;
  double best = 1e300;
  int best_alpha = 0, best_path = 1, best_digits = 0;
  for (int alpha = 2; alpha <= 16; ++alpha) {
    const double S = std::ldexp(1.0, alpha);
    const uint64_t M = (n + (1ull << alpha) - 1) >> alpha;
    const bool f32 = dtype == DRTOPK_F32;
    if (alpha >= 2 && M >= k) {
      // the sampler's pass over the keys (at its measured speed) plus the tail
      const double c = sampler_bytes(dn, alpha, false, f32, (double)M) + tail_default(dn, dk, S) +
                       small_k_latency(dn, dk, S, 1, 0, p);
      if (c < best) { best = c; best_alpha = alpha; best_path = 1; best_digits = 0; }
    }
    if (2 * M >= k && p->beta == 2) {
      // float keys crowd into a few top bytes (sign and exponent): a one-digit
      // threshold would admit far more candidates than the model says
      const int maxd = p->nbits == 8 ? 2 : 1;
      const int mind = (p->nbits == 8 && dtype == DRTOPK_F32) ? 2 : 1;
      for (int d = mind; d <= maxd; ++d) {
        const int digits = p->nbits == 8 ? d : (32 / p->nbits - 3);
        const double c = sampler_bytes(dn, alpha, true, f32, (double)M) + tail_beta(dn, dk, S, digits) +
                         small_k_latency(dn, dk, S, 2, digits, p);
        if (c < best) { best = c; best_alpha = alpha; best_path = 2; best_digits = d; }
      }
    }
  }
  // the sampled-threshold path (path 4): one streaming pass that appends
  // every key at or above a threshold predicted from a strided key sample;
  // calibrated on B200: the pass streams at ~1.1 of the copy bandwidth,
  // ~50 us fixed (the sample passes, seven launches, the last levels), and
  // ~73 bytes' worth per candidate (append, level-0 split, last levels).
  // Candidates: k plus the six-sigma margin plus one 16-bit prefix bin.
  bool best_emit = false;
  if (p->algo == DRTOPK_ALGO_RADIX && n >= (1ull << 20)) {
    const double cand = emit_cand_estimate(n, k, pre_stride_for(n));
    const double c = 4.0 * dn / 1.1 + 50.0 * TAIL_BYTES_PER_US + 73.0 * cand;
    // float keys crowd into few exponent bins: the delegate paths' fixed
    // threshold digits can then admit a large share of the keys (uniform
    // [0,1) keys: ~1/512 per 16-bit bin), while the sampled threshold adapts
    // to the data and its tight level 0 spreads the candidates; from 2^22
    // float keys and k >= 2^13 the sampled-threshold path is taken whatever
    // the model says (below that the delegate paths, whose first select
    // refines past crowded bins, measured 1.1-2.8x faster on B200)
    if (c < best || (dtype == DRTOPK_F32 && n >= (1ull << 22) && k >= (1ull << 13))) { best = c; best_emit = true; }
  }
  if (best_emit) {
    p->path = 4;
    p->alpha = 0;
    return DRTOPK_OK;
  }
  if (best_alpha == 0) {  // nothing fits (k close to n): plain select
    p->algo = p->algo == DRTOPK_ALGO_BUCKET ? p->algo : DRTOPK_ALGO_PLAIN_RADIX;
    p->alpha = 0;
    return DRTOPK_OK;
  }
  p->alpha = best_alpha;
  p->path = best_path;
  if (best_path == 2) {
    p->beta = 2;
    if (p->nbits == 8) p->first_digits = -best_digits;  // at least best_digits, refined while crowded
  }
  return DRTOPK_OK;
}

// ------------------------------------------------------------ reference-compatible entry points
static std::mutex g_default_mu;
static drtopk_handle_t g_default[64];

static drtopk_status_t default_handle(drtopk_handle_t* out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DRTOPK_ECUDA;
  std::lock_guard<std::mutex> lk(g_default_mu);
  if (dev < 0 || dev >= 64) return DRTOPK_EINVAL;
  if (!g_default[dev]) {
    drtopk_status_t s = drtopk_create(&g_default[dev], dev, 0);
    if (s != DRTOPK_OK) return s;
  }
  *out = g_default[dev];
  return DRTOPK_OK;
}

static drtopk_status_t blocking_select(const uint32_t* vec_d, uint64_t n, uint64_t k, const drtopk_params_t* p,
                                       uint32_t* TopKElement, drtopk_stats_t* st) {
  drtopk_handle_t h;
  drtopk_status_t s = default_handle(&h);
  if (s != DRTOPK_OK) return s;
  uint32_t* d_kth = nullptr;
  if (cudaMalloc(&d_kth, 4) != cudaSuccess) return DRTOPK_ENOMEM;
  s = drtopk_select(h, vec_d, DRTOPK_U32, n, k, p, d_kth, nullptr, nullptr, nullptr);
  if (s == DRTOPK_OK) s = drtopk_sync_check(h, nullptr);
  if (s == DRTOPK_OK && cudaMemcpy(TopKElement, d_kth, 4, cudaMemcpyDeviceToHost) != cudaSuccess) s = DRTOPK_ECUDA;
  if (s == DRTOPK_OK && st) s = drtopk_last_stats(h, st);
  cudaFree(d_kth);
  return s;
}

namespace drtopk {
// SubrangeId_d as the reference's samplers leave it: SubrangeId_d[j] = j
// (sampleMax, radixselect.cuh:882-918), or SubrangeId_d[2j] =
// SubrangeId_d[2j+1] = j beside the (Max, Second) pairs
// (sampleMax_NoReduction_Beta2, :966-1041)
__global__ void k_subrange_ids(int* ids, uint64_t n_ids, int per) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_ids; i += (uint64_t)gridDim.x * blockDim.x)
    ids[i] = (int)(i / (uint64_t)per);
}
}  // namespace drtopk

// The reference's observable counters after a delegate select, from our
// stage statistics:
//   CountSelectedSubrange: subranges whose keys were concatenated
//     (FindTopKRanges + FillWithKElementsID, radixselect.cuh:412-427,602-618;
//     FindTopKRanges_beta, :560-598);
//   CountLonelyElements: beta path only, beta (= 2) per lonely subrange, since
//     the reference appends (Max, Second) for each (:585); the default path
//     leaves the caller-zeroed counter alone, as the reference does;
//   write_pos: the concatenated size, which on the beta path counts both
//     values appended per lonely subrange (:1870-1880).
// This build appends only Max for a lonely subrange (Second < threshold
// cannot reach the top k), so n_candidates + n_lonely is the reference's size.
static drtopk_status_t write_reference_counters(const Plan& P, const drtopk_stats_t& st, int* SubrangeId_d,
                                                int* CountSelectedSubrange_d, int* CountLonelyElements_d,
                                                int* write_pos_d) {
  const bool beta = P.path == PATH_BETA;
  const int sel = (int)st.n_selected;
  const int lonely = (int)(2 * st.n_lonely);
  const int wpos = (int)(st.n_candidates + (beta ? st.n_lonely : 0));
  if (CountSelectedSubrange_d && cudaMemcpy(CountSelectedSubrange_d, &sel, 4, cudaMemcpyHostToDevice) != cudaSuccess)
    return DRTOPK_ECUDA;
  if (beta && CountLonelyElements_d &&
      cudaMemcpy(CountLonelyElements_d, &lonely, 4, cudaMemcpyHostToDevice) != cudaSuccess)
    return DRTOPK_ECUDA;
  if (write_pos_d && cudaMemcpy(write_pos_d, &wpos, 4, cudaMemcpyHostToDevice) != cudaSuccess) return DRTOPK_ECUDA;
  if (SubrangeId_d && (P.path == PATH_BETA || P.path == PATH_DEFAULT)) {
    const int per = beta ? 2 : 1;
    const uint64_t n_ids = P.M * (uint64_t)per;
    const int grid = (int)std::min<uint64_t>(4096, (n_ids + 255) / 256);
    k_subrange_ids<<<grid, 256>>>(SubrangeId_d, n_ids, per);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return DRTOPK_ECUDA;
  }
  return DRTOPK_OK;
}

extern "C" drtopk_status_t drtopk_sample_radix_select(
    uint32_t* vec_d, int num_element, int k, int num_bucket, uint32_t* TopKElement, int NBitsperDigit,
    int CurrentDigit, int NSubranges, int SubRangesize, int alpha, double* timeforMaxsample,
    double* timeforFirstTopK, double* timeForsecondTopK, double* timeforConcatenation, uint32_t* Max_d,
    int* SubrangeId_d, int NSharedMemoryElements, int SizeOfSubWarp, int pow_size_Subwarp, int NSubWarps_InBlock,
    int NSubRangesPerBlock, int NElementsPerBlock_ReadFromGlobal, int TotalBlocksrequired, int SizeOfAllocation,
    int NThreadsPerBlock, int beta, int defaultContribution, int NthreadstoworkInreduction,
    int* SelectedSubrangeId_d, int* CountLonelyElements_d, int* write_pos_d, uint32_t* ConcatenatedRange_d,
    int* CountSelectedSubrange_d) {
  (void)CurrentDigit; (void)NSharedMemoryElements; (void)SizeOfSubWarp;
  (void)pow_size_Subwarp; (void)NSubWarps_InBlock; (void)NSubRangesPerBlock; (void)NElementsPerBlock_ReadFromGlobal;
  (void)TotalBlocksrequired; (void)SizeOfAllocation; (void)NThreadsPerBlock; (void)NthreadstoworkInreduction;
  (void)SelectedSubrangeId_d; (void)ConcatenatedRange_d;
  if (!vec_d || !TopKElement || num_element <= 0 || k <= 0 || k > num_element) return DRTOPK_EINVAL;
  if (num_bucket != (1 << NBitsperDigit)) return DRTOPK_EINVAL;
  if (SubRangesize != (1 << alpha) || NSubranges != num_element / SubRangesize) return DRTOPK_EINVAL;
  drtopk_params_t p;
  drtopk_params_default(&p);
  p.nbits = NBitsperDigit;
  p.alpha = alpha;
  p.beta = beta;
  p.path = defaultContribution ? 1 : 2;
  drtopk_stats_t st;
  drtopk_status_t s = blocking_select(vec_d, (uint64_t)num_element, (uint64_t)k, &p, TopKElement, &st);
  if (s != DRTOPK_OK) return s;
  if (timeforMaxsample) *timeforMaxsample = st.ms_sample * 1e-3;
  if (timeforFirstTopK) *timeforFirstTopK = st.ms_first * 1e-3;
  if (timeforConcatenation) *timeforConcatenation = st.ms_concat * 1e-3;
  if (timeForsecondTopK) *timeForsecondTopK = st.ms_second * 1e-3;
  drtopk_handle_t h;
  if (default_handle(&h) != DRTOPK_OK || !h->have_last) return DRTOPK_EINVAL;
  const Plan& P = h->last_plan;
  drtopk_status_t rs = write_reference_counters(P, st, SubrangeId_d, CountSelectedSubrange_d, CountLonelyElements_d,
                                                write_pos_d);
  if (rs != DRTOPK_OK) return rs;
  // the delegates in the caller's Max_d (the reference leaves them there)
  if (Max_d && P.path != PATH_PLAIN) {
    size_t bytes = P.M * (P.path == PATH_BETA ? 8 : 4);
    if (cudaMemcpy(Max_d, static_cast<char*>(h->ws) + P.off_del, bytes, cudaMemcpyDeviceToDevice) != cudaSuccess)
      return DRTOPK_ECUDA;
  }
  return DRTOPK_OK;
}

extern "C" drtopk_status_t drtopk_radix_select(uint32_t* vec_d, int num_element, int k, int num_bucket,
                                               uint32_t* TopKElement, int NBitsperDigit, int CurrentDigit) {
  (void)CurrentDigit;
  if (!vec_d || !TopKElement || num_element <= 0 || k <= 0 || k > num_element) return DRTOPK_EINVAL;
  if (num_bucket != (1 << NBitsperDigit)) return DRTOPK_EINVAL;
  drtopk_params_t p;
  drtopk_params_default(&p);
  p.nbits = NBitsperDigit;
  p.algo = DRTOPK_ALGO_PLAIN_RADIX;
  return blocking_select(vec_d, (uint64_t)num_element, (uint64_t)k, &p, TopKElement, nullptr);
}

extern "C" drtopk_status_t drtopk_sample_bucket_select(
    uint32_t* vec_d, int num_element, int k, int num_bucket, uint32_t* TopKElement, int NSubranges,
    int SubRangesize, int alpha, double* timeforMaxsample, double* timeforFirstTopK, double* timeForsecondTopK,
    double* timeforConcatenation, uint32_t* Max_d, int* SubrangeId_d, int beta, int defaultContribution,
    int NthreadstoworkInreduction, int NThreadsPerBlock, int SizeOfAllocation, int NSharedMemoryElements,
    int* SelectedSubrangeId_d, int* CountSelectedSubrange_d, int* CountLonelyElements_d, int* write_pos_d,
    uint32_t* ConcatenatedRange_d) {
  (void)Max_d; (void)NthreadstoworkInreduction; (void)NThreadsPerBlock; (void)SizeOfAllocation;
  (void)NSharedMemoryElements; (void)SelectedSubrangeId_d; (void)ConcatenatedRange_d;
  if (!vec_d || !TopKElement || num_element <= 0 || k <= 0 || k > num_element) return DRTOPK_EINVAL;
  if (SubRangesize != (1 << alpha) || NSubranges != num_element / SubRangesize) return DRTOPK_EINVAL;
  drtopk_params_t p;
  drtopk_params_default(&p);
  p.algo = DRTOPK_ALGO_BUCKET;
  p.num_bucket = num_bucket;
  p.alpha = alpha;
  p.beta = beta;
  p.path = defaultContribution ? 1 : 2;
  drtopk_stats_t st;
  drtopk_status_t s = blocking_select(vec_d, (uint64_t)num_element, (uint64_t)k, &p, TopKElement, &st);
  if (s != DRTOPK_OK) return s;
  if (timeforMaxsample) *timeforMaxsample = st.ms_sample * 1e-3;
  if (timeforFirstTopK) *timeforFirstTopK = st.ms_first * 1e-3;
  if (timeforConcatenation) *timeforConcatenation = st.ms_concat * 1e-3;
  if (timeForsecondTopK) *timeForsecondTopK = st.ms_second * 1e-3;
  drtopk_handle_t h;
  if (default_handle(&h) != DRTOPK_OK || !h->have_last) return DRTOPK_EINVAL;
  return write_reference_counters(h->last_plan, st, SubrangeId_d, CountSelectedSubrange_d, CountLonelyElements_d,
                                  write_pos_d);
}

extern "C" drtopk_status_t drtopk_bitonic_topk(const uint32_t* A_d, int N, int k, int alpha, int NormalBitonic,
                                               uint32_t* d_topk, int64_t* d_idx, uint32_t* TopKElement) {
  if (!A_d || N <= 0 || k <= 0 || k > N) return DRTOPK_EINVAL;
  drtopk_params_t p;
  drtopk_params_default(&p);
  p.algo = DRTOPK_ALGO_BITONIC;
  p.alpha = NormalBitonic ? 0 : alpha;
  p.path = NormalBitonic ? 3 : 0;
  drtopk_handle_t h;
  drtopk_status_t s = default_handle(&h);
  if (s != DRTOPK_OK) return s;
  uint32_t* d_kth = nullptr;
  if (cudaMalloc(&d_kth, 4) != cudaSuccess) return DRTOPK_ENOMEM;
  s = drtopk_select(h, A_d, DRTOPK_U32, (uint64_t)N, (uint64_t)k, &p, d_kth, d_topk, d_idx, nullptr);
  if (s == DRTOPK_OK) s = drtopk_sync_check(h, nullptr);
  if (s == DRTOPK_OK && TopKElement && cudaMemcpy(TopKElement, d_kth, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    s = DRTOPK_ECUDA;
  cudaFree(d_kth);
  return s;
}

// ------------------------------------------------------------ failure-detection self-test
namespace drtopk {
__global__ void k_wait_probe(GridBar gb) { grid_barrier(gb); }
}  // namespace drtopk

extern "C" drtopk_status_t drtopk_selftest_wait_timeout(int device, double* ms_waited) {
  int cur = 0;
  cudaGetDevice(&cur);
  if (cudaSetDevice(device) != cudaSuccess) return DRTOPK_EINVAL;
  drtopk_status_t s = DRTOPK_OK;
  uint32_t* w = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaMalloc(&w, 16) != cudaSuccess) s = DRTOPK_ENOMEM;
  if (s == DRTOPK_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) s = DRTOPK_ECUDA;
  if (s == DRTOPK_OK && cudaMemset(w, 0, 16) != cudaSuccess) s = DRTOPK_ECUDA;
  if (s == DRTOPK_OK) {
    GridBar gb;
    gb.count = w;
    gb.err = w + 2;
    gb.nblocks = 2;           // one CTA more than launched: nothing completes the barrier
    gb.spin_limit = 1u << 22; // ~0.5 s of polls
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(1);
    cfg.blockDim = dim3(32);
    cfg.stream = nullptr;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void* args[] = {&gb};
    cudaEventRecord(e0, nullptr);
    if (cudaLaunchKernelExC(&cfg, (void*)k_wait_probe, args) != cudaSuccess) s = DRTOPK_ECUDA;
    cudaEventRecord(e1, nullptr);
    if (s == DRTOPK_OK && cudaEventSynchronize(e1) != cudaSuccess) s = DRTOPK_ECUDA;
    uint32_t err = 0;
    if (s == DRTOPK_OK && cudaMemcpy(&err, w + 2, 4, cudaMemcpyDeviceToHost) != cudaSuccess) s = DRTOPK_ECUDA;
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms_waited) *ms_waited = ms;
    if (s == DRTOPK_OK) s = (err & DE_BARRIER_TIMEOUT) ? DRTOPK_ETIMEOUT : DRTOPK_EDEVICE;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (w) cudaFree(w);
  cudaSetDevice(cur);
  return s;
}
