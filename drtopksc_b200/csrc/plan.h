// plan.h -- host-side plan of one select: chosen path/parameters and the
// workspace layout (byte offsets into one device allocation).
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/drtopk.h"

namespace drtopk {

// control block words (zeroed by one memset per call)
enum CtrlWord : int {
  CW_ERR = 0,
  CW_BAR_COUNT = 1,   // grid barrier word: (generation << 16) | arrivals
  CW_DEL_MINMAX = 4,   // 2 words
  CW_CAND_MINMAX = 6,  // 2 words
  CW_CAND_COUNT = 8,
  CW_SEL_COUNT = 9,
  CW_THR = 10,         // first-select threshold handed between launches
  CW_TAIL = 11,        // shared-memory tail outcome
  CW_TIE_CUT = 12,     // beta path, ties at a one-value threshold: subrange-id bound of the tied ones kept
  CW_STATS = 16,       // 32 words
  CTRL_HDR_WORDS = 48
};

// stats slots >= 16 hold 64-bit %globaltimer stamps (lo, hi)
enum StatTime : int { ST_T0 = 16, ST_T1 = 18, ST_T2 = 20, ST_T3 = 22 };

struct Plan {
  uint64_t n, k;
  int km, algo, path, bucket, nbits, nb, alpha;
  uint64_t S, M;
  int first_levels;
  int has_pos;
  int sorted;
  uint64_t cand_cap;
  int fused_grid, sample_grid;
  int split;           // concatenation as separate kernels (large inputs)
  int cluster;         // > 0: phases after the sampler run in one thread-block cluster of this many CTAs
  int tail;            // 1: phases after the sampler run in one CTA with the sets in shared memory
  int one_cta;         // sampled-threshold path: the last levels run in one ordinary CTA (no co-residency)
  uint32_t adapt_first;  // autotuned beta path: the first select refines past first_levels while its
                         // chosen bin holds more delegates than this (0: the reference's digits)
  int bounded;         // ... with candidate buffers of cap_bound entries (served form; DE_RETRY on overflow)
  uint64_t cap_bound;
  int split_grid, filter_grid, hist_grid, split0_grid;
  int emit_grid, presample_grid;  // sampled-threshold path
  uint32_t pre_target;            // sampled keys required at or above its predicted threshold
  uint32_t pre_stride;            // one 512-key chunk in pre_stride is sampled
  int first_pre;       // split mode: first select in k_level_hist / k_filter (beta, radix, <= 2 levels)
  size_t fused_smem;
  size_t run_words;
  int hist_words;
  size_t off_ctrl, ctrl_bytes;
  size_t pre_hist_word;  // word offset of the sampled-threshold histograms in the control block
  size_t off_sel;
  size_t off_del, off_pos, off_Atop, off_Acbuf0, off_Acbuf1;
  size_t off_cand, off_Ccbuf0, off_Ctop;
  size_t off_sort0, off_sort1, off_sortcnt;
  // bitonic variant
  int normal;  // NormalBitonic: no delegates
  uint64_t bbuf_cap;
  size_t off_bbuf0, off_bbuf1;
  size_t ws_bytes;
};

drtopk_status_t make_plan(uint64_t n, uint64_t k, drtopk_dtype_t dtype, const drtopk_params_t* p, int sms,
                          int fused_grid, Plan* P);
void layout(Plan* P, bool want_idx);
drtopk_status_t plan_select(int device, uint64_t n, uint64_t k, drtopk_dtype_t dtype, const drtopk_params_t* p,
                            bool want_idx, Plan* P);
// Served form: as plan_select; a sampled-threshold plan with one-CTA last
// levels gets candidate buffers sized by the sample's estimate (bounded):
// such a select that cannot finish in them reports DE_RETRY instead of
// falling back on the device, and its caller runs it with a general plan.
drtopk_status_t plan_select_bounded(int device, uint64_t n, uint64_t k, drtopk_dtype_t dtype,
                                    const drtopk_params_t* p, bool want_idx, Plan* P);
drtopk_status_t enqueue_select(const Plan& P, int device, const void* d_keys, void* d_kth, void* d_vals,
                               int64_t* d_idx, char* ws, cudaStream_t st, cudaEvent_t* ev);
int ref_alpha(double log2n, double k);

// One select of a grouped launch (sampled-threshold plans with one_cta set,
// one key mode per group): its plan, input, outputs, workspace and its
// control block (zeroed by the caller before enqueue_group).
struct GroupItem {
  const Plan* P;
  const void* keys;
  void* d_kth;
  void* d_vals;
  int64_t* d_idx;
  char* ws;
  char* ctrl;
};
// bytes of the device descriptor area enqueue_group needs for nprob selects
// (and of the pinned host staging it fills)
size_t group_desc_bytes(int nprob);
// Enqueue nprob selects as one chain of grouped launches on st.  h_stage is
// pinned host memory and d_desc device memory, both group_desc_bytes(nprob)
// bytes; h_stage must stay untouched until the upload has run.  Every
// problem's device error word ends up in d_err_out[nprob].
drtopk_status_t enqueue_group(int device, int km, const GroupItem* items, int nprob, char* h_stage, char* d_desc,
                              uint32_t* d_err_out, cudaStream_t st);
// status of a device error word: 0 -> OK, a bounded wait that gave up ->
// ETIMEOUT, any other device-side check -> EDEVICE
drtopk_status_t device_error_status(uint32_t err);
// concatenation length (keys) up to which the automatic choice lets one CTA
// run the phases after the sampler
constexpr double TAIL_GATHER_AUTO = 32768.0;

}  // namespace drtopk
