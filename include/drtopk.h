/* drtopk.h -- C ABI of the B200-native Dr.Top-k selection library
 * (libdrtopk.so).
 *
 * Plain C types only (device pointers as void*, CUDA streams as void*), so
 * ctypes/cffi/JNI/cgo can bind it without CUDA headers.  All device pointers
 * must belong to the handle's device.  Every call is stream-ordered and
 * returns a status; nothing calls exit().  Results are exact: the k-th
 * largest key equals ascending_sorted[n-k] (the reference's Enabletest check,
 * baseline+filter+beta+shuffle/main.cu:281-296), and the top-k list is every
 * key above it plus the lowest-index copies of it.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   baseline+filter+beta+shuffle/radixselect.cuh:1782-1784 sample_radix_select
 *   baseline+filter+beta+shuffle/radixselect.cuh:1472      radix_select
 *   bucket_select/bucketselect_combined.cuh:1279-1280      sample_bucket_select
 *   bitonic/bitonic_com.cuh:609,668                        bitonic_firstTopk / bitonic
 *   baseline+filter+beta+shuffle/main.cu:56-323            the topk.bin CLI (see topk_cli.cpp)
 */
#ifndef DRTOPK_H
#define DRTOPK_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define DRTOPK_API __attribute__((visibility("default")))
#else
#define DRTOPK_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  DRTOPK_OK = 0,
  DRTOPK_EINVAL = 1,       /* invalid argument (k<1, k>n, bad nbits/alpha/...) */
  DRTOPK_ENOMEM = 2,       /* device allocation failed or caller workspace too small */
  DRTOPK_ECUDA = 3,        /* CUDA runtime error */
  DRTOPK_EDEVICE = 4,      /* device-side check failed (see drtopk_sync_check) */
  DRTOPK_EBUDGET = 5,      /* request exceeds the handle's / server's HBM budget */
  DRTOPK_EUNSUPPORTED = 6, /* valid request outside the library's limits */
  DRTOPK_ETIMEOUT = 7,     /* a bounded device wait gave up */
  DRTOPK_EAGAIN = 8,       /* server: nothing finished yet / queue full */
  DRTOPK_ECANCELLED = 9    /* server: request cancelled */
} drtopk_status_t;

typedef enum { DRTOPK_U32 = 0, DRTOPK_F32 = 1 } drtopk_dtype_t;

typedef enum {
  DRTOPK_ALGO_RADIX = 0,       /* Dr.Top-k radix (the reference's final version) */
  DRTOPK_ALGO_BUCKET = 1,      /* Dr.Top-k bucket select (integer-exact buckets) */
  DRTOPK_ALGO_BITONIC = 2,     /* Dr.Top-k bitonic top-k (k a power of two, k <= 2048) */
  DRTOPK_ALGO_PLAIN_RADIX = 3, /* radix select without delegates (reference alpha==0) */
  DRTOPK_ALGO_AUTO = 4         /* autotuner picks algorithm and parameters */
} drtopk_algo_t;

typedef struct {
  int nbits;        /* bits per radix digit: 1,2,4,8 (reference NBitsPerDigit; default 8) */
  int alpha;        /* log2 subrange size; -1: reference formula (main.cu:83); -2: autotuner */
  int beta;         /* delegates per subrange on the small-alpha path; only 2 is valid (default 2) */
  int path;         /* 0: reference rule (alpha>5 -> one delegate, else beta delegates); 1: one; 2: beta;
                       4: sampled threshold (radix only): the streaming pass appends every key at or
                       above a threshold predicted from a key sample (no delegate vector; exact, with
                       a plain radix select over all keys when the prediction overshoots) */
  int algo;         /* drtopk_algo_t (default RADIX) */
  int num_bucket;   /* bucket variant: buckets per level, 2..4096 (default 256) */
  int largest;      /* 1: k largest (reference semantics, default); 0: k smallest */
  int sorted;       /* 1: top-k sorted by key (best first), ties by index ascending */
  int first_digits; /* beta path: digits used by the first select; 0: reference (32/nbits-3);
                       > 0: exactly this many; < 0 (the autotuner's choice): at least -first_digits,
                       refined while the chosen bin still holds more than max(2k, 256) delegates */
  int team;         /* CTAs running the phases after the sampler: 0 auto, 1 the whole GPU
                       (cooperative grid), 2 one thread-block cluster, 3 one CTA with the sets
                       in shared memory (small problems), 4 shared GPU: as auto, but a
                       select that would take the whole GPU runs its phases in one cluster
                       of at most 8 CTAs, so that concurrent selects overlap (served form);
                       5 ordinary launches only (sampled-threshold path): the last levels run in
                       one CTA, so the select never waits for a share of the GPU */
} drtopk_params_t;

typedef struct {
  int alpha;                 /* subrange size used: 2^alpha */
  int beta;                  /* delegates per subrange used (1 or 2) */
  int algo;                  /* algorithm actually run */
  uint32_t first_threshold;  /* threshold from the first select (mapped key space) */
  uint64_t n_subranges;      /* delegate subranges */
  uint64_t n_selected;       /* subranges whose keys were concatenated */
  uint64_t n_lonely;         /* single keys taken from subranges with one qualifying delegate */
  uint64_t n_candidates;     /* size of the concatenated candidate vector */
  int levels_first;          /* select levels run on the delegates */
  int levels_second;         /* select levels run on the candidates */
  uint32_t device_error;     /* device error word (0 = none) */
  double ms_sample;          /* stage times of the last call (device clock) */
  double ms_first;
  double ms_concat;
  double ms_second;
  double ms_total;
  int team_ctas;             /* CTAs that ran the phases after the sampler */
  int team_cluster;          /* 0: the cooperative grid; 1: one thread-block cluster; 3: one CTA
                                (shared-memory tail); 5: one ordinary CTA */
  int kernel_launches;       /* kernels the last select launched (sampler included) */
  int sample_stride;         /* sampled-threshold path: one 512-key chunk in sample_stride was
                                sampled to predict the threshold (0 on the other paths) */
} drtopk_stats_t;

typedef struct drtopk_handle* drtopk_handle_t;

DRTOPK_API void drtopk_params_default(drtopk_params_t* p);
DRTOPK_API const char* drtopk_status_str(drtopk_status_t s);

/* A handle owns a resident device workspace (grown on demand, capped by
 * hbm_budget_bytes; 0 = no cap), stage timers and the device error word.
 * One handle serves one host thread at a time. */
DRTOPK_API drtopk_status_t drtopk_create(drtopk_handle_t* h, int device, size_t hbm_budget_bytes);
DRTOPK_API drtopk_status_t drtopk_destroy(drtopk_handle_t h);

/* Scratch bytes a select of (n, k, dtype, params) needs -- replaces the
 * caller-sized scratch of main.cu:205-250. */
DRTOPK_API drtopk_status_t drtopk_workspace_size(uint64_t n, uint64_t k, drtopk_dtype_t dtype, const drtopk_params_t* p,
                                      size_t* bytes);

/* Exact top-k of d_keys[0..n) (uint32 or float32).  Outputs (device, any may
 * be NULL): d_kth[1] the k-th key (same dtype as the input), d_vals[k] the
 * top-k keys, d_idx[k] their indices.  n < 2^32, 1 <= k <= n. */
DRTOPK_API drtopk_status_t drtopk_select(drtopk_handle_t h, const void* d_keys, drtopk_dtype_t dtype, uint64_t n, uint64_t k,
                              const drtopk_params_t* p, void* d_kth, void* d_vals, int64_t* d_idx, void* stream);

/* Same, with caller-owned scratch of at least drtopk_workspace_size bytes
 * (256-byte aligned); the handle's own workspace is not touched. */
DRTOPK_API drtopk_status_t drtopk_select_ws(drtopk_handle_t h, const void* d_keys, drtopk_dtype_t dtype, uint64_t n,
                                 uint64_t k, const drtopk_params_t* p, void* d_kth, void* d_vals, int64_t* d_idx,
                                 void* d_workspace, size_t workspace_bytes, void* stream);

/* No counterpart in the reference.  A select that allocates no device
 * memory, for callers that cannot allocate when they ask for a top-k (their
 * framework's allocator owns all device memory, cudaMalloc's device-wide
 * synchronisation is not acceptable on their path, or their host program
 * forbids allocation inside it).  Same inputs, outputs, parameters and
 * results as drtopk_select, on the current device; the scratch is one
 * 32 MiB (33554432-byte) array built into the library, held by every GPU
 * that uses the library until the process exits.
 * Requests whose workspace (drtopk_workspace_size) is larger return
 * DRTOPK_EUNSUPPORTED.  The first call on a device looks the array's
 * address up, and with CUDA's lazy module loading (the default) that first
 * use is also when the 32 MiB are taken from the device: make the first
 * call at initialisation, before the caller's allocator reserves the device
 * memory and before capturing any stream work (CUDA_MODULE_LOADING=EAGER
 * takes the memory at context creation instead).  Calls share the array:
 * calls whose GPU work overlaps race and must be serialised. */
DRTOPK_API drtopk_status_t drtopk_select_noalloc(const void* d_keys, drtopk_dtype_t dtype, uint64_t n, uint64_t k,
                                                 const drtopk_params_t* p, void* d_kth, void* d_vals,
                                                 int64_t* d_idx, void* stream);

/* Companion of drtopk_select_noalloc (no counterpart in the reference):
 * synchronise the stream and report device-side failures of the last
 * no-allocation select on the current device (a bounded wait that gave up:
 * DRTOPK_ETIMEOUT; an internal check: DRTOPK_EDEVICE).  Allocates nothing. */
DRTOPK_API drtopk_status_t drtopk_noalloc_sync_check(void* stream);

/* Synchronise the stream and report device-side failures of the last call
 * (bounded waits that gave up, internal checks). */
DRTOPK_API drtopk_status_t drtopk_sync_check(drtopk_handle_t h, void* stream);

/* Statistics and stage times of the handle's last select (synchronises). */
DRTOPK_API drtopk_status_t drtopk_last_stats(drtopk_handle_t h, drtopk_stats_t* st);

/* Per-call kernel timing: between profile_begin and profile_end every select
 * on this handle records CUDA events on its stream around the sampler and
 * the fused kernel (up to max_calls calls).  profile_end synchronises and
 * returns the summed device times (ms) of the two kernels and the number of
 * calls recorded. */
DRTOPK_API drtopk_status_t drtopk_profile_begin(drtopk_handle_t h, int max_calls);
DRTOPK_API drtopk_status_t drtopk_profile_end(drtopk_handle_t h, double* ms_sample, double* ms_fused, int* ncalls);

/* Failure-detection self-test: launches a one-CTA cooperative kernel whose
 * grid barrier waits for a second CTA that does not exist.  The bounded wait
 * gives up (about 0.5 s), records the timeout in the device error word and
 * the kernel returns, leaving the context usable.  Returns DRTOPK_ETIMEOUT
 * when the timeout was detected (the expected outcome); *ms_waited receives
 * the kernel's duration. */
DRTOPK_API drtopk_status_t drtopk_selftest_wait_timeout(int device, double* ms_waited);

/* Parameters the autotuner picks for (n, k, dtype); p is updated in place. */
DRTOPK_API drtopk_status_t drtopk_autotune(uint64_t n, uint64_t k, drtopk_dtype_t dtype, drtopk_params_t* p);

/* ---------------------------------------------------------------------
 * Reference-compatible entry points (same arguments, same meaning,
 * blocking like the reference; launch-shape arguments of the reference's
 * own kernels are accepted and ignored; status instead of exit()).
 * ------------------------------------------------------------------- */

/* baseline+filter+beta+shuffle/radixselect.cuh:1782-1784 sample_radix_select.
 * Max_d (NSubranges*beta keys) receives the delegates ((Max, Second) pairs on
 * the beta path) and SubrangeId_d their subrange ids, as the reference's
 * samplers leave them.  The counters receive the reference's values:
 * *CountSelectedSubrange_d the subranges whose keys were concatenated;
 * *CountLonelyElements_d (beta path) beta = 2 per subrange with only its Max
 * at or above the threshold, left untouched on the default path;
 * *write_pos_d the concatenated size, two per lonely subrange included.
 * SelectedSubrangeId_d and ConcatenatedRange_d (the reference's scratch,
 * filled in an unspecified order there) are not written.
 * Stage times are returned in seconds like the reference's wtime() deltas. */
DRTOPK_API drtopk_status_t drtopk_sample_radix_select(
    uint32_t* vec_d, int num_element, int k, int num_bucket, uint32_t* TopKElement, int NBitsperDigit,
    int CurrentDigit, int NSubranges, int SubRangesize, int alpha, double* timeforMaxsample,
    double* timeforFirstTopK, double* timeForsecondTopK, double* timeforConcatenation, uint32_t* Max_d,
    int* SubrangeId_d, int NSharedMemoryElements, int SizeOfSubWarp, int pow_size_Subwarp, int NSubWarps_InBlock,
    int NSubRangesPerBlock, int NElementsPerBlock_ReadFromGlobal, int TotalBlocksrequired, int SizeOfAllocation,
    int NThreadsPerBlock, int beta, int defaultContribution, int NthreadstoworkInreduction,
    int* SelectedSubrangeId_d, int* CountLonelyElements_d, int* write_pos_d, uint32_t* ConcatenatedRange_d,
    int* CountSelectedSubrange_d);

/* baseline+filter+beta+shuffle/radixselect.cuh:1472 radix_select (no delegates). */
DRTOPK_API drtopk_status_t drtopk_radix_select(uint32_t* vec_d, int num_element, int k, int num_bucket, uint32_t* TopKElement,
                                    int NBitsperDigit, int CurrentDigit);

/* bucket_select/bucketselect_combined.cuh:1279-1280 sample_bucket_select
 * (k is the k of the k-th largest, as at bucket_select/main.cu:166).  The
 * counters and SubrangeId_d are written as by drtopk_sample_radix_select;
 * their values follow this build's exact integer buckets. */
DRTOPK_API drtopk_status_t drtopk_sample_bucket_select(
    uint32_t* vec_d, int num_element, int k, int num_bucket, uint32_t* TopKElement, int NSubranges,
    int SubRangesize, int alpha, double* timeforMaxsample, double* timeforFirstTopK, double* timeForsecondTopK,
    double* timeforConcatenation, uint32_t* Max_d, int* SubrangeId_d, int beta, int defaultContribution,
    int NthreadstoworkInreduction, int NThreadsPerBlock, int SizeOfAllocation, int NSharedMemoryElements,
    int* SelectedSubrangeId_d, int* CountSelectedSubrange_d, int* CountLonelyElements_d, int* write_pos_d,
    uint32_t* ConcatenatedRange_d);

/* bitonic/sampleBitonic.cu:192 + bitonic_com.cuh:609-728: Dr.Top-k bitonic
 * top-k of A_d[0..N) with subranges of 2^alpha keys (NormalBitonic=1: no
 * delegates).  Writes the k largest keys sorted descending to d_topk (device)
 * and, if d_idx is not NULL, their indices.  k must be a power of two <= 2048
 * and N>>alpha >= k (sampleBitonic.cu:198-221). */
DRTOPK_API drtopk_status_t drtopk_bitonic_topk(const uint32_t* A_d, int N, int k, int alpha, int NormalBitonic,
                                    uint32_t* d_topk, int64_t* d_idx, uint32_t* TopKElement);

/* baseline+filter+beta+shuffle/RealDatasets/BinaryDataset/main.cu:109-148:
 * the reference's score-file readers (host only, no GPU needed).  Fills
 * h_keys[0..n) with uint32 keys; *n_read (may be NULL) receives the values
 * read from the file before any repetition.
 *   DRTOPK_DATASET_BIN_I32    raw little-endian int32 values, kept as their
 *                             bit patterns (the readBinary build); a short
 *                             file repeats its last value, as there
 *   DRTOPK_DATASET_TXT_REF    decimal scores read as the reference's default
 *                             build reads them ("%f" into its unsigned key
 *                             slots, then (1 - u) * 10^9 in unsigned 32-bit
 *                             arithmetic on the float's bit pattern u); at
 *                             most 2^26 scores, repeated in order up to n
 *   DRTOPK_DATASET_TXT_SCORE  the same file with the intended map
 *                             (1 - s) * 1e9 in float, truncated and clamped
 *                             to [0, 2^32 - 1]
 * DRTOPK_EINVAL if the file cannot be read or holds no value. */
typedef enum {
  DRTOPK_DATASET_BIN_I32 = 0,
  DRTOPK_DATASET_TXT_REF = 1,
  DRTOPK_DATASET_TXT_SCORE = 2
} drtopk_dataset_format_t;
DRTOPK_API drtopk_status_t drtopk_load_dataset(const char* path, int format, uint64_t n, uint32_t* h_keys,
                                               uint64_t* n_read);

/* BMW experiment (replaces BMW/radixselect.cuh:1746-1832 with BMW/PQ.h):
 * the device sampler writes one delegate (Max) per subrange of 2^alpha keys
 * of d_keys; the host then scans h_keys (the same n uint32 keys) in order,
 * keeping the k largest seen in a min-heap, and skips every subrange whose
 * Max is below the heap's minimum once the heap holds k keys.  *kth: the
 * k-th largest key (exact); *n_skipped: keys the scan never examined (the
 * reference's NSkipDocument); *ms_sample, *ms_scan (any may be NULL): the
 * sampler with its copy to the host, and the scan.  Blocking. */
DRTOPK_API drtopk_status_t drtopk_bmw_select(drtopk_handle_t h, const void* d_keys, const uint32_t* h_keys,
                                             uint64_t n, uint64_t k, int alpha, uint32_t* kth,
                                             uint64_t* n_skipped, double* ms_sample, double* ms_scan);

/* ---------------------------------------------------------------------
 * Batched form: many independent top-k problems in one persistent launch.
 * Segment s covers keys[offsets[s] .. offsets[s+1]) of one dtype; its k is
 * ks[s].  Outputs are packed at out_offsets[s] (exclusive scan of ks).
 * All arrays are device arrays except where noted.
 * ------------------------------------------------------------------- */
typedef struct drtopk_batch* drtopk_batch_t;

DRTOPK_API drtopk_status_t drtopk_batch_create(drtopk_batch_t* b, int device);
DRTOPK_API drtopk_status_t drtopk_batch_destroy(drtopk_batch_t b);
/* Plan a batch (host arrays h_offsets[nseg+1], h_ks[nseg], h_dtypes[nseg]):
 * autotunes per segment and sizes the resident workspace.  Re-plan only
 * when the segment layout changes; run() can then be graph-replayed. */
DRTOPK_API drtopk_status_t drtopk_batch_plan(drtopk_batch_t b, int nseg, const uint64_t* h_offsets, const uint32_t* h_ks,
                                  const int* h_dtypes, int sorted);
DRTOPK_API drtopk_status_t drtopk_batch_run(drtopk_batch_t b, const void* d_keys, void* d_kth, void* d_vals, int64_t* d_idx,
                                 void* stream);
/* Capture run() into a CUDA graph once and replay it (same pointers). */
DRTOPK_API drtopk_status_t drtopk_batch_run_graph(drtopk_batch_t b, const void* d_keys, void* d_kth, void* d_vals,
                                       int64_t* d_idx, void* stream);
DRTOPK_API drtopk_status_t drtopk_batch_sync_check(drtopk_batch_t b, void* stream);
/* Per-segment choice of the autotuner: h_algo[nseg], h_alpha[nseg], h_beta[nseg] (host). */
DRTOPK_API drtopk_status_t drtopk_batch_describe(drtopk_batch_t b, int* h_algo, int* h_alpha, int* h_beta);

/* Per-segment knobs of the batched form (the reference sets them per run:
 * alphaManualTuning/main.cu:83-84, bucket_select/main.cu:57-67,
 * bitonic/sampleBitonic.cu:194-204).  drtopk_batch_plan_params takes one per
 * segment (host array; NULL = all tuned) with -1 in any field the autotuner
 * should pick; drtopk_batch_describe_params returns the choice.
 *   algo        DRTOPK_ALGO_PLAIN_RADIX (block select over the raw keys),
 *               DRTOPK_ALGO_RADIX (delegates, then the block selects),
 *               DRTOPK_ALGO_BITONIC (every key sorted in shared memory;
 *               segments of <= 4096 keys)
 *   alpha       log2 subrange size (delegate segments; 0 otherwise)
 *   beta        delegates per subrange: 1 (Max) or 2 (Max, Second; k <= 1365)
 *   nbits       digit width of the block selects: 4 or 8 (2^nbits bins)
 *   bucket      0: radix digits; 1: min/max buckets (the reference's bucket
 *               select, exact) in the block selects
 *   chunk_log2  keys per sampler task, 2^chunk_log2 (13..20, >= alpha) */
typedef struct {
  int algo, alpha, beta, nbits, bucket, chunk_log2;
} drtopk_seg_params_t;
DRTOPK_API drtopk_status_t drtopk_batch_plan_params(drtopk_batch_t b, int nseg, const uint64_t* h_offsets,
                                                    const uint32_t* h_ks, const int* h_dtypes, int sorted,
                                                    const drtopk_seg_params_t* h_params);
DRTOPK_API drtopk_status_t drtopk_batch_describe_params(drtopk_batch_t b, drtopk_seg_params_t* h_params);

/* ---------------------------------------------------------------------
 * Served form: continuous batching of top-k requests under an HBM budget.
 * Requests carry host keys (copied into device buffers) or device-resident
 * keys; the server admits them when budget and slots allow, runs the
 * requests admitted together as one chain of grouped launches (several
 * chains overlap on the device), and returns exact results.
 * ------------------------------------------------------------------- */
typedef struct drtopk_server* drtopk_server_t;

typedef struct {
  uint64_t id;          /* request id returned by submit */
  int status;           /* drtopk_status_t of this request */
  uint32_t kth;         /* k-th key (raw bits of the request dtype) */
  double t_submit_ms;   /* server clock (ms since creation) */
  double t_start_ms;
  double t_done_ms;
} drtopk_result_t;

DRTOPK_API drtopk_status_t drtopk_server_create(drtopk_server_t* s, int device, size_t hbm_budget_bytes, int max_inflight);
DRTOPK_API drtopk_status_t drtopk_server_destroy(drtopk_server_t s);
/* Submit a request (keys are copied before return).  out_vals / out_idx are
 * host buffers of k entries, filled when the request completes (may be NULL). */
DRTOPK_API drtopk_status_t drtopk_server_submit(drtopk_server_t s, const void* h_keys, drtopk_dtype_t dtype, uint64_t n,
                                     uint64_t k, int sorted, void* out_vals, int64_t* out_idx, uint64_t* id);
/* Same for keys already resident in device memory (caller-owned, left
 * untouched until the request completes): no host copy, no upload. */
DRTOPK_API drtopk_status_t drtopk_server_submit_device(drtopk_server_t s, const void* d_keys, drtopk_dtype_t dtype,
                                                       uint64_t n, uint64_t k, int sorted, void* out_vals,
                                                       int64_t* out_idx, uint64_t* id);
/* Pop up to max finished results; *count receives how many (DRTOPK_EAGAIN
 * when none has finished yet). */
DRTOPK_API drtopk_status_t drtopk_server_poll(drtopk_server_t s, drtopk_result_t* results, int max, int* count);
/* Cancel a request that has not started. */
DRTOPK_API drtopk_status_t drtopk_server_cancel(drtopk_server_t s, uint64_t id);
/* Block until every submitted request has finished (bounded by timeout_ms; -1 = no bound). */
DRTOPK_API drtopk_status_t drtopk_server_drain(drtopk_server_t s, int timeout_ms);
/* Current resident bytes and in-flight request count. */
DRTOPK_API drtopk_status_t drtopk_server_usage(drtopk_server_t s, size_t* resident_bytes, int* inflight, int* queued);

/* Counters of the server's worker since creation (observability). */
typedef struct {
  uint64_t singles;          /* requests run as one select each (whole-GPU sorted output) */
  uint64_t batches;          /* worker ticks that issued grouped chains */
  uint64_t batched;          /* requests run inside grouped chains */
  uint64_t pinned_allocs;    /* pinned host buffers newly allocated (staging-cache misses) */
  uint64_t worker_ticks;     /* worker loop iterations that admitted or completed something */
  double host_ms_pinned;     /* worker time spent allocating pinned staging */
  double host_ms_launch;     /* worker time issuing device work */
  double host_ms_complete;   /* worker time copying results to the callers' buffers */
  uint64_t retries;          /* grouped selects run again with the general plan (DE_RETRY) */
  double host_ms_retry;      /* completion-thread time spent in those runs */
  double host_ms_alloc;      /* worker time in stream-ordered allocations (cudaMallocAsync) */
} drtopk_server_stats_t;
DRTOPK_API drtopk_status_t drtopk_server_stats(drtopk_server_t s, drtopk_server_stats_t* st);

#ifdef __cplusplus
}
#endif

#endif /* DRTOPK_H */
