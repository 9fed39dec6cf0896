// server.cu -- served form: continuous batching of top-k requests.
//
// A worker thread admits queued requests as in-flight slots and the HBM byte
// budget allow, and keeps admitting while earlier requests are still on the
// GPU:
//   * requests with n <= 2^22 and k <= 4096 admitted in the same tick are
//     grouped into ONE persistent segmented launch (segmented.cuh), each
//     segment reading and writing its request's own buffers;
//   * other requests run one select each: in order on the select stream
//     (the whole-GPU cooperative tail: one at a time), or on a stream of
//     their own when their tail is the one-CTA shared-memory kernel, which
//     then overlaps the other streams' work;
//   * each request's outputs come back with ONE device-to-host copy on the
//     copy stream paired with its compute stream, ordered after its kernels
//     by an event, so result copies never stall the compute streams.
// Device memory: a request's keys copy and workspace come from the
// stream-ordered pool and go back on the same compute stream right after its
// kernels; its outputs come from a per-server cache and go back when its
// completion event has fired.  The worker holds the server mutex only to
// move requests between the queue, the admitted set and the result list;
// CUDA calls run unlocked.
// Results are exact and identical to the plain call (same kernels / same
// integer arithmetic); results are copied into the caller's host buffers
// before poll() reports them.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "../../include/drtopk.h"
#include "plan.h"
#include "segmented.cuh"

using namespace drtopk;

namespace {

// stream roles: compute streams, each paired with its own copy stream for
// the result copies and completion events (a request's copy waits only for
// its own stream's kernels, never behind another stream's slower request)
constexpr int ST_BATCH = 0;    // micro-batches (segmented kernel, not cooperative)
constexpr int ST_TAIL = 1;     // single selects with the one-CTA shared-memory tail
constexpr int ST_SINGLE = 2;   // first of NSINGLE streams for the other single selects (dealt
                               // round-robin when NSINGLE > 1)
// Single selects run in order on one stream with the planner's own team
// choice (the whole-GPU cooperative tail for large problems: one at a time).
// Four streams with the shared-GPU team (SINGLE_TEAM 4: each tail in one
// 8-CTA cluster, overlapping the other streams' samplers) reached 14-17 K
// req/s on the bench mix against ~11.5 K, but under saturation a cluster
// launch could wait seconds for 8 free SMs of one GPC while the other
// streams' samplers kept arriving (p99 1.7-2.7 s, 0.7-1.2 K req/s in two
// runs), so it is not the default.
constexpr int NSINGLE = 1;
constexpr int SINGLE_TEAM = 0;
constexpr int NCOMPUTE = ST_SINGLE + NSINGLE;
constexpr int ST_COPY = NCOMPUTE;  // copy stream of compute stream i: ST_COPY + i
constexpr int NSTREAMS = 2 * NCOMPUTE;
constexpr uint64_t BATCH_MAX_N = 1ull << 22;  // larger inputs run as single selects

struct Req {
  uint64_t id = 0;
  drtopk_dtype_t dtype = DRTOPK_U32;
  uint64_t n = 0, k = 0;
  int sorted = 0;
  void* user_vals = nullptr;
  int64_t* user_idx = nullptr;
  const void* dkeys_user = nullptr;  // device-resident keys (caller-owned)
  void* hkeys = nullptr;             // pinned copy of host keys
  size_t hkeys_cap = 0;
  char* dmem = nullptr;              // keys copy (+ workspace when run alone): stream-ordered, freed
                                     // on the compute stream right after the request's kernels
  char* dout = nullptr;              // outputs (kth | values | indices) from the server's device cache
  size_t dout_cap = 0;
  size_t dbytes = 0;
  size_t ws_bytes = 0;
  uint32_t* d_keys = nullptr;
  uint32_t* d_kth = nullptr;
  uint32_t* d_vals = nullptr;
  int64_t* d_idx = nullptr;
  char* d_ws = nullptr;
  void* hout = nullptr;              // pinned staging of the outputs
  size_t hout_cap = 0;
  void* extra = nullptr;             // pinned batch-descriptor staging released with this request
  size_t extra_cap = 0;
  cudaEvent_t ev = nullptr;
  int stream = 0;
  int ev_stream = 0;                 // stream the completion event is recorded on
  drtopk_result_t res = {};
  double t_submit = 0, t_start = 0, t_done = 0;
  int status = DRTOPK_OK;
  bool small = false;
  bool planned = false;              // plan computed once, at first admission attempt
  Plan plan;
};

// Process-wide cache of pinned host buffers (size classes of powers of two),
// shared by all servers so pinning happens once per process, not per request.
struct PinnedCache {
  std::mutex mu;
  std::multimap<size_t, void*> free_;
  size_t cached = 0;
  std::atomic<uint64_t> allocs{0};
  std::atomic<uint64_t> alloc_ns{0};
  void* get(size_t bytes, size_t* cap) {
    std::lock_guard<std::mutex> lk(mu);
    size_t c = 4096;
    while (c < bytes) c <<= 1;
    auto it = free_.lower_bound(c);
    if (it != free_.end() && it->first <= 2 * c) {
      void* p = it->second;
      *cap = it->first;
      cached -= it->first;
      free_.erase(it);
      return p;
    }
    void* p = nullptr;
    const auto t0 = std::chrono::steady_clock::now();
    const cudaError_t e = cudaHostAlloc(&p, c, cudaHostAllocPortable);
    alloc_ns += (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0)
                    .count();
    allocs++;
    if (e != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    *cap = c;
    return p;
  }
  void put(void* p, size_t cap) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(mu);
    if (cached + cap > (size_t(8) << 30)) {
      cudaFreeHost(p);
      return;
    }
    free_.emplace(cap, p);
    cached += cap;
  }
};

// Process-wide cache of device output buffers, one per device (power-of-two
// size classes).  A buffer goes back to the cache only after its request's
// completion event has fired (its result copy is done), so reuse needs no
// stream ordering; servers created later reuse what earlier ones allocated,
// so a new server does not pay cudaMalloc in the middle of its traffic.
struct DevCache {
  std::mutex mu;
  std::multimap<size_t, void*> free_;
  void* get(size_t bytes, size_t* cap) {
    size_t c = 4096;
    while (c < bytes) c <<= 1;
    {
      std::lock_guard<std::mutex> lk(mu);
      auto it = free_.lower_bound(c);
      if (it != free_.end() && it->first <= 2 * c) {
        void* p = it->second;
        *cap = it->first;
        free_.erase(it);
        return p;
      }
    }
    void* p = nullptr;
    if (cudaMalloc(&p, c) != cudaSuccess) {  // on the calling thread's current device
      cudaGetLastError();
      return nullptr;
    }
    *cap = c;
    return p;
  }
  void put(void* p, size_t cap) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(mu);
    free_.emplace(cap, p);
  }
};

DevCache& dev_cache(int device) {
  static std::mutex mu;
  static DevCache* caches[64] = {};
  std::lock_guard<std::mutex> lk(mu);
  if (!caches[device]) caches[device] = new DevCache();  // lives until process exit
  return *caches[device];
}

PinnedCache& pinned_cache() {
  static PinnedCache* c = new PinnedCache();  // lives until process exit
  return *c;
}

inline size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

struct drtopk_server {
  int device = 0;
  size_t budget = 0;
  int max_inflight = 64;
  drtopk_handle_t h = nullptr;
  cudaStream_t streams[NSTREAMS] = {};
  uint64_t next_single = 0;  // round-robin over the single-select streams (worker thread only)
  cudaEvent_t ev_kernels = nullptr;  // kernels-done marker (re-recorded per launch)
  int seg_grid = 0;
  size_t seg_smem = 0;
  std::mutex mu;
  std::condition_variable cv, done_cv;
  std::deque<Req*> queue;           // guarded by mu
  std::mutex mu_run;                // guards `launched` and ev_free
  std::condition_variable cv_run;   // new work for the completion thread
  std::list<Req*> launched;         // launched, not yet taken by the completion thread
  std::deque<Req*> pending[NSTREAMS];  // completion thread only: per event stream, in record order
  std::deque<drtopk_result_t> results;
  size_t used = 0;
  int inflight = 0;                 // admitted, not yet published (guarded by mu)
  uint64_t next_id = 1;
  bool stop = false;
  std::thread worker, completer;
  std::chrono::steady_clock::time_point t0;
  PinnedCache& pinned = pinned_cache();
  DevCache* outs = nullptr;         // this device's process-wide output cache
  std::vector<cudaEvent_t> ev_free; // guarded by mu_run
  drtopk_server_stats_t stats = {}; // guarded by mu
  uint64_t pin_allocs0 = 0, pin_ns0 = 0;

  double now_ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  cudaEvent_t get_event() {
    {
      std::lock_guard<std::mutex> lk(mu_run);
      if (!ev_free.empty()) {
        cudaEvent_t e = ev_free.back();
        ev_free.pop_back();
        return e;
      }
    }
    cudaEvent_t e = nullptr;
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    return e;
  }
  // device bytes of a request: keys copy (host mode) + outputs (+ workspace when run alone)
  drtopk_status_t need_bytes(Req* r, size_t* out) {
    size_t b = 0;
    if (!r->dkeys_user) b += al256(r->n * 4);
    b += al256(4) + al256(r->k * 4) + al256(r->k * 8);
    if (!r->small) {
      // the request's one plan: autotuned parameters, SINGLE_TEAM
      if (!r->planned) {
        drtopk_params_t p;
        drtopk_params_default(&p);
        p.alpha = -2;
        p.sorted = r->sorted;
        p.team = SINGLE_TEAM;
        drtopk_status_t s = plan_select(device, r->n, r->k, r->dtype, &p, r->user_idx != nullptr, &r->plan);
        if (s != DRTOPK_OK) return s;
        r->planned = true;
      }
      r->ws_bytes = r->plan.ws_bytes;
      b += al256(r->ws_bytes);
    } else {
      // share of the batch workspace: delegates + candidates of its segment
      b += al256(r->n / 16 * 4) + al256(r->k * 8 * 256);
    }
    *out = b;
    return DRTOPK_OK;
  }
  void copy_out(Req* r, cudaError_t q);
  void publish(Req* r);
  void finish_on_copy_stream(Req* r, cudaEvent_t kernels_done);
  void copy_result(Req* r, int si);
  void admit(std::vector<Req*>& out);
  void launch_admitted(std::vector<Req*>& v);
  void complete_loop();
  void launch_single(Req* r);
  void launch_batch(std::vector<Req*>& v, int si);
  void loop();
};

// result of a finished request into the caller's buffers (worker thread, unlocked)
void drtopk_server::copy_out(Req* r, cudaError_t q) {
  r->t_done = now_ms();
  if (q != cudaSuccess) r->status = DRTOPK_ECUDA;
  drtopk_result_t& res = r->res;
  std::memset(&res, 0, sizeof(res));
  res.id = r->id;
  if (r->status == DRTOPK_OK) {
    const char* ho = static_cast<const char*>(r->hout);
    std::memcpy(&res.kth, ho, 4);
    if (r->user_vals) std::memcpy(r->user_vals, ho + al256(4), r->k * 4);
    if (r->user_idx) std::memcpy(r->user_idx, ho + al256(4) + al256(r->k * 4), r->k * 8);
  }
  res.status = r->status;
  res.t_submit_ms = r->t_submit;
  res.t_start_ms = r->t_start;
  res.t_done_ms = r->t_done;
  pinned.put(r->hkeys, r->hkeys_cap);
  pinned.put(r->hout, r->hout_cap);
  pinned.put(r->extra, r->extra_cap);
  r->hkeys = r->hout = r->extra = nullptr;
  outs->put(r->dout, r->dout_cap);
  r->dout = nullptr;
  if (r->ev) {
    std::lock_guard<std::mutex> lk(mu_run);
    ev_free.push_back(r->ev);
  }
  r->ev = nullptr;
}

// hand a finished request to poll() (mutex held)
void drtopk_server::publish(Req* r) {
  results.push_back(r->res);
  used -= r->dbytes;
  inflight--;
  delete r;
}

// result copy: one D2H of the request's contiguous output block (kth,
// values, indices when asked) on stream `xs` behind the kernels, then the
// completion event
void drtopk_server::copy_result(Req* r, int si) {
  cudaStream_t xs = streams[si];
  r->ev_stream = si;
  if (r->status == DRTOPK_OK && r->dout) {
    const size_t outb = al256(4) + al256(r->k * 4) + (r->user_idx ? al256(r->k * 8) : 0);
    if (cudaMemcpyAsync(r->hout, r->d_kth, outb, cudaMemcpyDeviceToHost, xs) != cudaSuccess) r->status = DRTOPK_ECUDA;
  }
  cudaEventRecord(r->ev, xs);
}

// a request's copy on its compute stream's own copy stream, after a wait for
// the kernels (one wait per request, or per micro-batch)
void drtopk_server::finish_on_copy_stream(Req* r, cudaEvent_t kernels_done) {
  cudaStreamWaitEvent(streams[ST_COPY + r->stream], kernels_done, 0);
  copy_result(r, ST_COPY + r->stream);
}

void drtopk_server::launch_single(Req* r) {
  cudaStream_t st = streams[r->stream];
  const uint32_t* keys = r->dkeys_user ? static_cast<const uint32_t*>(r->dkeys_user) : r->d_keys;
  if (!r->dkeys_user && cudaMemcpyAsync(r->d_keys, r->hkeys, r->n * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
    r->status = DRTOPK_ECUDA;
  // the plan made at admission, enqueued directly (no per-call statistics)
  if (r->status == DRTOPK_OK)
    r->status = enqueue_select(r->plan, device, keys, r->d_kth, r->d_vals, r->user_idx ? r->d_idx : nullptr,
                               r->d_ws, st, nullptr);
  if (r->dmem) cudaFreeAsync(r->dmem, st);  // same stream: reusable by the next request at once
  r->dmem = nullptr;
  // the result copy waits on the stream's own copy stream: the compute
  // stream never queues behind the device-to-host engine (copies on the
  // compute streams cut the served rate from ~14-17 K to ~9 K req/s)
  cudaEventRecord(ev_kernels, st);
  finish_on_copy_stream(r, ev_kernels);
}

void drtopk_server::launch_batch(std::vector<Req*>& v, int si) {
  cudaStream_t st = streams[si];
  const int nseg = (int)v.size();
  std::vector<SegDesc> seg(nseg);
  std::vector<uint2> tasks;
  uint64_t del_total = 0, cand_total = 0;
  for (int s = 0; s < nseg; ++s) {
    Req* r = v[s];
    r->stream = si;
    SegDesc& d = seg[s];
    std::memset(&d, 0, sizeof(d));
    d.len = (uint32_t)r->n;
    d.k = (uint32_t)r->k;
    d.km = r->dtype == DRTOPK_F32 ? KM_F32 : KM_U32;
    d.kptr = r->dkeys_user ? static_cast<const uint32_t*>(r->dkeys_user) : r->d_keys;
    d.okth = r->d_kth;
    d.ovals = r->d_vals;
    d.oidx = r->user_idx ? r->d_idx : nullptr;
    d.sorted = r->sorted;
    // same per-segment choice as the batched form
    if (d.len <= 32768) {
      d.mode = SEG_PLAIN;
    } else {
      int a = (int)std::lround(std::log2(std::max(2.0, std::sqrt(5.0 * d.len / d.k))));
      a = std::max(5, std::min(a, 15));
      while (a > 5 && ((((uint64_t)d.len + (1ull << a) - 1) >> a) < d.k)) a--;
      if ((((uint64_t)d.len + (1ull << a) - 1) >> a) < d.k) {
        d.mode = SEG_PLAIN;
      } else {
        d.mode = SEG_DELEGATE;
        d.alpha = a;
      }
    }
    if (d.mode == SEG_DELEGATE) {
      const uint64_t S = 1ull << d.alpha, M = (d.len + S - 1) >> d.alpha;
      d.del_off = del_total;
      del_total += M;
      d.cand_off = cand_total;
      cand_total += (uint64_t)d.k * S;
      d.ntasks = (int)((d.len + SEG_CH - 1) / SEG_CH);
      for (int c = 0; c < d.ntasks; ++c) tasks.push_back(make_uint2((uint32_t)s, (uint32_t)c));
    }
  }
  size_t off = 0;
  const size_t o_seg = off;
  off += al256(sizeof(SegDesc) * nseg);
  const size_t o_tasks = off;
  off += al256(sizeof(uint2) * std::max<size_t>(1, tasks.size()));
  const size_t o_del = off;
  off += al256(4 * std::max<uint64_t>(1, del_total));
  const size_t o_cand = off;
  off += al256(8 * std::max<uint64_t>(1, cand_total));
  const size_t o_ctrl = off;
  const size_t ctrl_bytes = 4 * (8 + 2 * (size_t)nseg);
  off += al256(ctrl_bytes);
  const size_t hbytes = o_del;  // descriptors + tasks are staged from host
  char* ws = nullptr;
  size_t hcap = 0;
  char* hst = static_cast<char*>(pinned.get(hbytes, &hcap));
  bool ok = hst && cudaMallocAsync(reinterpret_cast<void**>(&ws), off, st) == cudaSuccess;
  if (ok) {
    std::memcpy(hst + o_seg, seg.data(), sizeof(SegDesc) * nseg);
    if (!tasks.empty()) std::memcpy(hst + o_tasks, tasks.data(), sizeof(uint2) * tasks.size());
    for (Req* r : v)
      if (!r->dkeys_user) cudaMemcpyAsync(r->d_keys, r->hkeys, r->n * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(ws, hst, hbytes, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(ws + o_ctrl, 0, ctrl_bytes, st);
    uint32_t* ctrl = reinterpret_cast<uint32_t*>(ws + o_ctrl);
    SegArgs a;
    std::memset(&a, 0, sizeof(a));
    a.keys = nullptr;
    a.seg = reinterpret_cast<const SegDesc*>(ws + o_seg);
    a.tasks = reinterpret_cast<const uint2*>(ws + o_tasks);
    a.n_sampler_tasks = (uint32_t)tasks.size();
    a.nseg = (uint32_t)nseg;
    a.del_pool = reinterpret_cast<uint32_t*>(ws + o_del);
    a.cand_pool = reinterpret_cast<uint2*>(ws + o_cand);
    a.ticket = ctrl;
    a.err = ctrl + 1;
    a.done = ctrl + 8;
    a.seg_err = ctrl + 8 + nseg;
    const int grid = std::min<int>(seg_grid, (int)(tasks.size() + nseg));
    if (launch_segmented(a, std::max(1, grid), seg_smem, st) != cudaSuccess) ok = false;
    cudaFreeAsync(ws, st);
  }
  for (Req* r : v) {
    if (r->dmem) cudaFreeAsync(r->dmem, st);
    r->dmem = nullptr;
  }
  cudaEventRecord(ev_kernels, st);
  for (Req* r : v) {
    if (!ok) r->status = DRTOPK_ENOMEM;
    finish_on_copy_stream(r, ev_kernels);
  }
  // the descriptor staging buffer may be reused only after its copy ran:
  // it is released with the last request of the batch (completion event
  // recorded later on the copy stream)
  if (hst) {
    v.back()->extra = hst;
    v.back()->extra_cap = hcap;
  }
}

// Admission (mutex held): move requests from the queue into `out` while the
// in-flight limit and the byte budget allow; no CUDA calls here.
void drtopk_server::admit(std::vector<Req*>& out) {
  int scanned = 0;
  const double t = now_ms();
  for (auto it = queue.begin(); it != queue.end() && inflight < max_inflight && scanned < 256; ++scanned) {
    Req* r = *it;
    size_t need = 0;
    drtopk_status_t s = need_bytes(r, &need);
    if (s == DRTOPK_OK && budget && need > budget) s = DRTOPK_EBUDGET;
    if (s != DRTOPK_OK) {
      it = queue.erase(it);
      r->status = s;
      r->t_start = t;
      r->dbytes = 0;
      inflight++;
      copy_out(r, cudaSuccess);
      publish(r);
      continue;
    }
    if (budget && used + need > budget) {
      // head-of-line request too large for now: smaller ones may pass it,
      // unless it has waited for 50 ms (then it goes first)
      if (it == queue.begin() && t - r->t_submit > 50.0) break;
      ++it;
      continue;
    }
    it = queue.erase(it);
    r->t_start = t;
    r->dbytes = need;
    used += need;
    inflight++;
    out.push_back(r);
  }
}

// Device work of the admitted requests (worker thread, unlocked): small
// requests of this tick form one micro-batch, the others run one select each.
void drtopk_server::launch_admitted(std::vector<Req*>& v) {
  std::vector<Req*> small;
  for (Req* r : v) {
    r->ev = get_event();
    const size_t outb = al256(4) + al256(r->k * 4) + al256(r->k * 8);
    r->hout = pinned.get(outb, &r->hout_cap);
    r->stream = r->small ? ST_BATCH : ST_SINGLE + (int)(next_single++ % NSINGLE);
    // a select whose tail is the one-CTA kernel holds few SMs and never
    // waits on other CTAs: it runs on its own stream, beside the others
    if (!r->small && r->plan.tail) r->stream = ST_TAIL;
    cudaStream_t st = streams[r->stream];
    // keys copy (host mode) and, for a request run alone, its workspace
    const size_t kb = r->dkeys_user ? 0 : al256(r->n * 4);
    const size_t dev = kb + (r->small ? 0 : al256(r->ws_bytes));
    r->dout = static_cast<char*>(r->hout ? outs->get(outb, &r->dout_cap) : nullptr);
    if (!r->dout || (dev && cudaMallocAsync(reinterpret_cast<void**>(&r->dmem), dev, st) != cudaSuccess)) {
      cudaGetLastError();
      r->dmem = nullptr;
      r->status = DRTOPK_ENOMEM;
      r->ev_stream = ST_COPY + r->stream;
      cudaEventRecord(r->ev, streams[r->ev_stream]);
      continue;
    }
    if (!r->dkeys_user) r->d_keys = reinterpret_cast<uint32_t*>(r->dmem);
    r->d_ws = r->dmem + kb;
    char* p = r->dout;
    r->d_kth = reinterpret_cast<uint32_t*>(p);
    p += al256(4);
    r->d_vals = reinterpret_cast<uint32_t*>(p);
    p += al256(r->k * 4);
    r->d_idx = reinterpret_cast<int64_t*>(p);
    if (r->small) small.push_back(r);
    else launch_single(r);
  }
  if (!small.empty()) launch_batch(small, ST_BATCH);
  // hand the requests (all with their completion events recorded) to the
  // completion thread
  {
    std::lock_guard<std::mutex> lk(mu_run);
    for (Req* r : v) launched.push_back(r);
  }
  cv_run.notify_one();
}

// Launch thread: admission and launches.  Completions run on their own
// thread (complete_loop), so result copies into the caller's buffers never
// hold up the next launches.
void drtopk_server::loop() {
  cudaSetDevice(device);
  std::vector<Req*> admitted;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(mu);
      if (stop && queue.empty()) break;
      if (!queue.empty()) admit(admitted);
      if (inflight == 0) done_cv.notify_all();  // requests refused at admission are already published
      if (admitted.empty()) {
        // woken by submit() and by every publish (a slot or budget freed)
        cv.wait_for(lk, std::chrono::milliseconds(queue.empty() ? 5 : 1));
        continue;
      }
    }
    const auto tl0 = std::chrono::steady_clock::now();
    uint64_t ns = 0, nbr = 0;
    for (Req* r : admitted) (r->small ? nbr : ns)++;
    launch_admitted(admitted);
    admitted.clear();
    const double ms_launch = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tl0).count();
    {
      std::lock_guard<std::mutex> lk(mu);
      stats.host_ms_launch += ms_launch;
      stats.singles += ns;
      stats.batches += nbr ? 1 : 0;
      stats.batched += nbr;
      stats.worker_ticks++;
    }
  }
}

// Completion thread: polls the launched requests' completion events, copies
// finished results into the caller's buffers and publishes them.
void drtopk_server::complete_loop() {
  cudaSetDevice(device);
  std::vector<Req*> finished;
  std::vector<cudaError_t> fq;
  for (;;) {
    bool any = false;
    {
      std::unique_lock<std::mutex> lk(mu_run);
      for (Req* r : launched) pending[r->ev_stream].push_back(r);
      launched.clear();
      for (const auto& q : pending) any = any || !q.empty();
      if (!any) {
        {
          std::lock_guard<std::mutex> lk2(mu);
          if (stop && queue.empty() && inflight == 0) break;
        }
        cv_run.wait_for(lk, std::chrono::milliseconds(2));
        continue;
      }
    }
    // events on one stream complete in record order: only the oldest
    // pending request of each stream needs a query
    finished.clear();
    fq.clear();
    for (auto& q : pending) {
      while (!q.empty()) {
        const cudaError_t e = cudaEventQuery(q.front()->ev);
        if (e == cudaErrorNotReady) break;
        if (e != cudaSuccess) cudaGetLastError();
        finished.push_back(q.front());
        fq.push_back(e);
        q.pop_front();
      }
    }
    if (finished.empty()) {
      std::this_thread::sleep_for(std::chrono::microseconds(10));
      continue;
    }
    const auto tc0 = std::chrono::steady_clock::now();
    for (size_t i = 0; i < finished.size(); ++i) copy_out(finished[i], fq[i]);
    const double ms_complete =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tc0).count();
    {
      std::lock_guard<std::mutex> lk(mu);
      stats.host_ms_complete += ms_complete;
      for (Req* r : finished) publish(r);
    }
    cv.notify_one();
    done_cv.notify_all();
  }
  done_cv.notify_all();
}

extern "C" drtopk_status_t drtopk_server_create(drtopk_server_t* out, int device, size_t hbm_budget_bytes,
                                                int max_inflight) {
  if (!out) return DRTOPK_EINVAL;
  *out = nullptr;
  int cur = 0;
  cudaGetDevice(&cur);
  if (device < 0 || device >= 64 || cudaSetDevice(device) != cudaSuccess) return DRTOPK_EINVAL;
  drtopk_server* s = new (std::nothrow) drtopk_server();
  if (!s) return DRTOPK_ENOMEM;
  s->device = device;
  s->outs = &dev_cache(device);
  s->budget = hbm_budget_bytes;
  s->max_inflight = max_inflight > 0 ? max_inflight : 64;
  s->t0 = std::chrono::steady_clock::now();
  drtopk_status_t st = drtopk_create(&s->h, device, 0);
  for (int i = 0; st == DRTOPK_OK && i < NSTREAMS; ++i)
    if (cudaStreamCreateWithFlags(&s->streams[i], cudaStreamNonBlocking) != cudaSuccess) st = DRTOPK_ECUDA;
  if (st == DRTOPK_OK && cudaEventCreateWithFlags(&s->ev_kernels, cudaEventDisableTiming) != cudaSuccess)
    st = DRTOPK_ECUDA;
  if (st == DRTOPK_OK) {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    if (segmented_shape(device, &s->seg_grid, &s->seg_smem) != cudaSuccess) st = DRTOPK_ECUDA;
  }
  cudaSetDevice(cur);
  if (st != DRTOPK_OK) {
    if (s->h) drtopk_destroy(s->h);
    for (auto& x : s->streams)
      if (x) cudaStreamDestroy(x);
    if (s->ev_kernels) cudaEventDestroy(s->ev_kernels);
    delete s;
    return st;
  }
  s->pin_allocs0 = s->pinned.allocs.load();
  s->pin_ns0 = s->pinned.alloc_ns.load();
  s->worker = std::thread([s]() { s->loop(); });
  s->completer = std::thread([s]() { s->complete_loop(); });
  *out = s;
  return DRTOPK_OK;
}

extern "C" drtopk_status_t drtopk_server_destroy(drtopk_server_t s) {
  if (!s) return DRTOPK_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    // queued requests are cancelled
    for (Req* r : s->queue) {
      s->pinned.put(r->hkeys, r->hkeys_cap);
      delete r;
    }
    s->queue.clear();
  }
  s->cv.notify_all();
  if (s->worker.joinable()) s->worker.join();
  s->cv_run.notify_all();
  if (s->completer.joinable()) s->completer.join();
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(s->device);
  for (auto& x : s->streams)
    if (x) cudaStreamSynchronize(x);
  for (auto& x : s->streams)
    if (x) cudaStreamDestroy(x);
  for (auto e : s->ev_free) cudaEventDestroy(e);
  if (s->ev_kernels) cudaEventDestroy(s->ev_kernels);
  drtopk_destroy(s->h);
  cudaSetDevice(cur);
  delete s;
  return DRTOPK_OK;
}

static drtopk_status_t submit_impl(drtopk_server_t s, const void* h_keys, const void* d_keys, drtopk_dtype_t dtype,
                                   uint64_t n, uint64_t k, int sorted, void* out_vals, int64_t* out_idx,
                                   uint64_t* id) {
  if (!s || (!h_keys && !d_keys) || n == 0 || k < 1 || k > n || n > 0xffffffffull) return DRTOPK_EINVAL;
  if (dtype != DRTOPK_U32 && dtype != DRTOPK_F32) return DRTOPK_EINVAL;
  Req* r = new (std::nothrow) Req();
  if (!r) return DRTOPK_ENOMEM;
  r->dtype = dtype;
  r->n = n;
  r->k = k;
  r->sorted = sorted;
  r->user_vals = out_vals;
  r->user_idx = out_idx;
  r->dkeys_user = d_keys;
  r->small = n <= BATCH_MAX_N && k <= (uint64_t)SEG_MAX_K;  // micro-batched through the segmented kernel
  // coarse check here (the exact workspace is sized at admission, on the
  // worker thread): the keys alone must fit the budget
  if (s->budget && (d_keys ? 0 : n * 4) + k * 12 > s->budget) {
    delete r;
    return DRTOPK_EBUDGET;
  }
  if (h_keys) {
    r->hkeys = s->pinned.get(n * 4, &r->hkeys_cap);
    if (!r->hkeys) {
      delete r;
      return DRTOPK_ENOMEM;
    }
  }
  if (h_keys) std::memcpy(r->hkeys, h_keys, n * 4);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    r->t_submit = s->now_ms();
    s->queue.push_back(r);
  }
  if (id) *id = r->id;
  s->cv.notify_all();
  return DRTOPK_OK;
}

extern "C" drtopk_status_t drtopk_server_submit(drtopk_server_t s, const void* h_keys, drtopk_dtype_t dtype,
                                                uint64_t n, uint64_t k, int sorted, void* out_vals, int64_t* out_idx,
                                                uint64_t* id) {
  if (!h_keys) return DRTOPK_EINVAL;
  return submit_impl(s, h_keys, nullptr, dtype, n, k, sorted, out_vals, out_idx, id);
}

extern "C" drtopk_status_t drtopk_server_submit_device(drtopk_server_t s, const void* d_keys, drtopk_dtype_t dtype,
                                                       uint64_t n, uint64_t k, int sorted, void* out_vals,
                                                       int64_t* out_idx, uint64_t* id) {
  if (!d_keys) return DRTOPK_EINVAL;
  return submit_impl(s, nullptr, d_keys, dtype, n, k, sorted, out_vals, out_idx, id);
}

extern "C" drtopk_status_t drtopk_server_poll(drtopk_server_t s, drtopk_result_t* results, int max, int* count) {
  if (!s || !count || (max > 0 && !results)) return DRTOPK_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  int c = 0;
  while (c < max && !s->results.empty()) {
    results[c++] = s->results.front();
    s->results.pop_front();
  }
  *count = c;
  return c ? DRTOPK_OK : DRTOPK_EAGAIN;
}

extern "C" drtopk_status_t drtopk_server_cancel(drtopk_server_t s, uint64_t id) {
  if (!s) return DRTOPK_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
    if ((*it)->id == id) {
      Req* r = *it;
      s->queue.erase(it);
      drtopk_result_t res;
      std::memset(&res, 0, sizeof(res));
      res.id = id;
      res.status = DRTOPK_ECANCELLED;
      res.t_submit_ms = r->t_submit;
      res.t_done_ms = s->now_ms();
      s->results.push_back(res);
      s->pinned.put(r->hkeys, r->hkeys_cap);
      delete r;
      s->done_cv.notify_all();
      return DRTOPK_OK;
    }
  }
  return DRTOPK_EAGAIN;  // already started or unknown
}

extern "C" drtopk_status_t drtopk_server_drain(drtopk_server_t s, int timeout_ms) {
  if (!s) return DRTOPK_EINVAL;
  std::unique_lock<std::mutex> lk(s->mu);
  auto pred = [&]() { return s->queue.empty() && s->inflight == 0; };
  if (timeout_ms < 0) {
    s->done_cv.wait(lk, pred);
    return DRTOPK_OK;
  }
  return s->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred) ? DRTOPK_OK : DRTOPK_ETIMEOUT;
}

extern "C" drtopk_status_t drtopk_server_usage(drtopk_server_t s, size_t* resident_bytes, int* inflight, int* queued) {
  if (!s) return DRTOPK_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  if (resident_bytes) *resident_bytes = s->used;
  if (inflight) *inflight = s->inflight;
  if (queued) *queued = (int)s->queue.size();
  return DRTOPK_OK;
}

extern "C" drtopk_status_t drtopk_server_stats(drtopk_server_t s, drtopk_server_stats_t* st) {
  if (!s || !st) return DRTOPK_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  *st = s->stats;
  // the staging cache is process-wide: report what it did since this server started
  st->pinned_allocs = s->pinned.allocs.load() - s->pin_allocs0;
  st->host_ms_pinned = (double)(s->pinned.alloc_ns.load() - s->pin_ns0) * 1e-6;
  return DRTOPK_OK;
}
