// server.cu -- served form: continuous batching of top-k requests.
//
// A worker thread admits queued requests as in-flight slots and the HBM byte
// budget allow, and keeps admitting while earlier requests are still on the
// GPU.  The requests admitted in one tick become, per key mode, ONE chain of
// grouped launches of the sampled-threshold select (enqueue_group): every
// launch covers all of the chain's problems, each problem getting the CTAs
// its size calls for, and the last levels run one CTA per problem -- no
// launch needs the whole GPU, so chains on different streams overlap.  A
// chain's control blocks, workspaces (candidate buffers sized by the key
// sample's estimate), host-mode keys and outputs live in one stream-ordered
// arena; its outputs come back with one device-to-host copy.  A select whose
// sample misjudged the input (DE_RETRY) runs again on the completion thread
// with the general plan.  Sorted requests of more than 4096 keys keep the
// whole-GPU sort and run one at a time on their own stream.
// Host time per request is its share of one chain's launches, which is what
// lets the server outrun a loop of plain calls.  The completion thread polls
// the chains' events, copies results into the callers' buffers and publishes
// them (the copies spread over a few helper threads); neither thread holds
// the server mutex during CUDA calls.
// Results are exact and identical to the plain call (same integer
// arithmetic).
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
#include "fused.cuh"

using namespace drtopk;

namespace {

// stream roles: compute streams, each paired with its own copy stream for
// the result copies and completion events (a request's copy waits only for
// its own stream's kernels, never behind another stream's slower request)
constexpr int ST_AUX = 0;      // server set-up work (memory pool warm-up)
constexpr int ST_TAIL = 1;     // single selects with the one-CTA shared-memory tail
constexpr int ST_SINGLE = 2;   // first of NSINGLE streams for the other single selects (dealt
                               // round-robin when NSINGLE > 1)
// Single selects take the sampled-threshold path with every launch an
// ordinary one (sample passes, the appending pass and the level-0 split over
// the whole GPU, the last levels in one CTA, team 5): no launch waits for a
// share of the GPU, so the selects of NSINGLE - 1 streams overlap, one's
// streaming filling the SMs another's last levels leave free.  Cooperative
// or cluster tails on several streams starve under load (a cluster launch
// waited seconds for 8 free SMs of one GPC while other streams' samplers
// kept arriving), so the one kind of single that keeps a cooperative kernel
// -- sorted output of more than SINGLE_ONE_CTA_SORT_K keys, sorted over the
// whole GPU -- runs in order on the first single stream.
constexpr int NSINGLE = 8;
constexpr int SINGLE_TEAM = 0;
constexpr int NCOMPUTE = ST_SINGLE + NSINGLE;
constexpr int ST_COPY = NCOMPUTE;  // copy stream of compute stream i: ST_COPY + i
constexpr int NSTREAMS = 2 * NCOMPUTE;
constexpr uint64_t SINGLE_ONE_CTA_SORT_K = 4096;     // sorted outputs larger than this keep the whole-GPU sort
constexpr size_t GROUP_OUT_CAP = size_t(32) << 20;   // output bytes of one grouped launch chain
constexpr size_t PREWARM_POOL = size_t(8) << 30;     // device pool bytes mapped at server creation

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
  bool planned = false;              // plan computed once, at first admission attempt
  Plan plan;
  const uint32_t* errp = nullptr;    // grouped: the device error word, in the group's staging
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
    if (!p || cap == 0) return;  // cap 0: a view into a buffer another request owns
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

// Helper threads for the completion thread's result copies: the copies of
// the requests finished together are cut into pieces of up to COPY_PIECE
// bytes and spread over the helpers and the completion thread itself.  One
// host thread copies far slower than a saturated server returns results,
// and an in-flight slot frees only once its copy is done (with one thread
// the server ran at 24 K requests/s, with three helpers at 36 K, on the
// same B200 and request mix).
constexpr size_t COPY_PIECE = size_t(1) << 20;
constexpr int COPY_HELPERS = 3;
struct CopyPiece {
  void* dst;
  const void* src;
  size_t n;
};
class CopyPool {
 public:
  CopyPool() {
    for (int i = 0; i < COPY_HELPERS; ++i) th_.emplace_back([this] { run(); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  // copies every piece; returns once all are done
  void copy(const std::vector<CopyPiece>& pieces) {
    if (pieces.empty()) return;
    {
      std::lock_guard<std::mutex> lk(mu_);
      work_ = &pieces;
      next_ = 0;
      left_ = pieces.size();
    }
    cv_.notify_all();
    drain();
    std::unique_lock<std::mutex> lk(mu_);
    done_.wait(lk, [&] { return left_ == 0; });
    work_ = nullptr;
  }

 private:
  void drain() {
    for (;;) {
      CopyPiece p;
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (!work_ || next_ >= work_->size()) return;
        p = (*work_)[next_++];
      }
      std::memcpy(p.dst, p.src, p.n);
      std::lock_guard<std::mutex> lk(mu_);
      if (--left_ == 0) done_.notify_all();
    }
  }
  void run() {
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || (work_ && next_ < work_->size()); });
        if (stop_) return;
      }
      drain();
    }
  }
  std::mutex mu_;
  std::condition_variable cv_, done_;
  const std::vector<CopyPiece>* work_ = nullptr;
  size_t next_ = 0, left_ = 0;
  bool stop_ = false;
  std::vector<std::thread> th_;
};

void add_pieces(std::vector<CopyPiece>& v, void* dst, const void* src, size_t n) {
  for (size_t o = 0; o < n; o += COPY_PIECE)
    v.push_back({static_cast<char*>(dst) + o, static_cast<const char*>(src) + o, std::min(COPY_PIECE, n - o)});
}

}  // namespace

struct drtopk_server {
  int device = 0;
  size_t budget = 0;
  int max_inflight = 64;
  drtopk_handle_t h = nullptr;
  cudaStream_t streams[NSTREAMS] = {};
  uint64_t next_single = 0;  // round-robin over the single-select streams (worker thread only)
  cudaEvent_t ev_kernels = nullptr;  // kernels-done marker (re-recorded per launch)
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
  CopyPool copies;                  // completion thread's result copies
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
    {
      // the request's one plan: autotuned parameters, SINGLE_TEAM
      if (!r->planned) {
        drtopk_params_t p;
        drtopk_params_default(&p);
        p.alpha = -2;
        p.sorted = r->sorted;
        p.team = SINGLE_TEAM;
        if (!r->sorted || r->k <= SINGLE_ONE_CTA_SORT_K) {
          // the sampled-threshold path with every launch an ordinary one (the
          // last levels in one CTA): no launch waits for a share of the GPU,
          // so the single streams' selects overlap
          p.alpha = 0;
          p.path = 4;
          p.team = 5;
        }
        drtopk_status_t s = plan_select_bounded(device, r->n, r->k, r->dtype, &p, r->user_idx != nullptr, &r->plan);
        if (s != DRTOPK_OK) return s;
        r->planned = true;
      }
      r->ws_bytes = r->plan.ws_bytes;
      b += al256(r->ws_bytes);
    }
    *out = b;
    return DRTOPK_OK;
  }
  void copy_out(Req* r, cudaError_t q, std::vector<CopyPiece>& pieces);
  void release(Req* r);
  void publish(Req* r);
  void finish_on_copy_stream(Req* r, cudaEvent_t kernels_done);
  void copy_result(Req* r, int si);
  void admit(std::vector<Req*>& out);
  void launch_admitted(std::vector<Req*>& v);
  void complete_loop();
  void launch_single(Req* r);
  void launch_group(std::vector<Req*>& v, int si);
  void prewarm();
  void retry_general(Req* r);
  void retry_general_run(Req* r);
  drtopk_handle_t h_retry = nullptr;  // completion thread only
  double alloc_ms = 0;                // worker thread: time in cudaMallocAsync (read under mu via stats)
  uint64_t retries = 0;               // completion thread
  double retry_ms = 0;
  void loop();
};

// result of a finished request into the caller's buffers (completion
// thread, unlocked); the values and indices go to `pieces` for the copy pool
void drtopk_server::copy_out(Req* r, cudaError_t q, std::vector<CopyPiece>& pieces) {
  r->t_done = now_ms();
  if (q != cudaSuccess) r->status = DRTOPK_ECUDA;
  drtopk_result_t& res = r->res;
  std::memset(&res, 0, sizeof(res));
  res.id = r->id;
  if (r->status == DRTOPK_OK) {
    const char* ho = static_cast<const char*>(r->hout);
    std::memcpy(&res.kth, ho, 4);
    if (r->user_vals) add_pieces(pieces, r->user_vals, ho + al256(4), r->k * 4);
    if (r->user_idx) add_pieces(pieces, r->user_idx, ho + al256(4) + al256(r->k * 4), r->k * 8);
  }
}

// after the copies: staging, outputs and the event go back to their caches
void drtopk_server::release(Req* r) {
  drtopk_result_t& res = r->res;
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

// Sampled-threshold singles of one key mode admitted in the same tick: one
// device arena (control blocks, workspaces, host-mode keys, outputs, launch
// descriptors), one chain of grouped launches (enqueue_group), one copy of
// all outputs back, one free.  Host work per request drops to filling its
// descriptor; the grouped kernels keep the GPU busy across problems.
void drtopk_server::launch_group(std::vector<Req*>& v, int si) {
  cudaStream_t st = streams[si];
  const int np = (int)v.size();
  std::vector<size_t> o_ctrl(np), o_ws(np), o_keys(np), o_out(np);
  size_t off = 0;
  for (int i = 0; i < np; ++i) {
    o_ctrl[i] = off;
    off += al256(v[i]->plan.ctrl_bytes);
  }
  const size_t ctrl_total = off;
  for (int i = 0; i < np; ++i) {
    o_ws[i] = off;
    off += al256(v[i]->plan.ws_bytes);
  }
  for (int i = 0; i < np; ++i) {
    o_keys[i] = off;
    if (!v[i]->dkeys_user) off += al256(v[i]->n * 4);
  }
  const size_t out0 = off;
  for (int i = 0; i < np; ++i) {
    Req* r = v[i];
    o_out[i] = off - out0;
    off += al256(4) + al256(r->k * 4) + (r->user_idx ? al256(r->k * 8) : 0);
  }
  const size_t o_err = off - out0;  // the problems' error words, copied back with the outputs
  off += al256(4 * (size_t)np);
  const size_t out_total = off - out0;
  const size_t o_desc = off;
  const size_t desc = group_desc_bytes(np);
  off += desc;
  size_t hcap = 0;
  char* hst = static_cast<char*>(pinned.get(out_total + desc, &hcap));
  char* arena = nullptr;
  const auto ta0 = std::chrono::steady_clock::now();
  bool ok = hst && cudaMallocAsync(reinterpret_cast<void**>(&arena), off, st) == cudaSuccess;
  if (!ok) cudaGetLastError();
  alloc_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ta0).count();
  if (ok && cudaMemsetAsync(arena, 0, ctrl_total, st) != cudaSuccess) ok = false;
  std::vector<GroupItem> items(np);
  for (int i = 0; ok && i < np; ++i) {
    Req* r = v[i];
    r->stream = si;
    const void* keys = r->dkeys_user;
    if (!keys) {
      keys = arena + o_keys[i];
      if (cudaMemcpyAsync(arena + o_keys[i], r->hkeys, r->n * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
        ok = false;
    }
    char* o = arena + out0 + o_out[i];
    items[i] = {&r->plan, keys, o, o + al256(4), r->user_idx ? reinterpret_cast<int64_t*>(o + al256(4) + al256(r->k * 4))
                                                              : nullptr,
                arena + o_ws[i], arena + o_ctrl[i]};
  }
  if (ok && enqueue_group(device, v[0]->plan.km, items.data(), np, hst + out_total, arena + o_desc,
                         reinterpret_cast<uint32_t*>(arena + out0 + o_err), st) != DRTOPK_OK)
    ok = false;
  // the outputs' copy back and the arena's release on the compute stream's
  // own copy stream: the next chain's kernels do not queue behind the
  // device-to-host engine
  const int xsi = ST_COPY + si;
  cudaStream_t xs = streams[xsi];
  cudaEventRecord(ev_kernels, st);
  cudaStreamWaitEvent(xs, ev_kernels, 0);
  if (ok && cudaMemcpyAsync(hst, arena + out0, out_total, cudaMemcpyDeviceToHost, xs) != cudaSuccess) ok = false;
  if (arena) cudaFreeAsync(arena, xs);
  for (int i = 0; i < np; ++i) {
    Req* r = v[i];
    r->stream = si;
    r->ev_stream = xsi;
    r->hout = hst ? hst + o_out[i] : nullptr;
    r->hout_cap = 0;  // a view into the group's staging (owned by the last request)
    r->errp = hst ? reinterpret_cast<const uint32_t*>(hst + o_err) + i : nullptr;
    if (!ok) r->status = DRTOPK_ECUDA;
    cudaEventRecord(r->ev, xs);
  }
  // the staging is released with the last request (its completion event is
  // recorded after the copy)
  if (hst) {
    v.back()->extra = hst;
    v.back()->extra_cap = hcap;
  }
}

// A grouped select whose device error word is set (DE_RETRY: its bounded
// candidate buffers could not hold the select; any other bit) runs again
// here, on the completion thread, with its general plan (autotuned,
// full-size workspace on the retry handle), and its results replace the
// staged ones.  Rare: the sample must have badly misjudged the input (heavy
// ties around the predicted threshold, an adversarial layout).
void drtopk_server::retry_general(Req* r) {
  const auto t0r = std::chrono::steady_clock::now();
  retry_general_run(r);
  retries++;
  retry_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0r).count();
}

void drtopk_server::retry_general_run(Req* r) {
  r->status = DRTOPK_ECUDA;
  if (!h_retry && drtopk_create(&h_retry, device, 0) != DRTOPK_OK) return;
  const size_t outb = al256(4) + al256(r->k * 4) + (r->user_idx ? al256(r->k * 8) : 0);
  char* d = nullptr;
  const size_t kb = r->dkeys_user ? 0 : al256(r->n * 4);
  if (cudaMalloc(&d, kb + outb) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  const void* keys = r->dkeys_user;
  drtopk_status_t s = DRTOPK_OK;
  if (!keys) {
    keys = d;
    if (cudaMemcpy(d, r->hkeys, r->n * 4, cudaMemcpyHostToDevice) != cudaSuccess) s = DRTOPK_ECUDA;
  }
  char* o = d + kb;
  drtopk_params_t p;
  drtopk_params_default(&p);
  p.alpha = -2;
  p.sorted = r->sorted;
  if (s == DRTOPK_OK)
    s = drtopk_select(h_retry, keys, r->dtype, r->n, r->k, &p, o, o + al256(4),
                      r->user_idx ? reinterpret_cast<int64_t*>(o + al256(4) + al256(r->k * 4)) : nullptr, nullptr);
  if (s == DRTOPK_OK) s = drtopk_sync_check(h_retry, nullptr);
  if (s == DRTOPK_OK && cudaMemcpy(r->hout, o, outb, cudaMemcpyDeviceToHost) != cudaSuccess) s = DRTOPK_ECUDA;
  cudaFree(d);
  r->status = s;
}

// Memory the worker would otherwise allocate in the middle of traffic
// (blocking its launches for milliseconds): the stream-ordered pool keeps
// PREWARM_POOL bytes mapped (its release threshold is unlimited), and the
// process-wide pinned cache gets two staging buffers of every size class up
// to four times the chain output cap (a chain's staging is its outputs plus
// its launch descriptors), once per process.
void drtopk_server::prewarm() {
  cudaStream_t st = streams[ST_AUX];
  const size_t want = std::min<size_t>(PREWARM_POOL, budget ? budget / 4 : PREWARM_POOL);
  void* p = nullptr;
  if (cudaMallocAsync(&p, want, st) == cudaSuccess) cudaFreeAsync(p, st);
  else cudaGetLastError();
  cudaStreamSynchronize(st);
  static std::once_flag once;
  std::call_once(once, [this]() {
    // pinned staging of every size class a chain's results can need, more
    // copies of the small classes (at light load many small chains are in
    // flight at once); a miss on the serving path costs a cudaHostAlloc of
    // milliseconds
    std::vector<std::pair<void*, size_t>> got;
    for (size_t c = size_t(64) << 10; c <= 4 * GROUP_OUT_CAP; c <<= 1)
      for (int i = 0, copies = c <= (size_t(4) << 20) ? 8 : (c <= GROUP_OUT_CAP ? 4 : 2); i < copies; ++i) {
        size_t cap = 0;
        void* b = pinned.get(c, &cap);
        if (b) got.emplace_back(b, cap);
      }
    for (auto& g : got) pinned.put(g.first, g.second);
  });
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
      std::vector<CopyPiece> none;
      copy_out(r, cudaSuccess, none);
      release(r);
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

// Device work of the admitted requests (worker thread, unlocked): per key
// mode one grouped chain; a request whose plan keeps a cooperative kernel
// runs as a select of its own.
void drtopk_server::launch_admitted(std::vector<Req*>& v) {
  std::vector<Req*> group[4];  // sampled-threshold selects by key mode
  for (Req* r : v) {
    r->ev = get_event();
    if (r->plan.one_cta) {
      group[r->plan.km].push_back(r);
      continue;
    }
    const size_t outb = al256(4) + al256(r->k * 4) + al256(r->k * 8);
    r->hout = pinned.get(outb, &r->hout_cap);
    // ordinary-launch singles round-robin over streams 1.. of the singles;
    // a single that keeps a cooperative kernel runs in order on stream 0
    r->stream = ST_SINGLE;
    // a select whose tail is the one-CTA kernel holds few SMs and never
    // waits on other CTAs: it runs on its own stream, beside the others
    if (r->plan.tail) r->stream = ST_TAIL;
    cudaStream_t st = streams[r->stream];
    // keys copy (host mode) and, for a request run alone, its workspace
    const size_t kb = r->dkeys_user ? 0 : al256(r->n * 4);
    const size_t dev = kb + al256(r->ws_bytes);
    r->dout = static_cast<char*>(r->hout ? outs->get(outb, &r->dout_cap) : nullptr);
    const auto ta0 = std::chrono::steady_clock::now();
    const bool got = r->dout && (!dev || cudaMallocAsync(reinterpret_cast<void**>(&r->dmem), dev, st) == cudaSuccess);
    alloc_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ta0).count();
    if (!got) {
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
    launch_single(r);
  }
  for (auto& g : group) {
    // chains of at most GROUP_OUT_CAP output bytes (staging stays in the
    // warmed size classes)
    std::vector<Req*> part;
    size_t bytes = 0;
    for (size_t i = 0; i < g.size(); ++i) {
      Req* r = g[i];
      const size_t ob = al256(4) + al256(r->k * 4) + (r->user_idx ? al256(r->k * 8) : 0);
      if (!part.empty() && bytes + ob > GROUP_OUT_CAP) {
        launch_group(part, ST_SINGLE + 1 + (int)(next_single++ % (NSINGLE - 1)));
        part.clear();
        bytes = 0;
      }
      part.push_back(r);
      bytes += ob;
    }
    if (!part.empty()) launch_group(part, ST_SINGLE + 1 + (int)(next_single++ % (NSINGLE - 1)));
  }
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
    for (Req* r : admitted) (r->plan.one_cta ? nbr : ns)++;
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
  std::vector<CopyPiece> pieces;
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
    for (size_t i = 0; i < finished.size(); ++i) {
      Req* r = finished[i];
      if (fq[i] == cudaSuccess && r->status == DRTOPK_OK && r->errp && *r->errp) retry_general(r);
    }
    pieces.clear();
    for (size_t i = 0; i < finished.size(); ++i) copy_out(finished[i], fq[i], pieces);
    copies.copy(pieces);
    for (Req* r : finished) release(r);
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
  }
  if (st == DRTOPK_OK) s->prewarm();
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
  if (s->h_retry) drtopk_destroy(s->h_retry);
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
  st->retries = s->retries;
  st->host_ms_retry = s->retry_ms;
  st->host_ms_alloc = s->alloc_ms;
  return DRTOPK_OK;
}
