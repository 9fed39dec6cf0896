// engine.cuh -- device-side k-th-largest select over (key, payload) sets,
// shared by the first select (on delegates), the second select (on the
// concatenated candidates), plain radix select and the integer bucket select.
//
// One "level" = pick a bin from the histogram of the current set, then split
// the set: keys above the bin go to the top list, keys inside the bin form the
// next set (compacted) and are histogrammed for the next level.
//
// Radix mode reproduces the reference's digit loop exactly
// (baseline+filter+beta+shuffle/radixselect.cuh:191-220 CumulateCount_inplace,
// 352-410 CalculateOccurence_inplace, 1410-1470 / 1666-1780 the host digit
// loops): the bin chosen is the smallest i with CumCount[i] >= n-k+1, which is
// the largest bin whose count-from-the-top reaches the remaining rank R.  The
// range [lo,hi] of the chosen bin is the reference's flag with the digits
// below still zero.  Bucket mode uses the same loop with integer bucket width
// w = (hi-lo)/nb + 1 over a [min,max] range (exact restatement of
// bucket_select/bucketselect_combined.cuh).
//
// All CTAs of a team (the grid of a cooperative kernel, one thread-block
// cluster, or one CTA) execute the same sequence; the pick is recomputed
// redundantly in every CTA from the global histogram, so the replicated
// level state stays identical without extra broadcasts.
#pragma once

#include "common.cuh"

namespace drtopk {

constexpr int FUSED_THREADS = 256;
constexpr int MAX_BLOCK_WARPS = 16;  // CTAs of up to 512 threads (the shared-memory tail uses 512)
constexpr int MAX_LEVELS = 40;

constexpr int SMALL_SET = 4096;  // a set this small is finished by one CTA in shared memory

struct EngineCfg {
  int bucket;          // 0 radix, 1 bucket
  int nbits;           // radix digit width
  int nb;              // bins per level (1<<nbits, or bucket count <= 4096)
  int stop_single;     // stop when the chosen bin holds exactly one key
  int max_levels;      // stop after this many levels
  int thr_only;        // only the final range is wanted (histogram passes, no appends)
  int key_from_payload;  // key = ~payload (fill by lowest payload)
  int skip_split0;     // level 0's split (top list, next set, level-1 histogram) was made by another kernel
  uint32_t adapt_cnt;  // thr_only: after max_levels, keep refining while the chosen bin holds more
                       // than adapt_cnt entries (0: stop at max_levels)
};

struct RunBufs {
  uint32_t* H[3];       // rotating histograms (nb words each)
  uint32_t* set_count;  // [MAX_LEVELS+2]: size of the set entering level j
  uint2* cbuf[2];       // compact ping-pong buffers
  uint2* top;           // top list (capacity k)
  uint32_t* top_count;
  uint32_t* res;        // [4] result of a run finished inside one CTA: thr, kth, levels, ok
  uint64_t top_cap;     // entries the top list holds
  uint64_t cbuf_cap;    // entries each compact buffer holds
  uint32_t* err;        // error word: DE_OVERFLOW when an append would pass a capacity
  // caller's output (value bits / index, either may be null): a split made
  // with DIRECT output writes its top entries there instead of rb.top
  int out_km;
  uint32_t* out_vals;
  int64_t* out_idx;
};

struct Level {
  uint32_t lo, hi;  // range of the set entering this level (inclusive)
  uint32_t w;       // bucket width at this level
  int wshift;       // log2(w) in radix mode, -1 in bucket mode
  uint32_t R;       // remaining rank within the range
};

// Source set of a run: either a key array with implicit payload (index) or
// an array of (key, payload) pairs.
struct Src {
  const uint32_t* keys;   // form 1
  const uint2* pairs;     // form 2
  uint64_t count;         // form 1 count (host-known)
  const uint32_t* count_dev;  // form 2 count (device)
  int raw_input;          // form 1 keys are the raw input (apply key transform)
};

struct RunResult {
  uint32_t thr;     // final range lower bound
  uint32_t thr_hi;  // ... and upper bound (thr_only runs)
  uint32_t kth;     // exact k-th key when the run finished (collapse/single)
  int levels;
  int ok;
};

DRTOPK_DEV uint32_t bin_of(uint32_t k, uint32_t lo, uint32_t w, int wshift) {
  const uint32_t d = k - lo;
  if (wshift >= 0) return d >> wshift;  // radix levels (and width-1 bins below them)
  if (w == 1u) return d;
  return d / w;                         // bucket levels
}

// --------------------------------------------------------------- block pick
struct Pick {
  uint32_t b, cnt, above;
};

// Every CTA: find the largest bin b with (count of bins >= b) >= R.
// H in global memory (written by other CTAs) or, with SMEM, shared memory.
template <bool SMEM = false>
DRTOPK_DEV Pick block_pick(const uint32_t* H, int nb, uint32_t R) {
  __shared__ uint32_t s_part[32];
  __shared__ Pick s_pick;
  __shared__ int s_found;
  const int t = threadIdx.x;
  const int nthr = blockDim.x;
  const int q = (nb + nthr - 1) / nthr;
  const int b0 = min(nb, t * q), b1 = min(nb, b0 + q);
  auto hb = [&](int b) { return SMEM ? H[b] : ld_cg_u32(H + b); };
  uint32_t local = 0;
  for (int b = b0; b < b1; ++b) local += hb(b);
  // inclusive prefix over threads (ascending), then above_t = total - incl
  uint32_t incl = local;
  const unsigned lane = t & 31u;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
    if ((int)lane >= off) incl += y;
  }
  if (lane == 31) s_part[t >> 5] = incl;
  if (t == 0) s_found = 0;
  __syncthreads();
  uint32_t wbase = 0, total = 0;
  for (int w = 0; w < nthr / 32; ++w) {
    if (w < (t >> 5)) wbase += s_part[w];
    total += s_part[w];
  }
  incl += wbase;
  const uint32_t above_t = total - incl;
  if (local > 0 && above_t < R && R <= above_t + local) {
    uint32_t acc = above_t;
    for (int b = b1 - 1; b >= b0; --b) {
      uint32_t c = hb(b);
      if (acc + c >= R) {
        s_pick.b = b; s_pick.cnt = c; s_pick.above = acc;
        s_found = 1;
        break;
      }
      acc += c;
    }
  }
  __syncthreads();
  Pick p;
  if (s_found) p = s_pick;
  else {  // R exceeds the set: the reference's rule then picks bin 0
    uint32_t h0 = hb(0);
    p.b = 0; p.cnt = h0; p.above = total - h0;
  }
  __syncthreads();
  return p;
}

// next level state after picking bin p from level L; returns done flag
DRTOPK_DEV bool advance(const EngineCfg& c, const Level& L, const Pick& p, int level_index, Level& N) {
  uint64_t lo2 = (uint64_t)L.lo + (uint64_t)p.b * (uint64_t)L.w;
  uint64_t hi2 = min((uint64_t)L.hi, lo2 + (uint64_t)L.w - 1);
  N.lo = (uint32_t)lo2;
  N.hi = (uint32_t)hi2;
  N.R = L.R - p.above;
  if (c.bucket) {
    N.wshift = -1;
    N.w = (uint32_t)((uint64_t)(N.hi - N.lo) / (uint64_t)c.nb + 1);
  } else {
    N.wshift = L.wshift - c.nbits;
    N.w = N.wshift >= 0 ? (1u << N.wshift) : 1u;
  }
  bool done = (N.lo == N.hi) || (c.stop_single && p.cnt == 1) ||
              (level_index + 1 >= c.max_levels && !(c.adapt_cnt && p.cnt > c.adapt_cnt));
  return done;
}

// --------------------------------------------------------------- helpers
// Team-strided loop over [0, n) with U loads per thread in flight: ld(i) for
// every index of a round, then use(i, value).  Consecutive threads take
// consecutive indices within each of the U slices (coalesced).
template <int U, typename LD, typename USE>
DRTOPK_DEV void team_load_loop(const Team& tm, uint64_t n, LD&& ld, USE&& use) {
  using V = decltype(ld(uint64_t(0)));
  const uint64_t G = (uint64_t)tm.size * blockDim.x;
  for (uint64_t b = (uint64_t)tm.rank * blockDim.x + threadIdx.x; b < n; b += G * U) {
    V v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint64_t i = b + (uint64_t)u * G;
      if (i < n) v[u] = ld(i);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint64_t i = b + (uint64_t)u * G;
      if (i < n) use(i, v[u]);
    }
  }
}

DRTOPK_DEV void zero_words(const Team& tm, uint32_t* p, int n) {
  const uint64_t g = (uint64_t)tm.rank * blockDim.x + threadIdx.x;
  const uint64_t G = (uint64_t)tm.size * blockDim.x;
  for (uint64_t i = g; i < (uint64_t)n; i += G) p[i] = 0;
}

DRTOPK_DEV void flush_hist(uint32_t* s_hist, uint32_t* gH, int nb) {
  __syncthreads();
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    uint32_t v = s_hist[i];
    if (v) atomicAdd(gH + i, v);
  }
  __syncthreads();
}

DRTOPK_DEV void clear_hist(uint32_t* s_hist, int nb) {
  for (int i = threadIdx.x; i < nb; i += blockDim.x) s_hist[i] = 0;
  __syncthreads();
}

template <int KM>
DRTOPK_DEV uint32_t src_key1(const Src& s, uint64_t i) {
  uint32_t v = ld_cg_u32(s.keys + i);
  return s.raw_input ? to_key<KM>(v) : v;
}

// entry visitor over the source set, for histogram passes (no appends inside
// fn).  fn(key, payload, valid) may be called by a subset of a warp's lanes:
// warp-collective work inside it must use __activemask().  A 16-byte
// aligned source is read as 16-byte words (4 keys or 2 pairs), FOR_EACH_V
// per thread in flight; the < 4-entry remainder is visited by the team's
// first CTA.  Otherwise tiles of blockDim*16 entries with one 4- or 8-byte
// load each.
constexpr int FOR_EACH_V = 4;

template <int KM, typename F>
DRTOPK_DEV void for_each_src(const Team& tm, const Src& s, bool from_pairs, uint64_t count, F&& fn) {
  const uint32_t* base = from_pairs ? reinterpret_cast<const uint32_t*>(s.pairs) : s.keys;
  if ((reinterpret_cast<uintptr_t>(base) & 15u) == 0) {
    const int per = from_pairs ? 2 : 4;  // entries per 16-byte word
    const uint64_t nw = count / (uint64_t)per;
    const uint64_t T = (uint64_t)blockDim.x * FOR_EACH_V;
    for (uint64_t tb = (uint64_t)tm.rank * T; tb < nw; tb += (uint64_t)tm.size * T) {
      uint4 w[FOR_EACH_V];
#pragma unroll
      for (int v = 0; v < FOR_EACH_V; ++v) {
        const uint64_t q = tb + (uint64_t)v * blockDim.x + threadIdx.x;
        w[v] = q < nw ? ld_cg_v4(base + 4 * q) : make_uint4(0u, 0u, 0u, 0u);
      }
#pragma unroll
      for (int v = 0; v < FOR_EACH_V; ++v) {
        const uint64_t q = tb + (uint64_t)v * blockDim.x + threadIdx.x;
        const bool valid = q < nw;
        if (from_pairs) {
          fn(w[v].x, w[v].y, valid);
          fn(w[v].z, w[v].w, valid);
        } else {
          const uint32_t i0 = (uint32_t)(4 * q);
          const bool raw = s.raw_input;
          fn(raw ? to_key<KM>(w[v].x) : w[v].x, i0, valid);
          fn(raw ? to_key<KM>(w[v].y) : w[v].y, i0 + 1, valid);
          fn(raw ? to_key<KM>(w[v].z) : w[v].z, i0 + 2, valid);
          fn(raw ? to_key<KM>(w[v].w) : w[v].w, i0 + 3, valid);
        }
      }
    }
    const uint64_t i = nw * (uint64_t)per + threadIdx.x;
    if (tm.rank == 0 && i < count) {
      if (from_pairs) {
        const uint2 x = ld_cg_v2(reinterpret_cast<const uint32_t*>(s.pairs + i));
        fn(x.x, x.y, true);
      } else {
        fn(src_key1<KM>(s, i), (uint32_t)i, true);
      }
    }
    return;
  }
  constexpr int E = 16;
  const uint64_t T = (uint64_t)blockDim.x * E;
  for (uint64_t tb = (uint64_t)tm.rank * T; tb < count; tb += (uint64_t)tm.size * T) {
    uint32_t key[E], pay[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const uint64_t i = tb + (uint64_t)e * blockDim.x + threadIdx.x;
      key[e] = 0;
      pay[e] = (uint32_t)i;
      if (i < count) {
        if (from_pairs) {
          uint2 x = ld_cg_v2(reinterpret_cast<const uint32_t*>(s.pairs + i));
          key[e] = x.x;
          pay[e] = x.y;
        } else {
          key[e] = src_key1<KM>(s, i);
        }
      }
    }
#pragma unroll
    for (int e = 0; e < E; ++e) fn(key[e], pay[e], tb + (uint64_t)e * blockDim.x + threadIdx.x < count);
  }
}

// --------------------------------------------------------------- split
constexpr int SPLIT_E = 16;  // entries per thread per tile

// One level's split of a set: keys above N's range -> top list, keys inside
// -> next set (+ histogram of the next level).  Tiles of blockDim*SPLIT_E
// entries, coalesced loads, one block-aggregated append per tile.  Slots are
// numbered warp by warp and entry by entry (ballot ranks), so the lanes of a
// warp write consecutive slots: the appends leave as coalesced stores.
template <int KM, bool DIRECT = false, int SPLIT_E = drtopk::SPLIT_E>
DRTOPK_DEV void split_tiles(const Team& tm, const EngineCfg& c, const Src& s, bool pairs, uint64_t count,
                            const Level& N, bool want_hist, const RunBufs& ob, uint32_t* top_count, uint2* nxt,
                            uint32_t* nxt_count, uint32_t* s_hist, uint64_t top_cap, uint64_t nxt_cap,
                            uint32_t* err) {
  const uint64_t T = (uint64_t)blockDim.x * SPLIT_E;
  bool ovf = false;
  const uint32_t span = N.hi - N.lo;
  for (uint64_t tb = (uint64_t)tm.rank * T; tb < count; tb += (uint64_t)tm.size * T) {
    // entry offsets inside the tile are 32-bit; entries >= rem are padding
    const uint64_t rem = count - tb;
    const uint2* tp = s.pairs + tb;
    uint32_t val[SPLIT_E], pay[SPLIT_E];
    uint32_t up = 0, in = 0, ca = 0, cb = 0;
#pragma unroll
    for (int e = 0; e < SPLIT_E; ++e) {
      const uint32_t o = (uint32_t)e * blockDim.x + threadIdx.x;
      val[e] = 0; pay[e] = 0;
      if (o < rem) {
        if (pairs) {
          uint2 x = ld_cg_v2(reinterpret_cast<const uint32_t*>(tp + o));
          val[e] = x.x; pay[e] = x.y;
        } else {
          val[e] = src_key1<KM>(s, tb + o);
          pay[e] = (uint32_t)(tb + o);
        }
      }
    }
#pragma unroll
    for (int e = 0; e < SPLIT_E; ++e) {
      const uint32_t key = c.key_from_payload ? ~pay[e] : val[e];
      const bool valid = (uint32_t)e * blockDim.x + threadIdx.x < rem;
      const bool u = valid && key > N.hi;
      const bool w = valid && key - N.lo <= span;
      up |= (uint32_t)u << e;
      in |= (uint32_t)w << e;
      ca += u;
      cb += w;
    }
    // warp totals go in through lane 0; every lane then starts from the
    // warp's base
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t wa = __reduce_add_sync(0xffffffffu, ca), wb = __reduce_add_sync(0xffffffffu, cb);
    Slots2 sl = block_append2(lane == 0 ? wa : 0u, lane == 0 ? wb : 0u, top_count, nxt_count);
    sl.a = __shfl_sync(0xffffffffu, sl.a, 0);
    sl.b = __shfl_sync(0xffffffffu, sl.b, 0);
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int e = 0; e < SPLIT_E; ++e) {
      // the histogram bounds both counts; a capacity check still guards
      // every address computed from device data
      const bool ue = (up >> e) & 1u, ie = (in >> e) & 1u;
      const unsigned mu = __ballot_sync(0xffffffffu, ue), mi = __ballot_sync(0xffffffffu, ie);
      if (ue) {
        const uint32_t slot = sl.a + __popc(mu & lt);
        if (slot < top_cap) {
          if (DIRECT) {
            if (ob.out_vals) ob.out_vals[slot] = from_key(val[e], ob.out_km);
            if (ob.out_idx) ob.out_idx[slot] = (int64_t)pay[e];
          } else {
            ob.top[slot] = make_uint2(val[e], pay[e]);
          }
        }
        else ovf = true;
      }
      if (ie) {
        const uint32_t slot = sl.b + __popc(mi & lt);
        if (slot < nxt_cap) nxt[slot] = make_uint2(val[e], pay[e]);
        else ovf = true;
        const uint32_t key = c.key_from_payload ? ~pay[e] : val[e];
        if (want_hist) hist_add_warp(s_hist, bin_of(key, N.lo, N.w, N.wshift));
      }
      sl.a += __popc(mu);
      sl.b += __popc(mi);
    }
  }
  if (ovf && err) atomicOr(err, (uint32_t)DE_OVERFLOW);
}

// --------------------------------------------------------------- one run
// Runs levels until done.  H[0] of the run must hold the histogram of level
// 0 over the source (with range L0) and H[1] must be zero when called.
// Barrier after every level.  Appends the keys above the final range to
// rb.top; leaves the final range's members in a compact buffer.
// Returns the level index that finished and the final Level through Lout.
template <int KM>
DRTOPK_DEV int run_levels(const EngineCfg& c, const Src& src0, bool src0_pairs, const RunBufs& rb, Level L,
                          uint32_t* s_hist, const Team& tm, Level& Lout, Pick& last_pick, int& eq_buf,
                          uint64_t& eq_count, bool& ok, bool small_exit = false, bool* went_small = nullptr) {
  int j = 0;
  ok = true;
  if (went_small) *went_small = false;
  for (;; ++j) {
    if (j >= MAX_LEVELS) { ok = false; break; }
    Pick p = block_pick<false>(rb.H[j % 3], c.nb, L.R);
    Level N;
    bool done = advance(c, L, p, j, N);
    last_pick = p;
    zero_words(tm, rb.H[(j + 2) % 3], c.nb);
    uint32_t* Hn = rb.H[(j + 1) % 3];
    const bool want_hist = !done;
    clear_hist(s_hist, c.nb);
    if (c.thr_only) {
      if (done) { Lout = N; break; }
      // histogram the members of the new range over the level-0 source
      const uint64_t cnt = src0_pairs ? (uint64_t)ld_cg_u32(src0.count_dev) : src0.count;
      for_each_src<KM>(tm, src0, src0_pairs, cnt, [&](uint32_t key, uint32_t, bool valid) {
        if (valid && key >= N.lo && key <= N.hi) hist_add_warp(s_hist, bin_of(key, N.lo, N.w, N.wshift));
      });
      flush_hist(s_hist, Hn, c.nb);
      if (!team_sync(tm)) { ok = false; break; }
      L = N;
      continue;
    }
    // split
    const bool from_pairs = (j == 0) ? src0_pairs : true;
    Src s = src0;
    uint64_t cnt;
    if (j == 0) {
      cnt = src0_pairs ? (uint64_t)ld_cg_u32(src0.count_dev) : src0.count;
    } else {
      s.pairs = rb.cbuf[(j - 1) & 1];
      cnt = ld_cg_u32(rb.set_count + j);
    }
    if (!(c.skip_split0 && j == 0)) {
      split_tiles<KM>(tm, c, s, from_pairs, cnt, N, want_hist, rb, rb.top_count, rb.cbuf[j & 1],
                      rb.set_count + j + 1, s_hist, rb.top_cap, rb.cbuf_cap, rb.err);
      if (want_hist) flush_hist(s_hist, Hn, c.nb);
    }
    if (!team_sync(tm)) { ok = false; break; }
    L = N;
    if (done) {
      Lout = N;
      eq_buf = j & 1;
      eq_count = ld_cg_u32(rb.set_count + j + 1);
      break;
    }
    if (small_exit && ld_cg_u32(rb.set_count + j + 1) <= (uint32_t)SMALL_SET) {
      // the next set fits one CTA's shared memory: finish there
      Lout = N;
      eq_buf = j & 1;
      eq_count = ld_cg_u32(rb.set_count + j + 1);
      *went_small = true;
      break;
    }
  }
  return j;
}

// ascending bitonic sort of npow2 64-bit values in shared memory (one CTA)
DRTOPK_DEV void block_bitonic_asc(uint64_t* s, int npow2) {
  for (int size = 2; size <= npow2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      __syncthreads();
      for (int i = threadIdx.x; i < npow2 / 2; i += blockDim.x) {
        const int lo = 2 * stride * (i / stride) + (i % stride), hi = lo + stride;
        const bool asc = ((lo & size) == 0);
        const uint64_t x = s[lo], y = s[hi];
        if ((x > y) == asc) { s[lo] = y; s[hi] = x; }
      }
    }
  }
  __syncthreads();
}

// histogram of the bins of sA[0..n) in shared memory (one CTA), four
// independent entries per thread per round
DRTOPK_DEV void smem_hist(const uint2* sA, uint32_t n, const Level& L, uint32_t* s_hist) {
  for (uint32_t i0 = threadIdx.x; i0 < n; i0 += 4 * blockDim.x) {
    uint32_t b[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t i = i0 + u * blockDim.x;
      b[u] = i < n ? bin_of(sA[i].x, L.lo, L.w, L.wshift) : 0xffffffffu;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (b[u] != 0xffffffffu) hist_add_warp(s_hist, b[u]);
  }
}

// The pick rule of block_pick, by one warp scanning a shared-memory
// histogram (nb <= 4096): lane l owns bins [l*per, (l+1)*per); one block
// barrier publishes the result.
DRTOPK_DEV Pick warp_pick_smem(const uint32_t* H, int nb, uint32_t R) {
  __shared__ Pick s_wpick;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    const int per = (nb + 31) / 32;
    const int b0 = min(nb, lane * per), b1 = min(nb, b0 + per);
    uint32_t local = 0;
    for (int b = b0; b < b1; ++b) local += H[b];
    // suffix sum over lanes: bins at and above this lane's
    uint32_t suf = local;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_down_sync(0xffffffffu, suf, off);
      if (lane + off < 32) suf += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, suf, 0);
    const uint32_t above = suf - local;
    const bool mine = local > 0 && above < R && R <= above + local;
    if (mine) {
      uint32_t acc = above;
      for (int b = b1 - 1; b >= b0; --b) {
        const uint32_t c = H[b];
        if (acc + c >= R) {
          s_wpick.b = b;
          s_wpick.cnt = c;
          s_wpick.above = acc;
          break;
        }
        acc += c;
      }
    }
    if (__ballot_sync(0xffffffffu, mine) == 0u && lane == 0) {
      // R exceeds the set: the reference's rule then picks bin 0
      s_wpick.b = 0;
      s_wpick.cnt = H[0];
      s_wpick.above = total - H[0];
    }
  }
  __syncthreads();
  const Pick p = s_wpick;
  return p;
}

// min and max key of sA[0..n) (one CTA); ends with a block barrier
DRTOPK_DEV void block_minmax(const uint2* sA, uint32_t n, uint32_t& mn, uint32_t& mx) {
  __shared__ uint32_t s_mn[32], s_mx[32];
  uint32_t a = 0xffffffffu, b = 0u;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const uint32_t k = sA[i].x;
    a = min(a, k);
    b = max(b, k);
  }
  a = __reduce_min_sync(0xffffffffu, a);
  b = __reduce_max_sync(0xffffffffu, b);
  if ((threadIdx.x & 31u) == 0) {
    s_mn[threadIdx.x >> 5] = a;
    s_mx[threadIdx.x >> 5] = b;
  }
  __syncthreads();
  mn = 0xffffffffu;
  mx = 0u;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
    mn = min(mn, s_mn[w]);
    mx = max(mx, s_mx[w]);
  }
  __syncthreads();  // s_mn / s_mx may be rewritten by the next call
}

// Pick of one level over sA[0..n) in shared memory (one CTA): when the
// whole set lies in one bin (common for delegates, which crowd into the top
// bins) its min and max show it without a histogram; else histogram + pick.
DRTOPK_DEV Pick smem_level_pick(const uint2* sA, uint32_t n, const Level& L, int nb, uint32_t* s_hist) {
  uint32_t mn, mx;
  block_minmax(sA, n, mn, mx);
  if (n > 0 && L.R <= n && mn >= L.lo && mx <= L.hi &&
      bin_of(mn, L.lo, L.w, L.wshift) == bin_of(mx, L.lo, L.w, L.wshift)) {
    Pick p;
    p.b = bin_of(mn, L.lo, L.w, L.wshift);
    p.cnt = n;
    p.above = 0;
    return p;
  }
  clear_hist(s_hist, nb);
  smem_hist(sA, n, L, s_hist);
  __syncthreads();
  return warp_pick_smem(s_hist, nb, L.R);
}

// Stable two-way split of src[0..n) by one CTA: entries with key > hi (when
// want_a) are appended to outA at *cntA, entries with lo <= key <= hi to
// outB at *cntB (counters in shared or global memory, advanced by one atomic
// each).  Every warp owns a contiguous segment of the input and writes
// contiguous runs ranked by ballots: no shared-memory bank conflicts, index
// order kept.  Ends with a block barrier.
DRTOPK_DEV void split_block(const uint2* src, uint32_t n, uint32_t lo, uint32_t hi, bool want_a, uint2* outA,
                            uint32_t* cntA, uint2* outB, uint32_t* cntB, uint64_t capA = ~0ull,
                            uint32_t* err = nullptr) {
  __shared__ uint32_t s_wa[32], s_wb[32], s_base[2];
  const unsigned lane = threadIdx.x & 31u;
  const int w = threadIdx.x >> 5, W = blockDim.x >> 5;
  const uint32_t per = (((n + W - 1) / W) + 31u) & ~31u;
  const uint32_t b0 = min(n, (uint32_t)w * per), b1 = min(n, b0 + per);
  uint32_t ca = 0, cb = 0;
  for (uint32_t c = b0; c < b1; c += 32) {
    const uint32_t i = c + lane;
    const bool v = i < b1;
    const uint32_t key = v ? src[i].x : 0u;
    ca += __popc(__ballot_sync(0xffffffffu, v && want_a && key > hi));
    cb += __popc(__ballot_sync(0xffffffffu, v && key >= lo && key <= hi));
  }
  if (lane == 0) {
    s_wa[w] = ca;
    s_wb[w] = cb;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t ta = 0, tb = 0;
    for (int q = 0; q < W; ++q) {
      const uint32_t xa = s_wa[q], xb = s_wb[q];
      s_wa[q] = ta;
      s_wb[q] = tb;
      ta += xa;
      tb += xb;
    }
    s_base[0] = ta ? atomicAdd(cntA, ta) : 0u;
    s_base[1] = tb ? atomicAdd(cntB, tb) : 0u;
  }
  __syncthreads();
  uint32_t pa = s_base[0] + s_wa[w], pb = s_base[1] + s_wb[w];
  const unsigned lt = (1u << lane) - 1u;
  for (uint32_t c = b0; c < b1; c += 32) {
    const uint32_t i = c + lane;
    const bool v = i < b1;
    const uint2 e = v ? src[i] : make_uint2(0u, 0u);
    const bool ia = v && want_a && e.x > hi;
    const bool ib = v && e.x >= lo && e.x <= hi;
    const unsigned ma = __ballot_sync(0xffffffffu, ia), mb = __ballot_sync(0xffffffffu, ib);
    if (ia) {
      const uint32_t slot = pa + __popc(ma & lt);
      if (slot < capA) outA[slot] = e;
      else if (err) atomicOr(err, (uint32_t)DE_OVERFLOW);
    }
    if (ib) outB[pb + __popc(mb & lt)] = e;
    pa += __popc(ma);
    pb += __popc(mb);
  }
  __syncthreads();
}

// Completion of a run inside ONE CTA once its remaining set (cnt <=
// SMALL_SET entries) fits in shared memory: the same levels (pick /
// advance / split), then the tie fill by lowest payload, with block
// barriers only.  Results go to rb.top (global, after the entries already
// there) and rb.res.  Called by all threads of one CTA.
template <int KM>
DRTOPK_DEV void block_finish(const EngineCfg& c, const Src& src, bool pairs, uint32_t cnt, Level L, int j,
                             const RunBufs& rb, uint32_t* s_hist, uint2* sA, uint2* sB) {
  __shared__ uint32_t s_n;
  if (pairs)
    block_load_loop<8>(cnt, [&](uint32_t i) { return ld_cg_v2(reinterpret_cast<const uint32_t*>(src.pairs + i)); },
                       [&](uint32_t i, uint2 v) { sA[i] = v; });
  else
    block_load_loop<8>(cnt, [&](uint32_t i) { return src_key1<KM>(src, i); },
                       [&](uint32_t i, uint32_t v) { sA[i] = make_uint2(v, i); });
  __syncthreads();
  uint32_t n = cnt;
  bool ok = true;
  for (;;) {
    if (j >= MAX_LEVELS) { ok = false; break; }
    const Pick p = smem_level_pick(sA, n, L, c.nb, s_hist);
    Level N;
    const bool done = advance(c, L, p, j, N);
    if (p.cnt != n) {  // else the whole set is in the chosen bin: nothing moves
      if (threadIdx.x == 0) s_n = 0;
      __syncthreads();
      split_block(sA, n, N.lo, N.hi, true, rb.top, rb.top_count, sB, &s_n, rb.top_cap, rb.err);
      n = s_n;
      uint2* t = sA; sA = sB; sB = t;
    }
    L = N;
    ++j;
    if (done) break;
  }
  const uint32_t R = L.R;
  const uint32_t kth = (n == 1) ? sA[0].x : L.lo;
  __shared__ uint32_t s_tb;
  if (ok && n == R) {
    if (threadIdx.x == 0) s_tb = atomicAdd(rb.top_count, n);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
      if ((uint64_t)s_tb + i < rb.top_cap) rb.top[s_tb + i] = sA[i];
      else if (rb.err) atomicOr(rb.err, (uint32_t)DE_OVERFLOW);
    }
  } else if (ok && n > R) {
    // keep the R lowest payloads among the tied entries
    uint64_t* w = reinterpret_cast<uint64_t*>(sB);
    int np2 = 1;
    while (np2 < (int)n) np2 <<= 1;
    for (int i = threadIdx.x; i < np2; i += blockDim.x)
      w[i] = i < (int)n ? (((uint64_t)sA[i].y << 32) | sA[i].x) : ~0ull;
    block_bitonic_asc(w, np2);
    if (threadIdx.x == 0) s_tb = atomicAdd(rb.top_count, R);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < R; i += blockDim.x) {
      if ((uint64_t)s_tb + i < rb.top_cap) rb.top[s_tb + i] = make_uint2((uint32_t)w[i], (uint32_t)(w[i] >> 32));
      else if (rb.err) atomicOr(rb.err, (uint32_t)DE_OVERFLOW);
    }
  } else {
    ok = false;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    rb.res[0] = L.lo;
    rb.res[1] = kth;
    rb.res[2] = (uint32_t)j;
    rb.res[3] = ok ? 1u : 0u;
  }
}

// histogram pass of level 0 for a run: hist of bin_of(key, L0) over the source
template <int KM>
DRTOPK_DEV void hist_pass(const Team& tm, const Src& src, bool pairs, bool key_from_payload, const Level& L0, int nb,
                          uint32_t* gH, uint32_t* s_hist) {
  clear_hist(s_hist, nb);
  const uint64_t cnt = pairs ? (uint64_t)ld_cg_u32(src.count_dev) : src.count;
  for_each_src<KM>(tm, src, pairs, cnt, [&](uint32_t val, uint32_t pay, bool valid) {
    const uint32_t key = key_from_payload ? ~pay : val;
    if (valid && key >= L0.lo && key <= L0.hi) hist_add_warp(s_hist, bin_of(key, L0.lo, L0.w, L0.wshift));
  });
  flush_hist(s_hist, gH, nb);
}

DRTOPK_DEV Level radix_level0(int nbits, uint32_t R) {
  Level L;
  L.lo = 0; L.hi = 0xffffffffu; L.wshift = 32 - nbits; L.w = 1u << L.wshift; L.R = R;
  return L;
}

// Level 0 of a second select whose candidates are all >= thr: the range
// [thr, 2^32) in nb = 2^nbits bins of the narrowest power-of-two width that
// covers it (thr = 0 gives radix_level0).  Later levels take nbits off the
// width as usual.  The exact k-th and the top list do not depend on where
// the digit boundaries lie; anchoring them at thr spreads the candidates
// over all bins instead of the few top digits above thr.
DRTOPK_DEV int cand_shift(uint32_t thr, int nbits) {
  const uint32_t top = 0xffffffffu - thr;  // largest key - thr
  const int bits = 32 - __clz(top);
  return max(0, bits - nbits);
}

DRTOPK_DEV Level cand_level0(uint32_t thr, int nbits, uint32_t R) {
  Level L;
  L.lo = thr; L.hi = 0xffffffffu; L.wshift = cand_shift(thr, nbits); L.w = 1u << L.wshift; L.R = R;
  return L;
}

// Level 0 over candidates known to lie in [thr, mx]: the same power-of-two
// radix bins, cut to the candidates' span (keys that crowd just above the
// threshold -- float keys, narrow distributions -- spread over the bins
// instead of landing in the first few)
DRTOPK_DEV Level cand_level0_tight(uint32_t thr, uint32_t mx, int nbits, uint32_t R) {
  Level L;
  const uint32_t top = mx - thr;
  const int bits = 32 - __clz(top);
  L.lo = thr; L.hi = mx; L.wshift = max(0, bits - nbits); L.w = 1u << L.wshift; L.R = R;
  return L;
}

DRTOPK_DEV Level bucket_level0(uint32_t mn, uint32_t mx, int nb, uint32_t R) {
  Level L;
  L.lo = mn; L.hi = mx; L.wshift = -1;
  L.w = (uint32_t)((uint64_t)(mx - mn) / (uint64_t)nb + 1);
  L.R = R;
  return L;
}

// Full select run: levels, then the tie fill (lowest payloads among the
// keys equal to the k-th) so that rb.top ends with exactly R0 entries.
// fb: buffers of the fill sub-run (its own histograms and counts; its
// compact buffers alias rb's).
template <int KM>
DRTOPK_DEV RunResult run_select(const EngineCfg& c, const Src& src0, bool src0_pairs, const RunBufs& rb,
                                const RunBufs& fb, Level L0, uint32_t* s_hist, const Team& tm,
                                uint2* s_fast = nullptr) {
  RunResult res = {0u, 0u, 0u, 0, 1};
  const bool can_small = s_fast && !c.thr_only && !c.key_from_payload;
  auto finish_small = [&](const Src& s, bool pairs, uint32_t cnt, const Level& L, int j0) {
    if (tm.rank == 0) block_finish<KM>(c, s, pairs, cnt, L, j0, rb, s_hist, s_fast, s_fast + SMALL_SET);
    if (!team_sync(tm)) { res.ok = 0; return; }
    res.thr = ld_cg_u32(rb.res);
    res.kth = ld_cg_u32(rb.res + 1);
    res.levels = (int)ld_cg_u32(rb.res + 2);
    res.ok = ld_cg_u32(rb.res + 3) ? 1 : 0;
  };
  if (can_small && !c.skip_split0) {
    const uint64_t n0 = src0_pairs ? (uint64_t)ld_cg_u32(src0.count_dev) : src0.count;
    if (n0 <= (uint64_t)SMALL_SET) {
      finish_small(src0, src0_pairs, (uint32_t)n0, L0, 0);
      return res;
    }
  }
  Level Lf;
  Pick lp;
  int eqb = 0;
  uint64_t E = 0;
  bool ok = true, small = false;
  int j = run_levels<KM>(c, src0, src0_pairs, rb, L0, s_hist, tm, Lf, lp, eqb, E, ok, can_small, &small);
  res.levels = j + 1;
  res.thr = Lf.lo;
  res.thr_hi = Lf.hi;
  if (!ok) { res.ok = 0; return res; }
  if (c.thr_only) return res;
  if (small) {
    Src s = {};
    s.pairs = rb.cbuf[eqb];
    finish_small(s, true, (uint32_t)E, Lf, j + 1);
    return res;
  }
  const uint2* eq = rb.cbuf[eqb];
  res.kth = (E == 1) ? ld_cg_v2(reinterpret_cast<const uint32_t*>(eq)).x : Lf.lo;
  const uint32_t R = Lf.R;
  if (E == R) {
    // every tied entry is kept: they go after the G = k0 - R entries above
    const uint64_t G0 = (uint64_t)ld_cg_u32(rb.top_count);
    const uint64_t g = (uint64_t)tm.rank * blockDim.x + threadIdx.x;
    const uint64_t Gs = (uint64_t)tm.size * blockDim.x;
    (void)g; (void)Gs;
    team_load_loop<8>(tm, E, [&](uint64_t i) { return ld_cg_v2(reinterpret_cast<const uint32_t*>(eq + i)); },
                      [&](uint64_t i, uint2 v) {
                        if (G0 + i < rb.top_cap) rb.top[G0 + i] = v;
                        else if (rb.err) atomicOr(rb.err, (uint32_t)DE_OVERFLOW);
                      });
    if (!team_sync(tm)) { res.ok = 0; return res; }
    if (tm.rank == 0 && threadIdx.x == 0) atomicAdd(rb.top_count, (uint32_t)E);
    if (!team_sync(tm)) res.ok = 0;
    return res;
  }
  if (E < R) { res.ok = 0; return res; }
  // E > R: keep the R lowest payloads among the tied entries (key = ~payload)
  EngineCfg fc = {0, 8, 256, 1, 4, 0, 1};
  Src s = {};
  s.pairs = eq;
  s.count_dev = rb.set_count + j + 1;
  Level F0 = radix_level0(8, R);
  hist_pass<KM>(tm, s, true, true, F0, 256, fb.H[0], s_hist);
  if (!team_sync(tm)) { res.ok = 0; return res; }
  RunBufs fr = fb;
  fr.cbuf[0] = rb.cbuf[eqb ^ 1];
  fr.cbuf[1] = rb.cbuf[eqb];
  fr.top = rb.top;
  fr.top_count = rb.top_count;
  fr.top_cap = rb.top_cap;
  fr.cbuf_cap = rb.cbuf_cap;
  fr.err = rb.err;
  Level Lf2;
  Pick lp2;
  int eqb2 = 0;
  uint64_t E2 = 0;
  bool ok2 = true;
  int j2 = run_levels<KM>(fc, s, true, fr, F0, s_hist, tm, Lf2, lp2, eqb2, E2, ok2);
  (void)j2;
  if (!ok2 || E2 != 1 || Lf2.R != 1) { res.ok = 0; return res; }
  // append the single remaining entry
  if (tm.rank == 0 && threadIdx.x == 0) {
    uint2 e = ld_cg_v2(reinterpret_cast<const uint32_t*>(fr.cbuf[eqb2]));
    uint32_t slot = atomicAdd(rb.top_count, 1u);
    if (slot < rb.top_cap) rb.top[slot] = e;
    else if (rb.err) atomicOr(rb.err, (uint32_t)DE_OVERFLOW);
  }
  if (!team_sync(tm)) res.ok = 0;
  return res;
}

}  // namespace drtopk
