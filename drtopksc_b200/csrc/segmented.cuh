// segmented.cuh -- batched Dr.Top-k: many independent top-k problems of
// uneven length and k in ONE persistent launch driven by a ticket queue.
//
// Tasks, in ticket order:
//   [sampler tasks]  one per 2^chunk_log2-key chunk of every delegate
//                    segment: the chunk's subrange maxima (sampleMax,
//                    reference radixselect.cuh:882-918) or (Max, Second,
//                    position of Max) triples (sampleMax_NoReduction_Beta2,
//                    966-1041) into the segment's delegate slice; the task
//                    then bumps the segment's done counter.
//   [select tasks]   one per segment, one CTA each: waits (bounded) for the
//                    segment's sampler tasks, then runs the whole Dr.Top-k
//                    tail inside the CTA --
//                      first select   exact k-th largest delegate D
//                                     (block radix or bucket select)
//                      keep           beta 1: subranges with delegate > D,
//                                     then the lowest-id ones == D, up to k;
//                                     beta 2: Max > D and Second >= D whole,
//                                     Max > D alone as its Max, and of the
//                                     subranges with Max == D the k lowest-id
//                      concatenate    their keys >= D, in index order
//                      second select  exact k-th key K over the candidates
//                      top list       keys > K, then the lowest-index == K
//                    plain segments skip straight to the last two steps on
//                    the raw keys; bitonic segments (short ones) sort every
//                    key in shared memory.
// Per segment the host autotuner (batch.cu) picks the mode, alpha, beta, the
// digit width (bucket count) and radix or bucket levels of the block
// selects, and the sampler chunk size.
// A select task only waits on sampler tasks with smaller tickets, which were
// taken by CTAs already running, so the queue cannot deadlock; the wait is
// bounded anyway (error flag, segment marked failed).
// Every scan inside a CTA is in index order, so results are deterministic
// and ties go to the lowest index without any sort.
#pragma once

#include "common.cuh"

namespace drtopk {

constexpr int SEG_THREADS = 256;
constexpr int SEG_MAX_K = 4096;      // per-segment k limit of the batched form
constexpr int SEG_SORT_MAX = 4096;   // bitonic segments: every key sorted in shared memory
constexpr int SEG_B2_MAX_K = SEG_MAX_K / 3;  // beta 2: the kept-subrange list holds up to 3k entries

enum SegMode : int { SEG_PLAIN = 0, SEG_DELEGATE = 1, SEG_BITONIC = 2 };
enum SegSelect : int { SEG_RADIX = 0, SEG_BUCKET = 1 };

struct SegDesc {
  uint64_t key_off;   // first key of the segment in the batch key array
  uint64_t del_off;   // delegate slice (beta 1: M words; beta 2: 3M words)
  uint64_t cand_off;  // candidate slice
  uint64_t out_off;   // first output slot
  uint32_t len, k;
  int32_t km, mode, alpha, ntasks;
  int32_t sorted;      // 1: this segment's top-k sorted (value desc, index asc)
  int32_t beta;        // delegates per subrange: 1 (Max) or 2 (Max, Second)
  int32_t nbits;       // digit width of the block selects: 2^nbits bins (4 or 8)
  int32_t sel;         // block selects by radix digits or min/max buckets
  int32_t chunk_log2;  // keys per sampler task: 2^chunk_log2
  int32_t pad_;
  // optional absolute pointers (served form: every request owns its buffers);
  // when kptr is set the segment's keys are kptr[0..len) and its outputs go
  // to okth[0], ovals[0..k), oidx[0..k) instead of the packed batch arrays
  const uint32_t* kptr;
  uint32_t* okth;
  uint32_t* ovals;
  int64_t* oidx;
};

DRTOPK_DEV const uint32_t* seg_keys(const uint32_t* keys, const SegDesc& d) {
  return d.kptr ? d.kptr : keys + d.key_off;
}

struct SegArgs {
  const uint32_t* keys;
  const SegDesc* seg;
  const uint2* tasks;     // sampler tasks: (segment, chunk)
  uint32_t n_sampler_tasks;
  uint32_t nseg;
  uint32_t* del_pool;
  uint2* cand_pool;
  uint32_t* done;         // per segment: sampler tasks finished
  uint32_t* ticket;
  uint32_t* err;
  uint32_t* seg_err;      // per segment: nonzero = failed
  uint32_t* out_kth;
  uint32_t* out_vals;
  int64_t* out_idx;
};

DRTOPK_DEV uint32_t to_key_rt(uint32_t u, int km) {
  if (km == KM_F32 || km == KM_F32_MIN) u = f32_bits_to_key(u);
  if (km == KM_U32_MIN || km == KM_F32_MIN) u = ~u;
  return u;
}

// ------------------------------------------------------------ sampler task
// One warp per subrange (chunks are multiples of S).  beta 1: del[j] = Max;
// beta 2: del[3j..3j+2] = (Max, Second, offset of Max in the subrange), the
// lowest offset among equal Maxes; Second = 0 for a one-key subrange.
template <int BETA>
DRTOPK_DEV void seg_sample_body(const SegArgs& a, const SegDesc& d, uint32_t chunk) {
  const uint32_t* keys = seg_keys(a.keys, d);
  const uint64_t len = d.len;
  const int alpha = d.alpha;
  const uint64_t S = 1ull << alpha;
  const uint64_t CH = 1ull << d.chunk_log2;
  const uint64_t c0 = (uint64_t)chunk * CH, c1 = min(len, c0 + CH);
  uint32_t* del = a.del_pool + d.del_off;
  const bool vec = (reinterpret_cast<uintptr_t>(keys) & 15u) == 0;
  const unsigned lane = threadIdx.x & 31u;
  const int wid = threadIdx.x >> 5, nw = SEG_THREADS / 32;
  for (uint64_t j = (c0 >> alpha) + wid; j < ((c1 + S - 1) >> alpha); j += nw) {
    const uint64_t b = j << alpha, e = min(len, b + S);
    uint32_t m1 = 0, m2 = 0, p1 = 0xffffffffu;
    for (uint64_t p0 = b + lane * 4; p0 < e; p0 += 512) {
      uint4 v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint64_t p = p0 + 128 * u;
        if (vec && p + 4 <= e) v[u] = __ldg(reinterpret_cast<const uint4*>(keys + p));
        else {
          uint32_t t[4];
          for (int q = 0; q < 4; ++q) t[q] = (p + q < e) ? __ldg(keys + p + q) : 0u;
          v[u] = make_uint4(t[0], t[1], t[2], t[3]);
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint64_t p = p0 + 128 * u;
        if (BETA == 1) {
          // keys past the end read as 0, the max identity
          const uint32_t x0 = p < e ? to_key_rt(v[u].x, d.km) : 0u, x1 = p + 1 < e ? to_key_rt(v[u].y, d.km) : 0u;
          const uint32_t x2 = p + 2 < e ? to_key_rt(v[u].z, d.km) : 0u, x3 = p + 3 < e ? to_key_rt(v[u].w, d.km) : 0u;
          m1 = max(m1, max(max(x0, x1), max(x2, x3)));
        } else {
          // branch-free top two: Second takes the smaller of (Max, key);
          // the Max's offset moves only on a strictly larger key (or the
          // lane's first one), so ties keep the lowest offset
          const uint32_t w[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const bool in = p + q < e;
            const uint32_t x = to_key_rt(w[q], d.km);
            const bool up = in && (x > m1 || p1 == 0xffffffffu);
            if (in) m2 = max(m2, p1 == 0xffffffffu ? 0u : min(m1, x));
            p1 = up ? (uint32_t)(p + q - b) : p1;
            m1 = up ? x : m1;
          }
        }
      }
    }
    if (BETA == 2) {
      // merge the lanes' (Max, Second, offset): lanes without keys hold p1 = ~0
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const uint32_t o1 = __shfl_xor_sync(0xffffffffu, m1, off);
        const uint32_t o2 = __shfl_xor_sync(0xffffffffu, m2, off);
        const uint32_t op = __shfl_xor_sync(0xffffffffu, p1, off);
        if (op == 0xffffffffu) continue;
        if (p1 == 0xffffffffu) { m1 = o1; m2 = o2; p1 = op; continue; }
        if (o1 > m1 || (o1 == m1 && op < p1)) { m2 = max(m1, o2); m1 = o1; p1 = op; }
        else m2 = max(m2, o1);
      }
      if (lane == 0) { del[3 * j] = m1; del[3 * j + 1] = m2; del[3 * j + 2] = p1; }
    } else {
      m1 = __reduce_max_sync(0xffffffffu, m1);
      if (lane == 0) del[j] = m1;
    }
  }
}

DRTOPK_DEV void seg_sample_chunk(const SegArgs& a, const SegDesc& d, uint32_t chunk) {
  if (d.beta == 2) seg_sample_body<2>(a, d, chunk);
  else seg_sample_body<1>(a, d, chunk);
}

// ------------------------------------------------------------ block select
// Warp 0 picks the bin of rank R from the top of nb <= 256 bins (s_hist):
// s_bin and s_above (keys in higher bins).
DRTOPK_DEV void block_pick_rank(const uint32_t* s_hist, int nb, uint32_t R, uint32_t* s_bin, uint32_t* s_above) {
  if (threadIdx.x < 32) {
    const unsigned lane = threadIdx.x;
    const int per = nb >= 32 ? nb / 32 : 1;  // bins per lane, from the top
    uint32_t c[8], loc = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int bin = nb - 1 - ((int)lane * per + q);
      c[q] = (q < per && bin >= 0) ? s_hist[bin] : 0u;
      loc += c[q];
    }
    uint32_t incl = loc;
    for (int off = 1; off < 32; off <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
      if ((int)lane >= off) incl += y;
    }
    const uint32_t before = incl - loc;  // keys in bins above this lane's bins
    if (loc && before < R && R <= incl) {
      uint32_t acc = before;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        if (q < per && acc + c[q] >= R) {
          *s_bin = (uint32_t)(nb - 1 - ((int)lane * per + q));
          *s_above = acc;
          break;
        }
        acc += c[q];
      }
    }
  }
}

// Exact k-th largest key over a set given by get(i) -> key for i < n (keys
// that the caller maps); returns K and, through n_above, how many keys are
// > K.  Radix: nbits-wide digits from the top, 32/nbits passes.  Bucket:
// one min/max pass, then 2^nbits integer-width buckets over the remaining
// range [lo, hi] (width (hi - lo) / nb + 1) until one value is left -- the
// reference's bucket select made exact; few passes when the keys span a
// narrow range.  All threads.
template <int SEL, typename G>
DRTOPK_DEV uint32_t block_kth_sel(uint64_t n, uint32_t k, G&& get, uint32_t* s_hist, uint32_t& n_above, int nbits) {
  constexpr int sel = SEL;
  __shared__ uint32_t s_bin, s_above, s_mm[2];
  constexpr int U = 8;  // independent loads in flight per thread
  const int nb = 1 << nbits;
  uint32_t lo = 0, hi = 0xffffffffu, R = k;
  if constexpr (sel == SEG_BUCKET) {
    if (threadIdx.x < 2) s_mm[threadIdx.x] = 0;
    __syncthreads();
    uint32_t mlo = 0, mhi = 0;  // max(~v), max(v)
    for (uint64_t b = 0; b < n; b += (uint64_t)blockDim.x * U) {
      uint32_t v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const uint64_t i = b + (uint64_t)u * blockDim.x + threadIdx.x;
        v[u] = i < n ? get(i) : 0u;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const uint64_t i = b + (uint64_t)u * blockDim.x + threadIdx.x;
        if (i < n) { mlo = max(mlo, ~v[u]); mhi = max(mhi, v[u]); }
      }
    }
    mlo = __reduce_max_sync(0xffffffffu, mlo);
    mhi = __reduce_max_sync(0xffffffffu, mhi);
    if ((threadIdx.x & 31) == 0) { atomicMax(&s_mm[0], mlo); atomicMax(&s_mm[1], mhi); }
    __syncthreads();
    lo = ~s_mm[0];
    hi = s_mm[1];
    __syncthreads();
  }
  for (int d = 32 / nbits - 1;; --d) {
    // this level's bins: radix digit d, or buckets of width w over [lo, hi]
    uint32_t w = 0;
    int sh = 0;
    uint32_t mask_hi = 0;
    if constexpr (sel == SEG_BUCKET) {
      if (lo == hi) break;
      w = (hi - lo) / (uint32_t)nb + 1u;
    } else {
      if (d < 0) break;
      sh = nbits * d;
      mask_hi = (sh + nbits >= 32) ? 0u : (0xffffffffu << (sh + nbits));
    }
    for (int i = threadIdx.x; i < nb; i += blockDim.x) s_hist[i] = 0;
    __syncthreads();
    for (uint64_t b = 0; b < n; b += (uint64_t)blockDim.x * U) {
      uint32_t v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const uint64_t i = b + (uint64_t)u * blockDim.x + threadIdx.x;
        v[u] = i < n ? get(i) : 0u;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const uint64_t i = b + (uint64_t)u * blockDim.x + threadIdx.x;
        if (i >= n) continue;
        if constexpr (sel == SEG_BUCKET) {
          if (v[u] >= lo && v[u] <= hi) hist_add_warp(s_hist, (v[u] - lo) / w);
        } else if ((v[u] & mask_hi) == lo) {
          hist_add_warp(s_hist, (v[u] >> sh) & (uint32_t)(nb - 1));
        }
      }
    }
    __syncthreads();
    block_pick_rank(s_hist, nb, R, &s_bin, &s_above);
    __syncthreads();
    if constexpr (sel == SEG_BUCKET) {
      const uint64_t nlo = (uint64_t)lo + (uint64_t)s_bin * w;
      hi = (uint32_t)min((uint64_t)hi, nlo + w - 1);
      lo = (uint32_t)nlo;
    } else {
      lo |= s_bin << sh;
    }
    R -= s_above;
    __syncthreads();
  }
  n_above = k - R;
  return lo;
}

template <typename G>
DRTOPK_DEV uint32_t block_kth(uint64_t n, uint32_t k, G&& get, uint32_t* s_hist, uint32_t& n_above, int nbits = 8,
                              int sel = SEG_RADIX) {
  return sel == SEG_BUCKET ? block_kth_sel<SEG_BUCKET>(n, k, get, s_hist, n_above, nbits)
                           : block_kth_sel<SEG_RADIX>(n, k, get, s_hist, n_above, nbits);
}

// Ordered selection: walks i = 0..n-1 in order and keeps every i with
// key > K, plus the first `need_eq` with key == K; emit(slot, i) receives
// consecutive slots in index order.  Returns the number kept.
template <typename G, typename E>
DRTOPK_DEV uint32_t block_ordered_take(uint64_t n, uint32_t K, uint32_t need_eq, G&& get, E&& emit) {
  __shared__ uint32_t s_w[2][SEG_THREADS / 32];
  __shared__ uint32_t s_run[2];
  if (threadIdx.x == 0) { s_run[0] = 0; s_run[1] = 0; }
  __syncthreads();
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  constexpr int U = 4;  // loads issued together; ranked one sub-round at a time (index order)
  for (uint64_t base = 0; base < n; base += (uint64_t)blockDim.x * U) {
    uint32_t vv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint64_t i = base + (uint64_t)u * blockDim.x + threadIdx.x;
      vv[u] = i < n ? get(i) : 0u;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint64_t i = base + (uint64_t)u * blockDim.x + threadIdx.x;
      const uint32_t v = vv[u];
      const bool valid = i < n;
      const bool gt = valid && v > K, eq = valid && v == K;
      const unsigned bg = __ballot_sync(0xffffffffu, gt), be = __ballot_sync(0xffffffffu, eq);
      if (lane == 0) { s_w[0][wid] = __popc(bg); s_w[1][wid] = __popc(be); }
      __syncthreads();
      uint32_t pg = 0, pe = 0, tg = 0, te = 0;
      for (int w = 0; w < SEG_THREADS / 32; ++w) {
        if (w < (int)wid) { pg += s_w[0][w]; pe += s_w[1][w]; }
        tg += s_w[0][w];
        te += s_w[1][w];
      }
      const uint32_t lm = (1u << lane) - 1u;
      const uint32_t rg = s_run[0] + pg + __popc(bg & lm);   // rank among > K so far
      const uint32_t re = s_run[1] + pe + __popc(be & lm);   // rank among == K so far
      const bool take_eq = eq && re < need_eq;
      // slots: all > K and the taken == K, interleaved in index order
      const uint32_t eq_before = min(re, need_eq);
      if (gt) emit(rg + eq_before, i);
      if (take_eq) emit(rg + re, i);
      __syncthreads();
      if (threadIdx.x == 0) { s_run[0] += tg; s_run[1] += te; }
      __syncthreads();
    }
  }
  const uint32_t kept = s_run[0] + min(s_run[1], need_eq);
  __syncthreads();
  return kept;
}

// Exclusive prefix sum of v over the block (all threads), with the total.
DRTOPK_DEV uint32_t seg_block_excl_scan(uint32_t v, uint32_t& total) {
  __shared__ uint32_t s_w[SEG_THREADS / 32];
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
    if ((int)lane >= off) x += y;
  }
  if (lane == 31) s_w[wid] = x;
  __syncthreads();
  uint32_t before = 0;
  total = 0;
  for (int w = 0; w < SEG_THREADS / 32; ++w) {
    if (w < (int)wid) before += s_w[w];
    total += s_w[w];
  }
  __syncthreads();
  return before + x - v;
}

// Bitonic sort of np2 (a power of two) 64-bit values in shared memory,
// descending.  All threads.
DRTOPK_DEV void seg_bitonic_desc(uint64_t* c64, int np2) {
  for (int size = 2; size <= np2; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      __syncthreads();
      for (int i = threadIdx.x; i < np2 / 2; i += blockDim.x) {
        const int lo = 2 * stride * (i / stride) + (i % stride), hi = lo + stride;
        const bool desc = ((lo & size) == 0);
        const uint64_t x = c64[lo], y = c64[hi];
        if ((x < y) == desc) { c64[lo] = y; c64[hi] = x; }
      }
    }
  __syncthreads();
}

// Second select over nc candidates (key, index) in index order: the exact
// k-th key K, then the top list (keys > K, then the lowest-index == K) into
// s_top in index order.
DRTOPK_DEV void seg_finish_candidates(const SegDesc& d, const uint2* cand, uint32_t nc, uint32_t* s_hist, uint2* s_top,
                                      uint32_t* o_kth) {
  auto getc = [&](uint64_t i) { return ld_cg_v2(reinterpret_cast<const uint32_t*>(cand + i)).x; };
  uint32_t gtK = 0;
  const uint32_t K = block_kth(nc, d.k, getc, s_hist, gtK, d.nbits, d.sel);
  block_ordered_take(nc, K, d.k - gtK, getc, [&](uint32_t slot, uint64_t i) {
    s_top[slot] = ld_cg_v2(reinterpret_cast<const uint32_t*>(cand + i));
  });
  if (threadIdx.x == 0 && o_kth) *o_kth = from_key(K, d.km);
}

// host helpers (defined with the kernel in batch.cu)
cudaError_t launch_segmented(const SegArgs& a, int grid, size_t smem, cudaStream_t st);
cudaError_t segmented_shape(int device, int* grid, size_t* smem);

#ifdef DRTOPK_DEFINE_SEGMENTED_KERNEL
// ------------------------------------------------------------ kernel
__global__ void __launch_bounds__(SEG_THREADS, 4) k_segmented(SegArgs a) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  uint32_t* s_hist = s_dyn;                                              // 256
  uint2* s_top = reinterpret_cast<uint2*>(s_dyn + 256);                  // SEG_MAX_K
  uint32_t* s_sel = s_dyn + 256 + 2 * SEG_MAX_K;                         // SEG_MAX_K
  __shared__ uint32_t s_ticket;
  __shared__ uint32_t s_cnt;
  const uint32_t total = a.n_sampler_tasks + a.nseg;
  for (;;) {
    if (threadIdx.x == 0) s_ticket = atomicAdd(a.ticket, 1u);
    __syncthreads();
    const uint32_t t = s_ticket;
    __syncthreads();
    if (t >= total) break;
    if (t < a.n_sampler_tasks) {
      const uint2 task = a.tasks[t];
      const SegDesc d = a.seg[task.x];
      seg_sample_chunk(a, d, task.y);
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(a.done + task.x, 1u);
      }
      continue;
    }
    const uint32_t s = t - a.n_sampler_tasks;
    const SegDesc d = a.seg[s];
    const uint32_t* keys = seg_keys(a.keys, d);
    const uint32_t k = d.k;
    uint32_t* o_kth = d.kptr ? d.okth : a.out_kth + s;
    uint32_t* o_vals = d.kptr ? d.ovals : (a.out_vals ? a.out_vals + d.out_off : nullptr);
    int64_t* o_idx = d.kptr ? d.oidx : (a.out_idx ? a.out_idx + d.out_off : nullptr);
    if (d.mode == SEG_DELEGATE) {
      // wait for this segment's sampler tasks (bounded)
      if (threadIdx.x == 0) {
        uint32_t it = 0, ok = 1;
        while (ld_acquire_gpu(a.done + s) < (uint32_t)d.ntasks) {
          if (++it > (1u << 24)) { ok = 0; break; }
          __nanosleep(128);
        }
        if (!ok) { atomicOr(a.err, (uint32_t)DE_BARRIER_TIMEOUT); a.seg_err[s] = 1; }
        s_cnt = ok;
      }
      __syncthreads();
      if (!s_cnt) continue;
    }
    bool plain = d.mode == SEG_PLAIN;
    if (d.mode == SEG_DELEGATE && d.beta == 1) {
      const uint32_t* del = a.del_pool + d.del_off;
      const uint64_t S = 1ull << d.alpha;
      const uint64_t M = ((uint64_t)d.len + S - 1) >> d.alpha;
      auto getd = [&](uint64_t i) { return ld_cg_u32(del + i); };
      uint32_t gtD = 0;
      const uint32_t D = block_kth(M, k, getd, s_hist, gtD, d.nbits, d.sel);
      // keep: delegates > D, then the lowest ids == D, up to k (ascending ids)
      block_ordered_take(M, D, k - gtD, getd, [&](uint32_t slot, uint64_t i) { s_sel[slot] = (uint32_t)i; });
      __syncthreads();
      // concatenate keys >= D of the kept subranges, in index order; only the
      // last kept subrange can be the segment's partial tail, so the virtual
      // span is clipped there
      uint2* cand = a.cand_pool + d.cand_off;
      uint64_t vspan = (uint64_t)k << d.alpha;
      if (s_sel[k - 1] == M - 1) vspan -= (M << d.alpha) - d.len;
      auto getv = [&](uint64_t q) -> uint32_t {
        const uint64_t pos = ((uint64_t)s_sel[q >> d.alpha] << d.alpha) + (q & (S - 1));
        return to_key_rt(__ldg(keys + pos), d.km);
      };
      auto putv = [&](uint32_t slot, uint64_t q) {
        const uint64_t pos = ((uint64_t)s_sel[q >> d.alpha] << d.alpha) + (q & (S - 1));
        cand[slot] = make_uint2(getv(q), (uint32_t)pos);
      };
      // keys >= D: "> D-1", or everything when D == 0
      const uint32_t nc = (D == 0) ? block_ordered_take(vspan, 0u, 0xffffffffu, getv, putv)
                                   : block_ordered_take(vspan, D - 1, 0u, getv, putv);
      __syncthreads();
      seg_finish_candidates(d, cand, nc, s_hist, s_top, o_kth);
    } else if (d.mode == SEG_DELEGATE) {
      // beta 2: delegates (Max, Second, offset of Max) per subrange
      const uint32_t* del = a.del_pool + d.del_off;
      const uint64_t M = ((uint64_t)d.len + (1ull << d.alpha) - 1) >> d.alpha;
      auto getd2 = [&](uint64_t i) { return ld_cg_u32(del + 3 * (i >> 1) + (i & 1)); };
      uint32_t gtD = 0;
      const uint32_t D = block_kth(2 * M, k, getd2, s_hist, gtD, d.nbits, d.sel);
      if (D == 0) {
        plain = true;  // every key qualifies: select over the raw keys
      } else {
        // kept subranges in id order (s_sel; bit 31: only its Max, at the
        // offset the sampler recorded): Max > D and Second >= D whole; Max >
        // D alone as its Max; Max == D -- copies of D, nothing above it --
        // only the k lowest-id ones (the lowest-index copies of D the top k
        // can need lie there or in the whole ones); < 3k entries
        uint32_t* s_off = reinterpret_cast<uint32_t*>(s_top);  // free until the top list is built
        __shared__ uint32_t s_run3[3];
        if (threadIdx.x == 0) { s_run3[0] = 0; s_run3[1] = 0; s_run3[2] = 0; }
        __syncthreads();
        for (uint64_t j0 = 0; j0 < M; j0 += blockDim.x) {
          const uint64_t j = j0 + threadIdx.x;
          uint32_t m1 = 0, m2 = 0;
          if (j < M) { m1 = ld_cg_u32(del + 3 * j); m2 = ld_cg_u32(del + 3 * j + 1); }
          const bool tied = j < M && m1 == D;
          uint32_t ttot = 0;
          const uint32_t trank = s_run3[1] + seg_block_excl_scan(tied ? 1u : 0u, ttot);
          const bool keep = j < M && (m1 > D || (tied && trank < k));
          const bool single = m2 < D;  // only the Max reaches D
          const uint32_t sz =
              !keep ? 0u
                    : (single ? 1u : (uint32_t)(min((uint64_t)d.len, (j + 1) << d.alpha) - (j << d.alpha)));
          uint32_t ktot = 0, otot = 0;
          const uint32_t slot = s_run3[0] + seg_block_excl_scan(keep ? 1u : 0u, ktot);
          const uint32_t off = s_run3[2] + seg_block_excl_scan(sz, otot);
          if (keep) {
            s_sel[slot] = (uint32_t)j | (single ? 0x80000000u : 0u);
            s_off[slot] = off;
          }
          __syncthreads();
          if (threadIdx.x == 0) { s_run3[0] += ktot; s_run3[1] += ttot; s_run3[2] += otot; }
          __syncthreads();
        }
        const uint32_t nent = s_run3[0];
        const uint64_t vspan = s_run3[2];
        __syncthreads();
        // entry of virtual position q: the last entry whose offset is <= q
        auto entry = [&](uint64_t q) -> uint32_t {
          uint32_t lo2 = 0, hi2 = nent;
          while (hi2 - lo2 > 1) {
            const uint32_t mid = (lo2 + hi2) >> 1;
            if (s_off[mid] <= q) lo2 = mid;
            else hi2 = mid;
          }
          return lo2;
        };
        auto posv = [&](uint64_t q, uint32_t& key) -> uint32_t {
          const uint32_t e = entry(q);
          const uint32_t id = s_sel[e] & 0x7fffffffu;
          if (s_sel[e] >> 31) {
            key = ld_cg_u32(del + 3 * (uint64_t)id);
            return (uint32_t)(((uint64_t)id << d.alpha) + ld_cg_u32(del + 3 * (uint64_t)id + 2));
          }
          const uint64_t pos = ((uint64_t)id << d.alpha) + (q - s_off[e]);
          key = to_key_rt(__ldg(keys + pos), d.km);
          return (uint32_t)pos;
        };
        uint2* cand = a.cand_pool + d.cand_off;
        auto getv = [&](uint64_t q) -> uint32_t {
          uint32_t key;
          posv(q, key);
          return key;
        };
        auto putv = [&](uint32_t slot, uint64_t q) {
          uint32_t key;
          const uint32_t pos = posv(q, key);
          cand[slot] = make_uint2(key, pos);
        };
        const uint32_t nc = block_ordered_take(vspan, D - 1, 0u, getv, putv);
        __syncthreads();
        seg_finish_candidates(d, cand, nc, s_hist, s_top, o_kth);
      }
    }
    if (d.mode == SEG_BITONIC) {
      // every key (len <= SEG_SORT_MAX) as (key << 32 | ~index) in shared
      // memory, bitonic-sorted descending: the first k are the top-k in
      // output order
      uint64_t* c64 = reinterpret_cast<uint64_t*>(s_top);
      int np2 = 1;
      while (np2 < (int)d.len) np2 <<= 1;
      for (int i = threadIdx.x; i < np2; i += blockDim.x)
        c64[i] = i < (int)d.len ? (((uint64_t)to_key_rt(__ldg(keys + i), d.km) << 32) | (uint64_t)(~(uint32_t)i))
                                : 0ull;
      seg_bitonic_desc(c64, np2);
      for (int i = threadIdx.x; i < (int)k; i += blockDim.x) {
        const uint64_t v = c64[i];
        if (o_vals) o_vals[i] = from_key((uint32_t)(v >> 32), d.km);
        if (o_idx) o_idx[i] = (int64_t)(uint32_t)~(uint32_t)v;
      }
      if (threadIdx.x == 0 && o_kth) *o_kth = from_key((uint32_t)(c64[k - 1] >> 32), d.km);
      __syncthreads();
      continue;
    }
    if (plain) {
      auto getk = [&](uint64_t i) { return to_key_rt(__ldg(keys + i), d.km); };
      uint32_t gtK = 0;
      const uint32_t K = block_kth(d.len, k, getk, s_hist, gtK, d.nbits, d.sel);
      block_ordered_take(d.len, K, k - gtK, getk,
                         [&](uint32_t slot, uint64_t i) { s_top[slot] = make_uint2(getk(i), (uint32_t)i); });
      if (threadIdx.x == 0 && o_kth) *o_kth = from_key(K, d.km);
    }
    __syncthreads();
    // output (s_top holds the top-k in index order)
    if (d.sorted) {
      // bitonic sort of composites (key << 32 | ~idx), descending, in place
      uint64_t* c64 = reinterpret_cast<uint64_t*>(s_top);
      int np2 = 1;
      while (np2 < (int)k) np2 <<= 1;
      for (int i = threadIdx.x; i < np2; i += blockDim.x) {
        uint64_t v = 0;
        if (i < (int)k) { uint2 e = s_top[i]; v = ((uint64_t)e.x << 32) | (uint64_t)(~e.y); }
        c64[i] = v;
      }
      seg_bitonic_desc(c64, np2);
      for (int i = threadIdx.x; i < (int)k; i += blockDim.x) {
        const uint64_t v = c64[i];
        if (o_vals) o_vals[i] = from_key((uint32_t)(v >> 32), d.km);
        if (o_idx) o_idx[i] = (int64_t)(uint32_t)~(uint32_t)v;
      }
    } else {
      for (int i = threadIdx.x; i < (int)k; i += blockDim.x) {
        const uint2 e = s_top[i];
        if (o_vals) o_vals[i] = from_key(e.x, d.km);
        if (o_idx) o_idx[i] = (int64_t)e.y;
      }
    }
    __syncthreads();
  }
}

#endif  // DRTOPK_DEFINE_SEGMENTED_KERNEL

}  // namespace drtopk
