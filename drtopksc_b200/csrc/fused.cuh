// fused.cuh -- everything after the delegate sampler, in one persistent
// kernel with team barriers between phases (no host round trip; the
// reference makes ~30 synchronous calls here: radixselect.cuh:1782-1894).
// The team is the cooperative grid, one thread-block cluster, or one CTA.
//
//   phase 1  first select on the delegates
//            default path (beta=1): k-th largest delegate with the reference's
//            early stop; the k subranges kept are those above the final range
//            plus the lowest-id ties (FindTopKRanges 412-427 +
//            FillWithKElementsID 602-618, made deterministic).
//            beta path (beta=2): threshold only, from the top digits of the
//            (Max, Second) delegates (radix_select_inplace_firsttopk_beta
//            1727-1780).
//   phase 2  concatenation of candidates >= threshold
//            default: keys of the k kept subranges (CreateConcatenateRange_
//            optimized 1574-1607); beta: FindTopKRanges_beta 560-598 (Max and
//            Second >= thr -> whole subrange; Max only -> that one key) fused
//            with CreateConcatenateRange_Beta_optimized 1609-1639.  Appends
//            are block-aggregated; the same pass histograms the candidates
//            over the first level of phase 3, which spans [threshold, 2^32).
//   phase 3  second select over the candidates (radix_select_inplace
//            1410-1470): exact k-th largest, plus the top-k list with ties
//            broken by lowest index.
//   phase 4  output: k-th value, top-k values/indices (optionally sorted by
//            value desc, index asc).
#pragma once

#include "engine.cuh"

namespace drtopk {

enum Path : int { PATH_DEFAULT = 0, PATH_BETA = 1, PATH_PLAIN = 2, PATH_BITONIC = 3, PATH_EMIT = 4 };

constexpr int SMALL_SORT = 4096;  // top-k sorted in one CTA's shared memory up to this k
constexpr int TIE_RUN_MAX = 32;   // large-k sort: longest run of equal keys put in index order by one thread
constexpr int SORT_U = 4;         // large-k sort: keys per thread per scatter round
constexpr int SORT_LONG_WORD = 8 * 256;  // sort_tot word after the digit totals: a longer run was found

struct FusedArgs {
  const uint32_t* keys;
  uint64_t n;
  uint32_t k;
  int km;
  int path;
  int bucket;
  int nbits;
  int nb;
  int alpha;
  uint64_t M;
  int first_levels;  // level cap of the first select (beta path threshold levels)
  int vec_ok;
  const uint32_t* del;
  const uint16_t* pos;
  int has_pos;
  const uint32_t* del_minmax;  // [2] from the sampler (bucket mode)
  RunBufs A, AF, C, CF;
  uint32_t* sel;          // beta path: selected subrange ids [M]
  uint32_t* sel_count;
  uint2* cand;
  uint32_t* cand_count;
  uint64_t cand_cap;
  uint32_t* cand_minmax;  // [2] (bucket mode)
  uint32_t* out_kth;      // [1] original value bits
  uint32_t* out_vals;     // [k] or null
  int64_t* out_idx;       // [k] or null
  int sorted;
  uint64_t* sort_buf[2];  // [k] each (large sorted output)
  uint32_t* sort_cnt;     // [grid][256]
  uint32_t* sort_tot;     // [8][256] digit totals, then the long-run flag
  uint32_t* stats;        // [16]
  uint32_t* thr_word;     // threshold handed between launches in split mode
  uint32_t* tail_flag;    // shared-memory tail: 1 done, 2 fall back to the general path
  uint32_t* tie_cut;      // beta path: id bound of the subranges tied at a one-value threshold kept
  int phase_lo, phase_hi; // phases run by this launch of k_fused (1..3)
  int first_pre;          // split mode: the first select runs in k_level_hist / k_filter
  int split0;             // split mode: level 0 of the second select runs in k_split0
  int direct0;            // ... writing its top entries straight to the (unsorted) output
  uint32_t* pre_hist;     // [4][256] sampled-threshold path: byte-level counts of the key sample
  uint32_t pre_target;    // sampled keys that must lie at or above the predicted threshold
  uint32_t pre_stride;    // one 512-key chunk in pre_stride is sampled (a power of two)
  int bounded;            // candidate buffers sized by the sample's estimate: no device fallback
  uint32_t adapt_first;   // beta path (autotuned): the threshold-only first select keeps refining
                          // past first_levels while its chosen bin holds more delegates than this
  GridBar gb;
};

enum StatSlot : int {
  ST_THR1 = 0, ST_NSEL = 1, ST_NLONELY = 2, ST_NCAND = 3, ST_LVA = 4, ST_LVC = 5,
  ST_TOPA = 6, ST_TOPC = 7, ST_KTH = 8, ST_OK = 9, ST_FALLBACK = 10
};

// --------------------------------------------------------------- gathers
template <int KM>
DRTOPK_DEV void load4(const FusedArgs& a, uint64_t base, bool vec, uint32_t (&v)[4]) {
  if (vec) {
    uint4 q = __ldg(reinterpret_cast<const uint4*>(a.keys + base));
    v[0] = to_key<KM>(q.x); v[1] = to_key<KM>(q.y); v[2] = to_key<KM>(q.z); v[3] = to_key<KM>(q.w);
  } else {
#pragma unroll
    for (int e = 0; e < 4; ++e) v[e] = (base + e < a.n) ? to_key<KM>(__ldg(a.keys + base + e)) : 0u;
  }
}

// candidates >= thr of a list of kept subranges: the default path's k
// subranges (ids in the .y of the first select's top list) or the beta
// path's selected list.  Virtual space = count*S keys in uint4 granules (S>=4;
// S=2 uses 2-key granules); 4 granules per thread per tile, one
// block-aggregated append per tile.
constexpr int GATHER_U = 8;

template <int KM, int GATHER_U = drtopk::GATHER_U>
DRTOPK_DEV void gather_list(const Team& tm, const FusedArgs& a, const uint2* ids2, const uint32_t* ids1, uint64_t nsub,
                            uint32_t thr, uint32_t* s_hist, uint32_t& mlo, uint32_t& mhi, bool& ovf) {
  const uint64_t S = 1ull << a.alpha;
  const int gshift = a.alpha >= 2 ? 2 : a.alpha;  // log2 keys per granule
  const int gk = 1 << gshift;
  const uint64_t units = (nsub * S) >> gshift;
  const uint64_t T = (uint64_t)blockDim.x * GATHER_U;
  const int cs = cand_shift(thr, a.nbits);
  for (uint64_t tb = (uint64_t)tm.rank * T; tb < units; tb += (uint64_t)tm.size * T) {
    uint32_t v[GATHER_U][4];
    uint32_t base[GATHER_U];  // key index of the granule (n < 2^32)
    uint64_t take = 0;
    uint32_t cnt = 0;
#pragma unroll
    for (int q = 0; q < GATHER_U; ++q) {
      const uint64_t u = tb + (uint64_t)q * blockDim.x + threadIdx.x;
      base[q] = 0;
      v[q][0] = v[q][1] = v[q][2] = v[q][3] = 0u;
      if (u < units) {
        const uint64_t pos = u << gshift;
        const uint64_t sel = pos >> a.alpha;
        const uint32_t sub = ids2 ? ld_cg_v2(reinterpret_cast<const uint32_t*>(ids2 + sel)).y : ld_cg_u32(ids1 + sel);
        base[q] = (uint32_t)(((uint64_t)sub << a.alpha) + (pos & (S - 1)));
        if (gk == 4) {
          load4<KM>(a, base[q], a.vec_ok && (uint64_t)base[q] + 4 <= a.n, v[q]);
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e)
            v[q][e] = (e < gk && (uint64_t)base[q] + e < a.n) ? to_key<KM>(__ldg(a.keys + base[q] + e)) : 0u;
        }
      }
    }
#pragma unroll
    for (int q = 0; q < GATHER_U; ++q) {
      const uint64_t u = tb + (uint64_t)q * blockDim.x + threadIdx.x;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const bool t = u < units && e < gk && ((uint64_t)base[q] + e < a.n) && v[q][e] >= thr;
        take |= (uint64_t)t << (q * 4 + e);
        cnt += t;
      }
    }
    uint32_t slot = block_append1(cnt, a.cand_count);
#pragma unroll
    for (int q = 0; q < GATHER_U; ++q)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if ((take >> (q * 4 + e)) & 1ull) {
          const uint32_t key = v[q][e];
          if (slot < a.cand_cap) a.cand[slot] = make_uint2(key, base[q] + e);
          else ovf = true;
          ++slot;
          if (a.bucket) { mlo = max(mlo, ~key); mhi = max(mhi, key); }
          else hist_add_warp(s_hist, (key - thr) >> cs);
        }
      }
  }
}

constexpr int FILTER_E = 8;  // subranges per thread per tile of the beta filter

// Exclusive prefix sum of v over the block (all threads), with the total.
DRTOPK_DEV uint32_t block_excl_scan(uint32_t v, uint32_t& total) {
  __shared__ uint32_t s_w[MAX_BLOCK_WARPS];
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
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
  for (unsigned w = 0; w < nw; ++w) {
    if (w < wid) before += s_w[w];
    total += s_w[w];
  }
  __syncthreads();
  return before + x - v;
}

// Ties at a one-value threshold (the autotuned beta path's first select
// collapsed to the single value thr, as few-digit keys make it): every
// subrange whose Max equals thr holds copies of thr and nothing above it.
// The k-th largest key K is >= thr.  If K > thr those subranges hold no key
// of the top k; if K == thr, the lowest-index copies of thr the top k needs
// lie in subranges kept whole anyway (Max > thr, Second >= thr) or in the k
// lowest-id subranges with Max == thr, since each of those holds a copy
// with a lower index than any copy further on.  Returns the id bound
// (exclusive) of the tied subranges to keep: after the k-th one, or M.
// Scratch: one word per tile of blockDim * FILTER_E subranges.
DRTOPK_DEV uint32_t beta_tie_cut(const Team& tm, const FusedArgs& a, uint32_t thr, uint32_t* scratch) {
  const uint64_t T = (uint64_t)blockDim.x * FILTER_E;
  const uint64_t tiles = (a.M + T - 1) / T;
  uint32_t tot = 0;
  for (uint64_t t = tm.rank; t < tiles; t += tm.size) {
    uint32_t c = 0;
#pragma unroll
    for (int q = 0; q < FILTER_E; ++q) {
      const uint64_t j = t * T + (uint64_t)q * blockDim.x + threadIdx.x;
      if (j < a.M && a.del[2 * j] == thr) ++c;
    }
    block_excl_scan(c, tot);
    if (threadIdx.x == 0) scratch[t] = tot;
  }
  if (!team_sync(tm)) return (uint32_t)a.M;
  if (tm.rank == 0) {
    __shared__ uint32_t s_found, s_tile, s_rem, s_cut;
    if (threadIdx.x == 0) { s_found = 0; s_cut = (uint32_t)a.M; }
    __syncthreads();
    // the tile holding the k-th tied subrange (tiles in id order)
    uint32_t base = 0;
    for (uint64_t t0 = 0; t0 < tiles; t0 += blockDim.x) {
      const uint64_t t = t0 + threadIdx.x;
      const uint32_t v = t < tiles ? ld_cg_u32(scratch + t) : 0u;
      const uint32_t ex = base + block_excl_scan(v, tot);
      if (v && ex < a.k && ex + v >= a.k) { s_found = 1; s_tile = (uint32_t)t; s_rem = a.k - ex; }
      base += tot;
      __syncthreads();
      if (s_found) break;
    }
    if (s_found) {
      // inside it, the s_rem-th tied subrange in id order
      uint32_t run = 0;
      for (int q = 0; q < FILTER_E; ++q) {
        const uint64_t j = (uint64_t)s_tile * T + (uint64_t)q * blockDim.x + threadIdx.x;
        const uint32_t f = (j < a.M && a.del[2 * j] == thr) ? 1u : 0u;
        const uint32_t ex = run + block_excl_scan(f, tot);
        if (f && ex + 1 == s_rem) s_cut = (uint32_t)(j + 1);
        run += tot;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) *a.tie_cut = s_cut;
  }
  if (!team_sync(tm)) return (uint32_t)a.M;
  return ld_cg_u32(a.tie_cut);
}

// beta path filter (FindTopKRanges_beta, radixselect.cuh:560-598): per
// subrange, Max >= thr and Second >= thr -> subrange id to the selected
// list; Max >= thr only -> Max itself is a candidate (with its position).
// Subranges whose Max equals thr with an id at or past `cut` are dropped.
template <int KM>
DRTOPK_DEV void filter_beta(const Team& tm, const FusedArgs& a, uint32_t thr, uint32_t* s_hist, uint32_t& mlo,
                            uint32_t& mhi, bool& ovf, uint64_t cut = ~0ull) {
  const uint64_t T = (uint64_t)blockDim.x * FILTER_E;
  const int hsh = cand_shift(thr, a.nbits);
  for (uint64_t tb = (uint64_t)tm.rank * T; tb < a.M; tb += (uint64_t)tm.size * T) {
    uint32_t m1[FILTER_E];
    uint32_t lon = 0, sel = 0, cl = 0, cs = 0;
#pragma unroll
    for (int q = 0; q < FILTER_E; ++q) {
      const uint64_t j = tb + (uint64_t)q * blockDim.x + threadIdx.x;
      m1[q] = 0;
      if (j < a.M) {
        const uint2 d = *reinterpret_cast<const uint2*>(a.del + 2 * j);
        m1[q] = d.x;
        const bool keep = d.x != thr || j < cut;  // tied subranges past the cut hold no needed key
        const bool s1 = keep && d.x >= thr && d.y >= thr;
        const bool l1 = keep && d.x >= thr && d.y < thr;
        sel |= (uint32_t)s1 << q;
        lon |= (uint32_t)l1 << q;
        cs += s1;
        cl += l1;
      }
    }
    Slots2 sl = block_append2(cl, cs, a.cand_count, a.sel_count);
#pragma unroll
    for (int q = 0; q < FILTER_E; ++q) {
      const uint64_t j = tb + (uint64_t)q * blockDim.x + threadIdx.x;
      if ((lon >> q) & 1u) {
        uint32_t idx = (uint32_t)(j << a.alpha);
        if (a.has_pos) idx += a.pos[j];
        if (sl.a < a.cand_cap) a.cand[sl.a] = make_uint2(m1[q], idx);
        else ovf = true;
        ++sl.a;
        if (a.bucket) { mlo = max(mlo, ~m1[q]); mhi = max(mhi, m1[q]); }
        else hist_add_warp(s_hist, (m1[q] - thr) >> hsh);
      }
      if ((sel >> q) & 1u) a.sel[sl.b++] = (uint32_t)j;
    }
  }
}

// min/max pass over a key array (plain bucket path)
template <int KM>
DRTOPK_DEV void minmax_pass(const Team& tm, const FusedArgs& a, uint32_t* gmm) {
  __shared__ uint32_t s_mm[2];
  if (threadIdx.x < 2) s_mm[threadIdx.x] = 0;
  __syncthreads();
  uint32_t lo = 0, hi = 0;
  const uint64_t g = (uint64_t)tm.rank * blockDim.x + threadIdx.x;
  const uint64_t G = (uint64_t)tm.size * blockDim.x;
  for (uint64_t i = g; i < a.n; i += G) {
    uint32_t k = to_key<KM>(__ldg(a.keys + i));
    lo = max(lo, ~k);
    hi = max(hi, k);
  }
  atomicMax(&s_mm[0], lo);
  atomicMax(&s_mm[1], hi);
  __syncthreads();
  if (threadIdx.x == 0) { atomicMax(&gmm[0], s_mm[0]); atomicMax(&gmm[1], s_mm[1]); }
}

// --------------------------------------------------------------- sorting
// One CTA: bitonic sort of n64 (<= SMALL_SORT, padded to a power of two)
// 64-bit composites in shared memory, descending.
DRTOPK_DEV void block_bitonic_desc(uint64_t* s, int npow2) {
  for (int size = 2; size <= npow2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      __syncthreads();
      for (int i = threadIdx.x; i < npow2 / 2; i += blockDim.x) {
        int lo = 2 * stride * (i / stride) + (i % stride);
        int hi = lo + stride;
        bool desc = ((lo & size) == 0);
        uint64_t x = s[lo], y = s[hi];
        if ((x < y) == desc) { s[lo] = y; s[hi] = x; }
      }
    }
  }
  __syncthreads();
}

// Multi-CTA stable LSD radix sort of nk 64-bit keys ascending (8-bit
// digits), skipping digits that are constant over all keys.  Keys are
// (~value << 32) | index, so ascending order = value desc, index asc.
// Each CTA owns one contiguous range; per digit: CTA counts -> column scan
// over CTAs (one digit column per CTA) -> stable scatter.  Returns the
// buffer holding the result.
DRTOPK_DEV uint64_t* grid_lsd_sort(const Team& tm, const FusedArgs& a, uint64_t* src, uint64_t* dst, uint32_t nk,
                                   uint32_t* s_cnt, bool& ok) {
  const int C = (int)tm.size, c = (int)tm.rank, t = threadIdx.x;
  const uint32_t per = (nk + C - 1) / C;
  const uint32_t r0 = min(nk, per * c), r1 = min(nk, r0 + per);
  __shared__ uint32_t s_run[256];
  __shared__ uint32_t s_wcnt[MAX_BLOCK_WARPS][257];
  __shared__ int s_trivial;
  // totals of all 8 digits, in one pass over this CTA's range (8 x 256
  // counters in the scatter's per-warp count space, unused until then)
  uint32_t* s_tot8 = &s_wcnt[0][0];
  for (int i = t; i < 8 * 256; i += blockDim.x) s_tot8[i] = 0;
  __syncthreads();
  block_load_loop<8>(r1 - r0, [&](uint32_t i) { return ld_cg_u64(src + r0 + i); }, [&](uint32_t, uint64_t v) {
#pragma unroll
    for (int d = 0; d < 8; ++d) atomicAdd(&s_tot8[d * 256 + ((v >> (8 * d)) & 255u)], 1u);
  });
  __syncthreads();
  for (int i = t; i < 8 * 256; i += blockDim.x) {
    const uint32_t cnt = s_tot8[i];
    if (cnt) atomicAdd(&a.sort_tot[i], cnt);
  }
  __syncthreads();
  if (!team_sync(tm)) { ok = false; return src; }
  // one stable counting pass over digit d (src -> dst, then swapped); a
  // digit every key shares is skipped
  auto digit_pass = [&](int d) -> bool {
    if (t == 0) s_trivial = 0;
    __syncthreads();
    for (int i = t; i < 256; i += blockDim.x)
      if (ld_cg_u32(a.sort_tot + d * 256 + i) == nk) s_trivial = 1;
    __syncthreads();
    if (s_trivial) return true;
    const int sh = 8 * d;
    // 1) this CTA's digit counts
    for (int i = t; i < 256; i += blockDim.x) s_cnt[i] = 0;
    __syncthreads();
    block_load_loop<8>(r1 - r0, [&](uint32_t i) { return ld_cg_u64(src + r0 + i); },
                       [&](uint32_t, uint64_t v) { atomicAdd(&s_cnt[(v >> sh) & 255u], 1u); });
    __syncthreads();
    for (int i = t; i < 256; i += blockDim.x) a.sort_cnt[(uint64_t)c * 256 + i] = s_cnt[i];
    if (!team_sync(tm)) return false;
    // 2) exclusive scan of each digit column over the CTAs (in place)
    for (int col = c; col < 256; col += C) {
      if (t < 32) {
        uint32_t carry = 0;
        for (int c0 = 0; c0 < C; c0 += 32) {
          const int cc = c0 + t;
          uint32_t v = cc < C ? ld_cg_u32(a.sort_cnt + (uint64_t)cc * 256 + col) : 0u;
          uint32_t incl = v;
#pragma unroll
          for (int off = 1; off < 32; off <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
            if (t >= off) incl += y;
          }
          if (cc < C) a.sort_cnt[(uint64_t)cc * 256 + col] = carry + incl - v;
          carry += __shfl_sync(0xffffffffu, incl, 31);
        }
      }
    }
    if (!team_sync(tm)) return false;
    // 3) running offsets = digit base (scan of totals) + this CTA's column prefix
    if (t < 256) s_cnt[t] = ld_cg_u32(a.sort_tot + d * 256 + t);
    __syncthreads();
    if (t == 0) {
      uint32_t acc = 0;
      for (int i = 0; i < 256; ++i) { uint32_t v = s_cnt[i]; s_cnt[i] = acc; acc += v; }
    }
    __syncthreads();
    if (t < 256) s_run[t] = s_cnt[t] + ld_cg_u32(a.sort_cnt + (uint64_t)c * 256 + t);
    __syncthreads();
    // 4) stable scatter in chunks of SORT_U keys per thread: warp w takes
    // the chunk's w-th span of 32 * SORT_U keys, in SORT_U rounds of 32
    // consecutive ones, so its ranks follow position order; the warps'
    // counts then give each warp its prefix per digit
    const int wid = t >> 5;
    const int nwarps = (int)(blockDim.x >> 5);
    const unsigned lane = t & 31u;
    const uint32_t CHK = blockDim.x * SORT_U;
    for (uint32_t cb = r0; cb < r1; cb += CHK) {
      for (int q = lane; q < 257; q += 32) s_wcnt[wid][q] = 0;
      __syncwarp();
      uint64_t kv[SORT_U];
      uint32_t dgs[SORT_U], rk[SORT_U];
      const uint32_t wb = cb + (uint32_t)wid * 32u * SORT_U;
#pragma unroll
      for (int u = 0; u < SORT_U; ++u) {
        const uint32_t i = wb + (uint32_t)u * 32u + lane;
        kv[u] = i < r1 ? ld_cg_u64(src + i) : 0ull;
      }
#pragma unroll
      for (int u = 0; u < SORT_U; ++u) {
        const uint32_t i = wb + (uint32_t)u * 32u + lane;
        const uint32_t dg = i < r1 ? (uint32_t)((kv[u] >> sh) & 255u) : 256u;
        const unsigned peers = __match_any_sync(0xffffffffu, dg);
        const uint32_t lower = __popc(peers & ((1u << lane) - 1u));
        rk[u] = s_wcnt[wid][dg] + lower;
        dgs[u] = dg;
        __syncwarp();
        if (lower == 0) s_wcnt[wid][dg] += __popc(peers);
        __syncwarp();
      }
      __syncthreads();
      // per digit: the warps' counts become their exclusive prefixes
      uint32_t dtot = 0;
      if (t < 256) {
        for (int w2 = 0; w2 < nwarps; ++w2) {
          const uint32_t v = s_wcnt[w2][t];
          s_wcnt[w2][t] = dtot;
          dtot += v;
        }
      }
      __syncthreads();
#pragma unroll
      for (int u = 0; u < SORT_U; ++u)
        if (dgs[u] < 256u) dst[s_run[dgs[u]] + s_wcnt[wid][dgs[u]] + rk[u]] = kv[u];
      __syncthreads();
      if (t < 256) s_run[t] += dtot;
    }
    if (!team_sync(tm)) return false;
    uint64_t* tmp = src; src = dst; dst = tmp;
    return true;
  };
  // The key's digits first (4..7): the passes are stable, so equal keys
  // keep their input order; then every run of equal keys is put in index
  // order in place, one thread per run.  Runs longer than TIE_RUN_MAX (heavy
  // ties) set a flag, and the keys then go through all eight digits from
  // the least significant, the plain LSD order.
  for (int d = 4; d < 8; ++d)
    if (!digit_pass(d)) { ok = false; return src; }
  __shared__ int s_long;
  if (t == 0) s_long = 0;
  __syncthreads();
  const uint64_t g = (uint64_t)c * blockDim.x + t, G = (uint64_t)C * blockDim.x;
  for (uint64_t i = g; i < nk; i += G) {
    const uint32_t hk = (uint32_t)(ld_cg_u64(src + i) >> 32);
    if (i > 0 && (uint32_t)(ld_cg_u64(src + i - 1) >> 32) == hk) continue;  // not a run start
    uint64_t e = i + 1;
    while (e < nk && e - i <= (uint64_t)TIE_RUN_MAX && (uint32_t)(ld_cg_u64(src + e) >> 32) == hk) ++e;
    if (e - i > (uint64_t)TIE_RUN_MAX) { s_long = 1; continue; }
    // insertion sort of the run by index, in a thread-local copy (the run's
    // loads are independent; the sort's compares are not)
    uint64_t run[TIE_RUN_MAX];
    const int m = (int)(e - i);
    for (int x = 0; x < m; ++x) run[x] = ld_cg_u64(src + i + x);
    for (int x = 1; x < m; ++x) {
      const uint64_t v = run[x];
      int y = x;
      for (; y > 0 && run[y - 1] > v; --y) run[y] = run[y - 1];
      run[y] = v;
    }
    for (int x = 0; x < m; ++x) src[i + x] = run[x];
  }
  __syncthreads();
  if (t == 0 && s_long) atomicOr(a.sort_tot + SORT_LONG_WORD, 1u);
  if (!team_sync(tm)) { ok = false; return src; }
  if (ld_cg_u32(a.sort_tot + SORT_LONG_WORD))
    for (int d = 0; d < 8; ++d)
      if (!digit_pass(d)) { ok = false; return src; }
  return src;
}

DRTOPK_DEV void stamp(uint32_t* stats, int slot) {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  stats[slot] = (uint32_t)t;
  stats[slot + 1] = (uint32_t)(t >> 32);
}

// --------------------------------------------------------------- kernel
// The phases of one problem, run by one team (the whole cooperative grid,
// one thread-block cluster, or one CTA).
template <int KM>
DRTOPK_DEV void fused_body(const FusedArgs& a, const Team& tm, uint32_t* s_dyn) {
  uint32_t* s_hist = s_dyn;
  // two SMALL_SET-entry buffers after the histogram (runs finished in one CTA)
  uint2* s_fast = reinterpret_cast<uint2*>(s_dyn + ((max(a.nb, 256) + 3) & ~3));
  const bool lead = tm.rank == 0 && threadIdx.x == 0;
  const int D = 32 / a.nbits;
  uint32_t thr1 = 0, nsel = 0, nlonely = 0;
  int lvA = 0;
  bool thr_one = false;  // the threshold-only first select ended on a single value
  if (lead && a.phase_lo <= 1) stamp(a.stats, 16);

  // ---------------- phase 1: first select on the delegates
  if (a.phase_lo > 1) {
    thr1 = ld_cg_u32(a.thr_word);
  } else if (a.path == PATH_DEFAULT || a.path == PATH_BETA) {
    const uint64_t ndel = a.path == PATH_BETA ? 2 * a.M : a.M;
    Src s = {};
    s.keys = a.del;
    s.count = ndel;
    Level L0;
    if (a.bucket) {
      L0 = bucket_level0(~ld_cg_u32(a.del_minmax), ld_cg_u32(a.del_minmax + 1), a.nb, a.k);
      hist_pass<KM>(tm, s, false, false, L0, a.nb, a.A.H[0], s_hist);
      if (!team_sync(tm)) return;
    } else {
      L0 = radix_level0(a.nbits, a.k);
    }
    EngineCfg c = {};
    c.bucket = a.bucket; c.nbits = a.nbits; c.nb = a.nb; c.key_from_payload = 0;
    if (a.path == PATH_DEFAULT) {
      c.stop_single = 1; c.thr_only = 0;
      c.max_levels = a.bucket ? MAX_LEVELS : D;
    } else {
      c.stop_single = 0; c.thr_only = 1;
      c.max_levels = a.first_levels;
      c.adapt_cnt = a.adapt_first;
    }
    if (a.path == PATH_BETA && c.max_levels <= 0) {
      thr1 = 0;  // no digit processed: every subrange qualifies
    } else {
      RunResult r = run_select<KM>(c, s, false, a.A, a.AF, L0, s_hist, tm, s_fast);
      if (!r.ok) { if (lead) atomicOr(a.gb.err, (uint32_t)DE_INTERNAL); return; }
      lvA = r.levels;
      thr_one = c.thr_only && r.thr_hi == r.thr;
      // radix keeps the reference's flag (final range lower bound); the bucket
      // variant uses the exact k-th delegate on its default path
      thr1 = (a.path == PATH_DEFAULT && a.bucket) ? r.kth : r.thr;
    }
  }

  if (a.phase_lo <= 1 && lead) *a.thr_word = thr1;
  if (a.phase_hi == 1) {
    // split mode: the concatenation runs as separate kernels
    if (lead) {
      stamp(a.stats, 18);
      a.stats[ST_LVA] = lvA;
    }
    return;
  }
  // ---------------- phase 2: concatenation of candidates
  if (lead && a.phase_lo <= 2) stamp(a.stats, 18);
  clear_hist(s_hist, a.nb);
  uint32_t mlo = 0, mhi = 0;
  bool ovf = false;
  if (a.phase_lo > 2) {
    // concatenation already done by the split-mode kernels
  } else if (a.path == PATH_DEFAULT) {
    // the k kept subranges must all be there before their ids are used as
    // addresses (every CTA reads the same count after the last barrier)
    if (ld_cg_u32(a.A.top_count) != a.k) {
      if (lead) atomicOr(a.gb.err, (uint32_t)DE_INTERNAL);
      return;
    }
    gather_list<KM>(tm, a, a.A.top, nullptr, a.k, thr1, s_hist, mlo, mhi, ovf);
  } else if (a.path == PATH_BETA) {
    // autotuned select whose threshold collapsed to one value: keep only
    // the k lowest-id subranges tied at it (scratch: the second run's
    // compact buffer, unused until phase 3)
    const uint64_t cut = (a.adapt_first && !a.bucket && thr_one)
                             ? (uint64_t)beta_tie_cut(tm, a, thr1, reinterpret_cast<uint32_t*>(a.C.cbuf[0]))
                             : ~0ull;
    filter_beta<KM>(tm, a, thr1, s_hist, mlo, mhi, ovf, cut);
    if (!team_sync(tm)) return;
    const uint32_t nsel_sub = ld_cg_u32(a.sel_count);
    if (lead) {
      a.stats[ST_NSEL] = nsel_sub;
      a.stats[ST_NLONELY] = ld_cg_u32(a.cand_count);
    }
    if (nsel_sub > a.M) {
      if (lead) atomicOr(a.gb.err, (uint32_t)DE_INTERNAL);
      return;
    }
    gather_list<KM>(tm, a, nullptr, a.sel, nsel_sub, thr1, s_hist, mlo, mhi, ovf);
  }
  if (ovf) atomicOr(a.gb.err, (uint32_t)DE_OVERFLOW);
  if (a.phase_lo > 2) {
    // candidates' level-0 statistics were flushed by the split-mode kernels
  } else if (a.path != PATH_PLAIN) {
    if (a.bucket) {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        mlo = max(mlo, __shfl_xor_sync(0xffffffffu, mlo, off));
        mhi = max(mhi, __shfl_xor_sync(0xffffffffu, mhi, off));
      }
      if ((threadIdx.x & 31) == 0) { atomicMax(&a.cand_minmax[0], mlo); atomicMax(&a.cand_minmax[1], mhi); }
    } else {
      flush_hist(s_hist, a.C.H[0], a.nb);
    }
  } else {
    // plain select: level-0 statistics straight off the input
    if (a.bucket) minmax_pass<KM>(tm, a, a.cand_minmax);
    else {
      Src s = {};
      s.keys = a.keys; s.count = a.n; s.raw_input = 1;
      hist_pass<KM>(tm, s, false, false, radix_level0(a.nbits, a.k), a.nb, a.C.H[0], s_hist);
    }
  }
  if (!team_sync(tm)) return;

  // ---------------- phase 3: second select
  if (lead) {
    stamp(a.stats, 20);
    if (a.path == PATH_BETA && a.phase_lo > 2) a.stats[ST_NSEL] = ld_cg_u32(a.sel_count);
  }
  Src sc = {};
  bool pairs;
  // sampled-threshold path: fewer than k keys at or above the predicted
  // threshold means the prediction overshot the k-th key; the select then
  // runs over all keys (plain radix), so the answer stays exact
  const bool emit_fb = a.path == PATH_EMIT && (ld_cg_u32(a.cand_count) < a.k || ld_cg_u32(a.cand_count) > a.cand_cap);
  if (emit_fb && a.bounded) {
    // buffers sized by the estimate cannot hold the general select: the
    // caller runs this request again with its general plan
    if (lead) atomicOr(a.gb.err, (uint32_t)DE_RETRY);
    return;
  }
  if (emit_fb) {
    zero_words(tm, a.C.H[0], a.nb);
    if (!team_sync(tm)) return;
    Src s = {};
    s.keys = a.keys; s.count = a.n; s.raw_input = 1;
    hist_pass<KM>(tm, s, false, false, radix_level0(a.nbits, a.k), a.nb, a.C.H[0], s_hist);
    if (!team_sync(tm)) return;
    if (lead) a.stats[ST_FALLBACK] = 1;
  }
  if (a.path == PATH_PLAIN || emit_fb) {
    sc.keys = a.keys; sc.count = a.n; sc.raw_input = 1;
    pairs = false;
  } else {
    sc.pairs = a.cand; sc.count_dev = a.cand_count;
    pairs = true;
    if (ld_cg_u32(a.cand_count) < a.k || ld_cg_u32(a.cand_count) > a.cand_cap) {
      if (lead) atomicOr(a.gb.err, (uint32_t)DE_INTERNAL);
      return;
    }
  }
  Level L0c;
  if (a.bucket) {
    L0c = bucket_level0(~ld_cg_u32(a.cand_minmax), ld_cg_u32(a.cand_minmax + 1), a.nb, a.k);
    hist_pass<KM>(tm, sc, pairs, false, L0c, a.nb, a.C.H[0], s_hist);
    if (!team_sync(tm)) return;
  } else {
    // candidates of the sampled paths are all >= thr1 (their level-0
    // histogram was built against this level by the concatenation, or by
    // k_cand_hist)
    L0c = (a.path == PATH_PLAIN || emit_fb)
              ? radix_level0(a.nbits, a.k)
              : (a.path == PATH_EMIT ? cand_level0_tight(thr1, ld_cg_u32(a.cand_minmax + 1), a.nbits, a.k)
                                     : cand_level0(thr1, a.nbits, a.k));
  }
  EngineCfg cc = {};
  cc.bucket = a.bucket; cc.nbits = a.nbits; cc.nb = a.nb; cc.stop_single = 1;
  cc.max_levels = MAX_LEVELS; cc.thr_only = 0; cc.key_from_payload = 0; cc.skip_split0 = emit_fb ? 0 : a.split0;
  // entries k_split0 already wrote to the output (slots [0, c0) of the list)
  const uint32_t c0 = (a.direct0 && !emit_fb) ? ld_cg_u32(a.C.top_count) : 0u;
  RunResult rc = run_select<KM>(cc, sc, pairs, a.C, a.CF, L0c, s_hist, tm, s_fast);
  if (!rc.ok) { if (lead) atomicOr(a.gb.err, (uint32_t)DE_INTERNAL); return; }
  const uint32_t K = rc.kth;
  const uint32_t ntop = ld_cg_u32(a.C.top_count);
  if (lead) {
    stamp(a.stats, 22);
    if (a.out_kth) a.out_kth[0] = from_key(K, a.km);
    a.stats[ST_THR1] = thr1;
    if (a.path == PATH_DEFAULT) a.stats[ST_NSEL] = a.k;
    a.stats[ST_NCAND] = (a.path == PATH_PLAIN || emit_fb) ? (uint32_t)a.n : ld_cg_u32(a.cand_count);
    if (a.phase_lo <= 1) a.stats[ST_LVA] = lvA;
    a.stats[ST_LVC] = rc.levels;
    a.stats[ST_TOPA] = a.path == PATH_DEFAULT ? ld_cg_u32(a.A.top_count) : 0u;
    a.stats[ST_TOPC] = ntop;
    a.stats[ST_KTH] = K;
    a.stats[ST_OK] = 1;
    if (ntop != a.k) atomicOr(a.gb.err, (uint32_t)DE_INTERNAL);
  }
  if (!a.out_vals && !a.out_idx) return;
  if (ntop != a.k) return;

  // ---------------- phase 4: top-k output
  const uint64_t g = (uint64_t)tm.rank * blockDim.x + threadIdx.x;
  const uint64_t G = (uint64_t)tm.size * blockDim.x;
  if (!a.sorted) {
    team_load_loop<8>(tm, a.k - c0,
                      [&](uint64_t i) { return ld_cg_v2(reinterpret_cast<const uint32_t*>(a.C.top + c0 + i)); },
                      [&](uint64_t i, uint2 e) {
                        if (a.out_vals) a.out_vals[c0 + i] = from_key(e.x, a.km);
                        if (a.out_idx) a.out_idx[c0 + i] = (int64_t)e.y;
                      });
    return;
  }
  if (a.k <= SMALL_SORT) {
    if (tm.rank != 0) return;
    uint64_t* s = reinterpret_cast<uint64_t*>(s_dyn);
    int np2 = 1;
    while (np2 < (int)a.k) np2 <<= 1;
    for (int i = (int)a.k + threadIdx.x; i < np2; i += blockDim.x) s[i] = 0;
    block_load_loop<8>(a.k, [&](uint32_t i) { return ld_cg_v2(reinterpret_cast<const uint32_t*>(a.C.top + i)); },
                       [&](uint32_t i, uint2 e) { s[i] = ((uint64_t)e.x << 32) | (uint64_t)(~e.y); });
    block_bitonic_desc(s, np2);
    for (int i = threadIdx.x; i < (int)a.k; i += blockDim.x) {
      uint64_t v = s[i];
      if (a.out_vals) a.out_vals[i] = from_key((uint32_t)(v >> 32), a.km);
      if (a.out_idx) a.out_idx[i] = (int64_t)(uint32_t)(~(uint32_t)v);
    }
    return;
  }
  // large k: multi-CTA stable LSD radix sort of (~key << 32 | index)
  team_load_loop<8>(tm, a.k, [&](uint64_t i) { return ld_cg_v2(reinterpret_cast<const uint32_t*>(a.C.top + i)); },
                    [&](uint64_t i, uint2 e) { a.sort_buf[0][i] = ((uint64_t)(~e.x) << 32) | (uint64_t)e.y; });
  if (!team_sync(tm)) return;
  bool ok = true;
  uint64_t* res = grid_lsd_sort(tm, a, a.sort_buf[0], a.sort_buf[1], a.k, s_hist, ok);
  if (!ok) return;
  (void)g; (void)G;
  team_load_loop<8>(tm, a.k, [&](uint64_t i) { return ld_cg_u64(res + i); }, [&](uint64_t i, uint64_t v) {
    if (a.out_vals) a.out_vals[i] = from_key(~(uint32_t)(v >> 32), a.km);
    if (a.out_idx) a.out_idx[i] = (int64_t)(uint32_t)v;
  });
}

// cooperative launch: the whole grid is the team
template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS) k_fused(FusedArgs a) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  fused_body<KM>(a, grid_team(a.gb), s_dyn);
}

// one ordinary CTA is the team: no co-residency with other CTAs is needed, so
// the launch never waits for a share of the GPU and overlaps other streams'
// kernels (the served form's last levels of a sampled-threshold select)
template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS) k_fused_one(FusedArgs a) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  Team t = {};
  t.rank = 0;
  t.size = 1;
  t.cluster = 2;
  fused_body<KM>(a, t, s_dyn);
}

// cluster launch: every thread-block cluster is the team of one problem --
// problem clusterid.x of `list`, or the kernel argument when list is null
template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS) k_fused_cl(FusedArgs a0, const FusedArgs* list) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  __shared__ FusedArgs s_args;
  const FusedArgs* ap = &a0;
  if (list) {
    const uint32_t cid = cluster_id_x();
    const uint32_t* src = reinterpret_cast<const uint32_t*>(list + cid);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&s_args);
    for (int i = threadIdx.x; i < (int)(sizeof(FusedArgs) / 4); i += blockDim.x) dst[i] = __ldg(src + i);
    __syncthreads();
    ap = &s_args;
  }
  fused_body<KM>(*ap, cluster_team(), s_dyn);
}

// --------------------------------------------------------------- split mode
// For large concatenations the two streaming phases run as ordinary kernels
// (many more resident warps than the cooperative kernel) between two
// launches of k_fused (phase 1, then phase 3).  The threshold comes from
// a.thr_word; counts are read after the kernel boundary.
//
// Both kernels work warp by warp with no block barrier in the loop: a warp
// compacts what it keeps into its own stage in shared memory (one warp scan
// per round) and drains the stage to global memory in runs of up to
// SPLIT_STAGE entries with one atomic per run, so appends neither contend on
// the global counters nor stall the warp.  The second select's level-0
// histogram is taken from the stage as it drains.
constexpr int SPLIT_STAGE = 512;                 // staged entries per warp (k_filter)
constexpr int SPLIT_WARPS = FUSED_THREADS / 32;
constexpr int FILTER_Q = 8;                      // subranges per lane per batch (k_filter)
constexpr int GATHER_R = 4;                      // granules per lane per round (k_gather)
constexpr int GATHER_STAGE = 32 * 4 * GATHER_R;  // staged candidates per warp (k_gather): one round's worth
// shared memory of the split kernels after the histogram words
constexpr size_t SPLIT_FILTER_SMEM = (size_t)SPLIT_WARPS * SPLIT_STAGE * 12;  // candidate + selected-id stages
constexpr size_t SPLIT_GATHER_SMEM = (size_t)SPLIT_WARPS * GATHER_STAGE * 8;

DRTOPK_DEV int split_hist_words(int nb) { return (max(nb, 256) + 3) & ~3; }

// exclusive prefix of v over the warp; total in *tot
DRTOPK_DEV uint32_t warp_excl_scan(uint32_t v, uint32_t& tot) {
  const unsigned lane = lane_id();
  uint32_t x = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
    if ((int)lane >= off) x += y;
  }
  tot = __shfl_sync(0xffffffffu, x, 31);
  return x - v;
}

// A warp's stage of (key, index) candidates.  Every member is warp-uniform
// except the stage contents; all calls are made by the full warp.
struct CandStage {
  uint2* buf;
  uint32_t cap;
  uint32_t n;
  uint32_t thr;
  int cs;
  uint32_t mlo, mhi;
  bool ovf;
  bool track_max;  // record the largest key instead of the level-0 histogram

  DRTOPK_DEV void drain(const FusedArgs& a, uint32_t* s_hist) {
    __syncwarp();
    const unsigned lane = lane_id();
    if (n == 0) return;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(a.cand_count, n);
    base = __shfl_sync(0xffffffffu, base, 0);
    for (uint32_t i = lane; i < n; i += 32) {
      const uint2 v = buf[i];
      if ((uint64_t)base + i < a.cand_cap) a.cand[base + i] = v;
      else ovf = true;
      if (track_max) mhi = max(mhi, v.x);
      else if (a.bucket) { mlo = max(mlo, ~v.x); mhi = max(mhi, v.x); }
      else hist_add_warp(s_hist, (v.x - thr) >> cs);
    }
    __syncwarp();
    n = 0;
  }
  // room for `tot` more entries (tot <= cap); returns the first slot
  DRTOPK_DEV uint32_t reserve(const FusedArgs& a, uint32_t* s_hist, uint32_t tot) {
    if (n + tot > cap) drain(a, s_hist);
    const uint32_t at = n;
    n += tot;
    return at;
  }
};

DRTOPK_DEV void flush_cand_stats(const FusedArgs& a, uint32_t* s_hist, uint32_t mlo, uint32_t mhi) {
  if (a.bucket) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      mlo = max(mlo, __shfl_xor_sync(0xffffffffu, mlo, off));
      mhi = max(mhi, __shfl_xor_sync(0xffffffffu, mhi, off));
    }
    if ((threadIdx.x & 31) == 0) { atomicMax(&a.cand_minmax[0], mlo); atomicMax(&a.cand_minmax[1], mhi); }
  } else {
    flush_hist(s_hist, a.C.H[0], a.nb);
  }
}

// Convergent histogram increment (all 32 lanes call it; `in` selects the
// lanes that count): one atomic when every counting lane hits the same bin.
DRTOPK_DEV void hist_add_conv(uint32_t* h, bool in, uint32_t bin) {
  const unsigned m = __ballot_sync(0xffffffffu, in);
  if (m == 0u) return;
  const int leader = __ffs(m) - 1;
  const uint32_t b0 = __shfl_sync(0xffffffffu, bin, leader);
  if (__ballot_sync(0xffffffffu, in && bin == b0) == m) {
    if ((int)lane_id() == leader) atomicAdd(&h[b0], (uint32_t)__popc(m));
  } else if (in) {
    atomicAdd(&h[bin], 1u);
  }
}

// First select of the beta path in split mode (radix, first_levels <= 2):
// the threshold-only picks of radix_select_inplace_firsttopk_beta
// (radixselect.cuh:1727-1780) -- the same picks run_levels makes -- from
// the delegate histograms A.H[0] (sampler) and A.H[1] (k_level_hist).  Every
// CTA computes them redundantly; `upto` levels are picked.
DRTOPK_DEV Level beta_first_levels(const FusedArgs& a, int upto, int& levels) {
  EngineCfg c = {};
  c.bucket = 0; c.nbits = a.nbits; c.nb = a.nb; c.stop_single = 0; c.thr_only = 1;
  c.max_levels = a.first_levels; c.key_from_payload = 0;
  Level L = radix_level0(a.nbits, a.k);
  levels = 0;
  for (int j = 0; j < upto; ++j) {
    const Pick p = block_pick<false>(a.A.H[j], a.nb, L.R);
    Level N;
    const bool done = advance(c, L, p, j, N);
    L = N;
    levels = j + 1;
    if (done) break;
  }
  return L;
}

// Level-1 histogram of the delegates for the split-mode first select: every
// CTA picks the level-0 bin, then the delegates inside it are counted over
// the next digit into A.H[1] (16-byte loads, LEVEL_HIST_V per thread in flight).
constexpr int LEVEL_HIST_V = 8;

template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS) k_level_hist(FusedArgs a) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  uint32_t* s_hist = s_dyn;
  if (blockIdx.x == 0 && threadIdx.x == 0) stamp(a.stats, 16);
  clear_hist(s_hist, a.nb);
  int lv = 0;
  const Level N = beta_first_levels(a, 1, lv);
  const uint32_t span = N.hi - N.lo;
  const int sh = max(N.wshift, 0);  // radix: bins are power-of-two wide (width 1 below the last digit)
  const uint64_t nkeys = 2 * a.M;
  const uint64_t nw = nkeys / 4;
  const uint64_t T = (uint64_t)blockDim.x * LEVEL_HIST_V;
  for (uint64_t tb = (uint64_t)blockIdx.x * T; tb < nw; tb += (uint64_t)gridDim.x * T) {
    uint4 w[LEVEL_HIST_V];
#pragma unroll
    for (int v = 0; v < LEVEL_HIST_V; ++v) {
      const uint64_t q = tb + (uint64_t)v * blockDim.x + threadIdx.x;
      w[v] = q < nw ? __ldg(reinterpret_cast<const uint4*>(a.del) + q) : make_uint4(0u, 0u, 0u, 0u);
    }
#pragma unroll
    for (int v = 0; v < LEVEL_HIST_V; ++v) {
      const bool valid = tb + (uint64_t)v * blockDim.x + threadIdx.x < nw;
      const uint32_t kk[4] = {w[v].x, w[v].y, w[v].z, w[v].w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const uint32_t d = kk[e] - N.lo;
        const bool in = valid && d <= span;
        // plain shared atomics unless at least half the warp counts (then
        // one atomic when they all share a bin: crowded keys)
        if (__popc(__ballot_sync(0xffffffffu, in)) >= 16) hist_add_conv(s_hist, in, d >> sh);
        else if (in) atomicAdd(&s_hist[d >> sh], 1u);
      }
    }
  }
  if (blockIdx.x == 0 && threadIdx.x < nkeys - nw * 4) {
    const uint32_t d = __ldg(a.del + nw * 4 + threadIdx.x) - N.lo;
    if (d <= span) atomicAdd(&s_hist[d >> sh], 1u);
  }
  flush_hist(s_hist, a.A.H[1], a.nb);
}

// Level 0 of the second select (radix_select_inplace 1410-1470) over a large
// candidate set, as an ordinary kernel: every CTA makes the level-0 pick
// from C.H[0] (the concatenation's histogram) -- the pick the cooperative
// kernel then makes again -- and splits the candidates: above the chosen
// bin -> the top list, or straight to the output when it is unsorted
// (direct0); inside it -> the next set, with the level-1 histogram.
constexpr int SPLIT0_E = 8;  // entries per thread per tile (register budget of 4 CTAs / SM)

template <int KM>
DRTOPK_DEV void split0_body(const FusedArgs& a, uint32_t cta, uint32_t ncta, uint32_t* s_dyn) {
  uint32_t* s_hist = s_dyn;
  const uint32_t thr = ld_cg_u32(a.thr_word);
  const uint32_t ncand = ld_cg_u32(a.cand_count);
  if (ncand < a.k || ncand > a.cand_cap) return;  // uniform; the second select reports it
  EngineCfg cc = {};
  cc.bucket = 0; cc.nbits = a.nbits; cc.nb = a.nb; cc.stop_single = 1;
  cc.max_levels = MAX_LEVELS; cc.thr_only = 0; cc.key_from_payload = 0; cc.skip_split0 = 0;
  const Level L0 = a.path == PATH_EMIT ? cand_level0_tight(thr, ld_cg_u32(a.cand_minmax + 1), a.nbits, a.k)
                                       : cand_level0(thr, a.nbits, a.k);
  const Pick p = block_pick<false>(a.C.H[0], a.nb, L0.R);
  Level N;
  const bool done = advance(cc, L0, p, 0, N);
  clear_hist(s_hist, a.nb);
  Src sc = {};
  sc.pairs = a.cand;
  sc.count_dev = a.cand_count;
  Team tm = grid_team(a.gb);
  tm.rank = cta;
  tm.size = ncta;
  if (a.direct0)
    split_tiles<KM, true, SPLIT0_E>(tm, cc, sc, true, ncand, N, !done, a.C, a.C.top_count, a.C.cbuf[0], a.C.set_count + 1,
                          s_hist, a.C.top_cap, a.C.cbuf_cap, a.C.err);
  else
    split_tiles<KM, false, SPLIT0_E>(tm, cc, sc, true, ncand, N, !done, a.C, a.C.top_count, a.C.cbuf[0], a.C.set_count + 1,
                           s_hist, a.C.top_cap, a.C.cbuf_cap, a.C.err);
  if (!done) flush_hist(s_hist, a.C.H[1], a.nb);
}

template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS, 4) k_split0(FusedArgs a) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  split0_body<KM>(a, blockIdx.x, gridDim.x, s_dyn);
}

// Beta filter (FindTopKRanges_beta, radixselect.cuh:560-598) over batches of
// 32*FILTER_Q subranges per warp: Max and Second >= thr -> subrange id to
// the selected list; Max >= thr only -> Max is a candidate, at its position.
template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS) k_filter(FusedArgs a) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  uint32_t* s_hist = s_dyn;
  const int hw = split_hist_words(a.nb);
  const unsigned lane = lane_id();
  const int wib = threadIdx.x >> 5;
  uint2* cstage = reinterpret_cast<uint2*>(s_dyn + hw) + (size_t)wib * SPLIT_STAGE;
  uint32_t* sstage = reinterpret_cast<uint32_t*>(reinterpret_cast<uint2*>(s_dyn + hw) + (size_t)SPLIT_WARPS * SPLIT_STAGE) +
                     (size_t)wib * SPLIT_STAGE;
  uint32_t thr;
  if (a.first_pre) {
    // the first select ends here: every CTA picks the threshold itself
    int lv = 0;
    thr = a.first_levels > 0 ? beta_first_levels(a, a.first_levels, lv).lo : 0u;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      *a.thr_word = thr;
      a.stats[ST_LVA] = (uint32_t)lv;
      if (a.first_levels < 2) stamp(a.stats, 16);
      stamp(a.stats, 18);
    }
  } else {
    thr = ld_cg_u32(a.thr_word);
  }
  clear_hist(s_hist, a.nb);
  CandStage cst = {cstage, (uint32_t)SPLIT_STAGE, 0u, thr, cand_shift(thr, a.nbits), 0u, 0u, false, false};
  uint32_t ns = 0;               // staged selected ids (warp-uniform)
  uint32_t nsel = 0, nlone = 0;  // this warp's totals
  auto drain_sel = [&]() {
    __syncwarp();
    if (ns == 0) return;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(a.sel_count, ns);
    base = __shfl_sync(0xffffffffu, base, 0);
    for (uint32_t i = lane; i < ns; i += 32)
      if ((uint64_t)base + i < a.M) a.sel[base + i] = sstage[i];
      else cst.ovf = true;
    __syncwarp();
    ns = 0;
  };
  const uint64_t B = 32ull * FILTER_Q;
  const uint64_t nbatch = (a.M + B - 1) / B;
  const uint64_t gw = (uint64_t)blockIdx.x * SPLIT_WARPS + wib, nw = (uint64_t)gridDim.x * SPLIT_WARPS;
  const uint2* del2 = reinterpret_cast<const uint2*>(a.del);
  // subrange ids fit 32 bits (M <= n < 2^32); only the batch counter is 64-bit
  for (uint64_t bt = gw; bt < nbatch; bt += nw) {
    const uint64_t rem = a.M - bt * B;  // > 0
    const uint32_t j0 = (uint32_t)(bt * B);
    uint2 d[FILTER_Q];
    uint32_t ps[FILTER_Q];
#pragma unroll
    for (int q = 0; q < FILTER_Q; ++q) {
      const uint32_t o = (uint32_t)q * 32u + lane;
      d[q] = o < rem ? __ldg(del2 + j0 + o) : make_uint2(0u, 0u);
      ps[q] = (a.has_pos && o < rem) ? (uint32_t)__ldg(a.pos + j0 + o) : 0u;
    }
    uint32_t lone = 0, sel = 0;
#pragma unroll
    for (int q = 0; q < FILTER_Q; ++q) {
      const bool v = (uint32_t)q * 32u + lane < rem && d[q].x >= thr;
      sel |= (uint32_t)(v && d[q].y >= thr) << q;
      lone |= (uint32_t)(v && d[q].y < thr) << q;
    }
    uint32_t tl = 0, ts = 0;
    const uint32_t ol = warp_excl_scan(__popc(lone), tl);
    const uint32_t os = warp_excl_scan(__popc(sel), ts);
    nlone += tl;
    nsel += ts;
    if (tl) {
      uint32_t at = cst.reserve(a, s_hist, tl) + ol;
      if (lone) {
#pragma unroll
        for (int q = 0; q < FILTER_Q; ++q)
          if ((lone >> q) & 1u)
            cstage[at++] = make_uint2(d[q].x, ((j0 + (uint32_t)q * 32u + lane) << a.alpha) + ps[q]);
      }
    }
    if (ts) {
      if (ns + ts > (uint32_t)SPLIT_STAGE) drain_sel();
      uint32_t at = ns + os;
      if (sel) {
#pragma unroll
        for (int q = 0; q < FILTER_Q; ++q)
          if ((sel >> q) & 1u) sstage[at++] = j0 + (uint32_t)q * 32u + lane;
      }
      ns += ts;
    }
  }
  cst.drain(a, s_hist);
  drain_sel();
  if (lane == 0 && nlone) atomicAdd(a.stats + ST_NLONELY, nlone);
  (void)nsel;
  if (cst.ovf) atomicOr(a.gb.err, (uint32_t)DE_OVERFLOW);
  flush_cand_stats(a, s_hist, cst.mlo, cst.mhi);
}

// Keys >= thr of the kept subranges: the default path's k subranges (ids in
// the .y of the first select's top list) or the beta path's selected list.
// The virtual space of count*S keys is cut into granules of min(4, S) keys;
// each warp takes rounds of 32*GATHER_R granules.
template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS, 4) k_gather(FusedArgs a) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  uint32_t* s_hist = s_dyn;
  const int hw = split_hist_words(a.nb);
  const unsigned lane = lane_id();
  const int wib = threadIdx.x >> 5;
  uint2* cstage = reinterpret_cast<uint2*>(s_dyn + hw) + (size_t)wib * GATHER_STAGE;
  const uint32_t thr = ld_cg_u32(a.thr_word);
  const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
  uint64_t nsub;
  const uint2* ids2 = nullptr;
  const uint32_t* ids1 = nullptr;
  if (a.path == PATH_DEFAULT) {
    if (ld_cg_u32(a.A.top_count) != a.k) {  // uniform: written by the previous launch
      if (lead) atomicOr(a.gb.err, (uint32_t)DE_INTERNAL);
      return;
    }
    nsub = a.k;
    ids2 = a.A.top;
  } else {
    nsub = ld_cg_u32(a.sel_count);
    if (nsub > a.M) {
      if (lead) atomicOr(a.gb.err, (uint32_t)DE_INTERNAL);
      return;
    }
    ids1 = a.sel;
  }
  clear_hist(s_hist, a.nb);
  CandStage cst = {cstage, (uint32_t)GATHER_STAGE, 0u, thr, cand_shift(thr, a.nbits), 0u, 0u, false, false};
  // granule and key indices fit 32 bits (n < 2^32); only the round counter
  // is 64-bit
  const int alpha = a.alpha;
  const int gsh = alpha >= 2 ? 2 : alpha;  // log2 keys per granule
  const uint32_t gk = 1u << gsh;
  const int upg = alpha - gsh;             // log2 granules per subrange
  const uint32_t gmask = (1u << upg) - 1u;
  const uint64_t units = nsub << upg;
  const uint32_t R = 32u * GATHER_R;
  const uint64_t gw = (uint64_t)blockIdx.x * SPLIT_WARPS + wib, nw = (uint64_t)gridDim.x * SPLIT_WARPS;
  const uint32_t n32 = (uint32_t)a.n;
  // subrange ids of a round's granules; the next round's ids are loaded while
  // this round's keys are in flight
  auto load_ids = [&](uint64_t ub, uint32_t (&sub)[GATHER_R]) {
    const uint64_t rem = units - ub;  // > 0
    const uint32_t u32 = (uint32_t)ub;
#pragma unroll
    for (int r = 0; r < GATHER_R; ++r) {
      const uint32_t o = (uint32_t)r * 32u + lane;
      sub[r] = 0;
      if (o < rem) sub[r] = ids2 ? __ldg(ids2 + ((u32 + o) >> upg)).y : __ldg(ids1 + ((u32 + o) >> upg));
    }
  };
  uint32_t subn[GATHER_R];
  if (gw * R < units) load_ids(gw * R, subn);
  for (uint64_t u0 = gw * R; u0 < units; u0 += nw * R) {
    const uint64_t rem = units - u0;
    const uint32_t u32 = (uint32_t)u0;
    uint32_t v[GATHER_R][4];
    uint32_t kb[GATHER_R], lim[GATHER_R];
#pragma unroll
    for (int r = 0; r < GATHER_R; ++r) {
      const uint32_t o = (uint32_t)r * 32u + lane;
      const uint32_t u = u32 + o;
      kb[r] = (subn[r] << alpha) + ((u & gmask) << gsh);
      lim[r] = (o < rem && kb[r] < n32) ? min(gk, n32 - kb[r]) : 0u;  // keys of this granule inside [0, n)
      v[r][0] = v[r][1] = v[r][2] = v[r][3] = 0u;
      if (lim[r] == 4u && a.vec_ok) {
        const uint4 q = __ldg(reinterpret_cast<const uint4*>(a.keys + kb[r]));
        v[r][0] = q.x; v[r][1] = q.y; v[r][2] = q.z; v[r][3] = q.w;
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if ((uint32_t)e < lim[r]) v[r][e] = __ldg(a.keys + kb[r] + e);
      }
    }
    if (u0 + nw * R < units) load_ids(u0 + nw * R, subn);
    uint32_t take = 0;
#pragma unroll
    for (int r = 0; r < GATHER_R; ++r)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        v[r][e] = to_key<KM>(v[r][e]);
        take |= (uint32_t)((uint32_t)e < lim[r] && v[r][e] >= thr) << (r * 4 + e);
      }
    uint32_t tot = 0;
    const uint32_t off = warp_excl_scan(__popc(take), tot);
    if (tot) {
      uint32_t at = cst.reserve(a, s_hist, tot) + off;
      if (take) {
#pragma unroll
        for (int r = 0; r < GATHER_R; ++r)
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if ((take >> (r * 4 + e)) & 1u) cstage[at++] = make_uint2(v[r][e], kb[r] + e);
      }
    }
  }
  cst.drain(a, s_hist);
  if (cst.ovf) atomicOr(a.gb.err, (uint32_t)DE_OVERFLOW);
  flush_cand_stats(a, s_hist, cst.mlo, cst.mhi);
}

// --------------------------------------------------------------- sampled-threshold path
// For large k the filter and gather of the delegate paths re-read the
// delegate vector and the kept subranges after the streaming pass.  This
// path predicts the threshold before the pass instead and makes the pass
// itself the concatenation.  The concatenation of the beta path at a
// threshold t -- whole subranges whose Max and Second reach t, the lone Max
// of subranges where only Max does -- is exactly the set of keys >= t, so
// the pass appends every key >= t_pred together with its index:
//   k_presample   top-byte histogram of a strided sample of the keys (one
//                 512-key chunk in pre_stride, at a rotating offset);
//   k_prerefine   (levels 1..3) the bytes picked so far, then the next
//                 byte's histogram of the sampled keys under that prefix
//                 (the sample is L2-resident).  Levels 2 and 3 run only
//                 while the picked bin still holds more than
//                 PRE_REFINE_KEYS keys' worth of the sample -- inputs whose
//                 keys share their top bytes (few distinct values, narrow
//                 ranges) -- and return at once otherwise;
//   k_emit        t_pred = the prefix boundary at which the sample holds
//                 pre_target keys (k scaled to the sample plus a six-sigma
//                 margin, set by the host), then one streaming pass
//                 appending every key >= t_pred, with the level-0
//                 histogram of the second select, as the gather does.
// The last CTA to finish a sample pass makes the level's pick for all
// later kernels (pre_state): the next refine level's CTAs read one word to
// learn whether they have work, and k_emit reads the finished threshold.
// k_split0 and the last levels of k_fused then run as in split mode.  The
// count of appended keys proves the prediction: at least k of them means
// t_pred <= the k-th key, so every key of the top k is a candidate.  With
// fewer, k_split0 does nothing and k_fused selects over all keys (plain
// radix select), so the result is exact whatever the input.
constexpr uint32_t PRE_STRIDE_MIN = 64;    // the sample is at most 1/64 of the keys
constexpr uint32_t PRE_STRIDE_MAX = 512;   // and at least 1/512
constexpr uint64_t PRE_SAMPLE_CHUNKS = 4096;
constexpr int PRE_ROUND = 4;     // sampled chunks in flight per warp
constexpr int PRE_CTAS_PER_SM = 2;
constexpr int PRE_LEVELS = 4;    // byte levels of the predicted threshold (at least 2 are used)
// a picked bin holding more keys (estimated from the sample) than
// max(PRE_REFINE_KEYS, k / 4) is refined by one more sample pass: one pass
// over the L2-resident sample costs a few microseconds, about what
// appending and selecting over this many extra candidates does (float keys,
// whose top bytes are sign and exponent, and few-digit keys need it)
constexpr uint64_t PRE_REFINE_KEYS = 1ull << 16;
// control words after the PRE_LEVELS histograms (pre_hist + PRE_STATE):
// [0, PRE_LEVELS) CTAs done per level, then the walk's state
constexpr int PRE_STATE = 256 * PRE_LEVELS;
constexpr int PS_DONE = PRE_LEVELS;  // bytes of the finished threshold (0: not finished)
constexpr int PS_PREFIX = PRE_LEVELS + 1;  // picked bytes so far (the threshold once finished)
constexpr int PRE_STATE_WORDS = PRE_LEVELS + 2;

// sampling stride for n keys: the sparsest power of two in [PRE_STRIDE_MIN,
// PRE_STRIDE_MAX] that still samples PRE_SAMPLE_CHUNKS chunks
inline uint32_t pre_stride_for(uint64_t n) {
  uint32_t s = PRE_STRIDE_MIN;
  while (s < PRE_STRIDE_MAX && (n >> 9) / (2ull * s) >= PRE_SAMPLE_CHUNKS) s <<= 1;
  return s;
}

DRTOPK_DEV uint64_t pre_chunk(uint64_t i, uint32_t stride) {
  return i * stride + ((i * 37u) & (stride - 1));
}

// After the pass of byte level `level` (by `ncta` CTAs of this select): the
// last CTA to finish walks levels 0..level over the complete histograms and
// publishes the prefix (and, when the walk ends here, the threshold's byte
// count).  Level l picks the bin holding the remaining target rank; from
// level 1 on the walk ends once the picked bin is small enough, or at the
// last level.  Block-collective.
DRTOPK_DEV void pre_publish(const FusedArgs& a, int level, uint32_t ncta) {
  __shared__ uint32_t s_last;
  uint32_t* st = a.pre_hist + PRE_STATE;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&st[level], 1u) == ncta - 1 ? 1u : 0u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  uint32_t prefix = 0, r = a.pre_target;
  int done = 0;
  for (int l = 0; l <= level; ++l) {
    const Pick p = block_pick<false>(a.pre_hist + 256 * l, 256, r);
    prefix = (prefix << 8) | p.b;
    r = r > p.above ? r - p.above : 1u;
    if (l >= 1 && (l == PRE_LEVELS - 1 ||
                   (uint64_t)p.cnt * a.pre_stride <= max(PRE_REFINE_KEYS, (uint64_t)a.k / 4))) {
      done = l + 1;
      break;
    }
  }
  if (threadIdx.x == 0) {
    st[PS_PREFIX] = prefix;
    __threadfence();
    if (done) st[PS_DONE] = (uint32_t)done;
  }
}

// 16 keys of 512-key chunk `ch` held by this lane (load q: keys
// ch*512 + 128 q + 4 lane + e), mapped to keys; positions >= n read as key 0
template <int KM>
DRTOPK_DEV void chunk_keys(const FusedArgs& a, uint64_t ch, uint64_t pol, uint32_t (&k)[4][4]) {
  const uint64_t cb = ch << 9;
  const unsigned lane = lane_id();
  const bool full = a.vec_ok && cb + 512 <= a.n;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint64_t base = cb + 128 * q + 4 * lane;
    if (full) {
      const uint4 v = ld_stream_v4(a.keys + base, pol);
      k[q][0] = v.x; k[q][1] = v.y; k[q][2] = v.z; k[q][3] = v.w;
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) k[q][e] = base + e < a.n ? __ldg(a.keys + base + e) : 0u;
    }
  }
}

template <int KM>
// Histogram of byte `level` of the sampled keys whose higher bytes equal
// `prefix` (all keys at level 0), added to pre_hist row `level`.
DRTOPK_DEV void presample_pass(const FusedArgs& a, int level, uint32_t prefix, uint32_t (*s_h)[256], uint32_t cta,
                               uint32_t ncta) {
  const unsigned lane = lane_id();
  const int wib = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < SPLIT_WARPS * 256; i += blockDim.x) (&s_h[0][0])[i] = 0;
  __syncthreads();
  const uint64_t ns = (a.n >> 9) / a.pre_stride;
  const uint64_t gw = (uint64_t)cta * SPLIT_WARPS + wib, nw = (uint64_t)ncta * SPLIT_WARPS;
  // PRE_ROUND sampled chunks per warp and round, all loaded before any is
  // counted (the pass is latency-bound); a small persistent grid keeps the
  // histogram flushes few
  for (uint64_t i = gw; i < ns; i += PRE_ROUND * nw) {
    uint32_t k[PRE_ROUND][4][4];
#pragma unroll
    for (int c = 0; c < PRE_ROUND; ++c) {
      const uint64_t ic = i + (uint64_t)c * nw;
      const uint64_t cb = pre_chunk(ic < ns ? ic : i, a.pre_stride) << 9;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint64_t base = cb + 128 * q + 4 * lane;
        if (a.vec_ok) {
          const uint4 v = __ldg(reinterpret_cast<const uint4*>(a.keys + base));
          k[c][q][0] = v.x; k[c][q][1] = v.y; k[c][q][2] = v.z; k[c][q][3] = v.w;
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e) k[c][q][e] = __ldg(a.keys + base + e);
        }
      }
    }
    const int sh = 24 - 8 * level;  // the byte counted; the prefix is every bit above it
#pragma unroll
    for (int c = 0; c < PRE_ROUND; ++c) {
      if (i + (uint64_t)c * nw >= ns) break;  // warp-uniform
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const uint32_t key = to_key<KM>(k[c][q][e]);
          if (level == 0) {
            hist_add_warp(s_h[wib], key >> 24);
          } else {
            // the whole warp takes part: one vote when every matching lane
            // counts the same byte (keys crowding into a few values), else
            // one shared atomic per matching lane (sparse matches)
            const bool hit = (key >> (sh + 8)) == prefix;
            const uint32_t bin = (key >> sh) & 255u;
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (m) {
              const int lead = __ffs(m) - 1;
              const uint32_t b0 = __shfl_sync(0xffffffffu, bin, lead);
              if (__all_sync(0xffffffffu, !hit || bin == b0)) {
                if ((int)lane == lead) atomicAdd(&s_h[wib][b0], (uint32_t)__popc(m));
              } else if (hit) {
                atomicAdd(&s_h[wib][bin], 1u);
              }
            }
          }
        }
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < 256; b += blockDim.x) {
    uint32_t c = 0;
#pragma unroll
    for (int w = 0; w < SPLIT_WARPS; ++w) c += s_h[w][b];
    if (c) atomicAdd(&a.pre_hist[256 * level + b], c);
  }
}

template <int KM>
DRTOPK_DEV void presample_body(const FusedArgs& a, uint32_t cta, uint32_t ncta) {
  __shared__ uint32_t s_h[SPLIT_WARPS][256];
  if (cta == 0 && threadIdx.x == 0) stamp(a.stats, 16);
  presample_pass<KM>(a, 0, 0u, s_h, cta, ncta);
  pre_publish(a, 0, ncta);
}

template <int KM>
DRTOPK_DEV void prerefine_body(const FusedArgs& a, int level, uint32_t cta, uint32_t ncta) {
  __shared__ uint32_t s_h2[SPLIT_WARPS][256];
  const uint32_t* st = a.pre_hist + PRE_STATE;
  if (ld_cg_u32(st + PS_DONE)) return;  // the threshold needs no further byte
  presample_pass<KM>(a, level, ld_cg_u32(st + PS_PREFIX), s_h2, cta, ncta);
  pre_publish(a, level, ncta);
}

template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS) k_presample(FusedArgs a) {
  presample_body<KM>(a, blockIdx.x, gridDim.x);
}

template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS) k_prerefine(FusedArgs a, int level) {
  prerefine_body<KM>(a, level, blockIdx.x, gridDim.x);
}

template <int KM>
DRTOPK_DEV void emit_body(const FusedArgs& a, uint32_t cta, uint32_t ncta, uint32_t* s_dyn) {
  const unsigned lane = lane_id();
  const int wib = threadIdx.x >> 5;
  uint2* cstage = reinterpret_cast<uint2*>(s_dyn) + (size_t)wib * GATHER_STAGE;
  // the predicted threshold: the prefix boundary (2 to 4 bytes) holding
  // pre_target sampled keys at or above it, as the last sample pass left it
  const uint32_t levels = ld_cg_u32(a.pre_hist + PRE_STATE + PS_DONE);
  const uint32_t prefix = ld_cg_u32(a.pre_hist + PRE_STATE + PS_PREFIX);
  const uint32_t thr = levels >= 4 ? prefix : (levels ? prefix << (32 - 8 * levels) : 0u);
  if (levels == 0 && threadIdx.x == 0) atomicOr(a.gb.err, (uint32_t)DE_INTERNAL);
  if (cta == 0 && threadIdx.x == 0) {
    *a.thr_word = thr;
    a.stats[ST_LVA] = levels;
    stamp(a.stats, 18);
  }
  // the candidates' largest key bounds level 0 of the second select
  // (k_cand_hist builds its histogram once the span is known)
  CandStage cst = {cstage, (uint32_t)GATHER_STAGE, 0u, thr, 0, 0u, 0u, false, true};
  uint32_t* s_hist = nullptr;
  const uint64_t pol = make_evict_first_policy();
  const uint64_t nchunks = (a.n + 511) >> 9;
  const uint64_t gw = (uint64_t)cta * SPLIT_WARPS + wib, nw = (uint64_t)ncta * SPLIT_WARPS;
  // register double buffer: the next chunk's loads are in flight while this
  // chunk is compared and compacted
  uint32_t kn[4][4];
  uint64_t ch = gw;
  if (ch < nchunks) chunk_keys<KM>(a, ch, pol, kn);
  for (; ch < nchunks; ch += nw) {
    uint32_t k[4][4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int e = 0; e < 4; ++e) k[q][e] = kn[q][e];
    if (ch + nw < nchunks) chunk_keys<KM>(a, ch + nw, pol, kn);
    const uint64_t cb = ch << 9;
    uint32_t take = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        k[q][e] = to_key<KM>(k[q][e]);
        take |= (uint32_t)(k[q][e] >= thr) << (4 * q + e);
      }
    if (cb + 512 > a.n) {  // the partial last chunk: drop positions >= n
      const uint32_t lim = (uint32_t)(a.n - cb);
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (128u * q + 4u * lane + e >= lim) take &= ~(1u << (4 * q + e));
    }
    if (!__any_sync(0xffffffffu, take != 0u)) continue;
    uint32_t tot = 0;
    const uint32_t off = warp_excl_scan(__popc(take), tot);
    uint32_t at = cst.reserve(a, s_hist, tot) + off;
    // few lanes take a key, and rarely more than one: walk the set bits and
    // pick each key out of the 16 registers with a select tree (no
    // dynamically indexed register array)
    const uint32_t i0 = (uint32_t)cb + 4 * lane;
    for (uint32_t t = take; t; t &= t - 1) {
      const int b = __ffs(t) - 1;
      uint32_t s8[8], s4[4], s2[2];
#pragma unroll
      for (int j = 0; j < 8; ++j) s8[j] = (b & 1) ? k[(2 * j + 1) >> 2][(2 * j + 1) & 3] : k[(2 * j) >> 2][(2 * j) & 3];
#pragma unroll
      for (int j = 0; j < 4; ++j) s4[j] = (b & 2) ? s8[2 * j + 1] : s8[2 * j];
#pragma unroll
      for (int j = 0; j < 2; ++j) s2[j] = (b & 4) ? s4[2 * j + 1] : s4[2 * j];
      const uint32_t key = (b & 8) ? s2[1] : s2[0];
      cstage[at++] = make_uint2(key, i0 + 128u * (uint32_t)(b >> 2) + (uint32_t)(b & 3));
    }
  }
  cst.drain(a, s_hist);
  if (cst.ovf) atomicOr(a.gb.err, (uint32_t)DE_OVERFLOW);
  uint32_t mx = cst.mhi;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  if (lane == 0 && mx) atomicMax(&a.cand_minmax[1], mx);
}

template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS, 4) k_emit(FusedArgs a) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  emit_body<KM>(a, blockIdx.x, gridDim.x, s_dyn);
}

// Level-0 histogram of the sampled-threshold path's candidates over
// [thr, largest candidate] (cand_level0_tight), for k_split0's pick
template <int KM>
DRTOPK_DEV void cand_hist_body(const FusedArgs& a, uint32_t cta, uint32_t ncta, uint32_t* s_dyn) {
  uint32_t* s_hist = s_dyn;
  const uint32_t thr = ld_cg_u32(a.thr_word);
  const uint32_t ncand = ld_cg_u32(a.cand_count);
  if (ncand < a.k || ncand > a.cand_cap) return;  // uniform: the last kernel falls back
  const Level L0 = cand_level0_tight(thr, ld_cg_u32(a.cand_minmax + 1), a.nbits, a.k);
  clear_hist(s_hist, a.nb);
  const uint64_t T = (uint64_t)blockDim.x * 8;
  for (uint64_t tb = (uint64_t)cta * T; tb < ncand; tb += (uint64_t)ncta * T) {
    uint32_t v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const uint64_t i = tb + (uint64_t)u * blockDim.x + threadIdx.x;
      v[u] = i < ncand ? ld_cg_u32(reinterpret_cast<const uint32_t*>(a.cand + i)) : 0u;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const bool in = tb + (uint64_t)u * blockDim.x + threadIdx.x < ncand;
      hist_add_conv(s_hist, in, bin_of(v[u], L0.lo, L0.w, L0.wshift));
    }
  }
  flush_hist(s_hist, a.C.H[0], a.nb);
}

template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS) k_cand_hist(FusedArgs a) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  cand_hist_body<KM>(a, blockIdx.x, gridDim.x, s_dyn);
}

// ---------------------------------------------------------------- grouped launches
// The served form runs the sampled-threshold selects admitted together as
// one chain of launches: every kernel covers all problems of a group (one
// key mode), each problem getting the CTAs a prefix table assigns it, and
// the last levels run one CTA per problem.  A CTA finds its problem by
// binary search in the prefix (cta_prefix[p] <= blockIdx.x <
// cta_prefix[p+1]) and copies the problem's arguments into shared memory.
struct GroupArgs {
  const FusedArgs* probs;
  const uint32_t* prefix;  // [nprob + 1] CTA prefix of this launch
  uint32_t nprob;
};

DRTOPK_DEV const FusedArgs& group_problem(const GroupArgs& g, FusedArgs* s_args, uint32_t& cta, uint32_t& ncta) {
  __shared__ uint32_t s_p;
  if (threadIdx.x == 0) {
    uint32_t lo = 0, hi = g.nprob;  // largest p with prefix[p] <= blockIdx.x
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (__ldg(g.prefix + mid) <= blockIdx.x) lo = mid;
      else hi = mid;
    }
    s_p = lo;
  }
  __syncthreads();
  const uint32_t p = s_p;
  const uint32_t* src = reinterpret_cast<const uint32_t*>(g.probs + p);
  uint32_t* dst = reinterpret_cast<uint32_t*>(s_args);
  for (int i = threadIdx.x; i < (int)(sizeof(FusedArgs) / 4); i += blockDim.x) dst[i] = __ldg(src + i);
  cta = blockIdx.x - __ldg(g.prefix + p);
  ncta = __ldg(g.prefix + p + 1) - __ldg(g.prefix + p);
  __syncthreads();
  return *s_args;
}

template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS) k_presample_g(GroupArgs g) {
  __shared__ FusedArgs s_args;
  uint32_t cta, ncta;
  const FusedArgs& a = group_problem(g, &s_args, cta, ncta);
  presample_body<KM>(a, cta, ncta);
}

template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS) k_prerefine_g(GroupArgs g, int level) {
  __shared__ FusedArgs s_args;
  uint32_t cta, ncta;
  const FusedArgs& a = group_problem(g, &s_args, cta, ncta);
  prerefine_body<KM>(a, level, cta, ncta);
}

template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS, 4) k_emit_g(GroupArgs g) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  __shared__ FusedArgs s_args;
  uint32_t cta, ncta;
  const FusedArgs& a = group_problem(g, &s_args, cta, ncta);
  emit_body<KM>(a, cta, ncta, s_dyn);
}

template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS) k_cand_hist_g(GroupArgs g) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  __shared__ FusedArgs s_args;
  uint32_t cta, ncta;
  const FusedArgs& a = group_problem(g, &s_args, cta, ncta);
  cand_hist_body<KM>(a, cta, ncta, s_dyn);
}

template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS, 4) k_split0_g(GroupArgs g) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  __shared__ FusedArgs s_args;
  uint32_t cta, ncta;
  const FusedArgs& a = group_problem(g, &s_args, cta, ncta);
  split0_body<KM>(a, cta, ncta, s_dyn);
}

// the device error word of every problem of a group, gathered for one copy
// back (the served form retries problems flagged DE_RETRY)
static __global__ void k_group_errors(const FusedArgs* probs, uint32_t nprob, uint32_t* out) {
  for (uint32_t i = threadIdx.x; i < nprob; i += blockDim.x) out[i] = ld_cg_u32(probs[i].gb.err);
}

// the last levels: CTA p runs problem p alone
template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS) k_fused_one_g(GroupArgs g) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  __shared__ FusedArgs s_args;
  uint32_t cta, ncta;
  const FusedArgs& a = group_problem(g, &s_args, cta, ncta);
  Team t = {};
  t.rank = 0;
  t.size = 1;
  t.cluster = 2;
  fused_body<KM>(a, t, s_dyn);
}

}  // namespace drtopk
