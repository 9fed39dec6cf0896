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
//            are warp-aggregated; the same pass histograms the candidates'
//            top digit (first level of phase 3).
//   phase 3  second select over the candidates (radix_select_inplace
//            1410-1470): exact k-th largest, plus the top-k list with ties
//            broken by lowest index.
//   phase 4  output: k-th value, top-k values/indices (optionally sorted by
//            value desc, index asc).
#pragma once

#include "engine.cuh"

namespace drtopk {

enum Path : int { PATH_DEFAULT = 0, PATH_BETA = 1, PATH_PLAIN = 2, PATH_BITONIC = 3 };

constexpr int SMALL_SORT = 4096;  // top-k sorted in one CTA's shared memory up to this k

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
  uint32_t* sort_tot;     // [8][256]
  uint32_t* stats;        // [16]
  uint32_t* thr_word;     // threshold handed between launches in split mode
  uint32_t* tail_flag;    // shared-memory tail: 1 done, 2 fall back to the general path
  int phase_lo, phase_hi; // phases run by this launch of k_fused (1..3)
  GridBar gb;
};

enum StatSlot : int {
  ST_THR1 = 0, ST_NSEL = 1, ST_NLONELY = 2, ST_NCAND = 3, ST_LVA = 4, ST_LVC = 5,
  ST_TOPA = 6, ST_TOPC = 7, ST_KTH = 8, ST_OK = 9
};

// --------------------------------------------------------------- gathers
template <int KM>
DRTOPK_DEV void emit_candidate(const FusedArgs& a, bool take, uint32_t key, uint32_t idx, uint32_t* s_hist,
                               uint32_t& mlo, uint32_t& mhi, bool& ovf) {
  uint32_t slot = warp_append(take, a.cand_count);
  if (take) {
    if (slot < a.cand_cap) a.cand[slot] = make_uint2(key, idx);
    else ovf = true;
    if (a.bucket) { mlo = max(mlo, ~key); mhi = max(mhi, key); }
    else hist_add_warp(s_hist, key >> (32 - a.nbits));
  }
}

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
          else hist_add_warp(s_hist, key >> (32 - a.nbits));
        }
      }
  }
}

// beta path filter (FindTopKRanges_beta, radixselect.cuh:560-598): per
// subrange, Max >= thr and Second >= thr -> subrange id to the selected
// list; Max >= thr only -> Max itself is a candidate (with its position).
constexpr int FILTER_E = 8;

template <int KM>
DRTOPK_DEV void filter_beta(const Team& tm, const FusedArgs& a, uint32_t thr, uint32_t* s_hist, uint32_t& mlo,
                            uint32_t& mhi, bool& ovf) {
  const uint64_t T = (uint64_t)blockDim.x * FILTER_E;
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
        const bool s1 = d.x >= thr && d.y >= thr;
        const bool l1 = d.x >= thr && d.y < thr;
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
        else hist_add_warp(s_hist, m1[q] >> (32 - a.nbits));
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
  // totals of all 8 digits
  for (int d = 0; d < 8; ++d) {
    for (int i = t; i < 256; i += blockDim.x) s_cnt[i] = 0;
    __syncthreads();
    block_load_loop<8>(r1 - r0, [&](uint32_t i) { return ld_cg_u64(src + r0 + i); },
                       [&](uint32_t, uint64_t v) { atomicAdd(&s_cnt[(v >> (8 * d)) & 255u], 1u); });
    __syncthreads();
    for (int i = t; i < 256; i += blockDim.x)
      if (s_cnt[i]) atomicAdd(&a.sort_tot[d * 256 + i], s_cnt[i]);
    __syncthreads();
  }
  if (!team_sync(tm)) { ok = false; return src; }
  __shared__ uint32_t s_run[256];
  __shared__ uint32_t s_wcnt[MAX_BLOCK_WARPS][257];
  __shared__ int s_trivial;
  for (int d = 0; d < 8; ++d) {
    if (t == 0) s_trivial = 0;
    __syncthreads();
    for (int i = t; i < 256; i += blockDim.x)
      if (ld_cg_u32(a.sort_tot + d * 256 + i) == nk) s_trivial = 1;
    __syncthreads();
    if (s_trivial) continue;
    const int sh = 8 * d;
    // 1) this CTA's digit counts
    for (int i = t; i < 256; i += blockDim.x) s_cnt[i] = 0;
    __syncthreads();
    block_load_loop<8>(r1 - r0, [&](uint32_t i) { return ld_cg_u64(src + r0 + i); },
                       [&](uint32_t, uint64_t v) { atomicAdd(&s_cnt[(v >> sh) & 255u], 1u); });
    __syncthreads();
    for (int i = t; i < 256; i += blockDim.x) a.sort_cnt[(uint64_t)c * 256 + i] = s_cnt[i];
    if (!team_sync(tm)) { ok = false; return src; }
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
    if (!team_sync(tm)) { ok = false; return src; }
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
    // 4) stable scatter in chunks of blockDim keys
    const int wid = t >> 5;
    const unsigned lane = t & 31u;
    for (uint32_t cb = r0; cb < r1; cb += blockDim.x) {
      const uint32_t i = cb + t;
      const bool valid = i < r1;
      const uint64_t key = valid ? ld_cg_u64(src + i) : 0ull;
      const uint32_t dg = valid ? (uint32_t)((key >> sh) & 255u) : 256u;
      for (int q = lane; q < 257; q += 32) s_wcnt[wid][q] = 0;
      __syncwarp();
      const unsigned peers = __match_any_sync(0xffffffffu, dg);
      const uint32_t rank_in_warp = __popc(peers & ((1u << lane) - 1u));
      if (rank_in_warp == 0) s_wcnt[wid][dg] = __popc(peers);
      __syncthreads();
      if (valid) {
        uint32_t before_w = 0;
        for (int w2 = 0; w2 < wid; ++w2) before_w += s_wcnt[w2][dg];
        dst[s_run[dg] + before_w + rank_in_warp] = key;
      }
      __syncthreads();
      for (int q = t; q < 256; q += blockDim.x) {
        uint32_t add = 0;
        for (int w2 = 0; w2 < (int)(blockDim.x / 32); ++w2) add += s_wcnt[w2][q];
        s_run[q] += add;
      }
      __syncthreads();
    }
    if (!team_sync(tm)) { ok = false; return src; }
    uint64_t* tmp = src; src = dst; dst = tmp;
  }
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
  if (lead) stamp(a.stats, 16);

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
    EngineCfg c;
    c.bucket = a.bucket; c.nbits = a.nbits; c.nb = a.nb; c.key_from_payload = 0;
    if (a.path == PATH_DEFAULT) {
      c.stop_single = 1; c.thr_only = 0;
      c.max_levels = a.bucket ? MAX_LEVELS : D;
    } else {
      c.stop_single = 0; c.thr_only = 1;
      c.max_levels = a.first_levels;
    }
    if (a.path == PATH_BETA && c.max_levels <= 0) {
      thr1 = 0;  // no digit processed: every subrange qualifies
    } else {
      RunResult r = run_select<KM>(c, s, false, a.A, a.AF, L0, s_hist, tm, s_fast);
      if (!r.ok) { if (lead) atomicOr(a.gb.err, (uint32_t)DE_INTERNAL); return; }
      lvA = r.levels;
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
    filter_beta<KM>(tm, a, thr1, s_hist, mlo, mhi, ovf);
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
  if (a.path == PATH_PLAIN) {
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
    L0c = radix_level0(a.nbits, a.k);
  }
  EngineCfg cc;
  cc.bucket = a.bucket; cc.nbits = a.nbits; cc.nb = a.nb; cc.stop_single = 1;
  cc.max_levels = MAX_LEVELS; cc.thr_only = 0; cc.key_from_payload = 0;
  RunResult rc = run_select<KM>(cc, sc, pairs, a.C, a.CF, L0c, s_hist, tm, s_fast);
  if (!rc.ok) { if (lead) atomicOr(a.gb.err, (uint32_t)DE_INTERNAL); return; }
  const uint32_t K = rc.kth;
  const uint32_t ntop = ld_cg_u32(a.C.top_count);
  if (lead) {
    stamp(a.stats, 22);
    if (a.out_kth) a.out_kth[0] = from_key(K, a.km);
    a.stats[ST_THR1] = thr1;
    if (a.path == PATH_DEFAULT) a.stats[ST_NSEL] = a.k;
    a.stats[ST_NCAND] = a.path == PATH_PLAIN ? (uint32_t)a.n : ld_cg_u32(a.cand_count);
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
    team_load_loop<8>(tm, a.k, [&](uint64_t i) { return ld_cg_v2(reinterpret_cast<const uint32_t*>(a.C.top + i)); },
                      [&](uint64_t i, uint2 e) {
                        if (a.out_vals) a.out_vals[i] = from_key(e.x, a.km);
                        if (a.out_idx) a.out_idx[i] = (int64_t)e.y;
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

template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS) k_filter(FusedArgs a) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  uint32_t* s_hist = s_dyn;
  const uint32_t thr = ld_cg_u32(a.thr_word);
  clear_hist(s_hist, a.nb);
  uint32_t mlo = 0, mhi = 0;
  bool ovf = false;
  filter_beta<KM>(grid_team(a.gb), a, thr, s_hist, mlo, mhi, ovf);
  if (ovf) atomicOr(a.gb.err, (uint32_t)DE_OVERFLOW);
  flush_cand_stats(a, s_hist, mlo, mhi);
}

template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS) k_gather(FusedArgs a) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  uint32_t* s_hist = s_dyn;
  const uint32_t thr = ld_cg_u32(a.thr_word);
  const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
  uint64_t nsub;
  if (a.path == PATH_DEFAULT) {
    if (ld_cg_u32(a.A.top_count) != a.k) {  // uniform: written by the previous launch
      if (lead) atomicOr(a.gb.err, (uint32_t)DE_INTERNAL);
      return;
    }
    nsub = a.k;
  } else {
    nsub = ld_cg_u32(a.sel_count);
    if (nsub > a.M) {
      if (lead) atomicOr(a.gb.err, (uint32_t)DE_INTERNAL);
      return;
    }
    if (lead) a.stats[ST_NLONELY] = ld_cg_u32(a.cand_count);  // lonely candidates came first
  }
  clear_hist(s_hist, a.nb);
  uint32_t mlo = 0, mhi = 0;
  bool ovf = false;
  const Team tm = grid_team(a.gb);
  if (a.path == PATH_DEFAULT) gather_list<KM, 4>(tm, a, a.A.top, nullptr, nsub, thr, s_hist, mlo, mhi, ovf);
  else gather_list<KM, 4>(tm, a, nullptr, a.sel, nsub, thr, s_hist, mlo, mhi, ovf);
  if (ovf) atomicOr(a.gb.err, (uint32_t)DE_OVERFLOW);
  flush_cand_stats(a, s_hist, mlo, mhi);
}

}  // namespace drtopk
