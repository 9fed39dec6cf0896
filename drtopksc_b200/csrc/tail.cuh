// tail.cuh -- the phases after the sampler for SMALL problems, in one CTA
// and in shared memory.
//
// For a small problem the team kernel's cost is not bandwidth: every level
// of every select is a chain of dependent global-memory round trips
// (histogram flush, pick, append counters, barrier) of ~1 us each.  Here one
// CTA keeps the sets in shared memory instead, so the whole tail costs about
// two dependent global reads (the delegate vector, then the keys of the kept
// subranges):
//   1. first select on the delegates   -- levels in shared memory
//   2. keep / filter (beta)            -- in shared memory
//   3. concatenation                   -- keys >= threshold of the kept
//                                         subranges, appended in shared memory
//   4. second select                   -- one bitonic sort for small candidate
//                                         sets, else levels + tie fill
//   5. output (sorted in shared memory when asked)
// Same integer rules as the team path (engine.cuh / fused.cuh: the same pick,
// advance and lowest-payload tie fill), so thresholds, counts and results
// are identical.  If the candidates outgrow shared memory, the cluster that
// the CTA belongs to runs the general path (fused_body).
#pragma once

#include "fused.cuh"

namespace drtopk {

constexpr int TAIL_CAP = 8192;      // entries per shared-memory set buffer
constexpr int TAIL_THREADS = 512;
constexpr int TAIL_SORT = 2048;     // candidate sets up to this size are finished by one sort
constexpr int TAIL_CLUSTER = 8;     // CTAs of the cluster (rank 0 runs the tail)
// dynamic shared memory: 256-word histogram + three TAIL_CAP-entry buffers
constexpr size_t TAIL_SMEM = 256 * 4 + 3 * (size_t)TAIL_CAP * 8;

// Levels of a select over sA[0..n) in shared memory (one CTA): keys above the
// chosen range go to T (after *s_ntop entries; skipped with c.thr_only), the
// members of the range become the next set.  Returns with the final range's
// members in sA (count n), L the final level, j the levels run so far;
// false if the level cap was reached.
DRTOPK_DEV bool smem_levels(const EngineCfg& c, Level& L, int& j, uint2*& sA, uint2*& sB, uint32_t& n, uint2* T,
                            uint32_t* s_ntop, uint32_t* s_hist) {
  __shared__ uint32_t s_n;
  for (;;) {
    if (j >= MAX_LEVELS) return false;
    const Pick p = smem_level_pick(sA, n, L, c.nb, s_hist);
    Level N;
    const bool done = advance(c, L, p, j, N);
    if (p.cnt != n) {  // else the whole set is in the chosen bin: nothing moves
      if (threadIdx.x == 0) s_n = 0;
      __syncthreads();
      split_block(sA, n, N.lo, N.hi, !c.thr_only, T, s_ntop, sB, &s_n);
      n = s_n;
      uint2* t = sA; sA = sB; sB = t;
    }
    L = N;
    ++j;
    if (done) return true;
  }
}

// Tie fill after the levels: the R = L.R lowest payloads among the n entries
// of the final range (all of them when n == R) are appended to T.  scratch
// holds >= n 64-bit words.  false if n < R.
DRTOPK_DEV bool smem_fill(const Level& L, const uint2* sA, uint32_t n, uint2* T, uint32_t* s_ntop, uint2* scratch) {
  const uint32_t R = L.R;
  if (n < R) return false;
  const uint32_t base = *s_ntop;
  if (n == R) {
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) T[base + i] = sA[i];
  } else {
    uint64_t* w = reinterpret_cast<uint64_t*>(scratch);
    int np2 = 1;
    while (np2 < (int)n) np2 <<= 1;
    for (int i = threadIdx.x; i < np2; i += blockDim.x)
      w[i] = i < (int)n ? (((uint64_t)sA[i].y << 32) | sA[i].x) : ~0ull;
    block_bitonic_asc(w, np2);
    for (uint32_t i = threadIdx.x; i < R; i += blockDim.x)
      T[base + i] = make_uint2((uint32_t)w[i], (uint32_t)(w[i] >> 32));
  }
  __syncthreads();
  if (threadIdx.x == 0) *s_ntop = base + R;
  __syncthreads();
  return true;
}

// keys >= thr of the listed subranges (ids in T[i].y or ids1[i]) appended to
// cand[] with their indices; *s_ovf set if more than TAIL_CAP would be kept
template <int KM>
DRTOPK_DEV void smem_gather(const FusedArgs& a, const uint2* T, const uint32_t* ids1, uint32_t nsub, uint32_t thr,
                            uint2* cand, uint32_t* s_cnt, uint32_t* s_ovf) {
  const int alpha = a.alpha;
  const uint64_t S = 1ull << alpha;
  const int gshift = alpha >= 2 ? 2 : alpha;
  const int gk = 1 << gshift;
  const uint32_t units = (uint32_t)(((uint64_t)nsub * S) >> gshift);
  constexpr int U = 8;  // granules per thread in flight
  for (uint32_t tb = 0; tb < units; tb += blockDim.x * U) {
    uint32_t v[U][4];
    uint32_t base[U];
#pragma unroll
    for (int q = 0; q < U; ++q) {
      const uint32_t u = tb + q * blockDim.x + threadIdx.x;
      base[q] = 0;
      v[q][0] = v[q][1] = v[q][2] = v[q][3] = 0u;
      if (u < units) {
        const uint64_t pos = (uint64_t)u << gshift;
        const uint32_t sel = (uint32_t)(pos >> alpha);
        const uint32_t sub = T ? T[sel].y : ids1[sel];
        base[q] = (uint32_t)(((uint64_t)sub << alpha) + (pos & (S - 1)));
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
    for (int q = 0; q < U; ++q) {
      const uint32_t u = tb + q * blockDim.x + threadIdx.x;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const bool take = u < units && e < gk && (uint64_t)base[q] + e < a.n && v[q][e] >= thr;
        const uint32_t slot = warp_append(take, s_cnt);
        if (take) {
          if (slot < (uint32_t)TAIL_CAP) cand[slot] = make_uint2(v[q][e], base[q] + e);
          else *s_ovf = 1u;
        }
      }
    }
  }
}

// The whole tail in shared memory; false = the candidates did not fit (the
// caller runs the general path; nothing global has been written but stats).
template <int KM>
DRTOPK_DEV bool tail_small(const FusedArgs& a, uint32_t* s_dyn) {
  uint32_t* s_hist = s_dyn;
  uint2* bufA = reinterpret_cast<uint2*>(s_dyn + 256);
  uint2* bufB = bufA + TAIL_CAP;
  uint2* T = bufB + TAIL_CAP;
  __shared__ uint32_t s_ntop, s_cnt, s_nsel, s_ovf;
  const bool lead = threadIdx.x == 0;
  const int D = 32 / a.nbits;
  auto fail = [&]() {
    if (lead) atomicOr(a.gb.err, (uint32_t)DE_INTERNAL);
    return true;
  };
  if (lead) {
    stamp(a.stats, 16);
    s_ntop = 0; s_cnt = 0; s_nsel = 0; s_ovf = 0;
  }
  __syncthreads();
  // ---- 1-2: first select on the delegates, keep / filter
  uint32_t thr1 = 0, nsel = 0, nlonely = 0;
  int lvA = 0;
  uint2* sA = bufA;
  uint2* sB = bufB;
  uint32_t n = 0;
  if (a.path == PATH_DEFAULT || a.path == PATH_BETA) {
    const uint32_t Md = (uint32_t)(a.path == PATH_BETA ? 2 * a.M : a.M);
    block_load_loop<8>(Md, [&](uint32_t i) { return __ldg(a.del + i); },
                       [&](uint32_t i, uint32_t v) { sA[i] = make_uint2(v, i); });
    __syncthreads();
    n = Md;
    EngineCfg c = {};
    c.bucket = 0; c.nbits = a.nbits; c.nb = a.nb; c.key_from_payload = 0;
    if (a.path == PATH_DEFAULT) { c.stop_single = 1; c.thr_only = 0; c.max_levels = D; }
    else { c.stop_single = 0; c.thr_only = 1; c.max_levels = a.first_levels; c.adapt_cnt = a.adapt_first; }
    if (!(a.path == PATH_BETA && c.max_levels <= 0)) {
      Level L = radix_level0(a.nbits, a.k);
      int j = 0;
      if (!smem_levels(c, L, j, sA, sB, n, T, &s_ntop, s_hist)) return fail();
      lvA = j;
      thr1 = L.lo;
      if (a.path == PATH_DEFAULT) {
        if (!smem_fill(L, sA, n, T, &s_ntop, sB)) return fail();
        if (s_ntop != a.k) return fail();
      }
    }
    if (lead) stamp(a.stats, 18);
    if (a.path == PATH_DEFAULT) {
      smem_gather<KM>(a, T, nullptr, a.k, thr1, bufA, &s_cnt, &s_ovf);
    } else {
      // filter (FindTopKRanges_beta): Max and Second >= thr -> whole
      // subrange; Max only -> that key is a candidate
      uint32_t* selids = reinterpret_cast<uint32_t*>(T);
      block_load_loop<8>(
          (uint32_t)a.M, [&](uint32_t jj) { return __ldg(reinterpret_cast<const uint2*>(a.del) + jj); },
          [&](uint32_t jj, uint2 d) {
            const bool sel = d.x >= thr1 && d.y >= thr1;
            const bool lone = d.x >= thr1 && d.y < thr1;
            const uint32_t s1 = warp_append(sel, &s_nsel);
            const uint32_t s2 = warp_append(lone, &s_cnt);
            if (sel) selids[s1] = jj;
            if (lone) {
              uint32_t idx = jj << a.alpha;
              if (a.has_pos) idx += __ldg(a.pos + jj);
              if (s2 < (uint32_t)TAIL_CAP) bufA[s2] = make_uint2(d.x, idx);
              else s_ovf = 1u;
            }
          });
      __syncthreads();
      nsel = s_nsel;
      nlonely = min(s_cnt, (uint32_t)TAIL_CAP);
      smem_gather<KM>(a, nullptr, selids, nsel, thr1, bufA, &s_cnt, &s_ovf);
    }
  } else {
    // plain select: the keys themselves are the candidates
    if (a.n > (uint64_t)TAIL_CAP) return false;
    if (lead) stamp(a.stats, 18);
    block_load_loop<8>((uint32_t)a.n, [&](uint32_t i) { return __ldg(a.keys + i); },
                       [&](uint32_t i, uint32_t v) { bufA[i] = make_uint2(to_key<KM>(v), i); });
    if (lead) s_cnt = (uint32_t)a.n;
  }
  __syncthreads();
  if (s_ovf) return false;
  const uint32_t ncand = s_cnt;
  if (lead) stamp(a.stats, 20);
  // ---- 3: second select over the candidates
  if (ncand < a.k) return fail();
  uint32_t K = 0;
  int lvC = 0;
  bool in_order = false;  // T already sorted (value desc, index asc)
  if (ncand <= (uint32_t)TAIL_SORT) {
    // one bitonic sort of (key << 32 | ~index), descending: its first k
    // entries are exactly the top-k with ties broken by lowest index, and the
    // k-th key is the k-th largest -- the same answer as the levels
    uint64_t* w = reinterpret_cast<uint64_t*>(bufB);
    int np2 = 1;
    while (np2 < (int)ncand) np2 <<= 1;
    for (int i = threadIdx.x; i < np2; i += blockDim.x)
      w[i] = i < (int)ncand ? (((uint64_t)bufA[i].x << 32) | (uint64_t)(~bufA[i].y)) : 0ull;
    block_bitonic_desc(w, np2);
    for (uint32_t i = threadIdx.x; i < a.k; i += blockDim.x)
      T[i] = make_uint2((uint32_t)(w[i] >> 32), ~(uint32_t)w[i]);
    K = (uint32_t)(w[a.k - 1] >> 32);
    if (lead) s_ntop = a.k;
    in_order = true;
    __syncthreads();
  } else {
    sA = bufA;
    sB = bufB;
    n = ncand;
    __syncthreads();
    if (lead) s_ntop = 0;
    __syncthreads();
    EngineCfg cc = {};
    cc.bucket = 0; cc.nbits = a.nbits; cc.nb = a.nb; cc.stop_single = 1;
    cc.max_levels = MAX_LEVELS; cc.thr_only = 0; cc.key_from_payload = 0;
    Level L = cand_level0(thr1, a.nbits, a.k);  // every candidate is >= thr1 (0 on the plain path)
    int j = 0;
    if (!smem_levels(cc, L, j, sA, sB, n, T, &s_ntop, s_hist)) return fail();
    K = (n == 1) ? sA[0].x : L.lo;
    if (!smem_fill(L, sA, n, T, &s_ntop, sB)) return fail();
    lvC = j;
  }
  const uint32_t ntop = s_ntop;
  if (lead) {
    stamp(a.stats, 22);
    if (a.out_kth) a.out_kth[0] = from_key(K, a.km);
    a.stats[ST_THR1] = thr1;
    a.stats[ST_NSEL] = a.path == PATH_DEFAULT ? a.k : nsel;
    a.stats[ST_NLONELY] = nlonely;
    a.stats[ST_NCAND] = ncand;
    a.stats[ST_LVA] = lvA;
    a.stats[ST_LVC] = lvC;
    a.stats[ST_TOPA] = a.path == PATH_DEFAULT ? a.k : 0u;
    a.stats[ST_TOPC] = ntop;
    a.stats[ST_KTH] = K;
    a.stats[ST_OK] = 1;
    if (ntop != a.k) atomicOr(a.gb.err, (uint32_t)DE_INTERNAL);
  }
  if (ntop != a.k || (!a.out_vals && !a.out_idx)) return true;
  // ---- 4: output
  if (!a.sorted || in_order) {
    for (uint32_t i = threadIdx.x; i < a.k; i += blockDim.x) {
      const uint2 e = T[i];
      if (a.out_vals) a.out_vals[i] = from_key(e.x, a.km);
      if (a.out_idx) a.out_idx[i] = (int64_t)e.y;
    }
    return true;
  }
  uint64_t* s = reinterpret_cast<uint64_t*>(bufA);
  int np2 = 1;
  while (np2 < (int)a.k) np2 <<= 1;
  for (int i = threadIdx.x; i < np2; i += blockDim.x)
    s[i] = i < (int)a.k ? (((uint64_t)T[i].x << 32) | (uint64_t)(~T[i].y)) : 0ull;
  block_bitonic_desc(s, np2);
  for (int i = threadIdx.x; i < (int)a.k; i += blockDim.x) {
    const uint64_t v = s[i];
    if (a.out_vals) a.out_vals[i] = from_key((uint32_t)(v >> 32), a.km);
    if (a.out_idx) a.out_idx[i] = (int64_t)(uint32_t)(~(uint32_t)v);
  }
  return true;
}

// One thread-block cluster of TAIL_CLUSTER CTAs: rank 0 runs the
// shared-memory tail; if its candidates did not fit, the whole cluster runs
// the general path (the other CTAs only wait at one cluster barrier).
template <int KM>
__global__ void __launch_bounds__(TAIL_THREADS) k_tail(FusedArgs a) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  const Team tm = cluster_team();
  if (tm.rank == 0) {
    const bool done = tail_small<KM>(a, s_dyn);
    if (threadIdx.x == 0) *a.tail_flag = done ? 1u : 2u;
  }
  team_sync(tm);
  if (ld_cg_u32(a.tail_flag) == 1u) return;
  fused_body<KM>(a, tm, s_dyn);
}

}  // namespace drtopk
