// bitonic.cuh -- Dr.Top-k bitonic top-k variant
// (reference: bitonic/bitonic_com.cuh 609-728 bitonic_firstTopk / bitonic,
// kernels Combined_Sigmod_Merge(_firstTopK) 100-386 and
// Combined_Sigmod_MergeRebuild(_firstTopk) 387-608; driver
// bitonic/sampleBitonic.cu:192-336).
//
// The reference's network per shared-memory tile: sort runs of k with
// alternating direction, take the elementwise max of each (ascending,
// descending) run pair -- that is the top k of the 2k as a bitonic sequence
// -- rebuild it with a bitonic merge, and repeat until one run of k is left;
// tiles shrink the array by tile/k per pass.  Here the elements are 64-bit
// composites (key << 32 | ~index), so the network's max picks the larger key
// and, among equal keys, the lower index: the result is the exact top-k with
// lowest-index ties, already sorted.
//
// Path (one cooperative kernel, grid barriers between passes):
//   1. (sampler, beta=1) delegates;
//   2. bitonic top-k of (delegate, subrange id) -> the k subranges with the
//      largest delegates;
//   3. concatenation of their keys >= the k-th delegate (the reference copies
//      the k subranges whole; keys below the k-th delegate can never be in
//      the top k, so dropping them changes no result);
//   4. bitonic top-k of (key, index) over the concatenation -> sorted output.
// NormalBitonic=1 skips 1-3 and runs step 4 over all keys
// (sampleBitonic.cu:305-310).
#pragma once

#include "fused.cuh"

namespace drtopk {

constexpr int BITONIC_TILE = 4096;  // composites per CTA tile (32 KB of shared memory)
constexpr int BITONIC_MAX_K = 2048;

struct BitonicArgs {
  const uint32_t* keys;
  uint64_t n;
  uint32_t k;
  int km;
  int alpha;
  uint64_t M;
  int normal;            // 1: no delegates (plain bitonic top-k)
  int vec_ok;
  const uint32_t* del;   // [M] delegates (beta=1)
  uint64_t* buf[2];      // ping-pong composite buffers
  uint64_t buf_cap;
  uint32_t* cand_count;
  uint32_t* out_kth;
  uint32_t* out_vals;
  int64_t* out_idx;
  uint32_t* stats;
  GridBar gb;
};

// compare-exchange network helpers over s[0..T) with 256 threads
DRTOPK_DEV void cmpx(uint64_t* s, int i, int j, bool asc) {
  uint64_t a = s[i], b = s[j];
  if ((a > b) == asc) { s[i] = b; s[j] = a; }
}

// sort every run of k in s[0..T): run r ascending if r is even, else
// descending (the bitonic sort network stopped at size k leaves exactly this
// alternation, since the direction of a size block is (lo & size) == 0)
DRTOPK_DEV void sort_runs(uint64_t* s, int T, int k) {
  for (int size = 2; size <= k; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < T / 2; i += blockDim.x) {
        const int lo = 2 * stride * (i / stride) + (i % stride);
        cmpx(s, lo, lo + stride, (lo & size) == 0);
      }
      __syncthreads();
    }
  }
}

// bitonic merge (rebuild) of every run of k: run r ascending if r even
DRTOPK_DEV void rebuild_runs(uint64_t* s, int T, int k) {
  for (int stride = k >> 1; stride > 0; stride >>= 1) {
    for (int i = threadIdx.x; i < T / 2; i += blockDim.x) {
      const int lo = 2 * stride * (i / stride) + (i % stride);
      const int hi = lo + stride;
      const bool asc = ((lo / k) & 1) == 0;
      cmpx(s, lo, hi, asc);
    }
    __syncthreads();
  }
}

// top-k of a tile of T composites (T a power of two >= 2k); leaves the k
// largest in s[0..k) sorted ascending.
DRTOPK_DEV void tile_topk(uint64_t* s, int T, int k) {
  __syncthreads();
  sort_runs(s, T, k);
  int len = T;
  while (len > k) {
    // run pairs (2r ascending, 2r+1 descending): elementwise max -> run r
    const int half = len / 2;
    uint64_t v[BITONIC_TILE / 2 / FUSED_THREADS];
    int c = 0;
    for (int i = threadIdx.x; i < half; i += blockDim.x, ++c) {
      const int r = i / k, j = i % k;
      v[c] = max(s[2 * r * k + j], s[(2 * r + 1) * k + j]);
    }
    __syncthreads();
    c = 0;
    for (int i = threadIdx.x; i < half; i += blockDim.x, ++c) s[i] = v[c];
    __syncthreads();
    len = half;
    rebuild_runs(s, len, k);
  }
}

// one reduction pass: tiles of T over src[0..count) -> dst (k per tile)
// returns the output count (uniform).  Source entries are produced by `load`.
template <typename L>
DRTOPK_DEV uint64_t bitonic_pass(uint64_t count, int k, uint64_t* s, uint64_t* dst, L&& load) {
  const int T = BITONIC_TILE;
  const uint64_t ntiles = (count + T - 1) / T;
  for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    for (int i = threadIdx.x; i < T; i += blockDim.x) {
      const uint64_t g = t * T + i;
      s[i] = g < count ? load(g) : 0ull;
    }
    tile_topk(s, T, k);
    // keep the tile's k largest (s[0..k) ascending)
    for (int i = threadIdx.x; i < k; i += blockDim.x) dst[t * k + i] = s[i];
    __syncthreads();
  }
  return ntiles * (uint64_t)k;
}

template <int KM>
__global__ void __launch_bounds__(FUSED_THREADS) k_bitonic(BitonicArgs a) {
  extern __shared__ __align__(16) uint32_t s_dyn[];
  uint64_t* s = reinterpret_cast<uint64_t*>(s_dyn);
  const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
  const int k = (int)a.k;
  int cur = 0;
  uint64_t count;
  if (!a.normal) {
    // ---- top-k subranges by (delegate, lowest id)
    count = bitonic_pass(a.M, k, s, a.buf[0], [&](uint64_t j) {
      return ((uint64_t)a.del[j] << 32) | (uint64_t)(uint32_t)~(uint32_t)j;
    });
    if (!grid_barrier(a.gb)) return;
    while (count > (uint64_t)k) {
      const uint64_t* src = a.buf[cur];
      count = bitonic_pass(count, k, s, a.buf[cur ^ 1], [&](uint64_t g) { return ld_cg_u64(src + g); });
      cur ^= 1;
      if (!grid_barrier(a.gb)) return;
    }
    // buf[cur][0..k) ascending: [0] holds the k-th delegate
    const uint64_t* top = a.buf[cur];
    const uint32_t thr = (uint32_t)(ld_cg_u64(top) >> 32);
    // ---- concatenation of keys >= thr of the k subranges (composites)
    uint64_t* cand = a.buf[cur ^ 1];
    const uint64_t S = 1ull << a.alpha;
    const uint64_t units = ((uint64_t)k * S) >> 2;
    const uint64_t g0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t G = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t iters = (units + G - 1) / G;
    for (uint64_t it = 0; it < iters; ++it) {
      const uint64_t u = it * G + g0;
      const bool valid = u < units;
      uint64_t base = 0;
      uint32_t v[4] = {0u, 0u, 0u, 0u};
      if (valid) {
        const uint64_t q = u << 2;
        const uint32_t sub = ~(uint32_t)ld_cg_u64(top + (q >> a.alpha));
        base = ((uint64_t)sub << a.alpha) + (q & (S - 1));
        if (a.vec_ok && base + 4 <= a.n) {
          uint4 x = __ldg(reinterpret_cast<const uint4*>(a.keys + base));
          v[0] = to_key<KM>(x.x); v[1] = to_key<KM>(x.y); v[2] = to_key<KM>(x.z); v[3] = to_key<KM>(x.w);
        } else {
          for (int e = 0; e < 4; ++e) v[e] = (base + e < a.n) ? to_key<KM>(__ldg(a.keys + base + e)) : 0u;
        }
      }
      for (int e = 0; e < 4; ++e) {
        const bool take = valid && base + e < a.n && v[e] >= thr;
        const uint32_t slot = warp_append(take, a.cand_count);
        if (take && slot < a.buf_cap)
          cand[slot] = ((uint64_t)v[e] << 32) | (uint64_t)(uint32_t)~(uint32_t)(base + e);
      }
    }
    if (!grid_barrier(a.gb)) return;
    count = ld_cg_u32(a.cand_count);
    if (count > a.buf_cap || count < (uint64_t)k) {
      if (lead) atomicOr(a.gb.err, (uint32_t)DE_INTERNAL);
      return;
    }
    cur ^= 1;
    if (lead) { a.stats[ST_NSEL] = a.k; a.stats[ST_NCAND] = (uint32_t)count; a.stats[ST_THR1] = thr; }
  } else {
    count = bitonic_pass(a.n, k, s, a.buf[0], [&](uint64_t g) {
      return ((uint64_t)to_key<KM>(__ldg(a.keys + g)) << 32) | (uint64_t)(uint32_t)~(uint32_t)g;
    });
    cur = 0;
    if (!grid_barrier(a.gb)) return;
    if (lead) a.stats[ST_NCAND] = (uint32_t)a.n;
  }
  // ---- bitonic top-k of the candidates
  do {
    const uint64_t* src = a.buf[cur];
    count = bitonic_pass(count, k, s, a.buf[cur ^ 1], [&](uint64_t g) { return ld_cg_u64(src + g); });
    cur ^= 1;
    if (!grid_barrier(a.gb)) return;
  } while (count > (uint64_t)k);
  // buf[cur][0..k) ascending -> output descending
  const uint64_t* res = a.buf[cur];
  const uint64_t g0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t G = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = g0; i < (uint64_t)k; i += G) {
    const uint64_t c = ld_cg_u64(res + (k - 1 - i));
    if (a.out_vals) a.out_vals[i] = from_key((uint32_t)(c >> 32), a.km);
    if (a.out_idx) a.out_idx[i] = (int64_t)(uint32_t)~(uint32_t)c;
  }
  if (lead) {
    const uint64_t c = ld_cg_u64(res);
    if (a.out_kth) a.out_kth[0] = from_key((uint32_t)(c >> 32), a.km);
    a.stats[ST_KTH] = (uint32_t)(c >> 32);
    a.stats[ST_OK] = 1;
  }
}

}  // namespace drtopk
