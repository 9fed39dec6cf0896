// sampler.cuh -- delegate max-sampling, the streaming pass of Dr.Top-k.
//
// Semantics (reference: baseline+filter+beta+shuffle/radixselect.cuh):
//   beta=1  sampleMax (882-918): del[j] = max of subrange j = keys
//           [j*2^alpha, (j+1)*2^alpha) clipped to n.
//   beta=2  sampleMax_NoReduction_Beta2 (966-1041): del[2j] = Max,
//           del[2j+1] = Second (multiset second largest; 0 for a one-key
//           subrange, as the reference's Second=0 start gives).
// The reference launches one warp per subrange (beta=1) or stages 256
// subranges in padded shared memory (beta=2).  Here one kernel covers every
// alpha >= 1: warps walk 512-key chunks with four 128-bit evict-first loads
// per lane in flight, reduce inside the lane, then across the lanes that
// share a subrange with xor shuffles; small-subrange delegates are staged in
// shared memory so they leave as coalesced stores.  The same pass builds the
// histogram of the delegates' top digit (the first level of the first
// select) or, for bucket select, their min/max, so no extra pass over the
// delegate vector is needed to start the first select.
#pragma once

#include "common.cuh"

namespace drtopk {

struct SampleArgs {
  const uint32_t* keys;  // raw input (uint32 or float32 bits)
  uint64_t n;
  int alpha;             // log2 subrange size, >= 1
  int nbits;             // digit width for the fused histogram
  int hmode;             // 0 none, 1 top-digit histogram, 2 min/max
  int vec_ok;            // keys 16-byte aligned
  uint32_t* del;         // beta=1: [M]; beta=2: [2M] interleaved (Max, Second)
  uint16_t* pos;         // beta=2 with positions: offset of Max inside subrange j
  uint32_t* hist;        // [1<<nbits] (hmode 1)
  uint32_t* minmax;      // [2]: [0] = max(~v) (so min = ~[0]), [1] = max(v) (hmode 2)
  uint32_t* err;         // device error word
};

constexpr int SAMPLE_THREADS = 256;
constexpr int SAMPLE_WARPS = SAMPLE_THREADS / 32;

// lane-local accumulator: first, second (beta=2), position of first
struct Acc {
  uint32_t a1, a2, p1;
};

template <int BETA, bool POS>
DRTOPK_DEV void acc_push(Acc& s, uint32_t k, uint32_t p) {
  if (BETA == 2) {
    if (POS && k > s.a1) s.p1 = p;
    top2_push(s.a1, s.a2, k);
  } else {
    s.a1 = max(s.a1, k);
  }
}

template <int BETA, bool POS>
DRTOPK_DEV void acc_merge(Acc& s, const Acc& o) {
  if (BETA == 2) {
    if (POS && (o.a1 > s.a1 || (o.a1 == s.a1 && o.p1 < s.p1))) s.p1 = o.p1;
    top2_merge(s.a1, s.a2, o.a1, o.a2);
  } else {
    s.a1 = max(s.a1, o.a1);
  }
}

template <int BETA, bool POS>
DRTOPK_DEV Acc acc_shfl_xor(const Acc& s, int off) {
  Acc o;
  o.a1 = __shfl_xor_sync(0xffffffffu, s.a1, off);
  o.a2 = BETA == 2 ? __shfl_xor_sync(0xffffffffu, s.a2, off) : 0u;
  o.p1 = POS ? __shfl_xor_sync(0xffffffffu, s.p1, off) : 0u;
  return o;
}

// Four consecutive words [base, base+4).  A full row is returned RAW (the
// caller maps it to keys when it uses it, so the load can stay in flight
// meanwhile); a partial row is returned as keys, with positions >= n read
// as key 0 (the max identity).
template <int KM>
DRTOPK_DEV void load_row4(const SampleArgs& a, uint64_t base, uint64_t pol, bool full, uint32_t (&k)[4]) {
  if (full) {
    uint4 v = ld_stream_v4(a.keys + base, pol);
    k[0] = v.x; k[1] = v.y; k[2] = v.z; k[3] = v.w;
  } else {
#pragma unroll
    for (int e = 0; e < 4; ++e) k[e] = (base + e < a.n) ? to_key<KM>(ld_stream_u32(a.keys + base + e, pol)) : 0u;
  }
}

// A lane's 16 consecutive keys as 16/2^SA whole subranges of 2^SA keys
// (SA <= 3), with the lane's slot i holding its 128-bit word i ^ r (the
// rotation that makes the shared-memory transpose conflict-free).  The xor
// keeps every subrange inside one group of slots, so the groups are reduced
// in slot order and stored at their true subrange index.
template <int SA, int BETA, bool POS>
DRTOPK_DEV void small_subranges(const uint32_t (&k)[4][4], int r, uint32_t* stage, uint16_t* pstage, unsigned lane) {
  constexpr int S_ = 1 << SA, per = 16 >> SA;
#pragma unroll
  for (int j = 0; j < per; ++j) {
    Acc acc = {0u, 0u, 0u};
    int sub = 0;
#pragma unroll
    for (int t = 0; t < S_; ++t) {
      const int q = j * S_ + t;                     // slot-order key index
      const int key = 4 * ((q >> 2) ^ r) + (q & 3);  // index among the lane's 16 keys
      sub = key >> SA;
      acc_push<BETA, POS>(acc, k[q >> 2][q & 3], (uint32_t)(key & (S_ - 1)));
    }
    const int d = (int)lane * per + sub;
    if (BETA == 2) {
      stage[2 * d] = acc.a1;
      stage[2 * d + 1] = acc.a2;
      if (POS) pstage[d] = (uint16_t)acc.p1;
    } else {
      stage[d] = acc.a1;
    }
  }
}

// WIDE: subranges of >= 512 keys (alpha >= 9), one warp per subrange;
// otherwise 512-key chunks of 512/2^alpha subranges (alpha 1..8).  The two
// are separate kernels so that each gets its own registers, shared memory
// and occupancy.  Each warp counts the delegates' top digits in its own
// shared histogram (delegates crowd into a few top bins, so one histogram
// per CTA made every warp's atomics meet on the same word); the copies are
// summed once at the end.
template <int KM, int BETA, bool POS, bool WIDE>
__global__ void __launch_bounds__(SAMPLE_THREADS, POS ? 2 : 4) k_sample(SampleArgs a) {
  __shared__ uint32_t s_hist[SAMPLE_WARPS][256];
  __shared__ uint32_t s_stage[WIDE ? 1 : SAMPLE_WARPS][WIDE ? 1 : 256 * BETA];
  __shared__ uint16_t s_pstage[WIDE ? 1 : SAMPLE_WARPS][(POS && !WIDE) ? 256 : 1];
  __shared__ uint4 s_xpose[WIDE ? 1 : SAMPLE_WARPS][WIDE ? 1 : 128];  // per-warp transpose of one 512-key chunk
  __shared__ uint32_t s_mm[2];

  const int tid = threadIdx.x;
  const unsigned lane = tid & 31u;
  const int wib = tid >> 5;
  const int nb = 1 << a.nbits;
  const int dshift = 32 - a.nbits;
  if (a.hmode == 1)
    for (int i = tid; i < SAMPLE_WARPS * 256; i += SAMPLE_THREADS) (&s_hist[0][0])[i] = 0;
  if (tid < 2) s_mm[tid] = 0;
  __syncthreads();

  const uint64_t pol = make_evict_first_policy();
  const int alpha = a.alpha;
  const uint64_t S = 1ull << alpha;
  const uint64_t M = (a.n + S - 1) >> alpha;
  const uint64_t gwarp = (uint64_t)blockIdx.x * SAMPLE_WARPS + wib;
  const uint64_t nwarps = (uint64_t)gridDim.x * SAMPLE_WARPS;
  uint32_t mm_lo = 0, mm_hi = 0;  // lane-local max(~v), max(v) of emitted delegates

  auto emit_hist = [&](uint32_t v) {
    if (a.hmode == 1) hist_add_warp(s_hist[wib], v >> dshift);
    else if (a.hmode == 2) { mm_lo = max(mm_lo, ~v); mm_hi = max(mm_hi, v); }
  };

  if constexpr (WIDE) {
    // ---- one warp per subrange, 512-key chunks
    for (uint64_t j = gwarp; j < M; j += nwarps) {
      const uint64_t b = j << alpha;
      const uint64_t e = min(a.n, b + S);
      Acc s = {0u, 0u, 0u};
      for (uint64_t c = b; c < e; c += 512) {
        const bool full = a.vec_ok && (c + 512 <= e);
        uint32_t k[4][4];
#pragma unroll
        for (int r = 0; r < 4; ++r) load_row4<KM>(a, c + r * 128 + lane * 4, pol, full, k[r]);
        // full rows hold raw words (mapped here, after all four loads were issued)
        if (full) {
#pragma unroll
          for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int q = 0; q < 4; ++q)
              acc_push<BETA, POS>(s, to_key<KM>(k[r][q]), (uint32_t)(c - b) + r * 128 + lane * 4 + q);
        } else {
#pragma unroll
          for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc_push<BETA, POS>(s, k[r][q], (uint32_t)(c - b) + r * 128 + lane * 4 + q);
        }
      }
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) acc_merge<BETA, POS>(s, acc_shfl_xor<BETA, POS>(s, off));
      if (lane == 0) {
        if (BETA == 2) {
          *reinterpret_cast<uint2*>(a.del + 2 * j) = make_uint2(s.a1, s.a2);
          if (POS) a.pos[j] = (uint16_t)s.p1;
          emit_hist(s.a1);
          emit_hist(s.a2);
        } else {
          a.del[j] = s.a1;
          emit_hist(s.a1);
        }
      }
    }
  } else {
    // ---- 512-key chunks holding 512/S subranges (alpha 1..8).  Lane l
    // reduces keys [16 l, 16 l + 16) of the chunk: with G = max(1, S/16)
    // lanes per subrange its 16 keys belong to one subrange (reduced in-lane,
    // then log2(G) xor steps), and for S < 16 they are 16/S whole subranges
    // (no shuffles).  The keys arrive by fully coalesced 128-bit loads (load
    // i of lane l is the chunk's word 32 i + l, a 512-byte run per warp
    // instruction) and are regrouped through a 2 KB per-warp shared-memory
    // transpose; lane l reads its words back in the order (i ^ r), r = (l/2)
    // mod 4, which puts the 8 lanes of each quarter-warp on 8 distinct 16-byte
    // bank groups (no conflicts).  Loading the lane's 16 keys directly needs
    // 64-byte strides between lanes (16 cache lines per warp load) and
    // measured ~13 % slower even without any compute.
    const uint64_t nchunks = (a.n + 511) >> 9;
    const int G = alpha >= 4 ? min(32, 1 << (alpha - 4)) : 1;
    const int dpc = 512 >> alpha;  // delegates per chunk
    uint32_t* stage = s_stage[wib];
    uint4* xbuf = s_xpose[wib];
    const int grp = lane / G, gl = lane % G;
    const int r = (int)((lane >> 1) & 3u);
    // a full chunk is kept as raw words while its loads are in flight and
    // transposed and mapped when it is reduced; a partial (last) chunk is
    // loaded in the lane layout and mapped at load time, with positions >= n
    // as key 0
    auto load_chunk = [&](uint64_t ch, uint32_t (&k)[4][4]) {
      const uint64_t cb = ch << 9;
      const bool full = a.vec_ok && (cb + 512 <= a.n);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        if (full) {
          uint4 v = ld_stream_v4(a.keys + cb + 128 * i + 4 * lane, pol);
          k[i][0] = v.x; k[i][1] = v.y; k[i][2] = v.z; k[i][3] = v.w;
        } else {
          const uint64_t base = cb + 16 * (uint64_t)lane + 4 * (i ^ r);
#pragma unroll
          for (int e = 0; e < 4; ++e) k[i][e] = (base + e < a.n) ? to_key<KM>(ld_stream_u32(a.keys + base + e, pol)) : 0u;
        }
      }
    };
    // register double buffer: chunk ch+nwarps is in flight while ch is reduced
    uint32_t kn[4][4];
    uint64_t ch = gwarp;
    if (ch < nchunks) load_chunk(ch, kn);
    for (; ch < nchunks; ch += nwarps) {
      const bool full = a.vec_ok && ((ch << 9) + 512 <= a.n);
      uint32_t k[4][4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int e = 0; e < 4; ++e) k[i][e] = kn[i][e];
      const uint64_t chn = ch + nwarps;
      if (chn < nchunks) load_chunk(chn, kn);
      if (full) {
        // transpose through shared memory (word 32 i + l -> lane l's words),
        // then map the raw words to keys
#pragma unroll
        for (int i = 0; i < 4; ++i) xbuf[32 * i + lane] = make_uint4(k[i][0], k[i][1], k[i][2], k[i][3]);
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const uint4 v = xbuf[4 * lane + (i ^ r)];
          k[i][0] = to_key<KM>(v.x); k[i][1] = to_key<KM>(v.y); k[i][2] = to_key<KM>(v.z); k[i][3] = to_key<KM>(v.w);
        }
        __syncwarp();
      }
      if (alpha >= 4) {
        Acc acc = {0u, 0u, 0u};
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int e = 0; e < 4; ++e) acc_push<BETA, POS>(acc, k[i][e], (uint32_t)(16 * gl + 4 * (i ^ r) + e));
        for (int off = 1; off < G; off <<= 1) acc_merge<BETA, POS>(acc, acc_shfl_xor<BETA, POS>(acc, off));
        // the lanes holding a result (gl == 0) own consecutive subranges:
        // their stores are already coalesced, so they go straight to global
        // memory (no staging round trip through shared memory)
        const uint64_t j = ch * (uint64_t)dpc + grp;
        if (gl == 0 && j < M) {
          if (BETA == 2) {
            *reinterpret_cast<uint2*>(a.del + 2 * j) = make_uint2(acc.a1, acc.a2);
            if (POS) a.pos[j] = (uint16_t)acc.p1;
            emit_hist(acc.a1);
            emit_hist(acc.a2);
          } else {
            a.del[j] = acc.a1;
            emit_hist(acc.a1);
          }
        }
        continue;
      } else if (alpha == 3) {
        small_subranges<3, BETA, POS>(k, r, stage, s_pstage[wib], lane);
      } else if (alpha == 2) {
        small_subranges<2, BETA, POS>(k, r, stage, s_pstage[wib], lane);
      } else {
        small_subranges<1, BETA, POS>(k, r, stage, s_pstage[wib], lane);
      }
      __syncwarp();
      // coalesced copy-out of this chunk's delegates (skip subranges >= M)
      const uint64_t d0 = ch * (uint64_t)dpc;
      const int nd = (int)min((uint64_t)dpc, M - d0);
      for (int i = lane; i < nd * BETA; i += 32) {
        uint32_t v = stage[i];
        a.del[d0 * BETA + i] = v;
        emit_hist(v);
      }
      if (POS)
        for (int i = lane; i < nd; i += 32) a.pos[d0 + i] = s_pstage[wib][i];
      __syncwarp();
    }
  }

  if (a.hmode == 2) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      mm_lo = max(mm_lo, __shfl_xor_sync(0xffffffffu, mm_lo, off));
      mm_hi = max(mm_hi, __shfl_xor_sync(0xffffffffu, mm_hi, off));
    }
    if (lane == 0) { atomicMax(&s_mm[0], mm_lo); atomicMax(&s_mm[1], mm_hi); }
  }
  __syncthreads();
  if (a.hmode == 1) {
    for (int i = tid; i < nb; i += SAMPLE_THREADS) {
      uint32_t c = 0;
#pragma unroll
      for (int w = 0; w < SAMPLE_WARPS; ++w) c += s_hist[w][i];
      if (c) atomicAdd(&a.hist[i], c);
    }
  } else if (a.hmode == 2 && tid == 0) {
    atomicMax(&a.minmax[0], s_mm[0]);
    atomicMax(&a.minmax[1], s_mm[1]);
  }
}

}  // namespace drtopk
