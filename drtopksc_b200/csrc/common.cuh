// common.cuh -- shared device helpers for the B200 Dr.Top-k kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define DRTOPK_DEV __device__ __forceinline__

namespace drtopk {

// ------------------------------------------------------------------ keys
// Key modes: the kernels compare uint32 keys.  Float keys are mapped with the
// order-preserving transform (negative -> bit-inverted, non-negative -> sign
// bit set); "smallest" selection inverts the mapped key, so the same
// largest-first machinery returns the k smallest.
enum KeyMode : int { KM_U32 = 0, KM_F32 = 1, KM_U32_MIN = 2, KM_F32_MIN = 3 };

// float bits -> order-preserving key without a branch: negative values are
// inverted (xor with all ones), non-negative ones get the sign bit set
DRTOPK_DEV uint32_t f32_bits_to_key(uint32_t u) {
  const uint32_t neg = (uint32_t)((int32_t)u >> 31);  // all ones for negative values
  return u ^ (neg | 0x80000000u);
}

template <int KM>
DRTOPK_DEV uint32_t to_key(uint32_t u) {
  if (KM == KM_F32 || KM == KM_F32_MIN) u = f32_bits_to_key(u);
  if (KM == KM_U32_MIN || KM == KM_F32_MIN) u = ~u;
  return u;
}

DRTOPK_DEV uint32_t from_key(uint32_t k, int km) {
  if (km == KM_U32_MIN || km == KM_F32_MIN) k = ~k;
  if (km == KM_F32 || km == KM_F32_MIN) k = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  return k;
}

// ------------------------------------------------------------------ loads
// Streaming 128-bit load: read-only path, no L1 allocation, 256-byte L2
// prefetch, and an L2 evict-first policy so the stream does not push the
// (re-read) delegate vector out of L2.
DRTOPK_DEV uint64_t make_evict_first_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

DRTOPK_DEV uint4 ld_stream_v4(const uint32_t* p, uint64_t pol) {
  uint4 r;
  asm volatile(
      "ld.global.nc.L1::no_allocate.L2::cache_hint.L2::256B.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
      : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
      : "l"(p), "l"(pol));
  return r;
}

// Same read-only path but allocating in L1 (for warp layouts where two
// instructions split each 32-byte sector).
DRTOPK_DEV uint4 ld_l1_v4(const uint32_t* p, uint64_t pol) {
  uint4 r;
  asm volatile("ld.global.nc.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
               : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
               : "l"(p), "l"(pol));
  return r;
}

DRTOPK_DEV uint32_t ld_stream_u32(const uint32_t* p, uint64_t pol) {
  uint32_t r;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(r) : "l"(p), "l"(pol));
  return r;
}

// Loads of data written earlier in the same kernel (after a grid barrier):
// must not use the non-coherent path.
DRTOPK_DEV uint32_t ld_cg_u32(const uint32_t* p) {
  uint32_t r;
  asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(r) : "l"(p));
  return r;
}
DRTOPK_DEV uint2 ld_cg_v2(const uint32_t* p) {
  uint2 r;
  asm volatile("ld.global.cg.v2.u32 {%0,%1}, [%2];" : "=r"(r.x), "=r"(r.y) : "l"(p));
  return r;
}
DRTOPK_DEV uint4 ld_cg_v4(const uint32_t* p) {
  uint4 r;
  asm volatile("ld.global.cg.v4.u32 {%0,%1,%2,%3}, [%4];" : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w) : "l"(p));
  return r;
}

DRTOPK_DEV uint64_t ld_cg_u64(const uint64_t* p) {
  uint64_t r;
  asm volatile("ld.global.cg.u64 %0, [%1];" : "=l"(r) : "l"(p));
  return r;
}

DRTOPK_DEV uint32_t ld_acquire_gpu(const uint32_t* p) {
  uint32_t r;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(r) : "l"(p) : "memory");
  return r;
}
DRTOPK_DEV void st_release_gpu(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ------------------------------------------------------------------ warp
DRTOPK_DEV unsigned lane_id() { return threadIdx.x & 31u; }

// Top-2 (multiset) merge of two (first, second) pairs.
DRTOPK_DEV void top2_merge(uint32_t& a1, uint32_t& a2, uint32_t b1, uint32_t b2) {
  uint32_t hi = max(a1, b1), lo = min(a1, b1);
  a2 = max(lo, max(a2, b2));
  a1 = hi;
}
DRTOPK_DEV void top2_push(uint32_t& a1, uint32_t& a2, uint32_t v) {
  // same result as the reference's "if Max<v {Second=Max;Max=v} else if Second<v {Second=v}"
  uint32_t lo = min(a1, v);
  a1 = max(a1, v);
  a2 = max(a2, lo);
}

// Warp-aggregated append: every lane with pred reserves one slot of *counter;
// returns the slot (undefined for lanes without pred).  One atomic per warp.
DRTOPK_DEV uint32_t warp_append(bool pred, uint32_t* counter) {
  unsigned mask = __activemask();
  unsigned b = __ballot_sync(mask, pred);
  if (!b) return 0;
  unsigned lane = lane_id();
  int leader = __ffs(b) - 1;
  uint32_t base = 0;
  if ((int)lane == leader) base = atomicAdd(counter, (uint32_t)__popc(b));
  base = __shfl_sync(mask, base, leader);
  return base + __popc(b & ((1u << lane) - 1u));
}

// Histogram increment with a fast path for warps whose active lanes all hit
// one bin (one shared-memory atomic for the warp): skewed sets -- delegates
// are subrange maxima and crowd into the top bins -- would otherwise
// serialise 32 atomics on one address.  Mixed warps add per lane.
DRTOPK_DEV void hist_add_warp(uint32_t* h, uint32_t bin) {
  const unsigned mask = __activemask();
  const int leader = __ffs(mask) - 1;
  const uint32_t b0 = __shfl_sync(mask, bin, leader);
  if (__all_sync(mask, bin == b0)) {
    if ((int)lane_id() == leader) atomicAdd(&h[bin], (uint32_t)__popc(mask));
  } else {
    atomicAdd(&h[bin], 1u);
  }
}

// Block-aggregated append to two lists: every thread of the block passes the
// number of items it will write to list A and list B (each < 2^16 summed
// over the block); one atomic per list per call; returns this thread's
// first slot in each list.  Must be called by all threads of the block.
struct Slots2 {
  uint32_t a, b;
};
DRTOPK_DEV Slots2 block_append2(uint32_t ca, uint32_t cb, uint32_t* counter_a, uint32_t* counter_b) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_base[2];
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  uint32_t v = ca | (cb << 16);
  uint32_t incl = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
    if ((int)lane >= off) incl += y;
  }
  if (lane == 31) s_warp[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    uint32_t w = lane < nw ? s_warp[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, wi, off);
      if ((int)lane >= off) wi += y;
    }
    if (lane < nw) s_warp[lane] = wi - w;  // exclusive warp prefix
    if (lane == 31) {
      const uint32_t ta = wi & 0xffffu, tb = wi >> 16;
      s_base[0] = ta ? atomicAdd(counter_a, ta) : 0u;
      s_base[1] = tb ? atomicAdd(counter_b, tb) : 0u;
    }
  }
  __syncthreads();
  const uint32_t ex = s_warp[wid] + incl - v;
  Slots2 r;
  r.a = s_base[0] + (ex & 0xffffu);
  r.b = s_base[1] + (ex >> 16);
  __syncthreads();
  return r;
}

// single-list variant with 32-bit counts
DRTOPK_DEV uint32_t block_append1(uint32_t c, uint32_t* counter) {
  __shared__ uint32_t s_warp1[32];
  __shared__ uint32_t s_base1;
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  uint32_t incl = c;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
    if ((int)lane >= off) incl += y;
  }
  if (lane == 31) s_warp1[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    uint32_t w = lane < nw ? s_warp1[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, wi, off);
      if ((int)lane >= off) wi += y;
    }
    if (lane < nw) s_warp1[lane] = wi - w;
    if (lane == 31) s_base1 = wi ? atomicAdd(counter, wi) : 0u;
  }
  __syncthreads();
  const uint32_t r = s_base1 + s_warp1[wid] + incl - c;
  __syncthreads();
  return r;
}

// Block-strided loop over [0, n) that issues U loads per thread before
// using any of them: ld(i) for every index of a round, then use(i, value).
// A plain strided loop waits one memory round trip per iteration.
template <int U, typename LD, typename USE>
DRTOPK_DEV void block_load_loop(uint32_t n, LD&& ld, USE&& use) {
  using V = decltype(ld(0u));
  for (uint32_t b = 0; b < n; b += blockDim.x * U) {
    V v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint32_t i = b + u * blockDim.x + threadIdx.x;
      if (i < n) v[u] = ld(i);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint32_t i = b + u * blockDim.x + threadIdx.x;
      if (i < n) use(i, v[u]);
    }
  }
}

// ------------------------------------------------------------------ errors
enum DevErr : uint32_t {
  DE_BARRIER_TIMEOUT = 1u,   // a grid barrier gave up waiting
  DE_OVERFLOW = 2u,          // a bounded buffer would have overflowed (skipped)
  DE_INTERNAL = 4u,          // an invariant failed (result not trusted)
  DE_RETRY = 8u,             // a bounded select could not finish in its workspace: run it with the general plan
};

// Grid barrier for kernels launched cooperatively (all CTAs co-resident).
// One 32-bit word holds (generation << 16) | arrivals: a CTA arrives with one
// acq_rel atomic; the last arrival resets the count and opens the next
// generation with a second atomic, and the others poll the word for the
// generation change.  The spin is bounded: after ~2^26 polls (~seconds) the
// CTA records DE_BARRIER_TIMEOUT; a CTA that finds the flag set while it
// waits returns false at once, so a broken launch ends with an error
// instead of a hang.
struct GridBar {
  uint32_t* count;   // (generation << 16) | arrivals in this generation
  uint32_t* err;     // error word (host-visible)
  uint32_t nblocks;  // < 2^16
  uint32_t spin_limit;  // polls before giving up (0: default 2^26)
};

DRTOPK_DEV uint32_t atom_add_acq_rel_gpu(uint32_t* p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
DRTOPK_DEV void red_add_release_gpu(uint32_t* p, uint32_t v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

DRTOPK_DEV bool grid_barrier(const GridBar& gb) {
  __shared__ uint32_t s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t ok = 1;
    const uint32_t old = atom_add_acq_rel_gpu(gb.count, 1u);
    if ((old & 0xffffu) == gb.nblocks - 1) {
      red_add_release_gpu(gb.count, 0x10000u - gb.nblocks);
    } else {
      const uint32_t g = old >> 16;
      const uint32_t lim = gb.spin_limit ? gb.spin_limit : (1u << 26);
      uint32_t it = 0;
      while ((ld_acquire_gpu(gb.count) >> 16) == g) {
        if (++it > lim) {
          atomicOr(gb.err, (uint32_t)DE_BARRIER_TIMEOUT);
          ok = 0;
          break;
        }
        if ((it & 1023u) == 1u && (ld_acquire_gpu(gb.err) & DE_BARRIER_TIMEOUT)) { ok = 0; break; }
        __nanosleep(32);
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// A team of CTAs working on one problem: the whole grid of a cooperative
// launch (software grid barrier above), one thread-block cluster (hardware
// cluster barrier, ~0.2 us) or a single CTA.  Code written against a Team
// distributes work by (rank, size) and synchronises with team_sync; every
// CTA of a team must reach the same team_sync calls (control flow that
// leads to a team_sync depends only on kernel arguments and on values read
// after the previous team_sync).
struct Team {
  GridBar gb;     // grid teams: barrier words
  uint32_t rank;  // this CTA's index in the team
  uint32_t size;  // CTAs in the team
  int cluster;    // 0: grid team; 1: this CTA's thread-block cluster; 2: this CTA alone
};

DRTOPK_DEV uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
DRTOPK_DEV uint32_t cluster_nctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
DRTOPK_DEV uint32_t cluster_id_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}

DRTOPK_DEV Team grid_team(const GridBar& gb) {
  Team t;
  t.gb = gb;
  t.rank = blockIdx.x;
  t.size = gridDim.x;
  t.cluster = 0;
  return t;
}
DRTOPK_DEV Team cluster_team() {
  Team t = {};
  t.rank = cluster_ctarank();
  t.size = cluster_nctarank();
  t.cluster = 1;
  return t;
}

DRTOPK_DEV bool team_sync(const Team& t) {
  if (t.cluster == 2) {
    __syncthreads();  // one CTA: a block barrier orders its global-memory accesses
    return true;
  }
  if (t.cluster == 1) {
    // all threads of every CTA in the cluster arrive; release/acquire at
    // cluster scope orders the global-memory writes made before it
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
    return true;
  }
  return grid_barrier(t.gb);
}

}  // namespace drtopk
