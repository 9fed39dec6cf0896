// kernels_impl.cuh -- builds the KernelSet of one key mode; included only by
// the per-key-mode translation units km_*.cu.
#pragma once

#include "bitonic.cuh"
#include "fused.cuh"
#include "kernels.h"
#include "sampler.cuh"
#include "tail.cuh"

namespace drtopk {

template <int KM>
KernelSet make_kernel_set() {
  KernelSet s;
  s.fused = (const void*)k_fused<KM>;
  s.fused_cl = (const void*)k_fused_cl<KM>;
  s.tail = (const void*)k_tail<KM>;
  s.filter = (const void*)k_filter<KM>;
  s.gather = (const void*)k_gather<KM>;
  s.level_hist = (const void*)k_level_hist<KM>;
  s.split0 = (const void*)k_split0<KM>;
  s.bitonic = (const void*)k_bitonic<KM>;
  s.sample1 = (const void*)k_sample<KM, 1, false>;
  s.sample2 = (const void*)k_sample<KM, 2, false>;
  s.sample2pos = (const void*)k_sample<KM, 2, true>;
  return s;
}

}  // namespace drtopk
