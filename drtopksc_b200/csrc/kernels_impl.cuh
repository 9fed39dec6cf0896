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
  s.fused_one = (const void*)k_fused_one<KM>;
  s.tail = (const void*)k_tail<KM>;
  s.filter = (const void*)k_filter<KM>;
  s.gather = (const void*)k_gather<KM>;
  s.level_hist = (const void*)k_level_hist<KM>;
  s.split0 = (const void*)k_split0<KM>;
  s.bitonic = (const void*)k_bitonic<KM>;
  s.presample = (const void*)k_presample<KM>;
  s.prerefine = (const void*)k_prerefine<KM>;
  s.emit = (const void*)k_emit<KM>;
  s.cand_hist = (const void*)k_cand_hist<KM>;
  s.presample_g = (const void*)k_presample_g<KM>;
  s.prerefine_g = (const void*)k_prerefine_g<KM>;
  s.emit_g = (const void*)k_emit_g<KM>;
  s.cand_hist_g = (const void*)k_cand_hist_g<KM>;
  s.split0_g = (const void*)k_split0_g<KM>;
  s.fused_one_g = (const void*)k_fused_one_g<KM>;
  s.sample1 = (const void*)k_sample<KM, 1, false, false>;
  s.sample2 = (const void*)k_sample<KM, 2, false, false>;
  s.sample2pos = (const void*)k_sample<KM, 2, true, false>;
  s.sample1w = (const void*)k_sample<KM, 1, false, true>;
  s.sample2w = (const void*)k_sample<KM, 2, false, true>;
  s.sample2posw = (const void*)k_sample<KM, 2, true, true>;
  return s;
}

}  // namespace drtopk
