// kernels.h -- the device kernels of one key mode, as launchable pointers.
// Each key mode's kernels are instantiated in their own translation unit
// (km_*.cu) so that the four sets compile in parallel; the host code only
// sees these tables.
#pragma once

namespace drtopk {

struct KernelSet {
  const void* fused;       // k_fused<KM>
  const void* fused_cl;    // k_fused_cl<KM>
  const void* fused_one;   // k_fused_one<KM>
  const void* tail;        // k_tail<KM>
  const void* filter;      // k_filter<KM>
  const void* gather;      // k_gather<KM>
  const void* level_hist;  // k_level_hist<KM>
  const void* split0;      // k_split0<KM>
  const void* bitonic;     // k_bitonic<KM>
  const void* presample;   // k_presample<KM>   (sampled-threshold path)
  const void* prerefine;   // k_prerefine<KM>   (launched per byte level 1..3)
  const void* emit;        // k_emit<KM>
  const void* cand_hist;   // k_cand_hist<KM>
  // grouped forms of the sampled-threshold path (many problems per launch)
  const void* presample_g;
  const void* prerefine_g;
  const void* emit_g;
  const void* cand_hist_g;
  const void* split0_g;
  const void* fused_one_g;
  const void* sample1;     // k_sample<KM, 1, false, false>  (alpha <= 8)
  const void* sample2;     // k_sample<KM, 2, false, false>
  const void* sample2pos;  // k_sample<KM, 2, true, false>
  const void* sample1w;    // k_sample<KM, 1, false, true>   (alpha >= 9)
  const void* sample2w;    // k_sample<KM, 2, false, true>
  const void* sample2posw; // k_sample<KM, 2, true, true>
};

const KernelSet& kernels_u32();
const KernelSet& kernels_f32();
const KernelSet& kernels_u32_min();
const KernelSet& kernels_f32_min();

// key mode 0 u32, 1 f32, 2 u32 smallest, 3 f32 smallest
inline const KernelSet& kernels(int km) {
  switch (km) {
    case 0: return kernels_u32();
    case 1: return kernels_f32();
    case 2: return kernels_u32_min();
    default: return kernels_f32_min();
  }
}

}  // namespace drtopk
