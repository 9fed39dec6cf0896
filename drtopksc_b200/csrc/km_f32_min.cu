// km_f32_min.cu -- kernels of key mode KM_F32_MIN (see kernels.h).
#include "kernels_impl.cuh"

namespace drtopk {
const KernelSet& kernels_f32_min() {
  static const KernelSet s = make_kernel_set<KM_F32_MIN>();
  return s;
}
}  // namespace drtopk
