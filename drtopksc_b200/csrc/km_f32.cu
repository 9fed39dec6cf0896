// km_f32.cu -- kernels of key mode KM_F32 (see kernels.h).
#include "kernels_impl.cuh"

namespace drtopk {
const KernelSet& kernels_f32() {
  static const KernelSet s = make_kernel_set<KM_F32>();
  return s;
}
}  // namespace drtopk
