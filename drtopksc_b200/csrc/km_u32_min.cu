// km_u32_min.cu -- kernels of key mode KM_U32_MIN (see kernels.h).
#include "kernels_impl.cuh"

namespace drtopk {
const KernelSet& kernels_u32_min() {
  static const KernelSet s = make_kernel_set<KM_U32_MIN>();
  return s;
}
}  // namespace drtopk
