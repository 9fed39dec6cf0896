// km_u32.cu -- kernels of key mode KM_U32 (see kernels.h).
#include "kernels_impl.cuh"

namespace drtopk {
const KernelSet& kernels_u32() {
  static const KernelSet s = make_kernel_set<KM_U32>();
  return s;
}
}  // namespace drtopk
