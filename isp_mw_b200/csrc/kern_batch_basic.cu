// Persistent batched stage kernels, basic stage: register-resident (KS = 4
// and 1) and generic bodies.
#include "kern_unit.cuh"

BM3D_KERNEL_UNIT(batch_basic)

namespace bm3d {
template const void *batch_kernel_fn<false, 4, false>();
template const void *batch_kernel_fn<false, 1, false>();
template const void *batch_kernel_fn<false, 1, true>();
}  // namespace bm3d
