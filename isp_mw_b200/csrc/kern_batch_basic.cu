// Persistent batched stage kernels, basic stage: register-resident (KS = 4
// and 1) and generic bodies, one plane or three planes sharing luma groups.
#include "kern_unit.cuh"

BM3D_KERNEL_UNIT(batch_basic)

namespace bm3d {
template const void *batch_kernel_fn<false, 1, 4, false>();
template const void *batch_kernel_fn<false, 1, 1, false>();
template const void *batch_kernel_fn<false, 1, 1, true>();
template const void *batch_kernel_fn<false, 3, 4, false>();
template const void *batch_kernel_fn<false, 3, 1, false>();
template const void *batch_kernel_fn<false, 3, 1, true>();
}  // namespace bm3d
