// Register-resident stage kernels, double, final stage: one and three planes,
// block matching step 1 (KS = 4) and other steps (KS = 1).
#include "kern_unit.cuh"

BM3D_KERNEL_UNIT(stage_f64_final)

namespace bm3d {
template const void *stage_kernel_fn<double, true, 1, 1>();
template const void *stage_kernel_fn<double, true, 1, 4>();
template const void *stage_kernel_fn<double, true, 3, 1>();
template const void *stage_kernel_fn<double, true, 3, 4>();
}  // namespace bm3d
