// Register-resident stage kernels, double, basic stage: one and three planes,
// block matching step 1 (KS = 4) and other steps (KS = 1).
#include "kern_unit.cuh"

BM3D_KERNEL_UNIT(stage_f64_basic)

namespace bm3d {
template const void *stage_kernel_fn<double, false, 1, 1>();
template const void *stage_kernel_fn<double, false, 1, 4>();
template const void *stage_kernel_fn<double, false, 3, 1>();
template const void *stage_kernel_fn<double, false, 3, 4>();
}  // namespace bm3d
