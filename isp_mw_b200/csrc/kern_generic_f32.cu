// Generic-size stage kernels (BlockSize <= 16, GroupSize <= 32), float.
#include "kern_unit.cuh"

BM3D_KERNEL_UNIT(generic_f32)

namespace bm3d {
template const void *generic_kernel_fn<float, false, 1>();
template const void *generic_kernel_fn<float, false, 3>();
template const void *generic_kernel_fn<float, true, 1>();
template const void *generic_kernel_fn<float, true, 3>();
}  // namespace bm3d
