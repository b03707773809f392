// Generic-size stage kernels (BlockSize <= 16, GroupSize <= 32), double.
#include "kern_unit.cuh"

BM3D_KERNEL_UNIT(generic_f64)

namespace bm3d {
template const void *generic_kernel_fn<double, false, 1>();
template const void *generic_kernel_fn<double, false, 3>();
template const void *generic_kernel_fn<double, true, 1>();
template const void *generic_kernel_fn<double, true, 3>();
}  // namespace bm3d
