// Host-side handles of the stage kernels. Each kernel family is compiled in a
// translation unit of its own (kern_*.cu) so the library builds in parallel;
// the host launches through the returned pointers with cudaLaunchKernel.
// Every unit keeps its own copy of the constant cosine tables, which
// upload_dct_tables_all fills for the current device.
#pragma once

#include <cuda_runtime.h>

namespace bm3d {

// stage_kernel<T, W, NPL, KS> (bm3d_stage.cuh)
template <typename T, bool W, int NPL, int KS> const void *stage_kernel_fn();
// generic_stage_kernel<T, W, NPL> (bm3d_generic.cuh)
template <typename T, bool W, int NPL> const void *generic_kernel_fn();
// batch_stage_kernel<float, W, NPL, KS, GENERIC> (bm3d_batch.cuh)
template <bool W, int NPL, int KS, bool GENERIC> const void *batch_kernel_fn();

// Cosine matrices for group lengths 1..16, concatenated (1496 entries each).
struct DctTableData {
    const float *fwd_f, *inv_f;
    const double *fwd_d, *inv_d;
    const float *pad_fwd, *pad_inv;  // kPadTable entries each (bm3d_device.cuh)
    const float *d11_fwd, *d11_inv;  // length-11 matrices, 121 entries each
};
cudaError_t upload_dct_tables_all(const DctTableData &t);

}  // namespace bm3d

// The kernel units, each defining bm3d_upload_dct_tables_<name>.
#define BM3D_KERNEL_UNITS(X) \
    X(stage_f32_basic)       \
    X(stage_f32_final)       \
    X(stage_f64_basic)       \
    X(stage_f64_final)       \
    X(generic_f32)           \
    X(generic_f64)           \
    X(batch_basic)           \
    X(batch_final)
