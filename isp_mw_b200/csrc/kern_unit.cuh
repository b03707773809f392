// Shared part of the kernel translation units (kern_*.cu): the definitions
// behind the handles of bm3d_kernels.h and this unit's table upload.
#pragma once

#include "bm3d_batch.cuh"
#include "bm3d_kernels.h"

namespace bm3d {

template <typename T, bool W, int NPL, int KS> const void *stage_kernel_fn()
{
    return reinterpret_cast<const void *>(&stage_kernel<T, W, NPL, KS>);
}

template <typename T, bool W, int NPL> const void *generic_kernel_fn()
{
    return reinterpret_cast<const void *>(&generic_stage_kernel<T, W, NPL>);
}

template <bool W, int NPL, int KS, bool GENERIC> const void *batch_kernel_fn()
{
    return reinterpret_cast<const void *>(&batch_stage_kernel<float, W, NPL, KS, GENERIC>);
}

static cudaError_t upload_dct_tables_here(const DctTableData &t)
{
    cudaError_t e;
    if ((e = cudaMemcpyToSymbol(c_dct_fwd_f, t.fwd_f, sizeof(c_dct_fwd_f))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(c_dct_inv_f, t.inv_f, sizeof(c_dct_inv_f))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(c_dct_fwd_d, t.fwd_d, sizeof(c_dct_fwd_d))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(c_dct_pad_fwd, t.pad_fwd, sizeof(c_dct_pad_fwd))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(c_dct_pad_inv, t.pad_inv, sizeof(c_dct_pad_inv))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(c_dct11_fwd, t.d11_fwd, sizeof(c_dct11_fwd))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(c_dct11_inv, t.d11_inv, sizeof(c_dct11_inv))) != cudaSuccess) return e;
    return cudaMemcpyToSymbol(c_dct_inv_d, t.inv_d, sizeof(c_dct_inv_d));
}

}  // namespace bm3d

#define BM3D_KERNEL_UNIT(name)                                                      \
    cudaError_t bm3d_upload_dct_tables_##name(const bm3d::DctTableData &t)         \
    {                                                                               \
        return bm3d::upload_dct_tables_here(t);                                     \
    }
