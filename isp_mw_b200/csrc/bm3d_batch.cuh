// Batched BM3D stages: many planes of different sizes and noise levels in one
// persistent launch per stage. Each CTA pulls (image, tile) work items from a
// device counter; an image's items are its tiles, numbered after the items of
// the images before it (tile_base is the exclusive prefix sum). The per-tile
// work is the same body as the single-plane kernels, so results are
// bit-identical to per-plane calls.
#pragma once

#include "bm3d_generic.cuh"

namespace bm3d {

// The first 16 bytes of dynamic shared memory hold the CTA's current item.
constexpr int kBatchHeader = 16;

template <typename T, bool WIENER, int NPL, int KS, bool GENERIC>
__global__ void __launch_bounds__(GENERIC ? 256 : 512, 1)
    batch_stage_kernel(const StageArgs<T> *__restrict__ args, const int *__restrict__ tile_base,
                       int nimg, int *counter)
{
    extern __shared__ __align__(16) unsigned char smem[];
    int *item = reinterpret_cast<int *>(smem);
    const int total = tile_base[nimg];
    const unsigned avail = dynamic_smem_bytes() - kBatchHeader;
    for (;;) {
        if (threadIdx.x == 0) *item = atomicAdd(counter, 1);
        __syncthreads();
        const int it = *item;
        if (it >= total) break;
        int lo = 0, hi = nimg - 1;  // last image whose first item is <= it
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tile_base[mid] <= it) lo = mid;
            else hi = mid - 1;
        }
        const StageArgs<T> &a = args[lo];
        unsigned char *body = smem + kBatchHeader;
        if constexpr (GENERIC && NPL == 3) generic_tile_body_seq3<T, WIENER>(a, it - tile_base[lo], body, avail);
        else if constexpr (GENERIC) generic_tile_body<T, WIENER, NPL>(a, it - tile_base[lo], body, avail);
        else if constexpr (NPL == 3) stage_tile_body_seq3<T, WIENER, KS>(a, it - tile_base[lo], body, avail);
        else stage_tile_body<T, WIENER, NPL, KS>(a, it - tile_base[lo], body, avail);
        __syncthreads();  // every thread has read *item before it is replaced
    }
}

// One plane of a batch, for the per-pixel kernels.
template <typename T> struct BatchPlane {
    typename AccOf<T>::type *num, *den;
    const T *src;
    T *dst;
    long long src_stride, dst_stride;
    int width, height;
    int block_size;
    float *absmax;
};

// Zero each plane's sums and fold its max |src| (grid.y = plane).
template <typename T>
__global__ void prep_batch_kernel(const BatchPlane<T> *planes)
{
    const BatchPlane<T> q = planes[blockIdx.y];
    const long long n = static_cast<long long>(q.width) * q.height;
    float m = 0.0f;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        q.num[i] = 0;
        q.den[i] = 0;
        const long long y = i / q.width, x = i - y * q.width;
        const float v = fabsf(static_cast<float>(q.src[y * q.src_stride + x]));
        m = v > m ? v : m;
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        const float w = __shfl_xor_sync(0xffffffffu, m, o);
        m = w > m ? w : m;
    }
    if ((threadIdx.x & 31) == 0 && m > 0.0f)
        atomicMax(reinterpret_cast<int *>(q.absmax), __float_as_int(fminf(m, 3.0e38f)));
}

// dst = num / den for every plane (grid.y = plane); each CTA walks the
// plane's 32 x 32 tiles from blockIdx.x in steps of gridDim.x.
template <typename T>
__global__ void __launch_bounds__(256) normalize_batch_kernel(const BatchPlane<T> *planes)
{
    const BatchPlane<T> q = planes[blockIdx.y];
    const int tx = (q.width + kNormTile - 1) / kNormTile;
    const int ntiles = tx * ((q.height + kNormTile - 1) / kNormTile);
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int ty = tile / tx, txi = tile - ty * tx;
        normalize_tile<T>(q.dst, q.dst_stride, q.num, q.den, q.width, q.height, q.block_size,
                          ty * kNormTile, txi * kNormTile);
    }
}

}  // namespace bm3d
