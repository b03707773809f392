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
__global__ void __launch_bounds__(GENERIC ? (sizeof(T) == 4 ? 384 : 256) : 512, 1)
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
    const T *ref;              // counted for non-finite pixels too when not null
    T *dst;
    long long src_stride, dst_stride;
    int width, height;
    int block_size;
    float *absmax;
    int log2_bound, log2_corner;  // fixed-point bounds of the stage (StageArgs)
    unsigned *nonfinite;       // non-finite src / ref pixels (may be null)
    unsigned char *poison;     // pixels a non-finite term reached (may be null; all zero
                               // between stages: normalize_tile clears what it reads)
};

// Zero each plane's sums, fold its max finite |src| and count its non-finite
// pixels (grid.y = plane).
template <typename T>
__global__ void prep_batch_kernel(const BatchPlane<T> *planes)
{
    const BatchPlane<T> q = planes[blockIdx.y];
    prep_plane<T>(q.num, q.den, q.src, q.ref, q.src_stride, q.width, q.height, q.absmax,
                  q.nonfinite, blockIdx.x, gridDim.x);
}

// dst = num / den for every plane (grid.y = plane): fixed point by strips,
// warp w of the plane's CTAs taking strips w, w + warps, ...; FP64 by 32 x 32
// tiles, each CTA walking them from blockIdx.x in steps of gridDim.x.
template <typename T>
__global__ void __launch_bounds__(256) normalize_batch_kernel(const BatchPlane<T> *planes)
{
    const BatchPlane<T> q = planes[blockIdx.y];
    if constexpr (std::is_same<T, float>::value) {  // fixed point: one warp per strip
        normalize_plane_strips(q.dst, q.dst_stride, q.num, q.den, q.width, q.height, q.block_size,
                               q.poison, q.nonfinite, q.absmax, q.log2_bound, q.log2_corner,
                               static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) +
                                   (threadIdx.x >> 5),
                               static_cast<long long>(gridDim.x) * (blockDim.x >> 5));
        return;
    }
    const int tx = (q.width + kNormTile - 1) / kNormTile;
    const int ntiles = tx * ((q.height + kNormTile - 1) / kNormTile);
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int ty = tile / tx, txi = tile - ty * tx;
        normalize_tile<T>(q.dst, q.dst_stride, q.num, q.den, q.width, q.height, q.block_size,
                          ty * kNormTile, txi * kNormTile, q.poison, q.nonfinite, q.absmax,
                          q.log2_bound, q.log2_corner);
    }
}

}  // namespace bm3d
