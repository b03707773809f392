// Conversions between the reference's integer planes and the float planes the
// stage kernels filter: RangeConvert (include/Conversion.hpp:134-254) and the
// OPP colour matrices of MatrixConvert_RGB2YUV / MatrixConvert_YUV2RGB
// (include/Conversion.hpp:518-575, 661-748). Each pixel takes the same float
// operations in the same order as the reference (no contraction into FMA:
// the explicit _rn intrinsics), so results match it bit for bit. The
// coefficients are computed on the host, in float, as the reference does.
#pragma once

#include <cuda_runtime.h>

namespace bm3d {

// Y = (R + G + B) gainY + offsetY, U = (R - B) gainU + offsetC,
// V = (R - 2G + B) gainV + offsetC.
struct OppForward {
    float gainY, offsetY, gainU, gainV, offsetC;
};

// R = Ry Y + Ru U + Rv V + offR, G = Gy Y + Gv V + offG,
// B = By Y + Bu U + Bv V + offB, each clipped to [lo, hi] and truncated.
struct OppInverse {
    float Ry, Ru, Rv, Gy, Gv, By, Bu, Bv, offR, offG, offB, lo, hi;
};

// f = v gain + offset, clipped to [lo, hi] when `clip`.
struct RangeMap {
    float gain, offset, lo, hi;
    int clip;
};

__device__ __forceinline__ float clip_to(float t, float lo, float hi)
{
    return t <= lo ? lo : t >= hi ? hi : t;
}

// Rows are walked by grid.y (strided), columns by grid.x * blockDim.x.
template <typename F>
__device__ __forceinline__ void for_each_pixel(int width, int height, F f)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= width) return;
    for (int y = blockIdx.y; y < height; y += gridDim.y) f(y, x);
}

__global__ void rgb_to_opp_kernel(const int *__restrict__ r, const int *__restrict__ g,
                                  const int *__restrict__ b, long long istride,
                                  float *__restrict__ py, float *__restrict__ pu,
                                  float *__restrict__ pv, long long fpitch, int width, int height,
                                  OppForward c, int only_y)
{
    for_each_pixel(width, height, [&](int y, int x) {
        const long long i = y * istride + x, o = y * fpitch + x;
        const float R = static_cast<float>(r[i]), G = static_cast<float>(g[i]),
                    B = static_cast<float>(b[i]);
        py[o] = __fadd_rn(__fmul_rn(__fadd_rn(__fadd_rn(R, G), B), c.gainY), c.offsetY);
        if (only_y) return;
        pu[o] = __fadd_rn(__fmul_rn(__fsub_rn(R, B), c.gainU), c.offsetC);
        pv[o] = __fadd_rn(__fmul_rn(__fadd_rn(__fsub_rn(R, __fmul_rn(G, 2.0f)), B), c.gainV),
                          c.offsetC);
    });
}

__global__ void opp_to_rgb_kernel(const float *__restrict__ py, const float *__restrict__ pu,
                                  const float *__restrict__ pv, long long fpitch,
                                  int *__restrict__ r, int *__restrict__ g, int *__restrict__ b,
                                  long long ostride, int width, int height, OppInverse c)
{
    for_each_pixel(width, height, [&](int y, int x) {
        const long long i = y * fpitch + x, o = y * ostride + x;
        const float Y = py[i], U = pu[i], V = pv[i];
        float t = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(c.Ry, Y), __fmul_rn(c.Ru, U)),
                                      __fmul_rn(c.Rv, V)),
                            c.offR);
        r[o] = __float2int_rz(clip_to(t, c.lo, c.hi));
        t = __fadd_rn(__fadd_rn(__fmul_rn(c.Gy, Y), __fmul_rn(c.Gv, V)), c.offG);
        g[o] = __float2int_rz(clip_to(t, c.lo, c.hi));
        t = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(c.By, Y), __fmul_rn(c.Bu, U)),
                                __fmul_rn(c.Bv, V)),
                      c.offB);
        b[o] = __float2int_rz(clip_to(t, c.lo, c.hi));
    });
}

__global__ void int_to_float_kernel(const int *__restrict__ src, long long istride,
                                    float *__restrict__ dst, long long fpitch, int width,
                                    int height, RangeMap m)
{
    for_each_pixel(width, height, [&](int y, int x) {
        const float t =
            __fadd_rn(__fmul_rn(static_cast<float>(src[y * istride + x]), m.gain), m.offset);
        dst[y * fpitch + x] = m.clip ? clip_to(t, m.lo, m.hi) : t;
    });
}

__global__ void float_to_int_kernel(const float *__restrict__ src, long long fpitch,
                                    int *__restrict__ dst, long long ostride, int width,
                                    int height, RangeMap m)
{
    for_each_pixel(width, height, [&](int y, int x) {
        const float t = __fadd_rn(__fmul_rn(src[y * fpitch + x], m.gain), m.offset);
        dst[y * ostride + x] = __float2int_rz(clip_to(t, m.lo, m.hi));
    });
}

}  // namespace bm3d
