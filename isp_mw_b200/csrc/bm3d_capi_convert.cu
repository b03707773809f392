// C ABI, integer planes and RGB frames (declared in include/bm3d_b200.h):
// the reference's RangeConvert and OPP conversions as kernels around the
// float stage drivers.
#include "bm3d_capi_internal.h"
#include "bm3d_convert.cuh"

// ---------------------------------------------------------------------------
// Integer planes and RGB frames: conversion kernels around the float paths.

namespace {

// Quantisation of an integer plane (Floor, Neutral, Ceil) and of the float
// plane it maps to (the reference's default Plane_FL ranges,
// include/Image_Type.hpp:184-202): luma [0, 1], chroma [-0.5, 0.5].
struct Quant {
    int floor_, neutral, ceil_;
    bool chroma() const { return floor_ < neutral; }
    // isPCChroma (include/Image_Type.hpp:152-155)
    bool pc_chroma() const { return chroma() && (floor_ + ceil_) % 2 == 1; }
    float ffloor() const { return chroma() ? -0.5f : 0.0f; }
    float fceil() const { return chroma() ? 0.5f : 1.0f; }
};

// RangeConvert(float plane, int plane, clip = false)
// (include/Conversion.hpp:231-253): full-range chroma is clipped anyway.
RangeMap range_to_float(const Quant &q)
{
    const int sRange = q.ceil_ - q.floor_;
    const float dRange = q.fceil() - q.ffloor();
    const float dNeutral = 0.0f;
    RangeMap m;
    m.gain = dRange / static_cast<float>(sRange);
    m.offset = -static_cast<float>(q.neutral) * m.gain + dNeutral;
    m.lo = q.ffloor();
    m.hi = q.fceil();
    m.clip = q.pc_chroma() ? 1 : 0;
    return m;
}

// RangeConvert(int plane, float plane, clip = true): +0.5 (+0.499999 for
// full-range chroma) before truncation.
RangeMap range_to_int(const Quant &q)
{
    const float sRange = q.fceil() - q.ffloor();
    const int dRange = q.ceil_ - q.floor_;
    const float sNeutral = 0.0f;
    RangeMap m;
    m.gain = static_cast<float>(dRange) / sRange;
    m.offset = -sNeutral * m.gain + static_cast<float>(q.neutral);
    m.offset += q.pc_chroma() ? 0.499999f : 0.5f;
    m.lo = static_cast<float>(q.floor_);
    m.hi = static_cast<float>(q.ceil_);
    m.clip = 1;
    return m;
}

// MatrixConvert_RGB2YUV, ColorMatrix::OPP, float destination
// (include/Conversion.hpp:537-546): source Floor floor_, Ceil ceil_.
OppForward opp_forward(int floor_, int ceil_)
{
    const int sRange = ceil_ - floor_;
    const float dRangeY = 1.0f - 0.0f, dRangeC = 0.5f - -0.5f, dFloorY = 0.0f, dNeutralC = 0.0f;
    OppForward c;
    c.gainY = dRangeY / (static_cast<float>(sRange) * 3.0f);
    c.offsetY = -static_cast<float>(floor_) * 3.0f * c.gainY + dFloorY;
    c.gainU = dRangeC / (static_cast<float>(sRange) * 2.0f);
    c.gainV = dRangeC / (static_cast<float>(sRange) * 4.0f);
    c.offsetC = dNeutralC;
    return c;
}

// MatrixConvert_YUV2RGB, ColorMatrix::OPP, integer destination, clipping
// (include/Conversion.hpp:690-712, coefficients include/Specification.h:
// 468-484).
OppInverse opp_inverse(int floor_, int ceil_)
{
    const int dRange = ceil_ - floor_;
    const float sRangeY = 1.0f - 0.0f, sRangeC = 0.5f - -0.5f, sFloorY = 0.0f, sNeutralC = 0.0f;
    const float gainY = static_cast<float>(dRange) / sRangeY;
    const float gainC = static_cast<float>(dRange) / sRangeC;
    OppInverse c;
    c.Ry = static_cast<float>(1.0L) * gainY;
    c.Ru = static_cast<float>(1.0L) * gainC;
    c.Rv = static_cast<float>(2.0L / 3.0L) * gainC;
    c.Gy = static_cast<float>(1.0L) * gainY;
    const float Gu = static_cast<float>(0.0L) * gainC;
    c.Gv = static_cast<float>(-4.0L / 3.0L) * gainC;
    c.By = static_cast<float>(1.0L) * gainY;
    c.Bu = static_cast<float>(-1.0L) * gainC;
    c.Bv = static_cast<float>(2.0L / 3.0L) * gainC;
    const float dFloor = static_cast<float>(floor_);
    c.offR = -sFloorY * c.Ry - sNeutralC * (c.Ru + c.Rv) + dFloor;
    c.offR += 0.5f;
    c.offG = -sFloorY * c.Gy - sNeutralC * (Gu + c.Gv) + dFloor;
    c.offG += 0.5f;
    c.offB = -sFloorY * c.By - sNeutralC * (c.Bu + c.Bv) + dFloor;
    c.offB += 0.5f;
    c.lo = static_cast<float>(floor_);
    c.hi = static_cast<float>(ceil_);
    return c;
}

dim3 convert_grid(const bm3d_ctx *ctx, int width, int height)
{
    const int bx = (width + 255) / 256;
    const int rows = std::max(1, std::min(height, (ctx->sm_count * 16 + bx - 1) / bx));
    return dim3(static_cast<unsigned>(bx), static_cast<unsigned>(std::min(rows, 65535)));
}

// The guard of the stage-level integer and Frame filters
// (source/BM3D.cpp:250-256, 286-293): unlike BM3D_Base::Kernel's, it copies
// for GroupSize == 1, not 0.
bool int_path_rejected(const bm3d_stage_params *p, int nplanes)
{
    const bool sig = nplanes == 1 ? p->sigma[0] > 0
                                  : (p->sigma[0] > 0 || p->sigma[1] > 0 || p->sigma[2] > 0);
    return !sig || p->group_size == 1 || p->block_size <= 0 || p->bm_range <= 0 ||
           p->bm_range < p->bm_step || p->thMSE <= 0;
}

// Device-side integer planes of one call: the caller's (device mode) or the
// context's staging (host mode, pitch = width).
struct IntPlanes {
    const int *src[kMaxPlanes] = {nullptr, nullptr, nullptr};
    const int *ref[kMaxPlanes] = {nullptr, nullptr, nullptr};
    int *dst[kMaxPlanes] = {nullptr, nullptr, nullptr};
    size_t pitch = 0;
};

int stage_ints_in(bm3d_ctx *ctx, int nplanes, const int *const src[], const int *const ref[],
                  int width, int height, size_t stride, int mem, cudaStream_t s, IntPlanes &io)
{
    int rc;
    if (mem == BM3D_MEM_DEVICE) {
        io.pitch = stride;
        for (int c = 0; c < nplanes; ++c) {
            io.src[c] = src[c];
            io.ref[c] = ref ? ref[c] : nullptr;
        }
        return BM3D_OK;
    }
    io.pitch = static_cast<size_t>(width);
    const size_t bytes = sizeof(int) * static_cast<size_t>(width) * height;
    for (int c = 0; c < nplanes; ++c) {
        if ((rc = ensure(ctx, ctx->ints[c], bytes)) != BM3D_OK) return rc;
        int *d = static_cast<int *>(ctx->ints[c].ptr);
        if ((rc = copy_plane(ctx, d, io.pitch, src[c], stride, width, height,
                             cudaMemcpyHostToDevice, s)) != BM3D_OK)
            return rc;
        io.src[c] = d;
        if (ref && ref[c]) {
            if ((rc = ensure(ctx, ctx->ints[kMaxPlanes + c], bytes)) != BM3D_OK) return rc;
            int *r = static_cast<int *>(ctx->ints[kMaxPlanes + c].ptr);
            if ((rc = copy_plane(ctx, r, io.pitch, ref[c], stride, width, height,
                                 cudaMemcpyHostToDevice, s)) != BM3D_OK)
                return rc;
            io.ref[c] = r;
        }
    }
    return BM3D_OK;
}

int int_outputs(bm3d_ctx *ctx, int nplanes, int *const dst[], int width, int height, int mem,
                IntPlanes &io)
{
    int rc;
    const size_t bytes = sizeof(int) * static_cast<size_t>(width) * height;
    for (int c = 0; c < nplanes; ++c) {
        if (mem == BM3D_MEM_DEVICE) {
            io.dst[c] = dst[c];
        } else {
            if ((rc = ensure(ctx, ctx->ints[2 * kMaxPlanes + c], bytes)) != BM3D_OK) return rc;
            io.dst[c] = static_cast<int *>(ctx->ints[2 * kMaxPlanes + c].ptr);
        }
    }
    return BM3D_OK;
}

int finish_ints(bm3d_ctx *ctx, int nplanes, int *const dst[], int width, int height,
                size_t stride, int mem, cudaStream_t s, const IntPlanes &io, int status)
{
    if (mem == BM3D_MEM_DEVICE) return status;
    int rc;
    for (int c = 0; c < nplanes; ++c)
        if ((rc = copy_plane(ctx, dst[c], stride, static_cast<const int *>(io.dst[c]), io.pitch,
                             width, height, cudaMemcpyDeviceToHost, s)) != BM3D_OK)
            return rc;
    CK(ctx, cudaStreamSynchronize(s));
    rc = check_invariants(ctx);
    return rc != BM3D_OK ? rc : status;
}

// Float working planes (pitch = width): kind 0 = src, 1 = ref, 2 = dst.
int conv_planes(bm3d_ctx *ctx, int kind, int nplanes, int width, int height, float *out[])
{
    int rc;
    const size_t bytes = sizeof(float) * static_cast<size_t>(width) * height;
    for (int c = 0; c < nplanes; ++c) {
        if ((rc = ensure(ctx, ctx->conv[kind * kMaxPlanes + c], bytes)) != BM3D_OK) return rc;
        out[c] = static_cast<float *>(ctx->conv[kind * kMaxPlanes + c].ptr);
    }
    return BM3D_OK;
}

int check_int_call(bm3d_ctx *ctx, int nplanes, const void *const dst[], const void *const src[],
                   int width, int height, size_t stride, int floor_, int ceil_, int mem,
                   const bm3d_stage_params *const ps[], int nps)
{
    if (!ctx) return BM3D_ERR_INVALID;
    if (mem != BM3D_MEM_HOST && mem != BM3D_MEM_DEVICE) return BM3D_ERR_INVALID;
    for (int k = 0; k < nps; ++k)
        if (!ps[k]) return BM3D_ERR_INVALID;
    if (ceil_ <= floor_) return BM3D_ERR_INVALID;
    if (width < 1 || height < 1 || stride < static_cast<size_t>(width)) return BM3D_ERR_INVALID;
    for (int c = 0; c < nplanes; ++c)
        if (!dst[c] || !src[c]) return BM3D_ERR_INVALID;
    return BM3D_OK;
}

int copy_ints(bm3d_ctx *ctx, int nplanes, int *const dst[], const int *const src[], int width,
              int height, size_t stride, int mem, cudaStream_t s)
{
    int rc;
    for (int c = 0; c < nplanes; ++c) {
        if (dst[c] == src[c]) continue;
        if ((rc = copy_plane(ctx, dst[c], stride, src[c], stride, width, height,
                             mem == BM3D_MEM_HOST ? cudaMemcpyHostToHost : cudaMemcpyDeviceToDevice,
                             s)) != BM3D_OK)
            return rc;
    }
    if (mem == BM3D_MEM_HOST) CK(ctx, cudaStreamSynchronize(s));
    return BM3D_COPIED;
}

}  // namespace

extern "C" int bm3d_stage_int(bm3d_ctx *ctx, const bm3d_stage_params *params, int wiener,
                              int32_t *dst, const int32_t *src, const int32_t *ref, int width,
                              int height, size_t stride, int floor_, int neutral, int ceil_,
                              int mem, void *stream)
{
    const void *d[1] = {dst}, *sp[1] = {src};
    const bm3d_stage_params *ps[1] = {params};
    int rc = check_int_call(ctx, 1, d, sp, width, height, stride, floor_, ceil_, mem, ps, 1);
    if (rc != BM3D_OK) return rc;
    if (neutral < floor_ || neutral > ceil_) return BM3D_ERR_INVALID;
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int *dd[1] = {dst};
    const int *ss[1] = {src};
    if (int_path_rejected(params, 1)) return copy_ints(ctx, 1, dd, ss, width, height, stride, mem, s);
    const Quant q{floor_, neutral, ceil_};
    const int *rr[1] = {ref && ref != src ? ref : nullptr};
    IntPlanes io;
    if ((rc = stage_ints_in(ctx, 1, ss, rr, width, height, stride, mem, s, io)) != BM3D_OK) return rc;
    if ((rc = int_outputs(ctx, 1, dd, width, height, mem, io)) != BM3D_OK) return rc;
    float *fs[1], *fr[1], *fd[1];
    if ((rc = conv_planes(ctx, 0, 1, width, height, fs)) != BM3D_OK) return rc;
    if ((rc = conv_planes(ctx, 2, 1, width, height, fd)) != BM3D_OK) return rc;
    const dim3 grid = convert_grid(ctx, width, height);
    const RangeMap in = range_to_float(q);
    int_to_float_kernel<<<grid, 256, 0, s>>>(io.src[0], io.pitch, fs[0], width, width, height, in);
    CK(ctx, cudaGetLastError());
    fr[0] = fs[0];
    if (io.ref[0]) {
        if ((rc = conv_planes(ctx, 1, 1, width, height, fr)) != BM3D_OK) return rc;
        int_to_float_kernel<<<grid, 256, 0, s>>>(io.ref[0], io.pitch, fr[0], width, width, height,
                                                 in);
        CK(ctx, cudaGetLastError());
    }
    const float *cs[1] = {fs[0]}, *cr[1] = {fr[0]};
    const int st = stage_any<float>(ctx, params, wiener, 1, fd, cs, cr, width, height, width, 1.0,
                                    BM3D_MEM_DEVICE, stream);
    if (st < 0) return st;
    float_to_int_kernel<<<grid, 256, 0, s>>>(fd[0], width, io.dst[0], io.pitch, width, height,
                                             range_to_int(q));
    CK(ctx, cudaGetLastError());
    return finish_ints(ctx, 1, dd, width, height, stride, mem, s, io, st);
}

extern "C" int bm3d_plane_int(bm3d_ctx *ctx, const bm3d_stage_params *basic,
                              const bm3d_stage_params *final_, int32_t *dst, const int32_t *src,
                              const int32_t *ref, int width, int height, size_t stride,
                              int floor_, int neutral, int ceil_, int mem, void *stream)
{
    const void *d[1] = {dst}, *sp[1] = {src};
    const bm3d_stage_params *ps[2] = {basic, final_};
    int rc = check_int_call(ctx, 1, d, sp, width, height, stride, floor_, ceil_, mem, ps, 2);
    if (rc != BM3D_OK) return rc;
    if (neutral < floor_ || neutral > ceil_) return BM3D_ERR_INVALID;
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int *dd[1] = {dst};
    const int *ss[1] = {src};
    const Quant q{floor_, neutral, ceil_};
    const int *rr[1] = {ref && ref != src ? ref : nullptr};
    IntPlanes io;
    if ((rc = stage_ints_in(ctx, 1, ss, rr, width, height, stride, mem, s, io)) != BM3D_OK)
        return rc;
    if ((rc = int_outputs(ctx, 1, dd, width, height, mem, io)) != BM3D_OK) return rc;
    float *fs[1], *fd[1], *fr[1];
    if ((rc = conv_planes(ctx, 0, 1, width, height, fs)) != BM3D_OK) return rc;
    if ((rc = conv_planes(ctx, 2, 1, width, height, fd)) != BM3D_OK) return rc;
    const dim3 grid = convert_grid(ctx, width, height);
    const RangeMap in = range_to_float(q);
    int_to_float_kernel<<<grid, 256, 0, s>>>(io.src[0], io.pitch, fs[0], width, width, height, in);
    CK(ctx, cudaGetLastError());
    fr[0] = fs[0];
    if (io.ref[0]) {
        if ((rc = conv_planes(ctx, 1, 1, width, height, fr)) != BM3D_OK) return rc;
        int_to_float_kernel<<<grid, 256, 0, s>>>(io.ref[0], io.pitch, fr[0], width, width, height,
                                                 in);
        CK(ctx, cudaGetLastError());
    }
    const float *cs[1] = {fs[0]}, *cr[1] = {fr[0]};
    const int st = full_any<float>(ctx, basic, final_, 1, fd, cs, cr, width, height, width, 1.0,
                                   BM3D_MEM_DEVICE, stream);
    if (st < 0) return st;
    float_to_int_kernel<<<grid, 256, 0, s>>>(fd[0], width, io.dst[0], io.pitch, width, height,
                                             range_to_int(q));
    CK(ctx, cudaGetLastError());
    return finish_ints(ctx, 1, dd, width, height, stride, mem, s, io, st);
}

extern "C" int bm3d_frame(bm3d_ctx *ctx, const bm3d_stage_params *basic,
                          const bm3d_stage_params *final_, int32_t *const dst[3],
                          const int32_t *const src[3], const int32_t *const ref[3], int width,
                          int height, size_t stride, int floor_, int ceil_, int mem,
                          void *stream)
{
    if (!dst || !src) return BM3D_ERR_INVALID;
    const void *d[3] = {dst[0], dst[1], dst[2]}, *sp[3] = {src[0], src[1], src[2]};
    const bm3d_stage_params *ps[2] = {basic, final_};
    int rc = check_int_call(ctx, 3, d, sp, width, height, stride, floor_, ceil_, mem, ps, 2);
    if (rc != BM3D_OK) return rc;
    if (ref && (!ref[0] || !ref[1] || !ref[2])) return BM3D_ERR_INVALID;
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // a distinct ref frame (the reference compares the three plane pointers)
    const bool own_ref = ref && !(ref[0] == src[0] && ref[1] == src[1] && ref[2] == src[2]);
    IntPlanes io;
    if ((rc = stage_ints_in(ctx, 3, src, own_ref ? ref : nullptr, width, height, stride, mem, s,
                            io)) != BM3D_OK)
        return rc;
    if ((rc = int_outputs(ctx, 3, dst, width, height, mem, io)) != BM3D_OK) return rc;
    float *fs[3], *fd[3], *fr[1];
    if ((rc = conv_planes(ctx, 0, 3, width, height, fs)) != BM3D_OK) return rc;
    if ((rc = conv_planes(ctx, 2, 3, width, height, fd)) != BM3D_OK) return rc;
    const dim3 grid = convert_grid(ctx, width, height);
    rgb_to_opp_kernel<<<grid, 256, 0, s>>>(io.src[0], io.src[1], io.src[2], io.pitch, fs[0], fs[1],
                                           fs[2], width, width, height, opp_forward(floor_, ceil_),
                                           0);
    CK(ctx, cudaGetLastError());
    fr[0] = fs[0];
    if (own_ref) {  // only Y of ref (BM3D_Basic::RGB2YUV, source/BM3D.cpp:333)
        if ((rc = conv_planes(ctx, 1, 1, width, height, fr)) != BM3D_OK) return rc;
        rgb_to_opp_kernel<<<grid, 256, 0, s>>>(io.ref[0], io.ref[1], io.ref[2], io.pitch, fr[0],
                                               fr[0], fr[0], width, width, height,
                                               opp_forward(floor_, ceil_), 1);
        CK(ctx, cudaGetLastError());
    }
    const float *cs[3] = {fs[0], fs[1], fs[2]}, *cr[3] = {fr[0], fs[1], fs[2]};
    const int st = full_any<float>(ctx, basic, final_, 3, fd, cs, cr, width, height, width, 1.0,
                                   BM3D_MEM_DEVICE, stream);
    if (st < 0) return st;
    opp_to_rgb_kernel<<<grid, 256, 0, s>>>(fd[0], fd[1], fd[2], width, io.dst[0], io.dst[1],
                                           io.dst[2], io.pitch, width, height,
                                           opp_inverse(floor_, ceil_));
    CK(ctx, cudaGetLastError());
    return finish_ints(ctx, 3, dst, width, height, stride, mem, s, io, st);
}

extern "C" int bm3d_stage_frame(bm3d_ctx *ctx, const bm3d_stage_params *params, int wiener,
                                int32_t *const dst[3], const int32_t *const src[3],
                                const int32_t *const ref[3], int width, int height, size_t stride,
                                int floor_, int ceil_, int mem, void *stream)
{
    if (!dst || !src) return BM3D_ERR_INVALID;
    const void *d[3] = {dst[0], dst[1], dst[2]}, *sp[3] = {src[0], src[1], src[2]};
    const bm3d_stage_params *ps[1] = {params};
    int rc = check_int_call(ctx, 3, d, sp, width, height, stride, floor_, ceil_, mem, ps, 1);
    if (rc != BM3D_OK) return rc;
    if (ref && (!ref[0] || !ref[1] || !ref[2])) return BM3D_ERR_INVALID;
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (int_path_rejected(params, 3)) return copy_ints(ctx, 3, dst, src, width, height, stride, mem, s);
    // a distinct ref frame (the reference compares the three plane pointers)
    const bool own_ref = ref && !(ref[0] == src[0] && ref[1] == src[1] && ref[2] == src[2]);
    IntPlanes io;
    if ((rc = stage_ints_in(ctx, 3, src, own_ref ? ref : nullptr, width, height, stride, mem, s,
                            io)) != BM3D_OK)
        return rc;
    if ((rc = int_outputs(ctx, 3, dst, width, height, mem, io)) != BM3D_OK) return rc;
    float *fs[3], *fr[3];
    if ((rc = conv_planes(ctx, 0, 3, width, height, fs)) != BM3D_OK) return rc;
    const dim3 grid = convert_grid(ctx, width, height);
    rgb_to_opp_kernel<<<grid, 256, 0, s>>>(io.src[0], io.src[1], io.src[2], io.pitch, fs[0], fs[1],
                                           fs[2], width, width, height, opp_forward(floor_, ceil_),
                                           0);
    CK(ctx, cudaGetLastError());
    for (int c = 0; c < 3; ++c) fr[c] = fs[c];
    if (own_ref) {
        if ((rc = conv_planes(ctx, 1, wiener ? 3 : 1, width, height, fr)) != BM3D_OK) return rc;
        if (!wiener) fr[1] = fr[2] = fr[0];  // the basic stage reads only Y of ref
        rgb_to_opp_kernel<<<grid, 256, 0, s>>>(io.ref[0], io.ref[1], io.ref[2], io.pitch, fr[0],
                                               fr[1], fr[2], width, width, height,
                                               opp_forward(floor_, ceil_), wiener ? 0 : 1);
        CK(ctx, cudaGetLastError());
    }
    // in place on the YUV source, as the reference (planes a stage leaves
    // alone keep their converted values)
    const float *cs[3] = {fs[0], fs[1], fs[2]}, *cr[3] = {fr[0], fr[1], fr[2]};
    const int st = stage_any<float>(ctx, params, wiener, 3, fs, cs, cr, width, height, width, 1.0,
                                    BM3D_MEM_DEVICE, stream);
    if (st < 0) return st;
    opp_to_rgb_kernel<<<grid, 256, 0, s>>>(fs[0], fs[1], fs[2], width, io.dst[0], io.dst[1],
                                           io.dst[2], io.pitch, width, height,
                                           opp_inverse(floor_, ceil_));
    CK(ctx, cudaGetLastError());
    return finish_ints(ctx, 3, dst, width, height, stride, mem, s, io, st);
}

