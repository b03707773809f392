/* Oracle (test infrastructure only): a C entry layer around the reference's
 * own BM3D classes, compiled together with the reference's unmodified
 * source/BM3D.cpp and source/Image_Type.cpp into oracle/_ref/libbm3d_ref_*.so.
 * Tests and the CPU-baseline leg of bench.py load it with ctypes; the product
 * never does.
 *
 * Entry points follow the reference's working call sequences:
 *   - one stage:  BM3D_Basic(p).process(dst, src, ref) / BM3D_Final(p).process(...)
 *                 through FilterIF2::process (include/Filter.h:174) with a
 *                 pre-sized dst (the reference's combined BM3D::process_Plane_FL,
 *                 source/BM3D.cpp:464-472, passes an empty tmp and is not used);
 *   - three planes sharing luma groups: the public 9-plane BM3D_Base::Kernel
 *                 (source/BM3D.cpp:139-218);
 *   - the group list of every reference block: BM3D_Base::BlockMatching
 *                 (source/BM3D.cpp:221-236) over the scan of source/BM3D.cpp:98-121.
 * FLType is float when built with -D_CUDA_ and double otherwise
 * (include/Type.h:26-30). */
#include "BM3D.h"
#include "Conversion.hpp"

#include <cstring>

extern "C" {

/* Mirrors the numeric fields of BM3D_Para_Base (include/BM3D.h:15-45). */
typedef struct ref_stage_params {
    int block_size;
    int block_step;
    int group_size;
    int bm_range;
    int bm_step;
    double thMSE;
    double lambda;
    double sigma[3];
} ref_stage_params;

int ref_flt_size(void) { return (int)sizeof(FLType); }

/* Profile defaults from the reference's own parameter constructors
 * (include/BM3D.h:54-97 basic, 107-150 final), with sigma set and
 * thMSE_Default() re-run as BM3D_IO does (include/BM3D.h:492-504). */
int ref_stage_default(const char *profile, int wiener, const double sigma[3],
                      ref_stage_params *out)
{
    std::string prof(profile);
    if (prof != "fast" && prof != "lc" && prof != "np" && prof != "high" && prof != "vn") return 1;
    BM3D_Para_Base *p;
    BM3D_Basic_Para b(prof);
    BM3D_Final_Para f(prof);
    p = wiener ? static_cast<BM3D_Para_Base *>(&f) : static_cast<BM3D_Para_Base *>(&b);
    p->sigma = {sigma[0], sigma[1], sigma[2]};
    p->thMSE_Default();
    out->block_size = p->BlockSize;
    out->block_step = p->BlockStep;
    out->group_size = p->GroupSize;
    out->bm_range = p->BMrange;
    out->bm_step = p->BMstep;
    out->thMSE = p->thMSE;
    out->lambda = p->lambda;
    for (int i = 0; i < 3; ++i) out->sigma[i] = p->sigma[i];
    return 0;
}

}  // extern "C"

template <typename P>
static void fill_para(P &p, const ref_stage_params *s)
{
    p.sigma = {s->sigma[0], s->sigma[1], s->sigma[2]};
    p.BlockSize = s->block_size;
    p.BlockStep = s->block_step;
    p.GroupSize = s->group_size;
    p.BMrange = s->bm_range;
    p.BMstep = s->bm_step;
    p.thMSE = s->thMSE;
    p.lambda = s->lambda;
}

static Plane_FL make_plane(const FLType *data, int w, int h, double value_range, bool chroma)
{
    FLType range = static_cast<FLType>(value_range);
    FLType floor = chroma ? -range / 2 : 0;
    FLType ceil = chroma ? range / 2 : range;
    Plane_FL p(FLType(0), w, h, floor, FLType(0), ceil, TransferChar::linear, false);
    if (data) std::memcpy(p.data(), data, sizeof(FLType) * (size_t)w * (size_t)h);
    return p;
}

namespace {

/* Exposes the protected BlockMatching of each stage for the group dump. */
class BasicProbe : public BM3D_Basic
{
public:
    explicit BasicProbe(const BM3D_Basic_Para &p) : BM3D_Basic(p) {}
    PosPairCode match(const Plane_FL &ref, PCType j, PCType i) const { return BlockMatching(ref, j, i); }
    const BM3D_Para_Base &params() const { return para; }
};

class FinalProbe : public BM3D_Final
{
public:
    explicit FinalProbe(const BM3D_Final_Para &p) : BM3D_Final(p) {}
    PosPairCode match(const Plane_FL &ref, PCType j, PCType i) const { return BlockMatching(ref, j, i); }
    const BM3D_Para_Base &params() const { return para; }
};

template <typename Probe>
long long dump_groups(const Probe &probe, const Plane_FL &ref, int max_refs, int max_group,
                      int *counts, int *pos_yx, FLType *keys)
{
    const BM3D_Para_Base &para = probe.params();
    const PCType width = ref.Width(), height = ref.Height();
    const PCType right = width - para.BlockSize, bottom = height - para.BlockSize;
    long long r = 0;
    /* Same reference-block scan as BM3D_Base::Kernel (source/BM3D.cpp:98-121). */
    for (PCType j = 0;; j += para.BlockStep) {
        if (j >= bottom + para.BlockStep) break;
        if (j > bottom) j = bottom;
        for (PCType i = 0;; i += para.BlockStep) {
            if (i >= right + para.BlockStep) break;
            if (i > right) i = right;
            auto code = probe.match(ref, j, i);
            if (r < max_refs) {
                int n = (int)code.size();
                if (para.GroupSize > 0 && n > para.GroupSize) n = para.GroupSize;
                counts[r] = n;
                for (int z = 0; z < n && z < max_group; ++z) {
                    pos_yx[(r * max_group + z) * 2 + 0] = code[z].second.y;
                    pos_yx[(r * max_group + z) * 2 + 1] = code[z].second.x;
                    keys[r * max_group + z] = code[z].first;
                }
            }
            ++r;
        }
    }
    return r;
}

}  // namespace

extern "C" {

/* One stage on one plane: dst = BM3D_{Basic|Final}(params).process(src, ref). */
int ref_bm3d_stage(int wiener, const ref_stage_params *s, FLType *dst, const FLType *src,
                   const FLType *ref, int width, int height, double value_range)
{
    Plane_FL srcP = make_plane(src, width, height, value_range, false);
    Plane_FL refP = make_plane(ref, width, height, value_range, false);
    Plane_FL dstP(srcP, false);
    if (wiener) {
        BM3D_Final_Para p("fast");
        fill_para(p, s);
        BM3D_Final filter(p);
        filter.process(dstP, srcP, refP);
    } else {
        BM3D_Basic_Para p("fast");
        fill_para(p, s);
        BM3D_Basic filter(p);
        filter.process(dstP, srcP, refP);
    }
    std::memcpy(dst, dstP.data(), sizeof(FLType) * (size_t)width * (size_t)height);
    return 0;
}

/* Three planes sharing the luma groups: the public 9-plane BM3D_Base::Kernel. */
int ref_bm3d_stage3(int wiener, const ref_stage_params *s, FLType *const dst[3],
                    const FLType *const src[3], const FLType *const ref[3], int width, int height,
                    double value_range)
{
    Plane_FL sY = make_plane(src[0], width, height, value_range, false);
    Plane_FL sU = make_plane(src[1], width, height, value_range, true);
    Plane_FL sV = make_plane(src[2], width, height, value_range, true);
    Plane_FL rY = make_plane(ref[0], width, height, value_range, false);
    Plane_FL rU = make_plane(ref[1], width, height, value_range, true);
    Plane_FL rV = make_plane(ref[2], width, height, value_range, true);
    Plane_FL dY(sY, false), dU(sU, false), dV(sV, false);
    if (wiener) {
        BM3D_Final_Para p("fast");
        fill_para(p, s);
        BM3D_Final(p).Kernel(dY, dU, dV, sY, sU, sV, rY, rU, rV);
    } else {
        BM3D_Basic_Para p("fast");
        fill_para(p, s);
        BM3D_Basic(p).Kernel(dY, dU, dV, sY, sU, sV, rY, rU, rV);
    }
    const size_t n = sizeof(FLType) * (size_t)width * (size_t)height;
    std::memcpy(dst[0], dY.data(), n);
    std::memcpy(dst[1], dU.data(), n);
    std::memcpy(dst[2], dV.data(), n);
    return 0;
}

/* Group of every reference block in scan order: count, (y, x) and key of each
 * member. Returns the number of reference blocks (arrays hold max_refs). */
long long ref_bm3d_groups(int wiener, const ref_stage_params *s, const FLType *ref, int width,
                          int height, double value_range, int max_refs, int max_group, int *counts,
                          int *pos_yx, FLType *keys)
{
    Plane_FL refP = make_plane(ref, width, height, value_range, false);
    if (wiener) {
        BM3D_Final_Para p("fast");
        fill_para(p, s);
        FinalProbe probe(p);
        return dump_groups(probe, refP, max_refs, max_group, counts, pos_yx, keys);
    }
    BM3D_Basic_Para p("fast");
    fill_para(p, s);
    BasicProbe probe(p);
    return dump_groups(probe, refP, max_refs, max_group, counts, pos_yx, keys);
}

}  // extern "C"

extern "C" {

/* BM3D on an RGB Frame: FilterIF2::operator()(Frame) -> BM3D::process_Frame
 * (source/BM3D.cpp:501-527): OPP RGB->YUV, three-plane basic then final,
 * YUV->RGB with clipping. Planes are the reference's DType (int32) with the
 * Frame's quantisation: bit depth `bits`, full (PC) range when `pc`. `ref`
 * may be null (ref = src). */
int ref_bm3d_frame(const ref_stage_params *b, const ref_stage_params *f, int *const dst[3],
                   const int *const src[3], const int *const ref[3], int width, int height,
                   int bits, int pc)
{
    const QuantRange q = pc ? QuantRange::PC : QuantRange::TV;
    Frame in(0, PixelType::RGB, width, height, bits, q);
    Frame rf(0, PixelType::RGB, width, height, bits, q);
    const size_t n = sizeof(int) * (size_t)width * (size_t)height;
    std::memcpy(in.R().data(), src[0], n);
    std::memcpy(in.G().data(), src[1], n);
    std::memcpy(in.B().data(), src[2], n);
    if (ref) {
        std::memcpy(rf.R().data(), ref[0], n);
        std::memcpy(rf.G().data(), ref[1], n);
        std::memcpy(rf.B().data(), ref[2], n);
    }
    BM3D_Para para("fast");
    fill_para(para.basic, b);
    fill_para(para.final, f);
    BM3D filter(para);
    Frame out = ref ? filter(in, rf) : filter(in);
    std::memcpy(dst[0], out.R().data(), n);
    std::memcpy(dst[1], out.G().data(), n);
    std::memcpy(dst[2], out.B().data(), n);
    return 0;
}

/* BM3D (basic then final) on an integer Plane. BM3D::process_Plane
 * (source/BM3D.cpp:475-497) converts with RangeConvert to a float plane of
 * range 1 and back with clipping, but its process_Plane_FL (464-472) hands
 * the basic stage a default-constructed 0x0 `tmp`, so the reference fails
 * its size check there. This entry runs the same sequence from the
 * reference's own pieces with `tmp` sized like the source, the evident
 * intent. The plane's quantisation is (bits, floor, neutral, ceil);
 * neutral > floor marks a chroma plane. `ref` may be null (ref = src). */
int ref_bm3d_plane_int(const ref_stage_params *b, const ref_stage_params *f, int *dst,
                       const int *src, const int *ref, int width, int height, int bits,
                       int floor_, int neutral, int ceil_)
{
    Plane in(0, width, height, bits, floor_, neutral, ceil_, TransferChar::linear, false);
    std::memcpy(in.data(), src, sizeof(int) * (size_t)width * (size_t)height);
    Plane out(in, false);
    BM3D_Para para("fast");
    fill_para(para.basic, b);
    fill_para(para.final, f);
    BM3D_Basic basic(para.basic);
    BM3D_Final final(para.final);
    Plane_FL dst_data(out, false);
    Plane_FL src_data(in, false);
    RangeConvert(src_data, in, false);
    Plane_FL tmp(src_data, false);
    if (ref) {
        Plane rp(in, false);
        std::memcpy(rp.data(), ref, sizeof(int) * (size_t)width * (size_t)height);
        Plane_FL ref_data(rp, false);
        RangeConvert(ref_data, rp, false);
        basic.Kernel(tmp, src_data, ref_data);
    } else {
        basic.Kernel(tmp, src_data, src_data);
    }
    final.Kernel(dst_data, src_data, tmp);
    RangeConvert(out, dst_data, true);
    std::memcpy(dst, out.data(), sizeof(int) * (size_t)width * (size_t)height);
    return 0;
}

/* One stage on an integer Plane: BM3D_Basic or BM3D_Final used as a filter,
 * BM3D_Base::process_Plane (source/BM3D.cpp:248-281). `ref` may be null
 * (ref = src). */
int ref_bm3d_stage_int(int wiener, const ref_stage_params *p, int *dst, const int *src,
                       const int *ref, int width, int height, int bits, int floor_, int neutral,
                       int ceil_)
{
    const size_t n = sizeof(int) * (size_t)width * (size_t)height;
    Plane in(0, width, height, bits, floor_, neutral, ceil_, TransferChar::linear, false);
    std::memcpy(in.data(), src, n);
    Plane rf(in, false);
    if (ref) std::memcpy(rf.data(), ref, n);
    BM3D_Para para("fast");
    Plane out;
    if (!wiener) {
        fill_para(para.basic, p);
        BM3D_Basic filt(para.basic);
        out = ref ? filt(in, rf) : filt(in);
    } else {
        fill_para(para.final, p);
        BM3D_Final filt(para.final);
        out = ref ? filt(in, rf) : filt(in);
    }
    std::memcpy(dst, out.data(), n);
    return 0;
}

/* One stage on an RGB Frame: BM3D_Basic or BM3D_Final used as a filter,
 * BM3D_Base::process_Frame (source/BM3D.cpp:284-313) with the stage's
 * RGB2YUV (320-336 basic: Y of ref only; 392-408 final: all of ref). `ref`
 * may be null (ref = src). */
int ref_bm3d_stage_frame(int wiener, const ref_stage_params *p, int *const dst[3],
                         const int *const src[3], const int *const ref[3], int width, int height,
                         int bits, int pc)
{
    const size_t n = sizeof(int) * (size_t)width * (size_t)height;
    const QuantRange q = pc ? QuantRange::PC : QuantRange::TV;
    Frame in(0, PixelType::RGB, width, height, bits, q);
    Frame rf(0, PixelType::RGB, width, height, bits, q);
    std::memcpy(in.R().data(), src[0], n);
    std::memcpy(in.G().data(), src[1], n);
    std::memcpy(in.B().data(), src[2], n);
    if (ref) {
        std::memcpy(rf.R().data(), ref[0], n);
        std::memcpy(rf.G().data(), ref[1], n);
        std::memcpy(rf.B().data(), ref[2], n);
    }
    BM3D_Para para("fast");
    Frame out;
    if (!wiener) {
        fill_para(para.basic, p);
        BM3D_Basic filt(para.basic);
        out = ref ? filt(in, rf) : filt(in);
    } else {
        fill_para(para.final, p);
        BM3D_Final filt(para.final);
        out = ref ? filt(in, rf) : filt(in);
    }
    std::memcpy(dst[0], out.R().data(), n);
    std::memcpy(dst[1], out.G().data(), n);
    std::memcpy(dst[2], out.B().data(), n);
    return 0;
}

}  // extern "C"
