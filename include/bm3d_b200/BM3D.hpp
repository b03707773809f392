// C++ drop-in for the BM3D filter classes of mawen1250/ISP_MW
// (include/BM3D.h, include/Filter.h, include/Image_Type.h), implemented on the
// C ABI of bm3d_b200.h. Code written against the reference's
//
//     BM3D_Para para("fast");
//     para.basic.sigma = {s, s, s}; para.final.sigma = para.basic.sigma;
//     para.thMSE_Default();
//     Plane_FL tmp(src, false), dst(src, false);
//     BM3D_Basic(para.basic).process(tmp, src, src);
//     BM3D_Final(para.final).process(dst, src, tmp);
//
// compiles unchanged against this header and runs on the GPU.
//
// Differences from the reference, all deliberate:
//   - Plane_FL here is a minimal float plane (size, range, data); FLType is float.
//   - Errors throw bm3d_b200::Error instead of exiting the process.
//   - BM3D::process(dst, src) sizes its intermediate from src (the reference's
//     BM3D::process_Plane_FL passes an empty plane, source/BM3D.cpp:464-472).
//   - Plane (int32) and Frame are minimal: size, quantisation (Floor, Neutral,
//     Ceil, bit depth) and data; a Frame here is always RGB, the only kind the
//     reference's BM3D::process_Frame handles (source/BM3D.cpp:501-527).
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../bm3d_b200.h"

namespace bm3d_b200 {

typedef float FLType;
typedef int PCType;

class Error : public std::runtime_error {
public:
    Error(int code, const std::string &msg)
        : std::runtime_error("bm3d_b200 status " + std::to_string(code) + ": " + msg), code(code)
    {}
    int code;
};

// Minimal counterpart of the reference's Plane_FL (include/Image_Type.h:176-291):
// row-major, stride = width, Floor/Neutral/Ceil with ValueRange = Ceil - Floor.
class Plane_FL {
public:
    typedef FLType value_type;

    Plane_FL() {}
    explicit Plane_FL(value_type value, PCType width = 1920, PCType height = 1080,
                      bool RGB = true, bool chroma = false, bool init = true)
        : w_(width), h_(height), data_(static_cast<size_t>(width) * height)
    {
        if (!RGB && chroma) {
            floor_ = -0.5f;
            ceil_ = 0.5f;
        }
        if (init) for (auto &x : data_) x = value;
    }
    Plane_FL(value_type value, PCType width, PCType height, value_type floor, value_type neutral,
             value_type ceil, bool init = true)
        : w_(width), h_(height), floor_(floor), neutral_(neutral), ceil_(ceil),
          data_(static_cast<size_t>(width) * height)
    {
        if (init) for (auto &x : data_) x = value;
    }
    // Same size and range as src; filled with `value` when init (include/Image_Type.h:220).
    Plane_FL(const Plane_FL &src, bool init, value_type value = 0)
        : w_(src.w_), h_(src.h_), floor_(src.floor_), neutral_(src.neutral_), ceil_(src.ceil_),
          data_(src.data_.size())
    {
        if (init) for (auto &x : data_) x = value;
    }
    Plane_FL(const Plane_FL &) = default;
    Plane_FL(Plane_FL &&) = default;
    Plane_FL &operator=(const Plane_FL &) = default;
    Plane_FL &operator=(Plane_FL &&) = default;

    PCType Width() const { return w_; }
    PCType Height() const { return h_; }
    PCType Stride() const { return w_; }
    PCType PixelCount() const { return w_ * h_; }
    size_t size() const { return data_.size(); }
    value_type Floor() const { return floor_; }
    value_type Neutral() const { return neutral_; }
    value_type Ceil() const { return ceil_; }
    value_type ValueRange() const { return ceil_ - floor_; }
    value_type *data() { return data_.data(); }
    const value_type *data() const { return data_.data(); }
    value_type &operator[](PCType i) { return data_[i]; }
    const value_type &operator[](PCType i) const { return data_[i]; }
    value_type &operator()(PCType j, PCType i) { return data_[static_cast<size_t>(j) * w_ + i]; }
    const value_type &operator()(PCType j, PCType i) const
    {
        return data_[static_cast<size_t>(j) * w_ + i];
    }
    Plane_FL &ReSize(PCType width, PCType height)
    {
        w_ = width;
        h_ = height;
        data_.resize(static_cast<size_t>(width) * height);
        return *this;
    }

private:
    PCType w_ = 0, h_ = 0;
    value_type floor_ = 0, neutral_ = 0, ceil_ = 1;
    std::vector<value_type> data_;
};

// Minimal counterpart of the reference's integer Plane (include/Image_Type.h:
// 46-173): row-major int32 (DType), stride = width, with its quantisation.
// Default quantisation: full range of `bits` (include/Image_Type.hpp:94-109);
// chroma planes have Neutral = 2^(bits-1).
class Plane {
public:
    typedef int32_t value_type;

    Plane() {}
    explicit Plane(value_type value, PCType width = 1920, PCType height = 1080,
                   value_type bits = 16, bool init = true)
        : w_(width), h_(height), bits_(bits), ceil_((1 << bits) - 1),
          data_(static_cast<size_t>(width) * height)
    {
        if (init) for (auto &x : data_) x = value;
    }
    Plane(value_type value, PCType width, PCType height, value_type bits, value_type floor,
          value_type neutral, value_type ceil, bool init = true)
        : w_(width), h_(height), bits_(bits), floor_(floor), neutral_(neutral), ceil_(ceil),
          data_(static_cast<size_t>(width) * height)
    {
        if (init) for (auto &x : data_) x = value;
    }
    // Same size and quantisation as src (include/Image_Type.h:95).
    Plane(const Plane &src, bool init, value_type value = 0)
        : w_(src.w_), h_(src.h_), bits_(src.bits_), floor_(src.floor_), neutral_(src.neutral_),
          ceil_(src.ceil_), data_(src.data_.size())
    {
        if (init) for (auto &x : data_) x = value;
    }
    Plane(const Plane &) = default;
    Plane(Plane &&) = default;
    Plane &operator=(const Plane &) = default;
    Plane &operator=(Plane &&) = default;

    PCType Width() const { return w_; }
    PCType Height() const { return h_; }
    PCType Stride() const { return w_; }
    PCType PixelCount() const { return w_ * h_; }
    value_type BitDepth() const { return bits_; }
    value_type Floor() const { return floor_; }
    value_type Neutral() const { return neutral_; }
    value_type Ceil() const { return ceil_; }
    value_type ValueRange() const { return ceil_ - floor_; }
    bool isChroma() const { return floor_ < neutral_; }
    value_type *data() { return data_.data(); }
    const value_type *data() const { return data_.data(); }
    value_type &operator[](PCType i) { return data_[i]; }
    const value_type &operator[](PCType i) const { return data_[i]; }
    value_type &operator()(PCType j, PCType i) { return data_[static_cast<size_t>(j) * w_ + i]; }
    const value_type &operator()(PCType j, PCType i) const
    {
        return data_[static_cast<size_t>(j) * w_ + i];
    }

private:
    PCType w_ = 0, h_ = 0;
    value_type bits_ = 16, floor_ = 0, neutral_ = 0, ceil_ = 65535;
    std::vector<value_type> data_;
};

// Minimal RGB Frame (include/Image_Type.h:294-420 with PixelType::RGB): three
// Planes of one quantisation; full range (PC) or limited range (TV,
// [16, 235] << (bits - 8)) as Quantize_Value gives RGB planes.
class Frame {
public:
    Frame() {}
    Frame(int32_t value, PCType width, PCType height, int32_t bits = 8, bool full_range = true)
    {
        const int32_t lo = full_range ? 0 : 16 << (bits - 8);
        const int32_t hi = full_range ? (1 << bits) - 1 : 235 << (bits - 8);
        for (auto &p : p_) p = Plane(value, width, height, bits, lo, lo, hi);
    }
    Frame(const Frame &src, bool init, int32_t value = 0)
    {
        for (int i = 0; i < 3; ++i) p_[i] = Plane(src.p_[i], init, value);
    }
    Frame(const Frame &) = default;
    Frame(Frame &&) = default;
    Frame &operator=(const Frame &) = default;
    Frame &operator=(Frame &&) = default;

    Plane &R() { return p_[0]; }
    Plane &G() { return p_[1]; }
    Plane &B() { return p_[2]; }
    const Plane &R() const { return p_[0]; }
    const Plane &G() const { return p_[1]; }
    const Plane &B() const { return p_[2]; }
    Plane &P(int i) { return p_[i]; }
    const Plane &P(int i) const { return p_[i]; }
    PCType Width() const { return p_[0].Width(); }
    PCType Height() const { return p_[0].Height(); }

private:
    Plane p_[3];
};

// Shared device context: one per process and device, created on first use.
inline bm3d_ctx *default_context(int device = 0)
{
    struct Holder {
        bm3d_ctx *ctx = nullptr;
        ~Holder()
        {
            if (ctx) bm3d_ctx_destroy(ctx);
        }
    };
    static Holder h;
    if (!h.ctx) {
        int rc = bm3d_ctx_create(&h.ctx, device);
        if (rc != BM3D_OK) throw Error(rc, bm3d_last_error(nullptr));
    }
    return h.ctx;
}

inline void check(bm3d_ctx *ctx, int rc)
{
    if (rc != BM3D_OK && rc != BM3D_COPIED) throw Error(rc, bm3d_last_error(ctx));
}

// BM3D_Para_Base (include/BM3D.h:15-45).
struct BM3D_Para_Base {
    std::string profile;
    std::vector<double> sigma;
    PCType BlockSize = 8;
    PCType BlockStep = 8;
    PCType GroupSize = 16;
    PCType BMrange = 9;
    PCType BMstep = 1;
    double thMSE = 0;
    double lambda = 0;

    explicit BM3D_Para_Base(std::string p = "fast", bool wiener = false)
        : profile(std::move(p)), sigma({10.0, 10.0, 10.0}), wiener_(wiener)
    {
        bm3d_stage_params s;
        if (bm3d_stage_params_default(profile.c_str(), wiener_, sigma.data(), &s) != BM3D_OK)
            throw Error(BM3D_ERR_INVALID, "unrecognized profile \"" + profile + "\"");
        BlockSize = s.block_size;
        BlockStep = s.block_step;
        GroupSize = s.group_size;
        BMrange = s.bm_range;
        BMstep = s.bm_step;
        thMSE = s.thMSE;
        lambda = s.lambda;
    }
    virtual ~BM3D_Para_Base() {}

    virtual void thMSE_Default()
    {
        bm3d_stage_params s = to_c();
        bm3d_stage_params_thmse_default(profile.c_str(), wiener_, &s);
        thMSE = s.thMSE;
    }

    bm3d_stage_params to_c() const
    {
        bm3d_stage_params s;
        s.block_size = BlockSize;
        s.block_step = BlockStep;
        s.group_size = GroupSize;
        s.bm_range = BMrange;
        s.bm_step = BMstep;
        s.thMSE = thMSE;
        s.lambda = lambda;
        for (int i = 0; i < 3; ++i)
            s.sigma[i] = i < static_cast<int>(sigma.size()) ? sigma[i]
                                                            : (sigma.empty() ? 0.0 : sigma.back());
        return s;
    }

protected:
    bool wiener_;
};

// BM3D_Basic_Para (include/BM3D.h:48-98).
struct BM3D_Basic_Para : BM3D_Para_Base {
    explicit BM3D_Basic_Para(std::string p = "fast") : BM3D_Para_Base(std::move(p), false) {}
};

// BM3D_Final_Para (include/BM3D.h:101-151).
struct BM3D_Final_Para : BM3D_Para_Base {
    explicit BM3D_Final_Para(std::string p = "fast") : BM3D_Para_Base(std::move(p), true) {}
};

// BM3D_Para (include/BM3D.h:154-168).
struct BM3D_Para {
    BM3D_Basic_Para basic;
    BM3D_Final_Para final;
    BM3D_Para(std::string p = "fast") : basic(p), final(p) {}
    void thMSE_Default()
    {
        basic.thMSE_Default();
        final.thMSE_Default();
    }
};

// FilterIF2-style stage (include/Filter.h:138-217; include/BM3D.h:217-334).
class BM3D_Base {
public:
    BM3D_Base(const BM3D_Para_Base &para, bool wiener, bm3d_ctx *ctx)
        : para_(para.to_c()), wiener_(wiener), ctx_(ctx)
    {}

    Plane_FL &process(Plane_FL &dst, const Plane_FL &src, const Plane_FL &ref)
    {
        if (dst.Width() != src.Width() || dst.Height() != src.Height())
            dst.ReSize(src.Width(), src.Height());
        bm3d_ctx *c = ctx();
        check(c, bm3d_stage(c, &para_, wiener_, dst.data(), src.data(), ref.data(), src.Width(),
                            src.Height(), static_cast<size_t>(src.Stride()), ref.ValueRange(),
                            BM3D_MEM_HOST, nullptr));
        return dst;
    }
    Plane_FL &process(Plane_FL &dst, const Plane_FL &src) { return process(dst, src, src); }
    Plane_FL operator()(const Plane_FL &src, const Plane_FL &ref)
    {
        Plane_FL dst(src, false);
        return process(dst, src, ref);
    }
    Plane_FL operator()(const Plane_FL &src)
    {
        Plane_FL dst(src, false);
        return process(dst, src, src);
    }

    // Integer plane: BM3D_Base::process_Plane (source/BM3D.cpp:248-281).
    Plane &process(Plane &dst, const Plane &src, const Plane &ref)
    {
        if (dst.Width() != src.Width() || dst.Height() != src.Height()) dst = Plane(src, false);
        bm3d_ctx *c = ctx();
        check(c, bm3d_stage_int(c, &para_, wiener_, dst.data(), src.data(),
                                &ref == &src ? nullptr : ref.data(), src.Width(), src.Height(),
                                static_cast<size_t>(src.Stride()), src.Floor(), src.Neutral(),
                                src.Ceil(), BM3D_MEM_HOST, nullptr));
        return dst;
    }
    Plane &process(Plane &dst, const Plane &src) { return process(dst, src, src); }
    Plane operator()(const Plane &src, const Plane &ref)
    {
        Plane dst(src, false);
        return process(dst, src, ref);
    }
    Plane operator()(const Plane &src)
    {
        Plane dst(src, false);
        return process(dst, src, src);
    }

    // RGB frame: BM3D_Base::process_Frame (source/BM3D.cpp:284-313).
    Frame &process(Frame &dst, const Frame &src, const Frame &ref)
    {
        if (dst.Width() != src.Width() || dst.Height() != src.Height()) dst = Frame(src, false);
        int32_t *d[3] = {dst.R().data(), dst.G().data(), dst.B().data()};
        const int32_t *s[3] = {src.R().data(), src.G().data(), src.B().data()};
        const int32_t *r[3] = {ref.R().data(), ref.G().data(), ref.B().data()};
        bm3d_ctx *c = ctx();
        check(c, bm3d_stage_frame(c, &para_, wiener_, d, s, r, src.Width(), src.Height(),
                                  static_cast<size_t>(src.R().Stride()), src.R().Floor(),
                                  src.R().Ceil(), BM3D_MEM_HOST, nullptr));
        return dst;
    }
    Frame &process(Frame &dst, const Frame &src) { return process(dst, src, src); }
    Frame operator()(const Frame &src, const Frame &ref)
    {
        Frame dst(src, false);
        return process(dst, src, ref);
    }
    Frame operator()(const Frame &src)
    {
        Frame dst(src, false);
        return process(dst, src, src);
    }

    // Three planes sharing luma groups: BM3D_Base::Kernel's 9-plane form
    // (source/BM3D.cpp:139-218).
    void Kernel(Plane_FL &dstY, Plane_FL &dstU, Plane_FL &dstV, const Plane_FL &srcY,
                const Plane_FL &srcU, const Plane_FL &srcV, const Plane_FL &refY,
                const Plane_FL &refU, const Plane_FL &refV)
    {
        float *d[3] = {dstY.data(), dstU.data(), dstV.data()};
        const float *s[3] = {srcY.data(), srcU.data(), srcV.data()};
        const float *r[3] = {refY.data(), refU.data(), refV.data()};
        bm3d_ctx *c = ctx();
        check(c, bm3d_stage3(c, &para_, wiener_, d, s, r, srcY.Width(), srcY.Height(),
                             static_cast<size_t>(srcY.Stride()), refY.ValueRange(), BM3D_MEM_HOST,
                             nullptr));
    }

protected:
    bm3d_ctx *ctx() { return ctx_ ? ctx_ : default_context(); }
    bm3d_stage_params para_;
    bool wiener_;
    bm3d_ctx *ctx_;
};

class BM3D_Basic : public BM3D_Base {
public:
    BM3D_Basic(const BM3D_Basic_Para &para = BM3D_Basic_Para(), bm3d_ctx *ctx = nullptr)
        : BM3D_Base(para, false, ctx)
    {}
};

class BM3D_Final : public BM3D_Base {
public:
    BM3D_Final(const BM3D_Final_Para &para = BM3D_Final_Para(), bm3d_ctx *ctx = nullptr)
        : BM3D_Base(para, true, ctx)
    {}
};

// BM3D (include/BM3D.h:337-357): basic then final.
class BM3D {
public:
    BM3D(const BM3D_Para &para = BM3D_Para(), bm3d_ctx *ctx = nullptr)
        : basic_(para.basic.to_c()), final_(para.final.to_c()), ctx_(ctx)
    {}

    // BM3D::process_Plane_FL (source/BM3D.cpp:464-472); the basic stage matches on ref.
    Plane_FL &process(Plane_FL &dst, const Plane_FL &src, const Plane_FL &ref)
    {
        if (dst.Width() != src.Width() || dst.Height() != src.Height())
            dst.ReSize(src.Width(), src.Height());
        bm3d_ctx *c = ctx();
        check(c, bm3d_full(c, &basic_, &final_, dst.data(), src.data(), ref.data(), src.Width(),
                           src.Height(), static_cast<size_t>(src.Stride()), src.ValueRange(),
                           BM3D_MEM_HOST, nullptr));
        return dst;
    }
    Plane_FL &process(Plane_FL &dst, const Plane_FL &src) { return process(dst, src, src); }
    Plane_FL operator()(const Plane_FL &src, const Plane_FL &ref)
    {
        Plane_FL dst(src, false);
        return process(dst, src, ref);
    }
    Plane_FL operator()(const Plane_FL &src)
    {
        Plane_FL dst(src, false);
        return process(dst, src, src);
    }

    // BM3D::process_Plane (source/BM3D.cpp:475-497).
    Plane &process(Plane &dst, const Plane &src, const Plane &ref)
    {
        if (dst.Width() != src.Width() || dst.Height() != src.Height()) dst = Plane(src, false);
        bm3d_ctx *c = ctx();
        check(c, bm3d_plane_int(c, &basic_, &final_, dst.data(), src.data(),
                                &ref == &src ? nullptr : ref.data(), src.Width(), src.Height(),
                                static_cast<size_t>(src.Stride()), src.Floor(), src.Neutral(),
                                src.Ceil(), BM3D_MEM_HOST, nullptr));
        return dst;
    }
    Plane &process(Plane &dst, const Plane &src) { return process(dst, src, src); }
    Plane operator()(const Plane &src, const Plane &ref)
    {
        Plane dst(src, false);
        return process(dst, src, ref);
    }
    Plane operator()(const Plane &src)
    {
        Plane dst(src, false);
        return process(dst, src, src);
    }

    // BM3D::process_Frame (source/BM3D.cpp:501-527).
    Frame &process(Frame &dst, const Frame &src, const Frame &ref)
    {
        if (dst.Width() != src.Width() || dst.Height() != src.Height()) dst = Frame(src, false);
        int32_t *d[3] = {dst.R().data(), dst.G().data(), dst.B().data()};
        const int32_t *s[3] = {src.R().data(), src.G().data(), src.B().data()};
        const int32_t *r[3] = {ref.R().data(), ref.G().data(), ref.B().data()};
        bm3d_ctx *c = ctx();
        check(c, bm3d_frame(c, &basic_, &final_, d, s, r, src.Width(), src.Height(),
                            static_cast<size_t>(src.R().Stride()), src.R().Floor(),
                            src.R().Ceil(), BM3D_MEM_HOST, nullptr));
        return dst;
    }
    Frame &process(Frame &dst, const Frame &src) { return process(dst, src, src); }
    Frame operator()(const Frame &src, const Frame &ref)
    {
        Frame dst(src, false);
        return process(dst, src, ref);
    }
    Frame operator()(const Frame &src)
    {
        Frame dst(src, false);
        return process(dst, src, src);
    }

private:
    bm3d_ctx *ctx() { return ctx_ ? ctx_ : default_context(); }
    bm3d_stage_params basic_, final_;
    bm3d_ctx *ctx_;
};

}  // namespace bm3d_b200

#ifndef BM3D_B200_NO_GLOBAL_NAMES
using bm3d_b200::BM3D;
using bm3d_b200::BM3D_Basic;
using bm3d_b200::BM3D_Basic_Para;
using bm3d_b200::BM3D_Final;
using bm3d_b200::BM3D_Final_Para;
using bm3d_b200::BM3D_Para;
using bm3d_b200::BM3D_Para_Base;
using bm3d_b200::FLType;
using bm3d_b200::Frame;
using bm3d_b200::PCType;
using bm3d_b200::Plane;
using bm3d_b200::Plane_FL;
#endif
