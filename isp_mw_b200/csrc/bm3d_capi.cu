// C ABI of the B200 BM3D path (declared in include/bm3d_b200.h): parameter
// mirroring, per-call constant setup, context scratch and kernel launches.
#include "bm3d_b200.h"
#include "bm3d_batch.cuh"
#include "bm3d_convert.cuh"
#include "bm3d_kernels.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

using namespace bm3d;

// ---------------------------------------------------------------------------
// Context

struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
};

struct bm3d_ctx {
    int device = 0;
    int sm_count = 0;
    size_t smem_optin = 0;
    std::string err;
    // scratch
    DevBuf acc[2 * kMaxPlanes];       // num / den per plane
    DevBuf basic[kMaxPlanes];         // basic estimate for bm3d_full*
    DevBuf stage_in[kMaxPlanes];      // host-mode staging of src
    DevBuf stage_ref[kMaxPlanes];     // host-mode staging of ref
    DevBuf stage_out[kMaxPlanes];     // host-mode staging of dst
    DevBuf groups[3];                 // debug group dump
    DevBuf conv[3 * kMaxPlanes];      // float working planes of the integer paths: src, ref, dst
    DevBuf ints[3 * kMaxPlanes];      // host-mode staging of integer planes: src, ref, dst
    unsigned long long *stats = nullptr;
    float *absmax = nullptr;          // per plane max |src| of the running stage
    float *gtab_f = nullptr;          // generic path cosine matrices: fwd | inv (float)
    double *gtab_d = nullptr;         // same in double
    cudaStream_t last_stream = nullptr;
    int tile_x = 8, tile_y = 8, warps = 16;
    // bm3d_full_many's copy pipeline: two slots of device planes, an upload
    // and a download stream, and the events that order slot reuse
    struct PipeSlot {
        DevBuf in, out;
        cudaEvent_t in_ready = nullptr, computed = nullptr, drained = nullptr;
        bool used = false;
    } pipe[2];
    cudaStream_t up = nullptr, down = nullptr;
    unsigned long long pipe_count = 0;
    // optional per-launch timing of the stage kernels: [0] basic, [1] final
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending[2];
    double time_ms[2] = {0, 0};
    long long launches[2] = {0, 0};
};

static void drain_timing(bm3d_ctx *ctx)
{
    for (int k = 0; k < 2; ++k) {
        for (auto &ev : ctx->pending[k]) {
            float ms = 0;
            if (cudaEventSynchronize(ev.second) == cudaSuccess &&
                cudaEventElapsedTime(&ms, ev.first, ev.second) == cudaSuccess) {
                ctx->time_ms[k] += ms;
                ctx->launches[k] += 1;
            }
            cudaEventDestroy(ev.first);
            cudaEventDestroy(ev.second);
        }
        ctx->pending[k].clear();
    }
}

static thread_local std::string g_create_error;
constexpr int kStats = 5;

static int cuda_fail(bm3d_ctx *ctx, cudaError_t e, const char *what)
{
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    if (ctx) ctx->err = buf;
    else g_create_error = buf;
    return e == cudaErrorMemoryAllocation ? BM3D_ERR_NOMEM : BM3D_ERR_CUDA;
}

#define CK(ctx, call)                                                                       \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call);                           \
    } while (0)

static int ensure(bm3d_ctx *ctx, DevBuf &b, size_t bytes)
{
    if (b.bytes >= bytes) return BM3D_OK;
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
    CK(ctx, cudaMalloc(&b.ptr, bytes));
    b.bytes = bytes;
    return BM3D_OK;
}

#define BM3D_DECLARE_UNIT(name) cudaError_t bm3d_upload_dct_tables_##name(const bm3d::DctTableData &);
BM3D_KERNEL_UNITS(BM3D_DECLARE_UNIT)
#undef BM3D_DECLARE_UNIT

namespace bm3d {

cudaError_t upload_dct_tables_all(const DctTableData &t)
{
    cudaError_t e = cudaSuccess;
#define BM3D_UPLOAD_UNIT(name) \
    if ((e = bm3d_upload_dct_tables_##name(t)) != cudaSuccess) return e;
    BM3D_KERNEL_UNITS(BM3D_UPLOAD_UNIT)
#undef BM3D_UPLOAD_UNIT
    return e;
}

}  // namespace bm3d

// Cosine matrices in long double, rounded once to each precision; length n
// starts at (n-1) n (2n-1) / 6.
static void make_dct_tables(float *ff, float *fi, double *df, double *di)
{
    const long double pi = 3.141592653589793238462643383279502884L;
    int o = 0;
    for (int n = 1; n <= 16; ++n) {
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j) {
                const long double cf = 2.0L * cosl(pi * (2 * j + 1) * k / (2.0L * n));
                const long double ci = j == 0 ? 1.0L : 2.0L * cosl(pi * j * (2 * k + 1) / (2.0L * n));
                ff[o + k * n + j] = static_cast<float>(cf);
                fi[o + k * n + j] = static_cast<float>(ci);
                df[o + k * n + j] = static_cast<double>(cf);
                di[o + k * n + j] = static_cast<double>(ci);
            }
        o += n * n;
    }
}

static float g_tab_ff[1496], g_tab_fi[1496];
static float g_pad_f[bm3d::kPadTable], g_pad_i[bm3d::kPadTable];
static float g_d32_f[32 * 32], g_d32_i[32 * 32];
static float g_d11_f[11 * 11], g_d11_i[11 * 11];
static double g_tab_df[1496], g_tab_di[1496];
static std::once_flag g_tab_once;

static void init_dct_tables()
{
    make_dct_tables(g_tab_ff, g_tab_fi, g_tab_df, g_tab_di);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < 32; ++k)
        for (int j = 0; j < 32; ++j) {
            g_d32_f[k * 32 + j] = static_cast<float>(2.0L * cosl(pi * (2 * j + 1) * k / 64.0L));
            g_d32_i[k * 32 + j] =
                static_cast<float>(j == 0 ? 1.0L : 2.0L * cosl(pi * j * (2 * k + 1) / 64.0L));
        }
    for (int k = 0; k < 11; ++k)
        for (int j = 0; j < 11; ++j) {
            g_d11_f[k * 11 + j] = static_cast<float>(2.0L * cosl(pi * (2 * j + 1) * k / 22.0L));
            g_d11_i[k * 11 + j] =
                static_cast<float>(j == 0 ? 1.0L : 2.0L * cosl(pi * j * (2 * k + 1) / 22.0L));
        }
    // column-major, 16 rows, zero past row n: the same FP32 values
    for (int n = 1; n <= 15; ++n) {
        if (n == 8) continue;
        const int src = (n - 1) * n * (2 * n - 1) / 6, dst = bm3d::pad_table_offset(n);
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < 16; ++k) {
                g_pad_f[dst + 16 * j + k] = k < n ? g_tab_ff[src + k * n + j] : 0.0f;
                g_pad_i[dst + 16 * j + k] = k < n ? g_tab_fi[src + k * n + j] : 0.0f;
            }
    }
}

static cudaError_t upload_dct_tables()
{
    std::call_once(g_tab_once, init_dct_tables);
    return upload_dct_tables_all(
        DctTableData{g_tab_ff, g_tab_fi, g_tab_df, g_tab_di, g_pad_f, g_pad_i, g_d32_f, g_d32_i,
                     g_d11_f, g_d11_i});
}

extern "C" int bm3d_ctx_create(bm3d_ctx **out, int device)
{
    if (!out) return BM3D_ERR_INVALID;
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetDeviceCount");
    if (device < 0 || device >= count) {
        g_create_error = "bm3d_ctx_create: no such CUDA device";
        return BM3D_ERR_CUDA;
    }
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetDeviceProperties");
    if (prop.major < 10) {
        g_create_error = "bm3d_ctx_create: this build targets sm_100a (B200)";
        return BM3D_ERR_CUDA;
    }
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaSetDevice");
    bm3d_ctx *ctx = new bm3d_ctx;
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    ctx->smem_optin = prop.sharedMemPerBlockOptin;
    e = upload_dct_tables();
    if (e != cudaSuccess) {
        delete ctx;
        return cuda_fail(nullptr, e, "upload_dct_tables");
    }
    e = cudaMalloc(&ctx->stats, kStats * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        delete ctx;
        return cuda_fail(nullptr, e, "cudaMalloc(stats)");
    }
    cudaMemset(ctx->stats, 0, kStats * sizeof(unsigned long long));
    e = cudaMalloc(&ctx->absmax, kMaxPlanes * sizeof(float));
    if (e != cudaSuccess) {
        cudaFree(ctx->stats);
        delete ctx;
        return cuda_fail(nullptr, e, "cudaMalloc(absmax)");
    }
    // cosine matrices of lengths 1..32 for the generic path
    {
        std::vector<float> tf(2 * kDctTableSize);
        std::vector<double> td(2 * kDctTableSize);
        const long double pi = 3.141592653589793238462643383279502884L;
        for (int n = 1; n <= kGSTab; ++n) {
            const int o = dct_table_offset(n);
            for (int k = 0; k < n; ++k)
                for (int j = 0; j < n; ++j) {
                    const long double cf = 2.0L * cosl(pi * (2 * j + 1) * k / (2.0L * n));
                    const long double ci = j == 0 ? 1.0L : 2.0L * cosl(pi * j * (2 * k + 1) / (2.0L * n));
                    tf[o + k * n + j] = static_cast<float>(cf);
                    tf[kDctTableSize + o + k * n + j] = static_cast<float>(ci);
                    td[o + k * n + j] = static_cast<double>(cf);
                    td[kDctTableSize + o + k * n + j] = static_cast<double>(ci);
                }
        }
        e = cudaMalloc(&ctx->gtab_f, tf.size() * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&ctx->gtab_d, td.size() * sizeof(double));
        if (e == cudaSuccess)
            e = cudaMemcpy(ctx->gtab_f, tf.data(), tf.size() * sizeof(float), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(ctx->gtab_d, td.data(), td.size() * sizeof(double), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(ctx->stats);
            cudaFree(ctx->absmax);
            cudaFree(ctx->gtab_f);
            cudaFree(ctx->gtab_d);
            delete ctx;
            return cuda_fail(nullptr, e, "generic cosine tables");
        }
    }
    *out = ctx;
    return BM3D_OK;
}

extern "C" void bm3d_ctx_destroy(bm3d_ctx *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    auto fr = [](DevBuf &b) {
        if (b.ptr) cudaFree(b.ptr);
        b.ptr = nullptr;
    };
    for (auto &b : ctx->acc) fr(b);
    for (auto &b : ctx->basic) fr(b);
    for (auto &b : ctx->stage_in) fr(b);
    for (auto &b : ctx->stage_ref) fr(b);
    for (auto &b : ctx->stage_out) fr(b);
    for (auto &b : ctx->groups) fr(b);
    for (auto &b : ctx->conv) fr(b);
    for (auto &b : ctx->ints) fr(b);
    for (auto &sl : ctx->pipe) {
        fr(sl.in);
        fr(sl.out);
        for (cudaEvent_t e : {sl.in_ready, sl.computed, sl.drained})
            if (e) cudaEventDestroy(e);
    }
    if (ctx->up) cudaStreamDestroy(ctx->up);
    if (ctx->down) cudaStreamDestroy(ctx->down);
    if (ctx->stats) cudaFree(ctx->stats);
    if (ctx->absmax) cudaFree(ctx->absmax);
    if (ctx->gtab_f) cudaFree(ctx->gtab_f);
    if (ctx->gtab_d) cudaFree(ctx->gtab_d);
    drain_timing(ctx);
    delete ctx;
}

extern "C" const char *bm3d_last_error(const bm3d_ctx *ctx)
{
    if (ctx) return ctx->err.c_str();
    return g_create_error.c_str();
}

extern "C" int bm3d_set_tiling(bm3d_ctx *ctx, int tile_x, int tile_y, int warps)
{
    if (!ctx || tile_x < 0 || tile_y < 0 || warps < 0 || warps > 16) return BM3D_ERR_INVALID;
    if (tile_x) ctx->tile_x = tile_x;
    if (tile_y) ctx->tile_y = tile_y;
    if (warps) ctx->warps = warps;
    return BM3D_OK;
}

// ---------------------------------------------------------------------------
// Parameters: the reference's profile constructors (include/BM3D.h:27-151).

static bool known_profile(const std::string &p)
{
    return p == "fast" || p == "lc" || p == "np" || p == "high" || p == "vn";
}

extern "C" int bm3d_stage_params_thmse_default(const char *profile, int wiener,
                                               bm3d_stage_params *p)
{
    if (!profile || !p || !known_profile(profile)) return BM3D_ERR_INVALID;
    const std::string prof(profile);
    if (!wiener) p->thMSE = prof == "vn" ? 1000 + p->sigma[0] * 150 : 400 + p->sigma[0] * 80;
    else p->thMSE = prof == "vn" ? 400 + p->sigma[0] * 40 : 200 + p->sigma[0] * 10;
    return BM3D_OK;
}

extern "C" int bm3d_stage_params_default(const char *profile, int wiener, const double sigma[3],
                                         bm3d_stage_params *out)
{
    if (!profile || !out || !known_profile(profile)) return BM3D_ERR_INVALID;
    const std::string prof(profile);
    bm3d_stage_params p;
    p.block_size = 8;
    p.bm_range = (prof == "fast" || prof == "lc") ? 9 : 16;
    p.bm_step = 1;
    if (!wiener) {
        p.block_step = 4;
        p.group_size = 16;
        p.lambda = 2.7;
        if (prof == "fast") p.block_step = 8;
        else if (prof == "lc") p.block_step = 6;
        else if (prof == "high") p.block_step = 3;
        else if (prof == "vn") {
            p.block_step = 4;
            p.group_size = 32;
            p.lambda = 2.8;
        }
    } else {
        p.block_step = 3;
        p.group_size = 32;
        p.lambda = 0;
        if (prof == "fast") {
            p.block_step = 7;
            p.group_size = 16;
        } else if (prof == "lc") {
            p.block_step = 5;
            p.group_size = 16;
        } else if (prof == "high") {
            p.block_step = 2;
        } else if (prof == "vn") {
            p.block_size = 11;
            p.block_step = 6;
        }
    }
    for (int i = 0; i < 3; ++i) p.sigma[i] = sigma ? sigma[i] : 10.0;
    bm3d_stage_params_thmse_default(profile, wiener, &p);
    *out = p;
    return BM3D_OK;
}

extern "C" long long bm3d_ref_block_count(const bm3d_stage_params *p, int width, int height)
{
    if (!p || p->block_size <= 0 || p->block_step <= 0 || width < p->block_size ||
        height < p->block_size)
        return -1;
    return static_cast<long long>(ref_count(width - p->block_size, p->block_step)) *
           ref_count(height - p->block_size, p->block_step);
}

// ---------------------------------------------------------------------------
// Stage setup: BM3D_Base ctor (include/BM3D.h:237-259) and BM3D_FilterData
// ctor (source/BM3D.cpp:9-73), evaluated in double exactly as the reference.

static void opp_norms(double norm[3])
{
    const double Yr = static_cast<double>(1.0L / 3.0L), Yg = Yr, Yb = Yr;
    const double Ur = static_cast<double>(1.0L / 2.0L), Ug = 0.0, Ub = static_cast<double>(-1.0L / 2.0L);
    const double Vr = static_cast<double>(1.0L / 4.0L), Vg = static_cast<double>(-1.0L / 2.0L),
                 Vb = static_cast<double>(1.0L / 4.0L);
    norm[0] = std::sqrt(Yr * Yr + Yg * Yg + Yb * Yb);
    norm[1] = std::sqrt(Ur * Ur + Ug * Ug + Ub * Ub);
    norm[2] = std::sqrt(Vr * Vr + Vg * Vg + Vb * Vb);
}

enum class Guard { Run, Copy, Invalid, Unsupported };

// The register-resident kernel covers BlockSize 8 with GroupSize <= 16 (the
// "fast" and "lc" profiles); everything else up to BlockSize 16 and GroupSize
// 32 runs on the generic kernel.
static bool fast_path(const bm3d_stage_params *p)
{
    return p->block_size == kBS && p->group_size <= kGSMax;
}

static Guard check_params(const bm3d_stage_params *p, int nplanes)
{
    if (!p) return Guard::Invalid;
    double norm[3];
    opp_norms(norm);
    const double thMSE = p->thMSE * norm[0];
    const bool sig = nplanes == 3 ? (p->sigma[0] <= 0 && p->sigma[1] <= 0 && p->sigma[2] <= 0)
                                  : (p->sigma[0] <= 0);
    if (sig || p->group_size == 0 || p->block_size <= 0 || p->bm_range <= 0 ||
        p->bm_range < p->bm_step || thMSE <= 0)
        return Guard::Copy;
    if (p->group_size < 0 || p->block_step <= 0 || p->bm_step <= 0) return Guard::Invalid;
    if (p->block_size > kBSMax || p->group_size > kGSTab) return Guard::Unsupported;
    return Guard::Run;
}

template <typename T>
static void fill_tables(StageArgs<T> &a, const bm3d_stage_params *p, bool wiener, int nplanes,
                        double value_range)
{
    double norm[3];
    opp_norms(norm);
    const double thMSE = p->thMSE * norm[0];
    const int GS = p->group_size, BS = p->block_size;
    a.active = 0;
    for (int c = 0; c < nplanes; ++c) {
        if (!(p->sigma[c] > 0)) continue;
        a.active |= 1 << c;
        const double sigma = p->sigma[c] / double(255) * norm[c];
        for (int i = 1; i <= GS; ++i) {
            const double finalAMP = 2 * i * 2 * BS * 2 * BS;
            const double forwardAMP = std::sqrt(finalAMP);
            a.wss[c][i - 1] = static_cast<T>(sigma * forwardAMP * sigma * forwardAMP);
            const double thrBase = sigma * p->lambda * forwardAMP;
            a.thr[c][i - 1][0] = static_cast<T>(thrBase);
            a.thr[c][i - 1][1] = static_cast<T>(thrBase * std::sqrt(double(2)));
            a.thr[c][i - 1][2] = static_cast<T>(thrBase * double(2));
            a.thr[c][i - 1][3] = static_cast<T>(thrBase * std::sqrt(double(8)));
        }
    }
    if (nplanes == 1) a.active = 1;
    for (int i = 1; i <= GS; ++i) a.finalAMP[i - 1] = 2 * i * 2 * BS * 2 * BS;
    (void)wiener;
    // Block::BlockMatchingMulti (include/Block.h:582-584); the plane range is
    // an FLType, promoted to double in the product.
    const T range = static_cast<T>(value_range);
    const double MSE2SSE = static_cast<double>(BS * BS) * range * range / double(255 * 255);
    a.distMul = double(1) / MSE2SSE;
    a.thSSE = static_cast<T>(thMSE * MSE2SSE);
    a.match = (GS == 1 || thMSE <= 0) ? 0 : 1;
}

template <typename T, bool W, int NPL, int KS>
static int launch_one(bm3d_ctx *ctx, StageArgs<T> &a, cudaStream_t s, int warps)
{
    const void *kern = stage_kernel_fn<T, W, NPL, KS>();
    const SmemPlan sp =
        plan_smem<T>(NPL, W, a.ref_alias_src, a.region_h, a.region_pitch, a.key_slots, warps,
                     false, kBS, kGSMax, a.tile_x * a.tile_y);
    CK(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(sp.total)));
    const int grid = a.tiles_x * ((a.ny + a.tile_y - 1) / a.tile_y);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ctx->timing && !a.bm_only) {
        CK(ctx, cudaEventCreate(&e0));
        CK(ctx, cudaEventCreate(&e1));
        CK(ctx, cudaEventRecord(e0, s));
    }
    void *args[] = {&a};
    CK(ctx, cudaLaunchKernel(kern, dim3(grid), dim3(warps * kWarp), args, sp.total, s));
    if (e0) {
        CK(ctx, cudaEventRecord(e1, s));
        ctx->pending[W ? 1 : 0].emplace_back(e0, e1);
    }
    return BM3D_OK;
}

template <typename T, bool W, int NPL>
static int launch_ks(bm3d_ctx *ctx, StageArgs<T> &a, cudaStream_t s, int warps)
{
    if (a.bm_step == 1) return launch_one<T, W, NPL, 4>(ctx, a, s, warps);
    return launch_one<T, W, NPL, 1>(ctx, a, s, warps);
}

template <typename T, bool W, int NPL>
static int launch_generic(bm3d_ctx *ctx, StageArgs<T> &a, cudaStream_t s, int warps)
{
    const void *kern = generic_kernel_fn<T, W, NPL>();
    const SmemPlan sp = plan_smem<T>(NPL, W, a.ref_alias_src, a.region_h, a.region_pitch,
                                     a.key_slots, warps, true, a.block_size, a.group_size);
    CK(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(sp.total)));
    const int grid = a.tiles_x * ((a.ny + a.tile_y - 1) / a.tile_y);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ctx->timing && !a.bm_only) {
        CK(ctx, cudaEventCreate(&e0));
        CK(ctx, cudaEventCreate(&e1));
        CK(ctx, cudaEventRecord(e0, s));
    }
    void *args[] = {&a};
    CK(ctx, cudaLaunchKernel(kern, dim3(grid), dim3(warps * kWarp), args, sp.total, s));
    if (e0) {
        CK(ctx, cudaEventRecord(e1, s));
        ctx->pending[W ? 1 : 0].emplace_back(e0, e1);
    }
    return BM3D_OK;
}

static bool fast_args(int block_size, int group_size)
{
    return block_size == kBS && group_size <= kGSMax;
}

template <typename T>
static int launch_stage(bm3d_ctx *ctx, StageArgs<T> &a, bool wiener, int nplanes, cudaStream_t s,
                        int warps)
{
    if (!fast_args(a.block_size, a.group_size)) {
        if (nplanes == 1)
            return wiener ? launch_generic<T, true, 1>(ctx, a, s, warps)
                          : launch_generic<T, false, 1>(ctx, a, s, warps);
        return wiener ? launch_generic<T, true, 3>(ctx, a, s, warps)
                      : launch_generic<T, false, 3>(ctx, a, s, warps);
    }
    if (nplanes == 1)
        return wiener ? launch_ks<T, true, 1>(ctx, a, s, warps) : launch_ks<T, false, 1>(ctx, a, s, warps);
    return wiener ? launch_ks<T, true, 3>(ctx, a, s, warps) : launch_ks<T, false, 3>(ctx, a, s, warps);
}

template <typename T> struct GenericTables;
template <> struct GenericTables<float> {
    static const float *fwd(const bm3d_ctx *c) { return c->gtab_f; }
    static const float *inv(const bm3d_ctx *c) { return c->gtab_f ? c->gtab_f + kDctTableSize : nullptr; }
};
template <> struct GenericTables<double> {
    static const double *fwd(const bm3d_ctx *c) { return c->gtab_d; }
    static const double *inv(const bm3d_ctx *c) { return c->gtab_d ? c->gtab_d + kDctTableSize : nullptr; }
};

// Geometry, tiling and shared-memory fit.
template <typename T>
static int plan_geometry(bm3d_ctx *ctx, StageArgs<T> &a, const bm3d_stage_params *p, bool wiener,
                         int nplanes, int width, int height, int &warps)
{
    const int BS = p->block_size;
    const bool generic = !fast_args(BS, p->group_size);
    a.width = width;
    a.height = height;
    a.block_size = BS;
    a.step = p->block_step;
    a.group_size = p->group_size;
    a.bm_step = p->bm_step;
    a.range = p->bm_range / p->bm_step * p->bm_step;
    a.nx = ref_count(width - BS, a.step);
    a.ny = ref_count(height - BS, a.step);
    const int span = 2 * (a.range / a.bm_step) + 1;
    a.key_slots = span * span + 1;
    // the generic kernel launches at most 8 warps (launch bounds 256) on 4x4 tiles
    int tx = generic ? 4 : ctx->tile_x, ty = generic ? 4 : ctx->tile_y;
    warps = generic ? 8 : ctx->warps;
    for (;;) {
        const int reach = a.match ? a.range : 0;
        a.region_w = std::min(width, (tx - 1) * a.step + 2 * reach + BS);
        a.region_h = std::min(height, (ty - 1) * a.step + 2 * reach + BS);
        // pitch = 5 (mod 8): block matching's lanes read window rows 4 apart,
        // and this residue keeps those lane groups on the fewest shared banks
        a.region_pitch = a.region_w + ((5 - a.region_w % 8) + 8) % 8;
        const SmemPlan sp = plan_smem<T>(nplanes, wiener, a.ref_alias_src, a.region_h,
                                         a.region_pitch, a.key_slots, warps, generic, BS,
                                         p->group_size, std::min(tx, a.nx) * std::min(ty, a.ny));
        if (sp.total <= ctx->smem_optin) break;
        // The generic kernel's per-warp group buffers dominate its footprint:
        // give up warps before tile size there.
        if (warps > 8 || (generic && warps > 1)) warps /= 2;
        else if (ty > 1 && ty >= tx) --ty;
        else if (tx > 1) --tx;
        else if (warps > 1) warps /= 2;
        else {
            ctx->err = "stage does not fit in shared memory";
            return BM3D_ERR_UNSUPPORTED;
        }
    }
    a.tile_x = std::min(tx, a.nx);
    a.tile_y = std::min(ty, a.ny);
    a.tiles_x = (a.nx + a.tile_x - 1) / a.tile_x;
    return BM3D_OK;
}

template <typename T>
static int copy_plane(bm3d_ctx *ctx, T *dst, size_t dpitch, const T *src, size_t spitch, int w,
                      int h, cudaMemcpyKind kind, cudaStream_t s)
{
    CK(ctx, cudaMemcpy2DAsync(dst, dpitch * sizeof(T), src, spitch * sizeof(T), w * sizeof(T), h,
                              kind, s));
    return BM3D_OK;
}

// One stage over device-resident planes (all with row pitch `stride`).
template <typename T>
static int run_stage_device(bm3d_ctx *ctx, const bm3d_stage_params *p, bool wiener, int nplanes,
                            T *const dst[], const T *const src[], const T *const ref[], int width,
                            int height, size_t stride, double value_range, cudaStream_t s,
                            int *gcount = nullptr, int *gpos = nullptr, T *gkey = nullptr,
                            bool bm_only = false)
{
    StageArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    fill_tables(a, p, wiener, nplanes, value_range);
    a.stride = static_cast<long long>(stride);
    a.ref_alias_src = 0;
    for (int c = 0; c < nplanes; ++c) {
        a.src[c] = src[c];
        a.ref[c] = ref[c];
        if (src[c] == ref[c]) a.ref_alias_src |= 1 << c;
    }
    int warps;
    int rc = plan_geometry(ctx, a, p, wiener, nplanes, width, height, warps);
    if (rc != BM3D_OK) return rc;
    a.dct_fwd = GenericTables<T>::fwd(ctx);
    a.dct_inv = GenericTables<T>::inv(ctx);
    using Acc = typename AccOf<T>::type;
    const size_t acc_bytes = sizeof(Acc) * static_cast<size_t>(width) * height;
    const long long npx = static_cast<long long>(width) * height;
    const int threads = 256;
    const int blocks = static_cast<int>(std::min<long long>((npx + threads - 1) / threads,
                                                            static_cast<long long>(ctx->sm_count) * 8));
    // At most 2 * (reference blocks) * GroupSize terms reach one pixel (block
    // (0, 0) can sit in every group, twice).
    const double terms = 2.0 * static_cast<double>(a.nx) * a.ny * std::max(1, p->group_size);
    a.log2_bound = static_cast<int>(std::ceil(std::log2(std::max(2.0, terms))));
    a.absmax = ctx->absmax;
    if (!bm_only) CK(ctx, cudaMemsetAsync(ctx->absmax, 0, kMaxPlanes * sizeof(float), s));
    for (int c = 0; c < nplanes; ++c) {
        if (!(a.active & (1 << c)) && !bm_only) continue;
        if ((rc = ensure(ctx, ctx->acc[2 * c], acc_bytes)) != BM3D_OK) return rc;
        if ((rc = ensure(ctx, ctx->acc[2 * c + 1], acc_bytes)) != BM3D_OK) return rc;
        a.num[c] = static_cast<Acc *>(ctx->acc[2 * c].ptr);
        a.den[c] = static_cast<Acc *>(ctx->acc[2 * c + 1].ptr);
        if (!bm_only) {
            prep_kernel<T><<<blocks, threads, 0, s>>>(a.num[c], a.den[c], src[c],
                                                      static_cast<long long>(stride), width,
                                                      height, ctx->absmax + c);
            CK(ctx, cudaGetLastError());
        }
    }
    a.group_count = gcount;
    a.group_pos = gpos;
    a.group_key = gkey;
    a.bm_only = bm_only ? 1 : 0;
    a.stats = ctx->stats;
    // per-stage counters; the invariant counter (stats[4]) is sticky
    CK(ctx, cudaMemsetAsync(ctx->stats, 0, 4 * sizeof(unsigned long long), s));
    if ((rc = launch_stage(ctx, a, wiener, nplanes, s, warps)) != BM3D_OK) return rc;
    ctx->last_stream = s;
    if (bm_only) return BM3D_OK;
    for (int c = 0; c < nplanes; ++c) {
        if (!(a.active & (1 << c))) continue;
        const dim3 ngrid((width + kNormTile - 1) / kNormTile, (height + kNormTile - 1) / kNormTile);
        normalize_kernel<T><<<ngrid, 256, 0, s>>>(dst[c], static_cast<long long>(stride), a.num[c],
                                                  a.den[c], width, height, a.block_size);
        CK(ctx, cudaGetLastError());
    }
    return BM3D_OK;
}

// Host-mode calls end synchronised; a nonzero invariant counter means a group
// member fell outside its tile's staged window and was skipped.
static int check_invariants(bm3d_ctx *ctx)
{
    unsigned long long v[kStats];
    CK(ctx, cudaMemcpy(v, ctx->stats, sizeof(v), cudaMemcpyDeviceToHost));
    if (v[4] != 0) {  // low 32 bits: group blocks outside the window; high: CTAs short of smem
        ctx->err = "internal error: " + std::to_string(v[4] & 0xffffffffull) +
                   " group blocks outside the staged window, " + std::to_string(v[4] >> 32) +
                   " tiles launched with too little shared memory";
        return BM3D_ERR_CUDA;
    }
    return BM3D_OK;
}

template <typename T>
static int passthrough(bm3d_ctx *ctx, int nplanes, T *const dst[], const T *const src[], int width,
                       int height, size_t stride, int mem, cudaStream_t s)
{
    for (int c = 0; c < nplanes; ++c) {
        if (dst[c] == src[c]) continue;
        int rc = copy_plane(ctx, dst[c], stride, src[c], stride, width, height,
                            mem == BM3D_MEM_HOST ? cudaMemcpyHostToHost : cudaMemcpyDeviceToDevice, s);
        if (rc != BM3D_OK) return rc;
    }
    if (mem == BM3D_MEM_HOST) CK(ctx, cudaStreamSynchronize(s));
    return BM3D_COPIED;
}

static int check_planes(int nplanes, const void *const dst[], const void *const src[],
                        const void *const ref[], int width, int height, size_t stride, int bs)
{
    if (width < bs || height < bs || stride < static_cast<size_t>(width)) return BM3D_ERR_INVALID;
    for (int c = 0; c < nplanes; ++c)
        if (!dst[c] || !src[c] || (ref && !ref[c])) return BM3D_ERR_INVALID;
    return BM3D_OK;
}

// A stage in either memory kind. In host mode planes go through context
// staging buffers with pitch = width.
template <typename T>
static int stage_any(bm3d_ctx *ctx, const bm3d_stage_params *p, int wiener, int nplanes,
                     T *const dst[], const T *const src[], const T *const ref[], int width,
                     int height, size_t stride, double value_range, int mem, void *stream)
{
    if (!ctx) return BM3D_ERR_INVALID;
    if (mem != BM3D_MEM_HOST && mem != BM3D_MEM_DEVICE) return BM3D_ERR_INVALID;
    const Guard g = check_params(p, nplanes);
    if (g == Guard::Invalid) return BM3D_ERR_INVALID;
    int rc = check_planes(nplanes, reinterpret_cast<const void *const *>(dst),
                          reinterpret_cast<const void *const *>(src),
                          reinterpret_cast<const void *const *>(ref), width, height, stride,
                          p->block_size > 0 ? p->block_size : 1);
    if (rc != BM3D_OK) return rc;
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (g == Guard::Copy) return passthrough(ctx, nplanes, dst, src, width, height, stride, mem, s);
    if (g == Guard::Unsupported) {
        ctx->err = "parameters outside this build (BlockSize <= 16, GroupSize <= 32)";
        return BM3D_ERR_UNSUPPORTED;
    }
    if (mem == BM3D_MEM_DEVICE)
        return run_stage_device(ctx, p, wiener != 0, nplanes, dst, src, ref, width, height, stride,
                                value_range, s);
    const size_t plane_bytes = sizeof(T) * static_cast<size_t>(width) * height;
    T *dd[kMaxPlanes];
    const T *ds[kMaxPlanes], *dr[kMaxPlanes];
    for (int c = 0; c < nplanes; ++c) {
        if ((rc = ensure(ctx, ctx->stage_in[c], plane_bytes)) != BM3D_OK) return rc;
        if ((rc = ensure(ctx, ctx->stage_out[c], plane_bytes)) != BM3D_OK) return rc;
        T *in = static_cast<T *>(ctx->stage_in[c].ptr);
        if ((rc = copy_plane(ctx, in, width, src[c], stride, width, height,
                             cudaMemcpyHostToDevice, s)) != BM3D_OK)
            return rc;
        ds[c] = in;
        if (ref[c] == src[c]) {
            dr[c] = in;
        } else {
            if ((rc = ensure(ctx, ctx->stage_ref[c], plane_bytes)) != BM3D_OK) return rc;
            T *r = static_cast<T *>(ctx->stage_ref[c].ptr);
            if ((rc = copy_plane(ctx, r, width, ref[c], stride, width, height,
                                 cudaMemcpyHostToDevice, s)) != BM3D_OK)
                return rc;
            dr[c] = r;
        }
        dd[c] = static_cast<T *>(ctx->stage_out[c].ptr);
        // planes this stage leaves alone (sigma <= 0) keep the caller's contents
        if (nplanes > 1 && !(p->sigma[c] > 0))
            if ((rc = copy_plane(ctx, dd[c], width, dst[c], stride, width, height,
                                 cudaMemcpyHostToDevice, s)) != BM3D_OK)
                return rc;
    }
    rc = run_stage_device(ctx, p, wiener != 0, nplanes, dd, ds, dr, width, height, width,
                          value_range, s);
    if (rc != BM3D_OK) return rc;
    for (int c = 0; c < nplanes; ++c)
        if ((rc = copy_plane(ctx, dst[c], stride, static_cast<const T *>(dd[c]), width, width,
                             height, cudaMemcpyDeviceToHost, s)) != BM3D_OK)
            return rc;
    CK(ctx, cudaStreamSynchronize(s));
    return check_invariants(ctx);
}

extern "C" int bm3d_stage(bm3d_ctx *ctx, const bm3d_stage_params *params, int wiener, float *dst,
                          const float *src, const float *ref, int width, int height,
                          size_t stride, float value_range, int mem, void *stream)
{
    float *d[1] = {dst};
    const float *s[1] = {src}, *r[1] = {ref ? ref : src};
    return stage_any<float>(ctx, params, wiener, 1, d, s, r, width, height, stride, value_range,
                            mem, stream);
}

extern "C" int bm3d_stage_f64(bm3d_ctx *ctx, const bm3d_stage_params *params, int wiener,
                              double *dst, const double *src, const double *ref, int width,
                              int height, size_t stride, double value_range, int mem,
                              void *stream)
{
    double *d[1] = {dst};
    const double *s[1] = {src}, *r[1] = {ref ? ref : src};
    return stage_any<double>(ctx, params, wiener, 1, d, s, r, width, height, stride, value_range,
                             mem, stream);
}

extern "C" int bm3d_stage3(bm3d_ctx *ctx, const bm3d_stage_params *params, int wiener,
                           float *const dst[3], const float *const src[3],
                           const float *const ref[3], int width, int height, size_t stride,
                           float value_range, int mem, void *stream)
{
    if (!dst || !src) return BM3D_ERR_INVALID;
    const float *const *r = ref ? ref : src;
    return stage_any<float>(ctx, params, wiener, 3, dst, src, r, width, height, stride,
                            value_range, mem, stream);
}

template <typename T>
static int full_any(bm3d_ctx *ctx, const bm3d_stage_params *basic, const bm3d_stage_params *fin,
                    int nplanes, T *const dst[], const T *const src[], const T *const ref[],
                    int width, int height, size_t stride, double value_range, int mem,
                    void *stream)
{
    if (!ctx || !basic || !fin) return BM3D_ERR_INVALID;
    if (mem != BM3D_MEM_HOST && mem != BM3D_MEM_DEVICE) return BM3D_ERR_INVALID;
    int rc = check_planes(nplanes, reinterpret_cast<const void *const *>(dst),
                          reinterpret_cast<const void *const *>(src), nullptr, width, height,
                          stride, 1);
    if (rc != BM3D_OK) return rc;
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t plane_bytes = sizeof(T) * static_cast<size_t>(width) * height;
    const size_t dpitch = mem == BM3D_MEM_HOST ? static_cast<size_t>(width) : stride;
    // Device-resident src and dst (context staging in host mode) and the basic
    // estimate, all with row pitch dpitch.
    const T *ds[kMaxPlanes], *dr[kMaxPlanes];
    T *tmp[kMaxPlanes], *dd[kMaxPlanes];
    for (int c = 0; c < nplanes; ++c) {
        if ((rc = ensure(ctx, ctx->basic[c], sizeof(T) * dpitch * height)) != BM3D_OK) return rc;
        tmp[c] = static_cast<T *>(ctx->basic[c].ptr);
    }
    // a distinct ref (the basic stage matches on it; src when absent)
    const bool own_ref = ref != nullptr && ref[0] != nullptr && ref[0] != src[0];
    if (mem == BM3D_MEM_HOST) {
        for (int c = 0; c < nplanes; ++c) {
            if ((rc = ensure(ctx, ctx->stage_in[c], plane_bytes)) != BM3D_OK) return rc;
            if ((rc = ensure(ctx, ctx->stage_out[c], plane_bytes)) != BM3D_OK) return rc;
            T *in = static_cast<T *>(ctx->stage_in[c].ptr);
            if ((rc = copy_plane(ctx, in, width, src[c], stride, width, height,
                                 cudaMemcpyHostToDevice, s)) != BM3D_OK)
                return rc;
            ds[c] = in;
            dr[c] = in;
            dd[c] = static_cast<T *>(ctx->stage_out[c].ptr);
        }
        if (own_ref) {
            if ((rc = ensure(ctx, ctx->stage_ref[0], plane_bytes)) != BM3D_OK) return rc;
            T *r = static_cast<T *>(ctx->stage_ref[0].ptr);
            if ((rc = copy_plane(ctx, r, width, ref[0], stride, width, height,
                                 cudaMemcpyHostToDevice, s)) != BM3D_OK)
                return rc;
            dr[0] = r;
        }
    } else {
        for (int c = 0; c < nplanes; ++c) {
            ds[c] = src[c];
            dr[c] = src[c];
            dd[c] = dst[c];
        }
        if (own_ref) dr[0] = ref[0];
    }
    // Planes a stage does not filter (sigma <= 0), or a stage whose parameters
    // the reference's guard rejects, pass src through: the basic estimate and
    // dst start as copies of src, as in the reference's in-place Frame path
    // (source/BM3D.cpp:512-521).
    for (int c = 0; c < nplanes; ++c) {
        if ((rc = copy_plane(ctx, tmp[c], dpitch, ds[c], dpitch, width, height,
                             cudaMemcpyDeviceToDevice, s)) != BM3D_OK)
            return rc;
        if (nplanes > 1 || check_params(fin, nplanes) != Guard::Run)
            if ((rc = copy_plane(ctx, dd[c], dpitch, ds[c], dpitch, width, height,
                                 cudaMemcpyDeviceToDevice, s)) != BM3D_OK)
                return rc;
    }
    {
        const Guard g = check_params(basic, nplanes);
        if (g == Guard::Invalid) return BM3D_ERR_INVALID;
        if (g == Guard::Unsupported) {
            ctx->err = "parameters outside this build (BlockSize <= 16, GroupSize <= 32)";
            return BM3D_ERR_UNSUPPORTED;
        }
        if (g == Guard::Run) {
            rc = run_stage_device(ctx, basic, false, nplanes, tmp, ds, dr, width, height, dpitch,
                                  value_range, s);
            if (rc != BM3D_OK) return rc;
        }
    }
    {
        const Guard g = check_params(fin, nplanes);
        if (g == Guard::Invalid) return BM3D_ERR_INVALID;
        if (g == Guard::Unsupported) {
            ctx->err = "parameters outside this build (BlockSize <= 16, GroupSize <= 32)";
            return BM3D_ERR_UNSUPPORTED;
        }
        const T *tr[kMaxPlanes];
        for (int c = 0; c < nplanes; ++c) tr[c] = tmp[c];
        if (g == Guard::Run) {
            rc = run_stage_device(ctx, fin, true, nplanes, dd, ds, tr, width, height, dpitch,
                                  value_range, s);
            if (rc != BM3D_OK) return rc;
        }
    }
    if (mem == BM3D_MEM_HOST) {
        for (int c = 0; c < nplanes; ++c)
            if ((rc = copy_plane(ctx, dst[c], stride, static_cast<const T *>(dd[c]), width, width,
                                 height, cudaMemcpyDeviceToHost, s)) != BM3D_OK)
                return rc;
        CK(ctx, cudaStreamSynchronize(s));
        return check_invariants(ctx);
    }
    return BM3D_OK;
}

extern "C" int bm3d_full(bm3d_ctx *ctx, const bm3d_stage_params *basic,
                         const bm3d_stage_params *final_, float *dst, const float *src,
                         const float *ref, int width, int height, size_t stride,
                         float value_range, int mem, void *stream)
{
    float *d[1] = {dst};
    const float *s[1] = {src}, *r[1] = {ref};
    return full_any<float>(ctx, basic, final_, 1, d, s, r, width, height, stride, value_range,
                           mem, stream);
}

extern "C" int bm3d_full3(bm3d_ctx *ctx, const bm3d_stage_params *basic,
                          const bm3d_stage_params *final_, float *const dst[3],
                          const float *const src[3], const float *const ref[3], int width,
                          int height, size_t stride, float value_range, int mem, void *stream)
{
    if (!dst || !src) return BM3D_ERR_INVALID;
    return full_any<float>(ctx, basic, final_, 3, dst, src, ref, width, height, stride,
                           value_range, mem, stream);
}

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

// ---------------------------------------------------------------------------
// Many host planes, copies overlapped with the filtering.

extern "C" int bm3d_full_many(bm3d_ctx *ctx, int count, const bm3d_stage_params *basic,
                              const bm3d_stage_params *final_, float *const dst[],
                              const float *const src[], const int width[], const int height[],
                              const size_t stride[], float value_range, int async, void *stream)
{
    if (!ctx || count < 0 || (count > 0 && (!basic || !final_ || !dst || !src || !width ||
                                            !height || !stride)))
        return BM3D_ERR_INVALID;
    for (int i = 0; i < count; ++i)
        if (!dst[i] || !src[i] || width[i] < 1 || height[i] < 1 ||
            stride[i] < static_cast<size_t>(width[i]))
            return BM3D_ERR_INVALID;
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!ctx->up) {
        CK(ctx, cudaStreamCreateWithFlags(&ctx->up, cudaStreamNonBlocking));
        CK(ctx, cudaStreamCreateWithFlags(&ctx->down, cudaStreamNonBlocking));
        for (auto &sl : ctx->pipe) {
            CK(ctx, cudaEventCreateWithFlags(&sl.in_ready, cudaEventDisableTiming));
            CK(ctx, cudaEventCreateWithFlags(&sl.computed, cudaEventDisableTiming));
            CK(ctx, cudaEventCreateWithFlags(&sl.drained, cudaEventDisableTiming));
        }
    }
    // Uploads run one plane ahead on `up`, downloads trail on `down`; a slot's
    // input is reused once its plane has been filtered, its output once it
    // has been copied out. `stream` does the filtering.
    int status = BM3D_OK;
    auto upload = [&](int i) -> int {
        auto &sl = ctx->pipe[(ctx->pipe_count + i) & 1];
        const size_t bytes = sizeof(float) * static_cast<size_t>(width[i]) * height[i];
        if (sl.used) CK(ctx, cudaStreamWaitEvent(ctx->up, sl.computed, 0));
        if (sl.in.bytes < bytes) {  // growing a buffer: let every use of it finish first
            if (sl.used) CK(ctx, cudaEventSynchronize(sl.computed));
            int rc = ensure(ctx, sl.in, bytes);
            if (rc != BM3D_OK) return rc;
        }
        CK(ctx, cudaMemcpy2DAsync(sl.in.ptr, sizeof(float) * width[i], src[i],
                                  sizeof(float) * stride[i], sizeof(float) * width[i], height[i],
                                  cudaMemcpyHostToDevice, ctx->up));
        CK(ctx, cudaEventRecord(sl.in_ready, ctx->up));
        return BM3D_OK;
    };
    if (count > 0) {
        int rc = upload(0);
        if (rc != BM3D_OK) return rc;
    }
    for (int i = 0; i < count; ++i) {
        if (i + 1 < count) {
            int rc = upload(i + 1);
            if (rc != BM3D_OK) return rc;
        }
        auto &sl = ctx->pipe[(ctx->pipe_count + i) & 1];
        const size_t bytes = sizeof(float) * static_cast<size_t>(width[i]) * height[i];
        if (sl.used) CK(ctx, cudaStreamWaitEvent(s, sl.drained, 0));
        if (sl.out.bytes < bytes) {
            if (sl.used) CK(ctx, cudaEventSynchronize(sl.drained));
            int rc = ensure(ctx, sl.out, bytes);
            if (rc != BM3D_OK) return rc;
        }
        CK(ctx, cudaStreamWaitEvent(s, sl.in_ready, 0));
        float *d[1] = {static_cast<float *>(sl.out.ptr)};
        const float *x[1] = {static_cast<const float *>(sl.in.ptr)};
        const int rc = full_any<float>(ctx, &basic[i], &final_[i], 1, d, x, nullptr, width[i],
                                       height[i], static_cast<size_t>(width[i]), value_range,
                                       BM3D_MEM_DEVICE, s);
        if (rc < 0) return rc;
        if (rc == BM3D_COPIED) status = BM3D_COPIED;
        CK(ctx, cudaEventRecord(sl.computed, s));
        CK(ctx, cudaStreamWaitEvent(ctx->down, sl.computed, 0));
        CK(ctx, cudaMemcpy2DAsync(dst[i], sizeof(float) * stride[i], sl.out.ptr,
                                  sizeof(float) * width[i], sizeof(float) * width[i], height[i],
                                  cudaMemcpyDeviceToHost, ctx->down));
        CK(ctx, cudaEventRecord(sl.drained, ctx->down));
        sl.used = true;
    }
    ctx->pipe_count += static_cast<unsigned long long>(count);
    if (count > 0) {
        // `stream` completes after the last download
        auto &last = ctx->pipe[(ctx->pipe_count - 1) & 1];
        CK(ctx, cudaStreamWaitEvent(s, last.drained, 0));
    }
    if (async) return status;
    CK(ctx, cudaStreamSynchronize(s));
    const int rc = check_invariants(ctx);
    return rc != BM3D_OK ? rc : status;
}

extern "C" int bm3d_debug_groups(bm3d_ctx *ctx, const bm3d_stage_params *p, int wiener,
                                 const float *ref, int width, int height, size_t stride,
                                 float value_range, int *counts, int *pos_yx, float *keys)
{
    if (!ctx || !p || !ref || !counts || !pos_yx || !keys) return BM3D_ERR_INVALID;
    const Guard g = check_params(p, 1);
    if (g == Guard::Invalid || g == Guard::Copy) return BM3D_ERR_INVALID;
    if (g == Guard::Unsupported) return BM3D_ERR_UNSUPPORTED;
    if (width < p->block_size || height < p->block_size || stride < static_cast<size_t>(width))
        return BM3D_ERR_INVALID;
    CK(ctx, cudaSetDevice(ctx->device));
    const long long nref = bm3d_ref_block_count(p, width, height);
    int rc;
    const size_t plane_bytes = sizeof(float) * static_cast<size_t>(width) * height;
    if ((rc = ensure(ctx, ctx->stage_in[0], plane_bytes)) != BM3D_OK) return rc;
    if ((rc = ensure(ctx, ctx->groups[0], sizeof(int) * nref)) != BM3D_OK) return rc;
    if ((rc = ensure(ctx, ctx->groups[1], sizeof(int) * nref * kGSTab * 2)) != BM3D_OK) return rc;
    if ((rc = ensure(ctx, ctx->groups[2], sizeof(float) * nref * kGSTab)) != BM3D_OK) return rc;
    cudaStream_t s = nullptr;
    float *in = static_cast<float *>(ctx->stage_in[0].ptr);
    if ((rc = copy_plane(ctx, in, width, ref, stride, width, height, cudaMemcpyHostToDevice, s)) !=
        BM3D_OK)
        return rc;
    float *d[1] = {in};
    const float *sp[1] = {in};
    rc = run_stage_device<float>(ctx, p, wiener != 0, 1, d, sp, sp, width, height, width,
                                 value_range, s, static_cast<int *>(ctx->groups[0].ptr),
                                 static_cast<int *>(ctx->groups[1].ptr),
                                 static_cast<float *>(ctx->groups[2].ptr), true);
    if (rc != BM3D_OK) return rc;
    CK(ctx, cudaMemcpyAsync(counts, ctx->groups[0].ptr, sizeof(int) * nref, cudaMemcpyDeviceToHost, s));
    CK(ctx, cudaMemcpyAsync(pos_yx, ctx->groups[1].ptr, sizeof(int) * nref * kGSTab * 2,
                            cudaMemcpyDeviceToHost, s));
    CK(ctx, cudaMemcpyAsync(keys, ctx->groups[2].ptr, sizeof(float) * nref * kGSTab,
                            cudaMemcpyDeviceToHost, s));
    CK(ctx, cudaStreamSynchronize(s));
    return BM3D_OK;
}

extern "C" int bm3d_set_kernel_timing(bm3d_ctx *ctx, int on)
{
    if (!ctx) return BM3D_ERR_INVALID;
    CK(ctx, cudaSetDevice(ctx->device));
    drain_timing(ctx);
    ctx->timing = on != 0;
    ctx->time_ms[0] = ctx->time_ms[1] = 0;
    ctx->launches[0] = ctx->launches[1] = 0;
    return BM3D_OK;
}

extern "C" int bm3d_kernel_time(bm3d_ctx *ctx, int wiener, double *ms, long long *launches)
{
    if (!ctx || !ms || !launches) return BM3D_ERR_INVALID;
    CK(ctx, cudaSetDevice(ctx->device));
    drain_timing(ctx);
    *ms = ctx->time_ms[wiener ? 1 : 0];
    *launches = ctx->launches[wiener ? 1 : 0];
    return BM3D_OK;
}

extern "C" int bm3d_last_stats(bm3d_ctx *ctx, unsigned long long out[4])
{
    if (!ctx || !out) return BM3D_ERR_INVALID;
    CK(ctx, cudaSetDevice(ctx->device));
    CK(ctx, cudaStreamSynchronize(ctx->last_stream));
    CK(ctx, cudaMemcpy(out, ctx->stats, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    return BM3D_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free stage: bm3d_stage_noalloc.
//
// For callers that must not allocate device memory after start-up, e.g. a
// filter plugin inside a host application that owns every device allocation,
// or a real-time video path where a cudaMalloc (which can synchronise the
// device and can fail under memory pressure) is not allowed per frame. The
// stage kernels' scratch -- the fixed-point numerator and weight planes, the
// per-plane |src| maximum and the counters -- lives in the file-scope array
// below instead of context buffers. Every GPU that loads this library holds
// the array until the process exits.

namespace {

constexpr size_t kNoAllocMaxPixels = size_t(1) << 21;  // 2,097,152 pixels (1920x1080 fits)
constexpr size_t kNoAllocAccBytes = kNoAllocMaxPixels * sizeof(long long);
// num (int64 per pixel) | den (int64 per pixel) | absmax (4 floats) | counters (8 x u64)
constexpr size_t kNoAllocBytes = 2 * kNoAllocAccBytes + 256 + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

struct NoAllocDevice {
    bool ready = false;
    unsigned char *scratch = nullptr;  // device address of g_noalloc_scratch
    int sm_count = 0;
    size_t smem_optin = 0;
};

constexpr int kNoAllocMaxDevices = 64;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
std::mutex g_noalloc_mu;

// Status for a failed step: CUDA errors map to BM3D_ERR_CUDA, everything else
// to the given code. (The message names the step for readers of this file.)
int noalloc_error(const char *, cudaError_t e = cudaSuccess, int code = BM3D_ERR_INVALID)
{
    return e == cudaSuccess ? code : BM3D_ERR_CUDA;
}

// Set-up once per device, with that device current: the device address of the
// scratch array (the host-side symbol is only a stand-in, not a device
// address), the cosine tables, and the device limits.
int noalloc_setup(int dev, NoAllocDevice **out)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoAllocDevice &d = g_noalloc_dev[dev];
    if (d.ready) {
        *out = &d;
        return BM3D_OK;
    }
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return noalloc_error("cudaGetSymbolAddress(g_noalloc_scratch)", e);
    // the cosine tables live in fixed-size host arrays (no heap), uploaded per device
    if ((e = upload_dct_tables()) != cudaSuccess)
        return noalloc_error("cudaMemcpyToSymbol(cosine tables)", e);
    int sm = 0, optin = 0;
    if ((e = cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) !=
            cudaSuccess)
        return noalloc_error("cudaDeviceGetAttribute", e);
    d.scratch = static_cast<unsigned char *>(ptr);
    d.sm_count = sm;
    d.smem_optin = static_cast<size_t>(optin);
    d.ready = true;
    *out = &d;
    return BM3D_OK;
}

}  // namespace

extern "C" int bm3d_stage_noalloc(const bm3d_stage_params *params, int wiener, float *dst,
                                  const float *src, const float *ref, int width, int height,
                                  size_t stride, float value_range, void *stream)
{
    if (!ref) ref = src;
    if (!params || !dst || !src) return noalloc_error("bm3d_stage_noalloc: null argument");
    const Guard g = check_params(params, 1);
    if (g == Guard::Invalid) return noalloc_error("bm3d_stage_noalloc: invalid parameters");
    // the register-resident kernel only: BlockSize 8, GroupSize <= 16
    if (g == Guard::Unsupported || !fast_path(params)) return BM3D_ERR_UNSUPPORTED;
    if (width < params->block_size || height < params->block_size ||
        stride < static_cast<size_t>(width))
        return noalloc_error("bm3d_stage_noalloc: width/height below BlockSize or stride < width");
    if (static_cast<size_t>(width) * static_cast<size_t>(height) > kNoAllocMaxPixels)
        return BM3D_ERR_TOO_LARGE;  // larger than the 2,097,152-pixel static scratch
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_error("cudaGetDevice", e);
    if (dev < 0 || dev >= kNoAllocMaxDevices) return noalloc_error("bm3d_stage_noalloc: device id");
    NoAllocDevice *d = nullptr;
    int rc = noalloc_setup(dev, &d);
    if (rc != BM3D_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (g == Guard::Copy) {
        if (dst != src &&
            (e = cudaMemcpy2DAsync(dst, stride * sizeof(float), src, stride * sizeof(float),
                                   width * sizeof(float), height, cudaMemcpyDeviceToDevice, s)) !=
                cudaSuccess)
            return noalloc_error("cudaMemcpy2DAsync", e);
        return BM3D_COPIED;
    }

    // The shared scratch: this call's accumulators start from zero below.
    long long *num = reinterpret_cast<long long *>(d->scratch);
    long long *den = reinterpret_cast<long long *>(d->scratch + kNoAllocAccBytes);
    float *absmax = reinterpret_cast<float *>(d->scratch + 2 * kNoAllocAccBytes);
    unsigned long long *stats =
        reinterpret_cast<unsigned long long *>(d->scratch + 2 * kNoAllocAccBytes + 256);

    StageArgs<float> a;
    std::memset(&a, 0, sizeof(a));
    fill_tables(a, params, wiener != 0, 1, value_range);
    a.stride = static_cast<long long>(stride);
    a.src[0] = src;
    a.ref[0] = ref;
    a.ref_alias_src = src == ref ? 1 : 0;
    bm3d_ctx info;  // device limits and default tiling only; owns no device memory
    info.device = dev;
    info.sm_count = d->sm_count;
    info.smem_optin = d->smem_optin;
    int warps;
    rc = plan_geometry(&info, a, params, wiener != 0, 1, width, height, warps);
    if (rc != BM3D_OK) return rc;
    const double terms = 2.0 * static_cast<double>(a.nx) * a.ny * std::max(1, params->group_size);
    a.log2_bound = static_cast<int>(std::ceil(std::log2(std::max(2.0, terms))));
    a.absmax = absmax;
    a.num[0] = num;
    a.den[0] = den;
    a.stats = stats;

    const long long npx = static_cast<long long>(width) * height;
    const int threads = 256;
    const int blocks = static_cast<int>(
        std::min<long long>((npx + threads - 1) / threads, static_cast<long long>(d->sm_count) * 8));
    if ((e = cudaMemsetAsync(absmax, 0, 256 + 256, s)) != cudaSuccess)
        return noalloc_error("cudaMemsetAsync(scratch header)", e);
    prep_kernel<float><<<blocks, threads, 0, s>>>(num, den, src, a.stride, width, height, absmax);
    if ((e = cudaGetLastError()) != cudaSuccess) return noalloc_error("prep_kernel", e);
    rc = launch_stage(&info, a, wiener != 0, 1, s, warps);
    if (rc != BM3D_OK) return rc;
    const dim3 ngrid((width + kNormTile - 1) / kNormTile, (height + kNormTile - 1) / kNormTile);
    normalize_kernel<float><<<ngrid, 256, 0, s>>>(dst, a.stride, num, den, width, height,
                                                  a.block_size);
    if ((e = cudaGetLastError()) != cudaSuccess) return noalloc_error("normalize_kernel", e);
    return BM3D_OK;
}

// ---------------------------------------------------------------------------
// Batches: bm3d_batch_create / bm3d_batch_run / bm3d_batch_destroy.

namespace {

struct StageBuild {
    int tile_x = 0, tile_y = 0, warps = 0;
    bool generic = false;
    int nact = 0;            // planes with work in this stage
    int total_tiles = 0;
    size_t smem = 0;         // dynamic shared memory of the persistent launch
    int grid = 0;
    DevBuf args, base;       // device StageArgs[nact], int[nact + 1]
};

}  // namespace

struct bm3d_batch {
    bm3d_ctx *ctx = nullptr;
    int n = 0;    // images
    int npl = 1;  // planes per image (1, or 3 sharing the luma groups)
    std::vector<int> w, h;
    std::vector<size_t> stride;
    std::vector<const float *> src;  // plane c of image i at [i * npl + c]
    std::vector<float *> dst;
    std::vector<bm3d_stage_params> pb, pf;
    std::vector<Guard> gb, gf;
    std::vector<size_t> acc_off, basic_off;  // per plane: offsets into acc (int64) and basic (float)
    DevBuf acc, basic, absmax, counters, planes_b, planes_f;
    int nq_b = 0, nq_f = 0;  // entries of planes_b / planes_f (planes each stage filters)
    StageBuild sb, sf;
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

int batch_fail(bm3d_ctx *ctx, const char *msg)
{
    ctx->err = msg;
    return BM3D_ERR_INVALID;
}

// Per-plane stage arguments of one stage at one tiling; uploads them and sizes
// the persistent launch. Returns BM3D_ERR_UNSUPPORTED when the tiling does
// not fit in shared memory.
int build_stage(bm3d_batch *B, bool wiener, int tx, int ty, int warps, StageBuild &out)
{
    bm3d_ctx *ctx = B->ctx;
    std::vector<StageArgs<float>> args;
    std::vector<int> base(1, 0);
    size_t smem = 0;
    bool generic = false;
    for (int i = 0; i < B->n; ++i) {
        const bm3d_stage_params *p = wiener ? &B->pf[i] : &B->pb[i];
        if ((wiener ? B->gf[i] : B->gb[i]) != Guard::Run) continue;
        StageArgs<float> a;
        std::memset(&a, 0, sizeof(a));
        const int npl = B->npl;
        fill_tables(a, p, wiener, npl, 1.0);
        generic = !fast_args(p->block_size, p->group_size);
        const int BS = p->block_size;
        a.width = B->w[i];
        a.height = B->h[i];
        a.block_size = BS;
        a.step = p->block_step;
        a.group_size = p->group_size;
        a.bm_step = p->bm_step;
        a.range = p->bm_range / p->bm_step * p->bm_step;
        a.nx = ref_count(a.width - BS, a.step);
        a.ny = ref_count(a.height - BS, a.step);
        const int span = 2 * (a.range / a.bm_step) + 1;
        a.key_slots = span * span + 1;
        const int reach = a.match ? a.range : 0;
        a.region_w = std::min(a.width, (tx - 1) * a.step + 2 * reach + BS);
        a.region_h = std::min(a.height, (ty - 1) * a.step + 2 * reach + BS);
        a.region_pitch = a.region_w + ((5 - a.region_w % 8) + 8) % 8;
        a.tile_x = std::min(tx, a.nx);
        a.tile_y = std::min(ty, a.ny);
        a.tiles_x = (a.nx + a.tile_x - 1) / a.tile_x;
        a.stride = static_cast<long long>(B->stride[i]);
        a.ref_alias_src = wiener ? 0 : (1 << npl) - 1;
        for (int c = 0; c < npl; ++c) {
            const int k = i * npl + c;
            a.src[c] = B->src[k];
            a.ref[c] = wiener ? static_cast<const float *>(B->basic.ptr) + B->basic_off[k]
                              : B->src[k];
            a.num[c] = static_cast<long long *>(B->acc.ptr) + B->acc_off[k];
            a.den[c] = a.num[c] + static_cast<size_t>(a.width) * a.height;
        }
        a.absmax = static_cast<float *>(B->absmax.ptr) + i * npl;
        const double terms = 2.0 * static_cast<double>(a.nx) * a.ny * std::max(1, p->group_size);
        a.log2_bound = static_cast<int>(std::ceil(std::log2(std::max(2.0, terms))));
        a.dct_fwd = ctx->gtab_f;
        a.dct_inv = ctx->gtab_f ? ctx->gtab_f + kDctTableSize : nullptr;
        const SmemPlan sp = plan_smem<float>(npl, wiener, a.ref_alias_src, a.region_h,
                                             a.region_pitch, a.key_slots, warps, generic, BS,
                                             p->group_size, a.tile_x * a.tile_y);
        smem = std::max(smem, sp.total + kBatchHeader);
        args.push_back(a);
        base.push_back(base.back() + a.tiles_x * ((a.ny + a.tile_y - 1) / a.tile_y));
    }
    if (smem > ctx->smem_optin) return BM3D_ERR_UNSUPPORTED;
    out.tile_x = tx;
    out.tile_y = ty;
    out.warps = warps;
    out.generic = generic;
    out.nact = static_cast<int>(args.size());
    out.total_tiles = base.back();
    out.smem = smem;
    int rc;
    if (out.nact > 0) {
        if ((rc = ensure(ctx, out.args, sizeof(StageArgs<float>) * args.size())) != BM3D_OK) return rc;
        if ((rc = ensure(ctx, out.base, sizeof(int) * base.size())) != BM3D_OK) return rc;
        CK(ctx, cudaMemcpy(out.args.ptr, args.data(), sizeof(StageArgs<float>) * args.size(),
                           cudaMemcpyHostToDevice));
        CK(ctx, cudaMemcpy(out.base.ptr, base.data(), sizeof(int) * base.size(),
                           cudaMemcpyHostToDevice));
    }
    return BM3D_OK;
}

template <bool W>
int launch_batch_stage(bm3d_batch *B, StageBuild &sbd, int *counter, cudaStream_t s)
{
    bm3d_ctx *ctx = B->ctx;
    if (sbd.nact == 0) return BM3D_OK;
    CK(ctx, cudaMemsetAsync(counter, 0, sizeof(int), s));
    const auto *args = static_cast<const StageArgs<float> *>(sbd.args.ptr);
    const int *base = static_cast<const int *>(sbd.base.ptr);
    int nimg = sbd.nact;
    auto go = [&](const void *kern) -> int {
        CK(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(sbd.smem)));
        int per_sm = 0;
        CK(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, sbd.warps * kWarp,
                                                              sbd.smem));
        sbd.grid = std::max(1, per_sm) * ctx->sm_count;
        void *kargs[] = {&args, &base, &nimg, &counter};
        CK(ctx, cudaLaunchKernel(kern, dim3(sbd.grid), dim3(sbd.warps * kWarp), kargs, sbd.smem, s));
        return BM3D_OK;
    };
    const bool ks4 = (W ? B->pf[0].bm_step : B->pb[0].bm_step) == 1;
    if (B->npl == 3) {
        if (sbd.generic) return go(batch_kernel_fn<W, 3, 1, true>());
        return go(ks4 ? batch_kernel_fn<W, 3, 4, false>() : batch_kernel_fn<W, 3, 1, false>());
    }
    if (sbd.generic) return go(batch_kernel_fn<W, 1, 1, true>());
    return go(ks4 ? batch_kernel_fn<W, 1, 4, false>() : batch_kernel_fn<W, 1, 1, false>());
}

int launch_planes(bm3d_batch *B, const DevBuf &planes, bool prep, cudaStream_t s)
{
    const int count = &planes == &B->planes_b ? B->nq_b : B->nq_f;
    if (count == 0) return BM3D_OK;
    long long maxpx = 0;
    for (int i = 0; i < B->n; ++i) maxpx = std::max(maxpx, static_cast<long long>(B->w[i]) * B->h[i]);
    // enough CTAs in all to fill the GPU a few times over, at least 64 per plane
    const long long tiles = (maxpx + kNormTile * kNormTile - 1) / (kNormTile * kNormTile);
    const long long cap = std::max<long long>(64, 8LL * B->ctx->sm_count / count);
    const dim3 grid(static_cast<unsigned>(std::min<long long>(prep ? (maxpx + 255) / 256 : tiles, cap)),
                    static_cast<unsigned>(count));
    const auto *q = static_cast<const BatchPlane<float> *>(planes.ptr);
    if (prep) prep_batch_kernel<float><<<grid, 256, 0, s>>>(q);
    else normalize_batch_kernel<float><<<grid, 256, 0, s>>>(q);
    CK(B->ctx, cudaGetLastError());
    return BM3D_OK;
}

// The whole pipeline, enqueued on s (captured into the graph).
int enqueue_batch(bm3d_batch *B, cudaStream_t s)
{
    bm3d_ctx *ctx = B->ctx;
    int rc;
    int *counters = static_cast<int *>(B->counters.ptr);
    for (int i = 0; i < B->n; ++i) {  // planes a stage passes through unfiltered
        for (int c = 0; c < B->npl; ++c) {
            const int k = i * B->npl + c;
            float *bi = static_cast<float *>(B->basic.ptr) + B->basic_off[k];
            const bool b_off = B->gb[i] != Guard::Run || !(B->pb[i].sigma[c] > 0 || B->npl == 1);
            const bool f_off = B->gf[i] != Guard::Run || !(B->pf[i].sigma[c] > 0 || B->npl == 1);
            if (b_off)
                CK(ctx, cudaMemcpy2DAsync(bi, B->stride[i] * 4, B->src[k], B->stride[i] * 4,
                                          B->w[i] * 4, B->h[i], cudaMemcpyDeviceToDevice, s));
            if (f_off && B->dst[k] != B->src[k])
                CK(ctx, cudaMemcpy2DAsync(B->dst[k], B->stride[i] * 4, B->src[k], B->stride[i] * 4,
                                          B->w[i] * 4, B->h[i], cudaMemcpyDeviceToDevice, s));
        }
    }
    CK(ctx, cudaMemsetAsync(B->absmax.ptr, 0, sizeof(float) * B->n * B->npl, s));
    if ((rc = launch_planes(B, B->planes_b, true, s)) != BM3D_OK) return rc;
    if ((rc = launch_batch_stage<false>(B, B->sb, counters, s)) != BM3D_OK) return rc;
    if ((rc = launch_planes(B, B->planes_b, false, s)) != BM3D_OK) return rc;
    if ((rc = launch_planes(B, B->planes_f, true, s)) != BM3D_OK) return rc;
    if ((rc = launch_batch_stage<true>(B, B->sf, counters + 1, s)) != BM3D_OK) return rc;
    if ((rc = launch_planes(B, B->planes_f, false, s)) != BM3D_OK) return rc;
    return BM3D_OK;
}

// Time one stage launch (after a prep) at the current build.
template <bool W>
int time_stage(bm3d_batch *B, StageBuild &sbd, const DevBuf &planes, cudaStream_t s, float &ms)
{
    bm3d_ctx *ctx = B->ctx;
    int rc;
    cudaEvent_t e0, e1;
    CK(ctx, cudaEventCreate(&e0));
    CK(ctx, cudaEventCreate(&e1));
    ms = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        if ((rc = launch_planes(B, planes, true, s)) != BM3D_OK) return rc;
        CK(ctx, cudaEventRecord(e0, s));
        if ((rc = launch_batch_stage<W>(B, sbd, static_cast<int *>(B->counters.ptr) + (W ? 1 : 0),
                                        s)) != BM3D_OK)
            return rc;
        CK(ctx, cudaEventRecord(e1, s));
        CK(ctx, cudaEventSynchronize(e1));
        float t = 0;
        CK(ctx, cudaEventElapsedTime(&t, e0, e1));
        if (rep > 0) ms = std::min(ms, t);  // first run warms up
    }
    if (!W) {  // leave the basic estimates in place for the final stage's tuning
        if ((rc = launch_planes(B, planes, false, s)) != BM3D_OK) return rc;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return BM3D_OK;
}

// Pick the tiling of one stage: the fastest candidate that fits, or the
// default when not autotuning.
template <bool W>
int tune_stage(bm3d_batch *B, StageBuild &sbd, const DevBuf &planes, bool autotune, cudaStream_t s,
               const int *force = nullptr)
{
    if (force) return build_stage(B, W, force[0], force[1], force[2], sbd);  // a known tiling
    const bm3d_stage_params &p = W ? B->pf[0] : B->pb[0];
    const bool generic = !fast_args(p.block_size, p.group_size);
    static const int fast_cand[][3] = {{8, 8, 16}, {7, 7, 16}, {6, 8, 12}, {8, 6, 12},
                                       {6, 6, 12}, {4, 4, 4}, {4, 4, 2}, {2, 2, 1}};
    static const int gen_cand[][3] = {{4, 4, 8}, {4, 4, 4}, {2, 2, 4}, {2, 2, 2}, {1, 1, 2}, {1, 1, 1}};
    const int (*cand)[3] = generic ? gen_cand : fast_cand;
    const int ncand = generic ? 6 : 8;
    int best = -1;
    float best_ms = 1e30f;
    for (int c = 0; c < ncand; ++c) {
        int rc = build_stage(B, W, cand[c][0], cand[c][1], cand[c][2], sbd);
        if (rc == BM3D_ERR_UNSUPPORTED) continue;
        if (rc != BM3D_OK) return rc;
        if (!autotune) {
            best = c;
            break;
        }
        float ms;
        if ((rc = time_stage<W>(B, sbd, planes, s, ms)) != BM3D_OK) return rc;
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    if (best < 0) {
        B->ctx->err = "batch stage does not fit in shared memory";
        return BM3D_ERR_UNSUPPORTED;
    }
    int rc = build_stage(B, W, cand[best][0], cand[best][1], cand[best][2], sbd);
    if (rc == BM3D_OK && !W && autotune) {
        float ms;  // re-run the chosen basic tiling so the final stage tunes on its output
        rc = time_stage<W>(B, sbd, planes, s, ms);
    }
    return rc;
}

}  // namespace

static int batch_create_any(bm3d_ctx *ctx, int npl, int count, const bm3d_stage_params *basic,
                            const bm3d_stage_params *final_, float *const dst[],
                            const float *const src[], const int width[], const int height[],
                            const size_t stride[], int autotune, bm3d_batch **out,
                            const int *force_tiling = nullptr)
{
    if (!ctx || !out || count < 1 || !basic || !final_ || !dst || !src || !width || !height ||
        !stride)
        return BM3D_ERR_INVALID;
    *out = nullptr;
    CK(ctx, cudaSetDevice(ctx->device));
    auto *B = new bm3d_batch;
    B->ctx = ctx;
    B->n = count;
    B->npl = npl;
    auto fail = [&](int rc) {
        bm3d_batch_destroy(B);
        return rc;
    };
    size_t acc_total = 0, basic_total = 0;
    for (int i = 0; i < count; ++i) {
        const Guard gb = check_params(&basic[i], npl), gf = check_params(&final_[i], npl);
        if (gb == Guard::Invalid || gf == Guard::Invalid) return fail(batch_fail(ctx, "invalid parameters"));
        if (gb == Guard::Unsupported || gf == Guard::Unsupported) {
            ctx->err = "parameters outside this build (BlockSize <= 16, GroupSize <= 32)";
            return fail(BM3D_ERR_UNSUPPORTED);
        }
        for (const auto *pp : {&basic[i], &final_[i]}) {
            const auto &q0 = pp == &basic[i] ? basic[0] : final_[0];
            if (pp->block_size != q0.block_size || pp->block_step != q0.block_step ||
                pp->group_size != q0.group_size || pp->bm_range != q0.bm_range ||
                pp->bm_step != q0.bm_step)
                return fail(batch_fail(ctx, "planes of a batch must share the stage geometry"));
        }
        const int bs = std::max(basic[i].block_size, final_[i].block_size);
        if (width[i] < bs || height[i] < bs || stride[i] < static_cast<size_t>(width[i]))
            return fail(batch_fail(ctx, "bad plane"));
        B->w.push_back(width[i]);
        B->h.push_back(height[i]);
        B->stride.push_back(stride[i]);
        B->pb.push_back(basic[i]);
        B->pf.push_back(final_[i]);
        B->gb.push_back(gb);
        B->gf.push_back(gf);
        for (int c = 0; c < npl; ++c) {
            const int k = i * npl + c;
            if (!src[k] || !dst[k]) return fail(batch_fail(ctx, "bad plane"));
            B->src.push_back(src[k]);
            B->dst.push_back(dst[k]);
            B->acc_off.push_back(acc_total);
            B->basic_off.push_back(basic_total);
            acc_total += 2 * static_cast<size_t>(width[i]) * height[i];
            basic_total += stride[i] * height[i];
        }
    }
    int rc;
    if ((rc = ensure(ctx, B->acc, sizeof(long long) * acc_total)) != BM3D_OK) return fail(rc);
    if ((rc = ensure(ctx, B->basic, sizeof(float) * basic_total)) != BM3D_OK) return fail(rc);
    if ((rc = ensure(ctx, B->absmax, sizeof(float) * count * npl)) != BM3D_OK) return fail(rc);
    if ((rc = ensure(ctx, B->counters, 2 * sizeof(int))) != BM3D_OK) return fail(rc);
    // per-pixel kernels' plane tables, active planes of each stage in batch order
    for (int st = 0; st < 2; ++st) {
        std::vector<BatchPlane<float>> q;
        for (int i = 0; i < count; ++i) {
            if ((st ? B->gf[i] : B->gb[i]) != Guard::Run) continue;
            const bm3d_stage_params &pp = st ? final_[i] : basic[i];
            for (int c = 0; c < npl; ++c) {
                if (npl > 1 && !(pp.sigma[c] > 0)) continue;  // plane left alone by the stage
                const int k = i * npl + c;
                BatchPlane<float> bp;
                bp.num = static_cast<long long *>(B->acc.ptr) + B->acc_off[k];
                bp.den = bp.num + static_cast<size_t>(width[i]) * height[i];
                bp.src = src[k];
                bp.dst = st ? dst[k] : static_cast<float *>(B->basic.ptr) + B->basic_off[k];
                bp.src_stride = static_cast<long long>(stride[i]);
                bp.dst_stride = static_cast<long long>(stride[i]);
                bp.width = width[i];
                bp.height = height[i];
                bp.block_size = pp.block_size;
                bp.absmax = static_cast<float *>(B->absmax.ptr) + k;
                q.push_back(bp);
            }
        }
        DevBuf &dbuf = st ? B->planes_f : B->planes_b;
        (st ? B->nq_f : B->nq_b) = static_cast<int>(q.size());
        if (!q.empty()) {
            if ((rc = ensure(ctx, dbuf, sizeof(BatchPlane<float>) * q.size())) != BM3D_OK) return fail(rc);
            CK(ctx, cudaMemcpy(dbuf.ptr, q.data(), sizeof(BatchPlane<float>) * q.size(),
                               cudaMemcpyHostToDevice));
        }
    }
    cudaError_t e = cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "cudaStreamCreate"));
    // planes whose basic stage is a copy must hold src before the final stage tunes
    for (int i = 0; i < count; ++i)
        for (int c = 0; c < npl; ++c) {
            if (B->gb[i] == Guard::Run && (npl == 1 || basic[i].sigma[c] > 0)) continue;
            const int k = i * npl + c;
            float *bi = static_cast<float *>(B->basic.ptr) + B->basic_off[k];
            e = cudaMemcpy2DAsync(bi, stride[i] * 4, src[k], stride[i] * 4, width[i] * 4, height[i],
                                  cudaMemcpyDeviceToDevice, B->cap);
            if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "cudaMemcpy2DAsync"));
        }
    e = cudaMemsetAsync(B->absmax.ptr, 0, sizeof(float) * count * npl, B->cap);
    if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "cudaMemsetAsync"));
    if ((rc = tune_stage<false>(B, B->sb, B->planes_b, autotune != 0, B->cap,
                                force_tiling)) != BM3D_OK)
        return fail(rc);
    if ((rc = tune_stage<true>(B, B->sf, B->planes_f, autotune != 0, B->cap,
                               force_tiling ? force_tiling + 3 : nullptr)) != BM3D_OK)
        return fail(rc);
    e = cudaStreamSynchronize(B->cap);
    if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "batch tuning"));
    // capture the pipeline once
    e = cudaStreamBeginCapture(B->cap, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "cudaStreamBeginCapture"));
    rc = enqueue_batch(B, B->cap);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(B->cap, &g);
    if (rc != BM3D_OK) {
        if (g) cudaGraphDestroy(g);
        return fail(rc);
    }
    if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "cudaStreamEndCapture"));
    B->graph = g;
    e = cudaGraphInstantiate(&B->exec, g, 0);
    if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "cudaGraphInstantiate"));
    *out = B;
    return BM3D_OK;
}

extern "C" int bm3d_batch_create(bm3d_ctx *ctx, int count, const bm3d_stage_params *basic,
                                 const bm3d_stage_params *final_, float *const dst[],
                                 const float *const src[], const int width[], const int height[],
                                 const size_t stride[], int autotune, bm3d_batch **out)
{
    return batch_create_any(ctx, 1, count, basic, final_, dst, src, width, height, stride,
                            autotune, out);
}

extern "C" int bm3d_batch3_create(bm3d_ctx *ctx, int count, const bm3d_stage_params *basic,
                                  const bm3d_stage_params *final_, float *const dst[],
                                  const float *const src[], const int width[], const int height[],
                                  const size_t stride[], int autotune, bm3d_batch **out)
{
    return batch_create_any(ctx, 3, count, basic, final_, dst, src, width, height, stride,
                            autotune, out);
}

extern "C" int bm3d_batch_run(bm3d_batch *B, void *stream)
{
    if (!B || !B->exec) return BM3D_ERR_INVALID;
    CK(B->ctx, cudaSetDevice(B->ctx->device));
    CK(B->ctx, cudaGraphLaunch(B->exec, static_cast<cudaStream_t>(stream)));
    B->ctx->last_stream = static_cast<cudaStream_t>(stream);
    return BM3D_OK;
}

extern "C" int bm3d_batch_tuning(const bm3d_batch *B, int out[6])
{
    if (!B || !out) return BM3D_ERR_INVALID;
    out[0] = B->sb.tile_x;
    out[1] = B->sb.tile_y;
    out[2] = B->sb.warps;
    out[3] = B->sf.tile_x;
    out[4] = B->sf.tile_y;
    out[5] = B->sf.warps;
    return BM3D_OK;
}

extern "C" void bm3d_batch_destroy(bm3d_batch *B)
{
    if (!B) return;
    cudaSetDevice(B->ctx->device);
    if (B->cap) cudaStreamSynchronize(B->cap);
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->graph) cudaGraphDestroy(B->graph);
    if (B->cap) cudaStreamDestroy(B->cap);
    for (DevBuf *b : {&B->acc, &B->basic, &B->absmax, &B->counters, &B->planes_b, &B->planes_f,
                      &B->sb.args, &B->sb.base, &B->sf.args, &B->sf.base})
        if (b->ptr) cudaFree(b->ptr);
    delete B;
}

// ---------------------------------------------------------------------------
// Batches fed from host memory: two device slots, each with its own batch
// graph; uploads, filtering and downloads of consecutive runs overlap.

struct bm3d_host_batch {
    bm3d_ctx *ctx = nullptr;
    int n = 0;    // images
    int npl = 1;  // planes per image
    std::vector<bm3d_stage_params> pb, pf;
    std::vector<int> w, h;
    std::vector<size_t> off;  // element offset of each plane (npl per image) in a slot's buffers
    size_t total = 0;         // floats per slot buffer
    int autotune = 1;
    struct Slot {
        bm3d_batch *batch = nullptr;
        DevBuf src, dst;
        cudaEvent_t uploaded = nullptr, filtered = nullptr, drained = nullptr;
        bool used = false;
    } slot[2];
    cudaStream_t up = nullptr, down = nullptr;
    unsigned long long runs = 0;
};

extern "C" void bm3d_host_batch_destroy(bm3d_host_batch *H)
{
    if (!H) return;
    cudaSetDevice(H->ctx->device);
    if (H->up) cudaStreamSynchronize(H->up);
    if (H->down) cudaStreamSynchronize(H->down);
    for (auto &sl : H->slot) {
        if (sl.batch) bm3d_batch_destroy(sl.batch);
        if (sl.src.ptr) cudaFree(sl.src.ptr);
        if (sl.dst.ptr) cudaFree(sl.dst.ptr);
        for (cudaEvent_t e : {sl.uploaded, sl.filtered, sl.drained})
            if (e) cudaEventDestroy(e);
    }
    if (H->up) cudaStreamDestroy(H->up);
    if (H->down) cudaStreamDestroy(H->down);
    delete H;
}

static int host_batch_create_any(bm3d_ctx *ctx, int npl, int count,
                                 const bm3d_stage_params *basic, const bm3d_stage_params *final_,
                                 const int width[], const int height[], int autotune,
                                 bm3d_host_batch **out)
{
    if (!ctx || !out || count < 1 || !basic || !final_ || !width || !height)
        return BM3D_ERR_INVALID;
    *out = nullptr;
    CK(ctx, cudaSetDevice(ctx->device));
    auto *H = new bm3d_host_batch;
    H->ctx = ctx;
    H->n = count;
    H->npl = npl;
    H->autotune = autotune;
    auto fail = [&](int rc) {
        bm3d_host_batch_destroy(H);
        return rc;
    };
    for (int i = 0; i < count; ++i) {
        if (width[i] < 1 || height[i] < 1) return fail(BM3D_ERR_INVALID);
        H->pb.push_back(basic[i]);
        H->pf.push_back(final_[i]);
        H->w.push_back(width[i]);
        H->h.push_back(height[i]);
        for (int c = 0; c < npl; ++c) {
            H->off.push_back(H->total);
            H->total += static_cast<size_t>(width[i]) * height[i];
        }
    }
    int rc;
    for (auto &sl : H->slot) {
        if ((rc = ensure(ctx, sl.src, sizeof(float) * H->total)) != BM3D_OK) return fail(rc);
        if ((rc = ensure(ctx, sl.dst, sizeof(float) * H->total)) != BM3D_OK) return fail(rc);
        cudaError_t e;
        if ((e = cudaEventCreateWithFlags(&sl.uploaded, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&sl.filtered, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&sl.drained, cudaEventDisableTiming)) != cudaSuccess)
            return fail(cuda_fail(ctx, e, "cudaEventCreate"));
    }
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&H->up, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&H->down, cudaStreamNonBlocking)) != cudaSuccess)
        return fail(cuda_fail(ctx, e, "cudaStreamCreate"));
    *out = H;
    return BM3D_OK;
}

extern "C" int bm3d_host_batch_create(bm3d_ctx *ctx, int count, const bm3d_stage_params *basic,
                                      const bm3d_stage_params *final_, const int width[],
                                      const int height[], int autotune, bm3d_host_batch **out)
{
    return host_batch_create_any(ctx, 1, count, basic, final_, width, height, autotune, out);
}

extern "C" int bm3d_host_batch3_create(bm3d_ctx *ctx, int count, const bm3d_stage_params *basic,
                                       const bm3d_stage_params *final_, const int width[],
                                       const int height[], int autotune, bm3d_host_batch **out)
{
    return host_batch_create_any(ctx, 3, count, basic, final_, width, height, autotune, out);
}

// The slot's batch graph over its device buffers; built on the first run that
// uses the slot, so the autotuner times real data (slot 1 reuses slot 0's
// tiling).
static int host_batch_bind(bm3d_host_batch *H, int k)
{
    auto &sl = H->slot[k];
    if (sl.batch) return BM3D_OK;
    const size_t planes = H->off.size();
    std::vector<float *> d(planes);
    std::vector<const float *> x(planes);
    std::vector<size_t> st(H->n);
    for (size_t j = 0; j < planes; ++j) {
        d[j] = static_cast<float *>(sl.dst.ptr) + H->off[j];
        x[j] = static_cast<const float *>(sl.src.ptr) + H->off[j];
    }
    for (int i = 0; i < H->n; ++i) st[i] = static_cast<size_t>(H->w[i]);
    int tiling[6];
    const int *force = nullptr;
    if (k == 1 && H->slot[0].batch) {
        bm3d_batch_tuning(H->slot[0].batch, tiling);
        force = tiling;
    }
    return batch_create_any(H->ctx, H->npl, H->n, H->pb.data(), H->pf.data(), d.data(), x.data(),
                            H->w.data(), H->h.data(), st.data(), H->autotune, &sl.batch, force);
}

extern "C" int bm3d_host_batch_run(bm3d_host_batch *H, float *const dst[],
                                   const float *const src[], const size_t stride[], int async,
                                   void *stream)
{
    if (!H || !dst || !src || !stride) return BM3D_ERR_INVALID;
    const int np = H->npl;
    for (int i = 0; i < H->n; ++i) {
        if (stride[i] < static_cast<size_t>(H->w[i])) return BM3D_ERR_INVALID;
        for (int c = 0; c < np; ++c)
            if (!dst[np * i + c] || !src[np * i + c]) return BM3D_ERR_INVALID;
    }
    bm3d_ctx *ctx = H->ctx;
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int k = static_cast<int>(H->runs & 1);
    auto &sl = H->slot[k];
    // inputs: once this slot's previous run has been filtered
    if (sl.used) CK(ctx, cudaStreamWaitEvent(H->up, sl.filtered, 0));
    for (int j = 0; j < np * H->n; ++j) {
        const int i = j / np;
        CK(ctx, cudaMemcpy2DAsync(static_cast<float *>(sl.src.ptr) + H->off[j],
                                  sizeof(float) * H->w[i], src[j], sizeof(float) * stride[i],
                                  sizeof(float) * H->w[i], H->h[i], cudaMemcpyHostToDevice, H->up));
    }
    CK(ctx, cudaEventRecord(sl.uploaded, H->up));
    if (!sl.batch) {  // first use: build (and tune) the slot's graph on these inputs
        CK(ctx, cudaEventSynchronize(sl.uploaded));
        const int rc = host_batch_bind(H, k);
        if (rc != BM3D_OK) return rc;
    }
    CK(ctx, cudaStreamWaitEvent(s, sl.uploaded, 0));
    if (sl.used) CK(ctx, cudaStreamWaitEvent(s, sl.drained, 0));  // outputs copied out
    int rc = bm3d_batch_run(sl.batch, s);
    if (rc != BM3D_OK) return rc;
    CK(ctx, cudaEventRecord(sl.filtered, s));
    CK(ctx, cudaStreamWaitEvent(H->down, sl.filtered, 0));
    for (int j = 0; j < np * H->n; ++j) {
        const int i = j / np;
        CK(ctx, cudaMemcpy2DAsync(dst[j], sizeof(float) * stride[i],
                                  static_cast<const float *>(sl.dst.ptr) + H->off[j],
                                  sizeof(float) * H->w[i], sizeof(float) * H->w[i], H->h[i],
                                  cudaMemcpyDeviceToHost, H->down));
    }
    CK(ctx, cudaEventRecord(sl.drained, H->down));
    sl.used = true;
    ++H->runs;
    if (async == 2) return BM3D_OK;  // the caller joins later (bm3d_host_batch_join)
    CK(ctx, cudaStreamWaitEvent(s, sl.drained, 0));  // `stream` completes after the download
    if (async) return BM3D_OK;
    CK(ctx, cudaStreamSynchronize(s));
    return BM3D_OK;
}

extern "C" int bm3d_host_batch_join(bm3d_host_batch *H, void *stream)
{
    if (!H) return BM3D_ERR_INVALID;
    if (H->runs == 0) return BM3D_OK;
    CK(H->ctx, cudaSetDevice(H->ctx->device));
    // downloads run in order on one stream: the last one covers them all
    CK(H->ctx, cudaStreamWaitEvent(static_cast<cudaStream_t>(stream),
                                   H->slot[(H->runs - 1) & 1].drained, 0));
    return BM3D_OK;
}
