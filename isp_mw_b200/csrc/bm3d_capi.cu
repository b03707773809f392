// C ABI of the B200 BM3D path (declared in include/bm3d_b200.h): parameter
// mirroring, per-call constant setup, context scratch and kernel launches.
// The integer / Frame entry points are in bm3d_capi_convert.cu, the batches
// in bm3d_capi_batch.cu.
#include "bm3d_capi_internal.h"

#include <atomic>
#include <type_traits>

static thread_local std::string g_create_error;

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

int bm3d::cuda_fail(bm3d_ctx *ctx, cudaError_t e, const char *what)
{
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    if (ctx) ctx->err = buf;
    else g_create_error = buf;
    return e == cudaErrorMemoryAllocation ? BM3D_ERR_NOMEM : BM3D_ERR_CUDA;
}

// Allocations still to fail on purpose (bm3d_inject_alloc_failures).
static std::atomic<int> g_fail_allocs{0};

extern "C" int bm3d_inject_alloc_failures(int count)
{
    if (count < 0) return BM3D_ERR_INVALID;
    g_fail_allocs.store(count);
    return BM3D_OK;
}

int bm3d::ensure(bm3d_ctx *ctx, DevBuf &b, size_t bytes)
{
    if (b.bytes >= bytes) return BM3D_OK;
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
    for (int left = g_fail_allocs.load(); left > 0; left = g_fail_allocs.load())
        if (g_fail_allocs.compare_exchange_weak(left, left - 1))
            return cuda_fail(ctx, cudaErrorMemoryAllocation, "cudaMalloc (injected failure)");
    CK(ctx, cudaMalloc(&b.ptr, bytes));
    b.bytes = bytes;
    return BM3D_OK;
}

cudaError_t bm3d::raise_smem_limit(const void *kern, size_t bytes)
{
    static std::mutex mu;  // read-compare-set must not interleave across threads
    std::lock_guard<std::mutex> lock(mu);
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, kern);
    if (e != cudaSuccess) return e;
    if (fa.maxDynamicSharedSizeBytes >= 0 &&
        static_cast<size_t>(fa.maxDynamicSharedSizeBytes) >= bytes)
        return cudaSuccess;
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(bytes));
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
static float g_d11_f[11 * 11], g_d11_i[11 * 11];
static double g_tab_df[1496], g_tab_di[1496];
static std::once_flag g_tab_once;

static void init_dct_tables()
{
    make_dct_tables(g_tab_ff, g_tab_fi, g_tab_df, g_tab_di);
    const long double pi = 3.141592653589793238462643383279502884L;
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
        DctTableData{g_tab_ff, g_tab_fi, g_tab_df, g_tab_di, g_pad_f, g_pad_i, g_d11_f, g_d11_i});
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
    if (e == cudaSuccess) e = cudaMalloc(&ctx->nonfinite, kMaxPlanes * sizeof(unsigned));
    if (e != cudaSuccess) {
        cudaFree(ctx->stats);
        if (ctx->absmax) cudaFree(ctx->absmax);
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
            cudaFree(ctx->nonfinite);
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
    for (auto &b : ctx->poison) fr(b);
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
    if (ctx->nonfinite) cudaFree(ctx->nonfinite);
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

// The register-resident kernel covers BlockSize 8 with GroupSize <= 16 (the
// "fast" and "lc" profiles); everything else up to BlockSize 16 and GroupSize
// 32 runs on the generic kernel.
static bool fast_path(const bm3d_stage_params *p)
{
    return p->block_size == kBS && p->group_size <= kGSMax;
}

Guard bm3d::check_params(const bm3d_stage_params *p, int nplanes)
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
void bm3d::fill_tables(StageArgs<T> &a, const bm3d_stage_params *p, bool wiener, int nplanes,
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
    CK(ctx, raise_smem_limit(kern, sp.total));
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
                                     a.key_slots, warps, true, a.block_size, a.group_size,
                                     a.tile_x * a.tile_y);
    CK(ctx, raise_smem_limit(kern, sp.total));
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

bool bm3d::fast_args(int block_size, int group_size)
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
    // The generic kernel (launch bounds 384 in FP32, 256 in FP64) takes the
    // first of these (tile_x, tile_y, warps) that fits: reference blocks per
    // tile a multiple of the warps, so no warp idles in a tile's last round.
    static const int gen32[][3] = {{6, 4, 12}, {4, 3, 12}, {4, 4, 8}, {4, 4, 4},
                                   {2, 2, 4},  {2, 2, 2},  {1, 1, 2}, {1, 1, 1}};
    static const int gen64[][3] = {{4, 4, 8}, {4, 4, 4}, {2, 2, 4}, {2, 2, 2}, {1, 1, 2}, {1, 1, 1}};
    const int (*gcand)[3] = sizeof(T) == 4 ? gen32 : gen64;
    const int ngcand = sizeof(T) == 4 ? 8 : 6;
    int gi = 0;
    int tx = generic ? gcand[0][0] : ctx->tile_x, ty = generic ? gcand[0][1] : ctx->tile_y;
    warps = generic ? gcand[0][2] : ctx->warps;
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
        if (generic) {
            if (++gi >= ngcand) {
                ctx->err = "stage does not fit in shared memory";
                return BM3D_ERR_UNSUPPORTED;
            }
            tx = gcand[gi][0];
            ty = gcand[gi][1];
            warps = gcand[gi][2];
        } else if (warps > 8) {
            warps /= 2;
        } else if (ty > 1 && ty >= tx) {
            --ty;
        } else if (tx > 1) {
            --tx;
        } else if (warps > 1) {
            warps /= 2;
        } else {
            ctx->err = "stage does not fit in shared memory";
            return BM3D_ERR_UNSUPPORTED;
        }
    }
    a.tile_x = std::min(tx, a.nx);
    a.tile_y = std::min(ty, a.ny);
    a.tiles_x = (a.nx + a.tile_x - 1) / a.tile_x;
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
    fixed_point_bounds(p, width, height, a.log2_bound, a.log2_corner);
    a.absmax = ctx->absmax;
    // FP32 sums are fixed point: planes with NaN / Inf pixels take the checking
    // aggregation (FP64 sums are doubles and carry them like the reference's)
    constexpr bool kFixed = std::is_same<Acc, long long>::value;
    a.nonfinite = kFixed ? ctx->nonfinite : nullptr;
    if (!bm_only) {
        CK(ctx, cudaMemsetAsync(ctx->absmax, 0, kMaxPlanes * sizeof(float), s));
        CK(ctx, cudaMemsetAsync(ctx->nonfinite, 0, kMaxPlanes * sizeof(unsigned), s));
    }
    for (int c = 0; c < nplanes; ++c) {
        if (!(a.active & (1 << c)) && !bm_only) continue;
        if ((rc = ensure(ctx, ctx->acc[2 * c], acc_bytes)) != BM3D_OK) return rc;
        if ((rc = ensure(ctx, ctx->acc[2 * c + 1], acc_bytes)) != BM3D_OK) return rc;
        a.num[c] = static_cast<Acc *>(ctx->acc[2 * c].ptr);
        a.den[c] = static_cast<Acc *>(ctx->acc[2 * c + 1].ptr);
        if (kFixed) {  // starts zeroed; normalisation leaves it zero
            const bool grow = ctx->poison[c].bytes < static_cast<size_t>(npx);
            if ((rc = ensure(ctx, ctx->poison[c], static_cast<size_t>(npx))) != BM3D_OK) return rc;
            if (grow) CK(ctx, cudaMemsetAsync(ctx->poison[c].ptr, 0, ctx->poison[c].bytes, s));
            a.poison[c] = static_cast<unsigned char *>(ctx->poison[c].ptr);
        }
        if (!bm_only) {
            prep_kernel<T><<<std::min(height, blocks), threads, 0, s>>>(
                a.num[c], a.den[c], src[c], static_cast<long long>(stride), width, height,
                ctx->absmax + c, ref[c] != src[c] ? ref[c] : nullptr,
                kFixed ? ctx->nonfinite + c : nullptr);
            CK(ctx, cudaGetLastError());
        }
    }
    a.group_count = gcount;
    a.group_pos = gpos;
    a.group_key = gkey;
    a.bm_only = bm_only ? 1 : 0;
    a.stats = ctx->stats;
    a.bad = ctx->stats + 4;
    // per-stage counters; the invariant counter (stats[4]) is sticky
    CK(ctx, cudaMemsetAsync(ctx->stats, 0, 4 * sizeof(unsigned long long), s));
    if ((rc = launch_stage(ctx, a, wiener, nplanes, s, warps)) != BM3D_OK) return rc;
    ctx->last_stream = s;
    if (bm_only) return BM3D_OK;
    for (int c = 0; c < nplanes; ++c) {
        if (!(a.active & (1 << c))) continue;
        const dim3 ngrid = normalize_grid<T>(width, height);
        const int nsmem = std::is_same<T, float>::value ? strip_smem_bytes(a.block_size) : 0;
        normalize_kernel<T><<<ngrid, 256, nsmem, s>>>(dst[c], static_cast<long long>(stride), a.num[c],
                                                  a.den[c], width, height, a.block_size,
                                                  a.poison[c], a.nonfinite ? a.nonfinite + c : nullptr,
                                                  ctx->absmax + c, a.log2_bound, a.log2_corner);
        CK(ctx, cudaGetLastError());
    }
    return BM3D_OK;
}

// Host-mode calls end synchronised; a nonzero invariant counter means a group
// member fell outside its tile's staged window and was skipped.
int bm3d::check_invariants(bm3d_ctx *ctx)
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
int bm3d::stage_any(bm3d_ctx *ctx, const bm3d_stage_params *p, int wiener, int nplanes,
              T *const dst[], const T *const src[], const T *const ref[], int width, int height,
              size_t stride, double value_range, int mem, void *stream)
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
int bm3d::full_any(bm3d_ctx *ctx, const bm3d_stage_params *basic, const bm3d_stage_params *fin,
             int nplanes, T *const dst[], const T *const src[], const T *const ref[], int width,
             int height, size_t stride, double value_range, int mem, void *stream)
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


// The float drivers the other translation units call.
template void bm3d::fill_tables<float>(StageArgs<float> &, const bm3d_stage_params *, bool, int,
                                 double);
template int bm3d::stage_any<float>(bm3d_ctx *, const bm3d_stage_params *, int, int, float *const[],
                              const float *const[], const float *const[], int, int, size_t,
                              double, int, void *);
template int bm3d::full_any<float>(bm3d_ctx *, const bm3d_stage_params *, const bm3d_stage_params *,
                             int, float *const[], const float *const[], const float *const[],
                             int, int, size_t, double, int, void *);

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

extern "C" int bm3d_check(bm3d_ctx *ctx)
{
    if (!ctx) return BM3D_ERR_INVALID;
    CK(ctx, cudaSetDevice(ctx->device));
    CK(ctx, cudaStreamSynchronize(ctx->last_stream));
    return check_invariants(ctx);
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
// num (int64 per pixel) | den (int64 per pixel) | header: absmax (4 floats) at 0,
// non-finite pixel count at 128 | counters (8 x u64) | poison map (1 byte per pixel)
constexpr size_t kNoAllocBytes = 2 * kNoAllocAccBytes + 256 + 256 + kNoAllocMaxPixels;

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
// to the given code. The message (with the CUDA error text, if any) becomes
// this thread's context-free error, which bm3d_last_error(NULL) returns.
int noalloc_error(const char *what, cudaError_t e = cudaSuccess, int code = BM3D_ERR_INVALID)
{
    if (e != cudaSuccess) {
        char buf[256];
        std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
        g_create_error = buf;
        return BM3D_ERR_CUDA;
    }
    g_create_error = what;
    return code;
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
    int major = 0, sm = 0, optin = 0;
    cudaError_t e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (e != cudaSuccess) return noalloc_error("cudaDeviceGetAttribute", e);
    if (major < 10)
        return noalloc_error("bm3d_stage_noalloc: this build targets sm_100a (B200)",
                             cudaSuccess, BM3D_ERR_CUDA);
    void *ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return noalloc_error("cudaGetSymbolAddress(g_noalloc_scratch)", e);
    // the cosine tables live in fixed-size host arrays (no heap), uploaded per device
    if ((e = upload_dct_tables()) != cudaSuccess)
        return noalloc_error("cudaMemcpyToSymbol(cosine tables)", e);
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

// Offsets inside the scratch array after the two accumulator planes: the
// per-call |src| maximum (256 bytes, cleared by every call), then the counters:
// four statistics (cleared by every call) and the consistency counter, which
// starts at zero when the library loads and is cleared only by
// bm3d_noalloc_check, so it covers every call since the last check.
constexpr size_t kNoAllocAbsmaxOff = 2 * kNoAllocAccBytes;
constexpr size_t kNoAllocNonfiniteOff = kNoAllocAbsmaxOff + 128;
constexpr size_t kNoAllocStatsOff = kNoAllocAbsmaxOff + 256;
constexpr size_t kNoAllocPoisonOff = kNoAllocStatsOff + 256;
constexpr size_t kNoAllocClearBytes = 256 + 4 * sizeof(unsigned long long);

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
    if (g == Guard::Unsupported || !fast_path(params))
        return noalloc_error("bm3d_stage_noalloc: only BlockSize 8 with GroupSize <= 16",
                             cudaSuccess, BM3D_ERR_UNSUPPORTED);
    if (width < params->block_size || height < params->block_size ||
        stride < static_cast<size_t>(width))
        return noalloc_error("bm3d_stage_noalloc: width/height below BlockSize or stride < width");
    if (static_cast<size_t>(width) * static_cast<size_t>(height) > kNoAllocMaxPixels)
        return noalloc_error("bm3d_stage_noalloc: plane larger than the 2,097,152-pixel static "
                             "scratch", cudaSuccess, BM3D_ERR_TOO_LARGE);
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
    float *absmax = reinterpret_cast<float *>(d->scratch + kNoAllocAbsmaxOff);
    unsigned *nonfinite = reinterpret_cast<unsigned *>(d->scratch + kNoAllocNonfiniteOff);
    unsigned char *poison = d->scratch + kNoAllocPoisonOff;
    unsigned long long *stats = reinterpret_cast<unsigned long long *>(d->scratch + kNoAllocStatsOff);

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
    if (rc != BM3D_OK) return noalloc_error(info.err.c_str(), cudaSuccess, rc);
    fixed_point_bounds(params, width, height, a.log2_bound, a.log2_corner);
    a.absmax = absmax;
    a.nonfinite = nonfinite;
    a.poison[0] = poison;
    a.num[0] = num;
    a.den[0] = den;
    a.stats = stats;
    a.bad = stats + 4;

    const long long npx = static_cast<long long>(width) * height;
    const int threads = 256;
    const int blocks = static_cast<int>(
        std::min<long long>((npx + threads - 1) / threads, static_cast<long long>(d->sm_count) * 8));
    // |src| maximum and statistics start at zero; the consistency counter
    // (stats[4]) is left alone so bm3d_noalloc_check sees every call
    if ((e = cudaMemsetAsync(absmax, 0, kNoAllocClearBytes, s)) != cudaSuccess)
        return noalloc_error("cudaMemsetAsync(scratch header)", e);
    prep_kernel<float><<<std::min(height, blocks), threads, 0, s>>>(
        num, den, src, a.stride, width, height, absmax, ref != src ? ref : nullptr, nonfinite);
    if ((e = cudaGetLastError()) != cudaSuccess) return noalloc_error("prep_kernel", e);
    rc = launch_stage(&info, a, wiener != 0, 1, s, warps);
    if (rc != BM3D_OK) return noalloc_error(info.err.c_str(), cudaSuccess, rc);
    const dim3 ngrid = normalize_grid<float>(width, height);
    normalize_kernel<float><<<ngrid, 256, strip_smem_bytes(a.block_size), s>>>(
        dst, a.stride, num, den, width, height,
                                                  a.block_size, poison, nonfinite, absmax,
                                                  a.log2_bound, a.log2_corner);
    if ((e = cudaGetLastError()) != cudaSuccess) return noalloc_error("normalize_kernel", e);
    return BM3D_OK;
}

extern "C" int bm3d_noalloc_check(void *stream)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_error("cudaGetDevice", e);
    if (dev < 0 || dev >= kNoAllocMaxDevices) return noalloc_error("bm3d_noalloc_check: device id");
    NoAllocDevice *d = nullptr;
    int rc = noalloc_setup(dev, &d);
    if (rc != BM3D_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess)
        return noalloc_error("cudaStreamSynchronize", e);
    unsigned long long *bad =
        reinterpret_cast<unsigned long long *>(d->scratch + kNoAllocStatsOff) + 4;
    unsigned long long v = 0;
    if ((e = cudaMemcpy(&v, bad, sizeof(v), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return noalloc_error("cudaMemcpy(consistency counter)", e);
    if (v == 0) return BM3D_OK;
    if ((e = cudaMemset(bad, 0, sizeof(v))) != cudaSuccess)
        return noalloc_error("cudaMemset(consistency counter)", e);
    const std::string msg = "internal error: " + std::to_string(v & 0xffffffffull) +
                            " group blocks outside the staged window, " +
                            std::to_string(v >> 32) +
                            " tiles launched with too little shared memory";
    return noalloc_error(msg.c_str(), cudaSuccess, BM3D_ERR_CUDA);
}

