// C ABI of the learned pilot (declared in include/bm3d_b200.h): an 8-layer
// 48-channel 3 x 3 convolutional network whose output stands in for the BM3D
// basic estimate that the final (Wiener) stage takes as its reference. The
// reference has no such network; the final stage it feeds is
// BM3D_Final::CollaborativeFilter (source/BM3D.cpp:411-457), run here by
// bm3d_stage with the pilot's estimate as `ref`.
#include "bm3d_capi_internal.h"
#include "pilot_kernels.cuh"

#include <cudaTypedefs.h>

#include <atomic>
#include <cstdio>
#include <mutex>
#include <random>

using namespace pilot;

struct bm3d_pilot {
    bm3d_ctx *ctx = nullptr;
    long long step = 0;
    DevBuf params, grad, adam_m, adam_v;  // FP32, kParams each
    DevBuf wpack;  // BF16 packed: forward (6 layers) | data-gradient (6) | forward, N = 144 (6)
    DevBuf act[7];                        // X1..X7 (inference uses act[0], act[1])
    DevBuf gbuf[2];                       // pre-activation gradients, ping-pong
    DevBuf dout, out, partial, loss, err, sigma;
    // per-layer timing of forward passes (bm3d_pilot_set_timing): events
    // before layer 1, after each of the eight layers
    bool timing = false;
    cudaEvent_t ev[9] = {};
};

namespace {

constexpr int kPackElems = 9 * kC * kC;  // per layer

int pilot_fail(bm3d_ctx *ctx, int code, const char *msg)
{
    ctx->err = msg;
    return code;
}

int grid_for(const bm3d_ctx *ctx, int tiles) { return std::max(1, std::min(tiles, ctx->sm_count)); }

// Which 48 -> 48 convolution kernel runs: 0 = the N = 144 TMA pipeline for
// forward layers and the N = 48 one for data gradients, when their tensor
// maps encode (else the cp.async kernel); 1 = the cp.async kernel; 2 = the
// N = 48 TMA pipeline only; 3 = the N = 144 pipeline for forward layers
// (data gradients on the N = 48 one). g_conv_last records the kernel last
// launched (3, 2 or 1).
std::atomic<int> g_conv_choice{0};
std::atomic<int> g_conv_last{0};

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library); null when the driver does not provide it.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    });
    return fn;
}

// The TMA pipelines' two views of n images of h x w x 48 BF16 (NHWC): the
// input as (channel % 8, x, channel / 8, y, image), box {8, in_cols, 6,
// in_rows, 1}, and the output as (channel, x, y, image), box {48, out_cols,
// 4, 1}: {8, 10, 6, 18, 1} / {48, 8, 4, 1} for conv48_tma_kernel,
// {8, 8, 6, 18, 1} / {48, 6, 4, 1} for conv48_n144_kernel.
bool encode_conv_maps(const void *x, void *y, int n, int h, int w, CUtensorMap &in, CUtensorMap &out,
                      int in_cols = kT2X + 2, int out_cols = kT2X, int in_rows = kT2Y + 2)
{
    auto enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t px = 2ull * kC;  // bytes per pixel
    const cuuint64_t gdim[5] = {8, static_cast<cuuint64_t>(w), 6, static_cast<cuuint64_t>(h),
                                static_cast<cuuint64_t>(n)};
    const cuuint64_t gstride[4] = {px, 16, px * w, px * w * h};
    const cuuint32_t box[5] = {8, static_cast<cuuint32_t>(in_cols), 6,
                               static_cast<cuuint32_t>(in_rows), 1};
    const cuuint32_t ones[5] = {1, 1, 1, 1, 1};
    if (enc(&in, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void *>(x), gdim, gstride, box, ones,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    const cuuint64_t odim[4] = {static_cast<cuuint64_t>(kC), static_cast<cuuint64_t>(w),
                                static_cast<cuuint64_t>(h), static_cast<cuuint64_t>(n)};
    const cuuint64_t ostride[3] = {px, px * w, px * w * h};
    const cuuint32_t obox[4] = {kC, static_cast<cuuint32_t>(out_cols), 4, 1};
    return enc(&out, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, y, odim, ostride, obox, ones,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// One 48 -> 48 layer on the tensor cores.
int run_conv48(bm3d_ctx *ctx, const __nv_bfloat16 *x, __nv_bfloat16 *y, const __nv_bfloat16 *w,
               const __nv_bfloat16 *w3, const float *bias, const __nv_bfloat16 *aux, int mode, int n,
               int h, int wd, unsigned *err, cudaStream_t s)
{
    ConvArgs a;
    a.x = x;
    a.y = y;
    a.wt = reinterpret_cast<const uint4 *>(w);
    a.bias = bias;
    a.aux = aux;
    a.n = n;
    a.h = h;
    a.w = wd;
    a.mode = mode;
    a.err = err;
    const int choice = g_conv_choice.load();
    CUtensorMap tin, tout;
    if (w3 != nullptr && mode != kMaskPrev && (choice == 0 || choice == 3) &&
        encode_conv_maps(x, y, n, h, wd, tin, tout, kIn3X, kT3X, kT3Y + 2)) {
        a.wt = reinterpret_cast<const uint4 *>(w3);
        a.tiles_x = (wd + kT3X - 1) / kT3X;
        a.tiles_y = (h + kT3Y - 1) / kT3Y;
        a.tiles = n * a.tiles_x * a.tiles_y;
        // more than half an SM's shared memory keeps one CTA (and its 512
        // TMEM columns) per SM, so no CTA's allocation waits on another's
        const int smem3 = std::max(kT3Smem, 120 * 1024);
        CK(ctx, raise_smem_limit(reinterpret_cast<const void *>(conv48_n144_kernel), smem3));
        conv48_n144_kernel<<<std::max(1, std::min(a.tiles, ctx->sm_count)), kT3Threads, smem3,
                             s>>>(tin, tout, a);
        CK(ctx, cudaGetLastError());
        g_conv_last.store(3);
        return BM3D_OK;
    }
    if (choice == 3 && mode != kMaskPrev)
        return pilot_fail(ctx, BM3D_ERR_CUDA,
                          "pilot: the N = 144 convolution's tensor maps did not encode");
    if (choice != 1 && encode_conv_maps(x, y, n, h, wd, tin, tout)) {
        a.tiles_x = (wd + kT2X - 1) / kT2X;
        a.tiles_y = (h + kT2Y - 1) / kT2Y;
        a.tiles = n * a.tiles_x * a.tiles_y;
        CK(ctx, raise_smem_limit(reinterpret_cast<const void *>(conv48_tma_kernel), kTmaSmem));
        conv48_tma_kernel<<<std::max(1, std::min(a.tiles, ctx->sm_count)), kTmaThreads, kTmaSmem,
                            s>>>(tin, tout, a);
        CK(ctx, cudaGetLastError());
        g_conv_last.store(2);
        return BM3D_OK;
    }
    if (choice == 2 || choice == 3)
        return pilot_fail(ctx, BM3D_ERR_CUDA, "pilot: the convolution's tensor maps did not encode");
    a.tiles_x = (wd + kTX - 1) / kTX;
    a.tiles_y = (h + kTY - 1) / kTY;
    a.tiles = n * a.tiles_x * a.tiles_y;
    CK(ctx, raise_smem_limit(reinterpret_cast<const void *>(conv48_kernel), kConvSmem));
    conv48_kernel<<<std::max(1, std::min(a.tiles, kConvCtasPerSm * ctx->sm_count)), kConvThreads,
                    kConvSmem, s>>>(a);
    CK(ctx, cudaGetLastError());
    g_conv_last.store(1);
    return BM3D_OK;
}

int run_wgrad48(bm3d_ctx *ctx, const __nv_bfloat16 *x, const __nv_bfloat16 *g, float *partial,
                int n, int h, int wd, unsigned *err, cudaStream_t s, int &parts)
{
    WgradArgs a;
    a.x = x;
    a.g = g;
    a.partial = partial;
    a.n = n;
    a.h = h;
    a.w = wd;
    a.tiles_x = (wd + kTX - 1) / kTX;
    a.tiles_y = (h + kTY - 1) / kTY;
    a.tiles = n * a.tiles_x * a.tiles_y;
    a.err = err;
    parts = grid_for(ctx, a.tiles);
    // more than half the shared memory per CTA keeps one CTA (and its 512 TMEM columns) per SM
    const int smem = std::max(kWgSmem, 120 * 1024);
    CK(ctx, raise_smem_limit(reinterpret_cast<const void *>(wgrad48_kernel), smem));
    wgrad48_kernel<<<parts, kConvThreads, smem, s>>>(a);
    CK(ctx, cudaGetLastError());
    return BM3D_OK;
}

int check_err_flag(bm3d_ctx *ctx, unsigned *err, cudaStream_t s)
{
    unsigned v = 0;
    CK(ctx, cudaMemcpyAsync(&v, err, sizeof(v), cudaMemcpyDeviceToHost, s));
    CK(ctx, cudaStreamSynchronize(s));
    if (v) return pilot_fail(ctx, BM3D_ERR_CUDA, "pilot: a tensor-core wait gave up (timeout)");
    return BM3D_OK;
}

// The pilot's workspace for `pixels` pixels of images.
int ensure_workspace(bm3d_pilot *p, long long pixels, bool training)
{
    bm3d_ctx *ctx = p->ctx;
    int rc;
    const size_t act = static_cast<size_t>(pixels) * kC * sizeof(__nv_bfloat16);
    for (int i = 0; i < (training ? 7 : 2); ++i)
        if ((rc = ensure(ctx, p->act[i], act)) != BM3D_OK) return rc;
    if (training) {
        for (auto &g : p->gbuf)
            if ((rc = ensure(ctx, g, act)) != BM3D_OK) return rc;
        if ((rc = ensure(ctx, p->dout, static_cast<size_t>(pixels) * sizeof(float))) != BM3D_OK)
            return rc;
        const size_t part = static_cast<size_t>(std::max(ctx->sm_count, 1024)) *
                            std::max({kWgPartial, kW8Partial, kW1Partial}) * sizeof(float);
        if ((rc = ensure(ctx, p->partial, part)) != BM3D_OK) return rc;
        if ((rc = ensure(ctx, p->loss, sizeof(double))) != BM3D_OK) return rc;
    }
    if ((rc = ensure(ctx, p->err, sizeof(unsigned))) != BM3D_OK) return rc;
    return BM3D_OK;
}

const __nv_bfloat16 *wfwd(const bm3d_pilot *p, int layer)
{
    return static_cast<const __nv_bfloat16 *>(p->wpack.ptr) + (layer - 2) * kPackElems;
}
const __nv_bfloat16 *wbwd(const bm3d_pilot *p, int layer)
{
    return static_cast<const __nv_bfloat16 *>(p->wpack.ptr) + (6 + layer - 2) * kPackElems;
}
const __nv_bfloat16 *wfwd3(const bm3d_pilot *p, int layer)
{
    return static_cast<const __nv_bfloat16 *>(p->wpack.ptr) + (12 + layer - 2) * kPackElems;
}
const float *param(const bm3d_pilot *p, int offset)
{
    return static_cast<const float *>(p->params.ptr) + offset;
}

int pack(bm3d_pilot *p, cudaStream_t s)
{
    __nv_bfloat16 *w = static_cast<__nv_bfloat16 *>(p->wpack.ptr);
    pack_weights_kernel<<<216, 256, 0, s>>>(static_cast<const float *>(p->params.ptr), w,
                                            w + 6 * kPackElems, w + 12 * kPackElems);
    CK(p->ctx, cudaGetLastError());
    return BM3D_OK;
}

// Forward pass over n images; keeps X1..X7 when training (act[i] = X(i+1)),
// else ping-pongs act[0] / act[1]. Writes out (= noisy + residual), and with a
// target dOut and the loss.
int forward(bm3d_pilot *p, const float *in, long long stride, long long img_stride,
            const float *sigma_dev, int n, int h, int w, float *out, const float *target,
            cudaStream_t s)
{
    bm3d_ctx *ctx = p->ctx;
    const bool training = target != nullptr;
    auto X = [&](int layer) {  // output of layer (1..7)
        const int i = training ? layer - 1 : (layer - 1) & 1;
        return static_cast<__nv_bfloat16 *>(p->act[i].ptr);
    };
    unsigned *err = static_cast<unsigned *>(p->err.ptr);
    const long long pixels = static_cast<long long>(n) * h * w;
    const int blocks = static_cast<int>(std::min<long long>((pixels + 255) / 256, 8LL * ctx->sm_count));
    InArgs ia;
    ia.in = in;
    ia.stride = stride;
    ia.img_stride = img_stride;
    ia.sigma = sigma_dev;
    ia.wb = param(p, 0);
    ia.y = X(1);
    ia.n = n;
    ia.h = h;
    ia.w = w;
    if (p->timing) CK(ctx, cudaEventRecord(p->ev[0], s));
    conv_in_kernel<<<blocks, 256, 0, s>>>(ia);
    CK(ctx, cudaGetLastError());
    if (p->timing) CK(ctx, cudaEventRecord(p->ev[1], s));
    int rc;
    for (int layer = 2; layer <= 7; ++layer) {
        if ((rc = run_conv48(ctx, X(layer - 1), X(layer), wfwd(p, layer), wfwd3(p, layer),
                             param(p, off_b(layer)), nullptr, kBiasRelu, n, h, w, err, s)) != BM3D_OK)
            return rc;
        if (p->timing) CK(ctx, cudaEventRecord(p->ev[layer], s));
    }
    OutArgs oa;
    oa.x = X(7);
    oa.noisy = in;
    oa.stride = stride;
    oa.img_stride = img_stride;
    oa.wb = param(p, kOffW8);
    oa.out = out;
    oa.target = target;
    oa.dout = training ? static_cast<float *>(p->dout.ptr) : nullptr;
    oa.loss = training ? static_cast<double *>(p->loss.ptr) : nullptr;
    oa.sigma = sigma_dev;
    oa.inv_count = 1.0f / static_cast<float>(pixels);
    oa.n = n;
    oa.h = h;
    oa.w = w;
    conv_out_kernel<<<blocks, 256, 0, s>>>(oa);
    CK(ctx, cudaGetLastError());
    if (p->timing) CK(ctx, cudaEventRecord(p->ev[8], s));
    return BM3D_OK;
}

}  // namespace

extern "C" int bm3d_pilot_param_count(void) { return kParams; }

extern "C" int bm3d_pilot_set_conv_kernel(int which)
{
    if (which < 0 || which > 3) return BM3D_ERR_INVALID;
    g_conv_choice.store(which);
    return BM3D_OK;
}

extern "C" int bm3d_pilot_conv_kernel(void) { return g_conv_last.load(); }

extern "C" int bm3d_pilot_create(bm3d_ctx *ctx, unsigned long long seed, bm3d_pilot **out)
{
    if (!ctx || !out) return BM3D_ERR_INVALID;
    *out = nullptr;
    CK(ctx, cudaSetDevice(ctx->device));
    bm3d_pilot *p = new bm3d_pilot;
    p->ctx = ctx;
    int rc;
    for (DevBuf *b : {&p->params, &p->grad, &p->adam_m, &p->adam_v})
        if ((rc = ensure(ctx, *b, kParams * sizeof(float))) != BM3D_OK) {
            bm3d_pilot_destroy(p);
            return rc;
        }
    if ((rc = ensure(ctx, p->wpack, 18 * kPackElems * sizeof(__nv_bfloat16))) != BM3D_OK) {
        bm3d_pilot_destroy(p);
        return rc;
    }
    // He-normal initialisation (std sqrt(2 / fan_in)); the last layer 10x
    // smaller so the network starts close to the identity (residual 0).
    std::vector<float> h(kParams, 0.0f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.0f, 1.0f);
    for (int i = 0; i < kW1; ++i) h[i] = nd(rng) * std::sqrt(2.0f / (2 * 9));
    for (int l = 2; l <= 7; ++l)
        for (int i = 0; i < kWmid; ++i) h[off_w(l) + i] = nd(rng) * std::sqrt(2.0f / (kC * 9));
    for (int i = 0; i < kW8; ++i) h[kOffW8 + i] = 0.1f * nd(rng) * std::sqrt(2.0f / (kC * 9));
    rc = bm3d_pilot_set_params(p, h.data(), kParams);
    if (rc != BM3D_OK) {
        bm3d_pilot_destroy(p);
        return rc;
    }
    *out = p;
    return BM3D_OK;
}

extern "C" int bm3d_pilot_set_timing(bm3d_pilot *p, int on)
{
    if (!p) return BM3D_ERR_INVALID;
    CK(p->ctx, cudaSetDevice(p->ctx->device));
    if (on)
        for (cudaEvent_t &e : p->ev)
            if (!e) CK(p->ctx, cudaEventCreate(&e));
    p->timing = on != 0;
    return BM3D_OK;
}

extern "C" int bm3d_pilot_layer_ms(bm3d_pilot *p, float *ms)
{
    if (!p || !ms || !p->ev[8]) return BM3D_ERR_INVALID;
    CK(p->ctx, cudaSetDevice(p->ctx->device));
    CK(p->ctx, cudaEventSynchronize(p->ev[8]));
    for (int i = 0; i < 8; ++i) CK(p->ctx, cudaEventElapsedTime(&ms[i], p->ev[i], p->ev[i + 1]));
    return BM3D_OK;
}

extern "C" void bm3d_pilot_destroy(bm3d_pilot *p)
{
    if (!p) return;
    cudaSetDevice(p->ctx->device);
    std::vector<DevBuf *> bufs = {&p->params, &p->grad, &p->adam_m,  &p->adam_v,   &p->wpack,
                                  &p->dout,   &p->out,  &p->partial, &p->loss,     &p->err,
                                  &p->sigma,  &p->gbuf[0], &p->gbuf[1]};
    for (auto &b : p->act) bufs.push_back(&b);
    for (DevBuf *b : bufs)
        if (b->ptr) cudaFree(b->ptr);
    for (cudaEvent_t e : p->ev)
        if (e) cudaEventDestroy(e);
    delete p;
}

extern "C" int bm3d_pilot_set_params(bm3d_pilot *p, const float *host, int count)
{
    if (!p || !host || count != kParams) return BM3D_ERR_INVALID;
    bm3d_ctx *ctx = p->ctx;
    CK(ctx, cudaSetDevice(ctx->device));
    CK(ctx, cudaMemcpy(p->params.ptr, host, kParams * sizeof(float), cudaMemcpyHostToDevice));
    CK(ctx, cudaMemset(p->adam_m.ptr, 0, kParams * sizeof(float)));
    CK(ctx, cudaMemset(p->adam_v.ptr, 0, kParams * sizeof(float)));
    CK(ctx, cudaMemset(p->grad.ptr, 0, kParams * sizeof(float)));
    p->step = 0;
    int rc = pack(p, nullptr);
    if (rc != BM3D_OK) return rc;
    CK(ctx, cudaDeviceSynchronize());
    return BM3D_OK;
}

extern "C" int bm3d_pilot_get_params(bm3d_pilot *p, float *host, int count)
{
    if (!p || !host || count != kParams) return BM3D_ERR_INVALID;
    bm3d_ctx *ctx = p->ctx;
    CK(ctx, cudaSetDevice(ctx->device));
    CK(ctx, cudaDeviceSynchronize());
    CK(ctx, cudaMemcpy(host, p->params.ptr, kParams * sizeof(float), cudaMemcpyDeviceToHost));
    return BM3D_OK;
}

extern "C" int bm3d_pilot_get_grad(bm3d_pilot *p, float *host, int count)
{
    if (!p || !host || count != kParams) return BM3D_ERR_INVALID;
    bm3d_ctx *ctx = p->ctx;
    CK(ctx, cudaSetDevice(ctx->device));
    CK(ctx, cudaDeviceSynchronize());
    CK(ctx, cudaMemcpy(host, p->grad.ptr, kParams * sizeof(float), cudaMemcpyDeviceToHost));
    return BM3D_OK;
}

// Checkpoint: "BM3DPLT1", int32 parameter count, int64 step, then the FP32
// parameters and the two Adam moment vectors.
extern "C" int bm3d_pilot_save(bm3d_pilot *p, const char *path)
{
    if (!p || !path) return BM3D_ERR_INVALID;
    bm3d_ctx *ctx = p->ctx;
    std::vector<float> buf(3 * static_cast<size_t>(kParams));
    CK(ctx, cudaSetDevice(ctx->device));
    CK(ctx, cudaDeviceSynchronize());
    CK(ctx, cudaMemcpy(buf.data(), p->params.ptr, kParams * sizeof(float), cudaMemcpyDeviceToHost));
    CK(ctx, cudaMemcpy(buf.data() + kParams, p->adam_m.ptr, kParams * sizeof(float),
                       cudaMemcpyDeviceToHost));
    CK(ctx, cudaMemcpy(buf.data() + 2 * kParams, p->adam_v.ptr, kParams * sizeof(float),
                       cudaMemcpyDeviceToHost));
    FILE *f = std::fopen(path, "wb");
    if (!f) return pilot_fail(ctx, BM3D_ERR_INVALID, "bm3d_pilot_save: cannot open file");
    const int32_t count = kParams;
    const int64_t step = p->step;
    bool ok = std::fwrite("BM3DPLT1", 1, 8, f) == 8 && std::fwrite(&count, 4, 1, f) == 1 &&
              std::fwrite(&step, 8, 1, f) == 1 &&
              std::fwrite(buf.data(), sizeof(float), buf.size(), f) == buf.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? BM3D_OK : pilot_fail(ctx, BM3D_ERR_INVALID, "bm3d_pilot_save: write failed");
}

extern "C" int bm3d_pilot_load(bm3d_pilot *p, const char *path)
{
    if (!p || !path) return BM3D_ERR_INVALID;
    bm3d_ctx *ctx = p->ctx;
    FILE *f = std::fopen(path, "rb");
    if (!f) return pilot_fail(ctx, BM3D_ERR_INVALID, "bm3d_pilot_load: cannot open file");
    char magic[8];
    int32_t count = 0;
    int64_t step = 0;
    std::vector<float> buf(3 * static_cast<size_t>(kParams));
    const bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "BM3DPLT1", 8) == 0 &&
                    std::fread(&count, 4, 1, f) == 1 && count == kParams &&
                    std::fread(&step, 8, 1, f) == 1 &&
                    std::fread(buf.data(), sizeof(float), buf.size(), f) == buf.size();
    std::fclose(f);
    if (!ok) return pilot_fail(ctx, BM3D_ERR_INVALID, "bm3d_pilot_load: not a pilot checkpoint");
    int rc = bm3d_pilot_set_params(p, buf.data(), kParams);
    if (rc != BM3D_OK) return rc;
    CK(ctx, cudaMemcpy(p->adam_m.ptr, buf.data() + kParams, kParams * sizeof(float),
                       cudaMemcpyHostToDevice));
    CK(ctx, cudaMemcpy(p->adam_v.ptr, buf.data() + 2 * kParams, kParams * sizeof(float),
                       cudaMemcpyHostToDevice));
    p->step = step;
    return BM3D_OK;
}

extern "C" int bm3d_pilot_estimate(bm3d_pilot *p, float *dst, const float *src, int count,
                                   int width, int height, size_t stride, size_t img_stride,
                                   const float *sigma, int mem, void *stream)
{
    if (!p || !dst || !src || !sigma || count < 1 || width < 1 || height < 1 ||
        stride < static_cast<size_t>(width) ||
        (count > 1 && img_stride < stride * static_cast<size_t>(height)))
        return BM3D_ERR_INVALID;
    bm3d_ctx *ctx = p->ctx;
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long pixels = static_cast<long long>(count) * width * height;
    int rc = ensure_workspace(p, pixels, false);
    if (rc != BM3D_OK) return rc;
    if ((rc = ensure(ctx, p->sigma, count * sizeof(float))) != BM3D_OK) return rc;
    const size_t istride = count > 1 ? img_stride : stride * height;
    const float *in = src;
    float *out = dst;
    if (mem == BM3D_MEM_HOST) {
        const size_t bytes = istride * count * sizeof(float);
        if ((rc = ensure(ctx, ctx->stage_in[0], bytes)) != BM3D_OK) return rc;
        if ((rc = ensure(ctx, ctx->stage_out[0], bytes)) != BM3D_OK) return rc;
        CK(ctx, cudaMemcpyAsync(ctx->stage_in[0].ptr, src, bytes, cudaMemcpyHostToDevice, s));
        in = static_cast<const float *>(ctx->stage_in[0].ptr);
        out = static_cast<float *>(ctx->stage_out[0].ptr);
    }
    CK(ctx, cudaMemcpyAsync(p->sigma.ptr, sigma, count * sizeof(float),
                            mem == BM3D_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                            s));
    CK(ctx, cudaMemsetAsync(p->err.ptr, 0, sizeof(unsigned), s));
    if ((rc = forward(p, in, static_cast<long long>(stride), static_cast<long long>(istride),
                      static_cast<const float *>(p->sigma.ptr), count, height, width, out, nullptr,
                      s)) != BM3D_OK)
        return rc;
    if (mem == BM3D_MEM_HOST) {
        CK(ctx, cudaMemcpyAsync(dst, out, istride * count * sizeof(float), cudaMemcpyDeviceToHost, s));
        return check_err_flag(ctx, static_cast<unsigned *>(p->err.ptr), s);
    }
    return BM3D_OK;
}

extern "C" int bm3d_pilot_train_step(bm3d_pilot *p, int count, int height, int width,
                                     const float *noisy, const float *target, const float *sigma,
                                     float lr, double *loss, void *stream)
{
    if (!p || !noisy || !target || !sigma || count < 1 || height < 1 || width < 1 || !(lr > 0))
        return BM3D_ERR_INVALID;
    bm3d_ctx *ctx = p->ctx;
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long pixels = static_cast<long long>(count) * height * width;
    int rc = ensure_workspace(p, pixels, true);
    if (rc != BM3D_OK) return rc;
    if ((rc = ensure(ctx, p->out, static_cast<size_t>(pixels) * sizeof(float))) != BM3D_OK) return rc;
    unsigned *err = static_cast<unsigned *>(p->err.ptr);
    CK(ctx, cudaMemsetAsync(err, 0, sizeof(unsigned), s));
    CK(ctx, cudaMemsetAsync(p->loss.ptr, 0, sizeof(double), s));
    const long long plane = static_cast<long long>(height) * width;
    if ((rc = forward(p, noisy, width, plane, sigma, count, height, width,
                      static_cast<float *>(p->out.ptr), target, s)) != BM3D_OK)
        return rc;
    auto X = [&](int layer) { return static_cast<__nv_bfloat16 *>(p->act[layer - 1].ptr); };
    float *grad = static_cast<float *>(p->grad.ptr);
    float *part = static_cast<float *>(p->partial.ptr);
    const float *dout = static_cast<const float *>(p->dout.ptr);
    const int blocks = static_cast<int>(std::min<long long>((pixels + 255) / 256, 8LL * ctx->sm_count));
    const int rblocks = std::min(2 * ctx->sm_count, 1024);
    // layer 8: weight gradient, then the gradient into layer 7's pre-activation
    wgrad_out_kernel<<<rblocks, 256, 0, s>>>(X(7), dout, count, height, width, part);
    CK(ctx, cudaGetLastError());
    reduce_partials_kernel<<<4, 128, 0, s>>>(part, rblocks, kW8Partial, kW8Partial, grad + kOffW8);
    CK(ctx, cudaGetLastError());
    __nv_bfloat16 *G[2] = {static_cast<__nv_bfloat16 *>(p->gbuf[0].ptr),
                           static_cast<__nv_bfloat16 *>(p->gbuf[1].ptr)};
    OutBackArgs ob;
    ob.x7 = X(7);
    ob.dout = dout;
    ob.wb = param(p, kOffW8);
    ob.g = G[1];
    ob.n = count;
    ob.h = height;
    ob.w = width;
    out_backward_kernel<<<blocks, 256, 0, s>>>(ob);
    CK(ctx, cudaGetLastError());
    // layers 7 .. 2: weight gradient (tensor cores), data gradient (tensor cores)
    int cur = 1;
    for (int layer = 7; layer >= 2; --layer) {
        int parts = 0;
        if ((rc = run_wgrad48(ctx, X(layer - 1), G[cur], part, count, height, width, err, s,
                              parts)) != BM3D_OK)
            return rc;
        reduce_partials_kernel<<<(kWgPartial + 255) / 256, 256, 0, s>>>(
            part, parts, kWgPartial, kWgPartial, grad + off_w(layer));
        CK(ctx, cudaGetLastError());
        if ((rc = run_conv48(ctx, G[cur], G[cur ^ 1], wbwd(p, layer), nullptr, nullptr, X(layer - 1),
                             kMaskPrev, count, height, width, err, s)) != BM3D_OK)
            return rc;
        cur ^= 1;
    }
    // layer 1
    InArgs ia;
    ia.in = noisy;
    ia.stride = width;
    ia.img_stride = plane;
    ia.sigma = sigma;
    ia.wb = param(p, 0);
    ia.y = nullptr;
    ia.n = count;
    ia.h = height;
    ia.w = width;
    wgrad_in_kernel<<<rblocks, 240, 0, s>>>(ia, G[cur], part);
    CK(ctx, cudaGetLastError());
    reduce_partials_kernel<<<4, 256, 0, s>>>(part, rblocks, kW1Partial, kW1Partial, grad);
    CK(ctx, cudaGetLastError());
    // Adam (bias-corrected step size), then the packed BF16 copies
    p->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const double c1 = 1.0 - std::pow(b1, static_cast<double>(p->step));
    const double c2 = 1.0 - std::pow(b2, static_cast<double>(p->step));
    const float lr_t = static_cast<float>(lr * std::sqrt(c2) / c1);
    adam_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(
        static_cast<float *>(p->params.ptr), grad, static_cast<float *>(p->adam_m.ptr),
        static_cast<float *>(p->adam_v.ptr), kParams, lr_t, b1, b2, 1e-8f);
    CK(ctx, cudaGetLastError());
    if ((rc = pack(p, s)) != BM3D_OK) return rc;
    if (loss) {
        double l = 0.0;
        CK(ctx, cudaMemcpyAsync(&l, p->loss.ptr, sizeof(double), cudaMemcpyDeviceToHost, s));
        if ((rc = check_err_flag(ctx, err, s)) != BM3D_OK) return rc;
        *loss = l / static_cast<double>(pixels);
    }
    return BM3D_OK;
}

extern "C" int bm3d_pilot_full(bm3d_ctx *ctx, bm3d_pilot *p, const bm3d_stage_params *final_,
                               float *dst, const float *src, int width, int height, size_t stride,
                               float value_range, int mem, void *stream)
{
    if (!ctx || !p || !final_ || !dst || !src) return BM3D_ERR_INVALID;
    if (p->ctx != ctx) return pilot_fail(ctx, BM3D_ERR_INVALID, "bm3d_pilot_full: pilot of another context");
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc;
    // the noise-level input: the true noise std (0-1 scale) of plane 0, i.e. the
    // parameter sigma with the reference's OPP luma scaling (include/BM3D.h:246-253) applied
    const float sig = static_cast<float>(final_->sigma[0] / std::sqrt(3.0) / 255.0);
    const float *in = src;
    float *out = dst;
    const size_t bytes = stride * height * sizeof(float);
    if (mem == BM3D_MEM_HOST) {
        if ((rc = ensure(ctx, ctx->stage_in[0], bytes)) != BM3D_OK) return rc;
        if ((rc = ensure(ctx, ctx->stage_out[0], bytes)) != BM3D_OK) return rc;
        CK(ctx, cudaMemcpyAsync(ctx->stage_in[0].ptr, src, bytes, cudaMemcpyHostToDevice, s));
        in = static_cast<const float *>(ctx->stage_in[0].ptr);
        out = static_cast<float *>(ctx->stage_out[0].ptr);
    }
    if ((rc = ensure(ctx, ctx->basic[0], bytes)) != BM3D_OK) return rc;
    if ((rc = ensure(ctx, p->sigma, sizeof(float))) != BM3D_OK) return rc;
    CK(ctx, cudaMemcpyAsync(p->sigma.ptr, &sig, sizeof(float), cudaMemcpyHostToDevice, s));
    if ((rc = ensure_workspace(p, static_cast<long long>(width) * height, false)) != BM3D_OK) return rc;
    CK(ctx, cudaMemsetAsync(p->err.ptr, 0, sizeof(unsigned), s));
    float *pilot_est = static_cast<float *>(ctx->basic[0].ptr);
    if ((rc = forward(p, in, static_cast<long long>(stride), static_cast<long long>(stride) * height,
                      static_cast<const float *>(p->sigma.ptr), 1, height, width, pilot_est,
                      nullptr, s)) != BM3D_OK)
        return rc;
    rc = bm3d_stage(ctx, final_, 1, out, in, pilot_est, width, height, stride, value_range,
                    BM3D_MEM_DEVICE, s);
    if (rc < 0) return rc;
    if (mem == BM3D_MEM_HOST) {
        CK(ctx, cudaMemcpyAsync(dst, out, bytes, cudaMemcpyDeviceToHost, s));
        int rc2 = check_err_flag(ctx, static_cast<unsigned *>(p->err.ptr), s);
        if (rc2 != BM3D_OK) return rc2;
        return check_invariants(ctx);
    }
    return rc;
}

// ---- layer-level entry points (device memory), for tests and tools ----------

extern "C" int bm3d_pilot_conv48(bm3d_ctx *ctx, int n, int h, int w, const void *x,
                                 const float *weight, const float *bias, const void *aux, int mode,
                                 void *y, void *stream)
{
    if (!ctx || !x || !weight || !y || n < 1 || h < 1 || w < 1 || mode < 0 || mode > 2 ||
        (mode == kMaskPrev && !aux) || (mode != kMaskPrev && !bias))
        return BM3D_ERR_INVALID;
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // weight: FP32 [48][48][3][3] (device); packed here into the operand layout
    DevBuf &wp = ctx->groups[0], &pp = ctx->groups[1], &eb = ctx->groups[2];
    int rc;
    if ((rc = ensure(ctx, wp, 18 * kPackElems * sizeof(__nv_bfloat16))) != BM3D_OK) return rc;
    if ((rc = ensure(ctx, pp, kParams * sizeof(float))) != BM3D_OK) return rc;
    if ((rc = ensure(ctx, eb, sizeof(unsigned))) != BM3D_OK) return rc;
    float *params = static_cast<float *>(pp.ptr);
    CK(ctx, cudaMemsetAsync(params, 0, kParams * sizeof(float), s));
    CK(ctx, cudaMemcpyAsync(params + off_w(2), weight, kWmid * sizeof(float),
                            cudaMemcpyDeviceToDevice, s));
    __nv_bfloat16 *packed = static_cast<__nv_bfloat16 *>(wp.ptr);
    pack_weights_kernel<<<216, 256, 0, s>>>(params, packed, packed + 6 * kPackElems,
                                            packed + 12 * kPackElems);
    CK(ctx, cudaGetLastError());
    unsigned *err = static_cast<unsigned *>(eb.ptr);
    CK(ctx, cudaMemsetAsync(err, 0, sizeof(unsigned), s));
    if ((rc = run_conv48(ctx, static_cast<const __nv_bfloat16 *>(x), static_cast<__nv_bfloat16 *>(y),
                         mode == kMaskPrev ? packed + 6 * kPackElems : packed,
                         mode == kMaskPrev ? nullptr : packed + 12 * kPackElems, bias,
                         static_cast<const __nv_bfloat16 *>(aux), mode, n, h, w, err, s)) != BM3D_OK)
        return rc;
    return check_err_flag(ctx, err, s);
}

extern "C" int bm3d_pilot_wgrad48(bm3d_ctx *ctx, int n, int h, int w, const void *x, const void *g,
                                  float *dw, float *db, void *stream)
{
    if (!ctx || !x || !g || !dw || !db || n < 1 || h < 1 || w < 1) return BM3D_ERR_INVALID;
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DevBuf &part = ctx->groups[0], &eb = ctx->groups[2];
    int rc;
    if ((rc = ensure(ctx, part, static_cast<size_t>(ctx->sm_count) * kWgPartial * sizeof(float))) !=
        BM3D_OK)
        return rc;
    if ((rc = ensure(ctx, eb, sizeof(unsigned))) != BM3D_OK) return rc;
    unsigned *err = static_cast<unsigned *>(eb.ptr);
    CK(ctx, cudaMemsetAsync(err, 0, sizeof(unsigned), s));
    int parts = 0;
    float *pt = static_cast<float *>(part.ptr);
    if ((rc = run_wgrad48(ctx, static_cast<const __nv_bfloat16 *>(x),
                          static_cast<const __nv_bfloat16 *>(g), pt, n, h, w, err, s, parts)) !=
        BM3D_OK)
        return rc;
    reduce_partials_kernel<<<(kWmid + 255) / 256, 256, 0, s>>>(pt, parts, kWmid, kWgPartial, dw);
    CK(ctx, cudaGetLastError());
    // the bias gradient follows dW in each partial
    reduce_partials_kernel<<<1, 64, 0, s>>>(pt + kWmid, parts, kC, kWgPartial, db);
    CK(ctx, cudaGetLastError());
    return check_err_flag(ctx, err, s);
}
