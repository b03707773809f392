// C ABI, many planes per call (declared in include/bm3d_b200.h): pipelined
// host planes (bm3d_full_many), device batches replayed from CUDA graphs
// (bm3d_batch_*), and host batches over two device slots (bm3d_host_batch_*).
#include "bm3d_capi_internal.h"

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
    DevBuf nonfinite, poison;  // per plane: non-finite input pixels; pixels they reached
    std::vector<size_t> poison_off;  // per plane: offset into poison (bytes)
    // final-stage-only batches: the caller's reference planes (e.g. the learned
    // pilot's estimates) stand in for the basic estimates; empty otherwise
    std::vector<const float *> ext_ref;
    DevBuf bad;  // the kernels' consistency counter (bm3d_batch_check)
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
        if (!wiener && !B->ext_ref.empty()) continue;  // no basic stage: references supplied
        StageArgs<float> a;
        std::memset(&a, 0, sizeof(a));
        a.bad = static_cast<unsigned long long *>(B->bad.ptr);
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
            a.ref[c] = !wiener ? B->src[k]
                       : !B->ext_ref.empty()
                           ? B->ext_ref[k]
                           : static_cast<const float *>(B->basic.ptr) + B->basic_off[k];
            a.num[c] = static_cast<long long *>(B->acc.ptr) + B->acc_off[k];
            a.den[c] = a.num[c] + static_cast<size_t>(a.width) * a.height;
        }
        a.absmax = static_cast<float *>(B->absmax.ptr) + i * npl;
        a.nonfinite = static_cast<const unsigned *>(B->nonfinite.ptr) + i * npl;
        for (int c = 0; c < npl; ++c)
            a.poison[c] = static_cast<unsigned char *>(B->poison.ptr) + B->poison_off[i * npl + c];
        fixed_point_bounds(p, a.width, a.height, a.log2_bound, a.log2_corner);
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
        CK(ctx, raise_smem_limit(kern, sbd.smem));
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
    int bsmax = 1;  // the strip ring holds the largest block size of the batch
    for (int i = 0; i < B->n; ++i)
        bsmax = std::max(bsmax, (&planes == &B->planes_b ? B->pb[i] : B->pf[i]).block_size);
    if (prep) prep_batch_kernel<float><<<grid, 256, 0, s>>>(q);
    else normalize_batch_kernel<float><<<grid, 256, strip_smem_bytes(bsmax), s>>>(q);
    CK(B->ctx, cudaGetLastError());
    return BM3D_OK;
}

// The whole pipeline, enqueued on s (captured into the graph). With `ev`,
// events ev[0] / ev[1] bracket the basic stage's persistent launch and ev[2] /
// ev[3] the final stage's (an eager run for timing; not used in the graph).
int enqueue_batch(bm3d_batch *B, cudaStream_t s, cudaEvent_t *ev = nullptr)
{
    bm3d_ctx *ctx = B->ctx;
    int rc;
    int *counters = static_cast<int *>(B->counters.ptr);
    for (int i = 0; i < B->n; ++i) {  // planes a stage passes through unfiltered
        for (int c = 0; c < B->npl; ++c) {
            const int k = i * B->npl + c;
            float *bi = static_cast<float *>(B->basic.ptr) + B->basic_off[k];
            const bool b_off = B->ext_ref.empty() &&
                               (B->gb[i] != Guard::Run || !(B->pb[i].sigma[c] > 0 || B->npl == 1));
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
    CK(ctx, cudaMemsetAsync(B->nonfinite.ptr, 0, sizeof(unsigned) * B->n * B->npl, s));
    if ((rc = launch_planes(B, B->planes_b, true, s)) != BM3D_OK) return rc;
    if (ev) CK(ctx, cudaEventRecord(ev[0], s));
    if ((rc = launch_batch_stage<false>(B, B->sb, counters, s)) != BM3D_OK) return rc;
    if (ev) CK(ctx, cudaEventRecord(ev[1], s));
    if ((rc = launch_planes(B, B->planes_b, false, s)) != BM3D_OK) return rc;
    if ((rc = launch_planes(B, B->planes_f, true, s)) != BM3D_OK) return rc;
    if (ev) CK(ctx, cudaEventRecord(ev[2], s));
    if ((rc = launch_batch_stage<true>(B, B->sf, counters + 1, s)) != BM3D_OK) return rc;
    if (ev) CK(ctx, cudaEventRecord(ev[3], s));
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
    // reference blocks per tile a multiple of the warps where it can be, so
    // the tile's last round keeps every warp busy
    static const int fast_cand[][3] = {{8, 8, 16}, {7, 7, 16}, {6, 8, 16}, {8, 6, 16},
                                       {8, 4, 16}, {6, 8, 12}, {8, 6, 12}, {6, 6, 12},
                                       {4, 4, 4},  {4, 4, 2},  {2, 2, 1}};
    static const int gen_cand[][3] = {{6, 4, 12}, {4, 3, 12}, {4, 4, 8}, {4, 4, 4},
                                      {2, 2, 4},  {2, 2, 2},  {1, 1, 2}, {1, 1, 1}};
    const int (*cand)[3] = generic ? gen_cand : fast_cand;
    const int ncand = generic ? 8 : 11;
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
                            const int *force_tiling = nullptr,
                            const float *const ext_ref[] = nullptr)
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
            if (ext_ref && !ext_ref[k]) return fail(batch_fail(ctx, "bad reference plane"));
            B->src.push_back(src[k]);
            B->dst.push_back(dst[k]);
            if (ext_ref) B->ext_ref.push_back(ext_ref[k]);
            B->acc_off.push_back(acc_total);
            B->basic_off.push_back(basic_total);
            B->poison_off.push_back(acc_total / 2);
            acc_total += 2 * static_cast<size_t>(width[i]) * height[i];
            if (!ext_ref) basic_total += stride[i] * height[i];
        }
    }
    int rc;
    if ((rc = ensure(ctx, B->acc, sizeof(long long) * acc_total)) != BM3D_OK) return fail(rc);
    if ((rc = ensure(ctx, B->basic, sizeof(float) * basic_total)) != BM3D_OK) return fail(rc);
    if ((rc = ensure(ctx, B->absmax, sizeof(float) * count * npl)) != BM3D_OK) return fail(rc);
    if ((rc = ensure(ctx, B->nonfinite, sizeof(unsigned) * count * npl)) != BM3D_OK) return fail(rc);
    if ((rc = ensure(ctx, B->poison, acc_total / 2)) != BM3D_OK) return fail(rc);
    // all zero between stages: the normalisation clears what it reads
    CK(ctx, cudaMemset(B->poison.ptr, 0, acc_total / 2));
    if ((rc = ensure(ctx, B->counters, 2 * sizeof(int))) != BM3D_OK) return fail(rc);
    if ((rc = ensure(ctx, B->bad, sizeof(unsigned long long))) != BM3D_OK) return fail(rc);
    CK(ctx, cudaMemset(B->bad.ptr, 0, sizeof(unsigned long long)));
    // per-pixel kernels' plane tables, active planes of each stage in batch order
    for (int st = 0; st < 2; ++st) {
        std::vector<BatchPlane<float>> q;
        for (int i = 0; i < count; ++i) {
            if ((st ? B->gf[i] : B->gb[i]) != Guard::Run) continue;
            if (!st && ext_ref) continue;  // no basic stage
            const bm3d_stage_params &pp = st ? final_[i] : basic[i];
            for (int c = 0; c < npl; ++c) {
                if (npl > 1 && !(pp.sigma[c] > 0)) continue;  // plane left alone by the stage
                const int k = i * npl + c;
                BatchPlane<float> bp;
                bp.num = static_cast<long long *>(B->acc.ptr) + B->acc_off[k];
                bp.den = bp.num + static_cast<size_t>(width[i]) * height[i];
                bp.src = src[k];
                // the final stage's Wiener weights come from the basic estimate
                bp.ref = !st ? nullptr
                         : ext_ref ? ext_ref[k]
                                   : static_cast<const float *>(B->basic.ptr) + B->basic_off[k];
                bp.dst = st ? dst[k] : static_cast<float *>(B->basic.ptr) + B->basic_off[k];
                bp.src_stride = static_cast<long long>(stride[i]);
                bp.dst_stride = static_cast<long long>(stride[i]);
                bp.width = width[i];
                bp.height = height[i];
                bp.block_size = pp.block_size;
                bp.absmax = static_cast<float *>(B->absmax.ptr) + k;
                fixed_point_bounds(&pp, width[i], height[i], bp.log2_bound, bp.log2_corner);
                bp.nonfinite = static_cast<unsigned *>(B->nonfinite.ptr) + k;
                bp.poison = static_cast<unsigned char *>(B->poison.ptr) + B->poison_off[k];
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
            if (ext_ref || (B->gb[i] == Guard::Run && (npl == 1 || basic[i].sigma[c] > 0)))
                continue;
            const int k = i * npl + c;
            float *bi = static_cast<float *>(B->basic.ptr) + B->basic_off[k];
            e = cudaMemcpy2DAsync(bi, stride[i] * 4, src[k], stride[i] * 4, width[i] * 4, height[i],
                                  cudaMemcpyDeviceToDevice, B->cap);
            if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "cudaMemcpy2DAsync"));
        }
    e = cudaMemsetAsync(B->absmax.ptr, 0, sizeof(float) * count * npl, B->cap);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(B->nonfinite.ptr, 0, sizeof(unsigned) * count * npl, B->cap);
    if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "cudaMemsetAsync"));
    if (!ext_ref && (rc = tune_stage<false>(B, B->sb, B->planes_b, autotune != 0, B->cap,
                                            force_tiling)) != BM3D_OK)
        return fail(rc);
    if ((rc = tune_stage<true>(B, B->sf, B->planes_f, autotune != 0, B->cap,
                               force_tiling ? force_tiling + 3 : nullptr)) != BM3D_OK)
        return fail(rc);
    // tuning runs stages without their normalisation, which is what clears
    // the poison marks; a mark left behind would poison the first real run
    e = cudaMemsetAsync(B->poison.ptr, 0, acc_total / 2, B->cap);
    if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "cudaMemsetAsync"));
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

extern "C" int bm3d_batch_final_create(bm3d_ctx *ctx, int count, const bm3d_stage_params *final_,
                                       float *const dst[], const float *const src[],
                                       const float *const ref[], const int width[],
                                       const int height[], const size_t stride[], int autotune,
                                       bm3d_batch **out)
{
    if (!ref) return BM3D_ERR_INVALID;
    return batch_create_any(ctx, 1, count, final_, final_, dst, src, width, height, stride,
                            autotune, out, nullptr, ref);
}

extern "C" int bm3d_batch3_final_create(bm3d_ctx *ctx, int count, const bm3d_stage_params *final_,
                                        float *const dst[], const float *const src[],
                                        const float *const ref[], const int width[],
                                        const int height[], const size_t stride[], int autotune,
                                        bm3d_batch **out)
{
    if (!ref) return BM3D_ERR_INVALID;
    return batch_create_any(ctx, 3, count, final_, final_, dst, src, width, height, stride,
                            autotune, out, nullptr, ref);
}

extern "C" int bm3d_batch_stage_times(bm3d_batch *B, void *stream, float ms[2])
{
    if (!B || !ms) return BM3D_ERR_INVALID;
    bm3d_ctx *ctx = B->ctx;
    CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    int rc = BM3D_OK;
    for (auto &e : ev)
        if (rc == BM3D_OK && cudaEventCreate(&e) != cudaSuccess) rc = BM3D_ERR_CUDA;
    if (rc == BM3D_OK) rc = enqueue_batch(B, s, ev);
    if (rc == BM3D_OK && cudaEventSynchronize(ev[3]) != cudaSuccess) rc = BM3D_ERR_CUDA;
    if (rc == BM3D_OK && (cudaEventElapsedTime(&ms[0], ev[0], ev[1]) != cudaSuccess ||
                          cudaEventElapsedTime(&ms[1], ev[2], ev[3]) != cudaSuccess))
        rc = BM3D_ERR_CUDA;
    for (auto &e : ev)
        if (e) cudaEventDestroy(e);
    if (rc == BM3D_ERR_CUDA && ctx->err.empty()) ctx->err = "bm3d_batch_stage_times: event failure";
    return rc;
}

extern "C" int bm3d_batch_run(bm3d_batch *B, void *stream)
{
    if (!B || !B->exec) return BM3D_ERR_INVALID;
    CK(B->ctx, cudaSetDevice(B->ctx->device));
    CK(B->ctx, cudaGraphLaunch(B->exec, static_cast<cudaStream_t>(stream)));
    B->ctx->last_stream = static_cast<cudaStream_t>(stream);
    return BM3D_OK;
}

extern "C" int bm3d_batch_check(bm3d_batch *B, void *stream)
{
    if (!B) return BM3D_ERR_INVALID;
    bm3d_ctx *ctx = B->ctx;
    CK(ctx, cudaSetDevice(ctx->device));
    CK(ctx, cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    unsigned long long v = 0;
    CK(ctx, cudaMemcpy(&v, B->bad.ptr, sizeof(v), cudaMemcpyDeviceToHost));
    if (v != 0) {
        ctx->err = "internal error: " + std::to_string(v & 0xffffffffull) +
                   " group blocks outside the staged window, " + std::to_string(v >> 32) +
                   " tiles launched with too little shared memory";
        return BM3D_ERR_CUDA;
    }
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
    for (DevBuf *b : {&B->acc, &B->basic, &B->absmax, &B->nonfinite, &B->poison, &B->counters,
                      &B->bad, &B->planes_b, &B->planes_f,
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

