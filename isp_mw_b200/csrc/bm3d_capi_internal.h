// Internal interface shared by the C ABI's translation units (bm3d_capi.cu,
// bm3d_capi_convert.cu, bm3d_capi_batch.cu): the context, status helpers and
// the float stage drivers the integer / Frame and batch entry points build
// on. Not installed; the public interface is include/bm3d_b200.h.
#pragma once

#include "bm3d_b200.h"
#include "bm3d_batch.cuh"
#include "bm3d_kernels.h"

#include <algorithm>
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
    DevBuf poison[kMaxPlanes];        // per plane: pixels a non-finite term reached (1 B / pixel)
    unsigned long long *stats = nullptr;
    float *absmax = nullptr;          // per plane max finite |src| of the running stage
    unsigned *nonfinite = nullptr;    // per plane non-finite src / ref pixels of the running stage
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


constexpr int kStats = 5;

namespace bm3d {

// Status for a failed CUDA call: the message goes to the context (or, with no
// context, to the thread's creation error).
int cuda_fail(bm3d_ctx *ctx, cudaError_t e, const char *what);

#define CK(ctx, call)                                                                       \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call);                           \
    } while (0)

// Grow a context buffer to at least `bytes`.
int ensure(bm3d_ctx *ctx, DevBuf &b, size_t bytes);

// Raise a kernel's dynamic shared memory limit to at least `bytes`; never
// lower it. The limit belongs to the kernel function and is shared by every
// context, batch and captured graph in the process: a graph node captured at
// a larger size must stay launchable after a later call (another batch's
// autotuning, a smaller tile) asks for less. A profiler that re-launches a
// graph node on its own checks the node's size against the function's
// current limit.
cudaError_t raise_smem_limit(const void *kern, size_t bytes);

template <typename T>
inline int copy_plane(bm3d_ctx *ctx, T *dst, size_t dpitch, const T *src, size_t spitch, int w,
                      int h, cudaMemcpyKind kind, cudaStream_t s)
{
    CK(ctx, cudaMemcpy2DAsync(dst, dpitch * sizeof(T), src, spitch * sizeof(T), w * sizeof(T), h,
                              kind, s));
    return BM3D_OK;
}

// The reference's parameter guard (source/BM3D.cpp:82-87) and this build's
// limits.
enum class Guard { Run, Copy, Invalid, Unsupported };
Guard check_params(const bm3d_stage_params *p, int nplanes);

// BlockSize 8 with GroupSize <= 16 runs on the register-resident kernel.
bool fast_args(int block_size, int group_size);

// Per-call constant setup of one stage (thresholds, Wiener sigmas, finalAMP).
template <typename T>
void fill_tables(StageArgs<T> &a, const bm3d_stage_params *p, bool wiener, int nplanes,
                 double value_range);

// Fixed-point bounds of one stage on a width x height plane (fixed_scale):
// ceil(log2) of the most terms that reach one pixel outside block (0, 0) --
// group members lie within BMrange of their reference block, so only the
// reference positions within BlockSize + 2 BMrange of the pixel, per axis,
// reach it, GroupSize terms each -- and of those that reach block (0, 0)'s
// pixels and its weight origin, which every group may also hold twice (the
// reference's trailing (0, 0) candidate, include/Block.h:668-687).
inline void fixed_point_bounds(const bm3d_stage_params *p, int width, int height, int &log2_bound,
                               int &log2_corner)
{
    const int bs = p->block_size, step = std::max(1, p->block_step);
    const int range = p->bm_step > 0 ? p->bm_range / p->bm_step * p->bm_step : p->bm_range;
    const int per_axis = (bs + 2 * std::max(0, range) + step - 1) / step + 1;
    const double local = static_cast<double>(per_axis) * per_axis * std::max(1, p->group_size);
    const double refs = static_cast<double>(ref_count(width - bs, step)) * ref_count(height - bs, step);
    log2_bound = static_cast<int>(std::ceil(std::log2(std::max(2.0, local))));
    log2_corner = static_cast<int>(std::ceil(std::log2(std::max(2.0, 2.0 * refs + local))));
}

// Host-mode calls end synchronised; fails if the kernels' invariant counter
// is nonzero.
int check_invariants(bm3d_ctx *ctx);

// One stage / basic + final over planes of either memory kind.
template <typename T>
int stage_any(bm3d_ctx *ctx, const bm3d_stage_params *p, int wiener, int nplanes,
              T *const dst[], const T *const src[], const T *const ref[], int width, int height,
              size_t stride, double value_range, int mem, void *stream);
template <typename T>
int full_any(bm3d_ctx *ctx, const bm3d_stage_params *basic, const bm3d_stage_params *fin,
             int nplanes, T *const dst[], const T *const src[], const T *const ref[], int width,
             int height, size_t stride, double value_range, int mem, void *stream);

}  // namespace bm3d
