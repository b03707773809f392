/* bm3d_b200: B200-native BM3D (basic hard-threshold estimate and final Wiener
 * estimate) behind a plain C ABI.
 *
 * This is the drop-in boundary for the BM3D path of mawen1250/ISP_MW. Each
 * entry point below names the reference interface it replaces. The C++
 * classes in bm3d_b200/BM3D.hpp (BM3D_Para, BM3D_Basic, BM3D_Final, BM3D)
 * mirror the reference's filter classes on top of these functions.
 *
 * Conventions
 *   - Planes are row-major float32 (or float64 for the *_f64 entry points)
 *     with a row pitch `stride` in elements (stride >= width).
 *   - `mem` says whether the plane pointers are host or device memory. With
 *     BM3D_MEM_HOST the call copies in, filters and copies out before it
 *     returns. With BM3D_MEM_DEVICE it only enqueues work on `stream`
 *     (a cudaStream_t, NULL = the legacy default stream) and returns.
 *   - The caller owns every plane. The context owns its device scratch
 *     (accumulators, staging, tables) and grows it on demand.
 *   - A context belongs to one host thread at a time.
 *   - No CPU fallback: without a usable sm_100 device every call fails with
 *     BM3D_ERR_CUDA.
 */
#ifndef BM3D_B200_H_
#define BM3D_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
enum {
    BM3D_OK = 0,
    /* The reference's parameter guard fired (sigma <= 0, GroupSize == 0,
     * BlockSize <= 0, BMrange <= 0, BMrange < BMstep or thMSE <= 0), so src was
     * copied to dst unchanged, as source/BM3D.cpp:82-87 and 143-151 do. */
    BM3D_COPIED = 1,
    BM3D_ERR_INVALID = -1,     /* null pointer, width/height < BlockSize, stride < width, ... */
    BM3D_ERR_UNSUPPORTED = -2, /* valid in the reference but not built here: BlockSize > 16 or
                                  GroupSize > 32 */
    BM3D_ERR_CUDA = -3,        /* CUDA runtime error (message via bm3d_last_error) */
    BM3D_ERR_NOMEM = -4,       /* device allocation failed */
    BM3D_ERR_TOO_LARGE = -5    /* plane exceeds bm3d_stage_noalloc's static scratch */
};

enum { BM3D_MEM_HOST = 0, BM3D_MEM_DEVICE = 1 };

/* Numeric fields of one stage's parameters.
 * Replaces BM3D_Para_Base / BM3D_Basic_Para / BM3D_Final_Para
 * (reference include/BM3D.h:15-151). `sigma` is on the 0-255 scale, one
 * value per plane; thMSE and sigma are the unscaled user values: the OPP
 * normalisation of include/BM3D.h:241-258 is applied inside. */
typedef struct bm3d_stage_params {
    int block_size;  /* BlockSize */
    int block_step;  /* BlockStep */
    int group_size;  /* GroupSize */
    int bm_range;    /* BMrange */
    int bm_step;     /* BMstep */
    double thMSE;    /* thMSE */
    double lambda;   /* lambda (hard-threshold multiplier; unused by the final stage) */
    double sigma[3]; /* sigma per plane, 0-255 scale */
} bm3d_stage_params;

/* Profile defaults of one stage ("fast", "lc", "np", "high", "vn"), with
 * `sigma` applied and thMSE recomputed from sigma[0] as thMSE_Default() does.
 * Replaces the BM3D_Basic_Para(profile) / BM3D_Final_Para(profile) constructors
 * and thMSE_Default() (reference include/BM3D.h:54-97, 107-150). The reference
 * never initialises the final stage's lambda; here it is 0.
 * Returns BM3D_OK or BM3D_ERR_INVALID for an unknown profile (the reference
 * exits the process, include/BM3D.h:79-84). */
int bm3d_stage_params_default(const char *profile, int wiener, const double sigma[3],
                              bm3d_stage_params *out);

/* Recompute thMSE from sigma[0] for the given profile (reference
 * BM3D_{Basic,Final}_Para::thMSE_Default, include/BM3D.h:89-97, 142-150). */
int bm3d_stage_params_thmse_default(const char *profile, int wiener, bm3d_stage_params *p);

typedef struct bm3d_ctx bm3d_ctx;

/* Create a context on CUDA device `device`. Replaces the per-filter FFTW
 * planning and table setup of the BM3D_Base constructor
 * (reference include/BM3D.h:237-259, source/BM3D.cpp:9-73), which here happens
 * per call from the parameters (a few hundred bytes of constants). */
int bm3d_ctx_create(bm3d_ctx **out, int device);
void bm3d_ctx_destroy(bm3d_ctx *ctx);

/* Last error message of this context; with ctx == NULL, of this thread's last
 * failed bm3d_ctx_create or context-free call (bm3d_stage_noalloc,
 * bm3d_noalloc_check). Never NULL. */
const char *bm3d_last_error(const bm3d_ctx *ctx);

/* One BM3D stage on one plane: dst = stage(src, ref).
 *   wiener = 0: basic estimate, matching and hard thresholding on `ref`
 *               (usually ref == src).
 *   wiener = 1: final estimate; `ref` is the basic estimate.
 * `value_range` is the plane's ValueRange() (Ceil - Floor, 1 for the
 * reference's default Plane_FL); it scales the matching threshold.
 * Replaces BM3D_Basic::process(dst, src, ref) / BM3D_Final::process(dst, src, ref)
 * through FilterIF2::process (reference include/Filter.h:174) and
 * BM3D_Base::Kernel(dst, src, ref) (source/BM3D.cpp:80-136). */
int bm3d_stage(bm3d_ctx *ctx, const bm3d_stage_params *params, int wiener, float *dst,
               const float *src, const float *ref, int width, int height, size_t stride,
               float value_range, int mem, void *stream);

/* Three planes (Y, U, V) sharing the groups matched on ref[0]; planes with
 * sigma[p] <= 0 are left untouched in dst. Replaces the 9-plane
 * BM3D_Base::Kernel (reference source/BM3D.cpp:139-218). */
int bm3d_stage3(bm3d_ctx *ctx, const bm3d_stage_params *params, int wiener, float *const dst[3],
                const float *const src[3], const float *const ref[3], int width, int height,
                size_t stride, float value_range, int mem, void *stream);

/* Basic then final on one plane, the basic estimate held in context scratch:
 * basic = stage(src, ref), dst = final(src, basic). `ref` may be NULL
 * (ref = src). Replaces BM3D::process(dst, src[, ref]) on Plane_FL,
 * BM3D::process_Plane_FL (reference source/BM3D.cpp:464-472), with the
 * intermediate sized from src (the reference passes an empty plane there). */
int bm3d_full(bm3d_ctx *ctx, const bm3d_stage_params *basic, const bm3d_stage_params *final_,
              float *dst, const float *src, const float *ref, int width, int height,
              size_t stride, float value_range, int mem, void *stream);

/* Three-plane basic then final (reference BM3D::process_Frame's YUV core,
 * source/BM3D.cpp:512-521); the basic stage matches on ref[0] (ref may be
 * NULL: ref = src). */
int bm3d_full3(bm3d_ctx *ctx, const bm3d_stage_params *basic, const bm3d_stage_params *final_,
               float *const dst[3], const float *const src[3], const float *const ref[3],
               int width, int height, size_t stride, float value_range, int mem, void *stream);

/* Basic then final on `count` planes in HOST memory, each with its own
 * parameters and size, with the copies overlapped with the filtering: plane
 * i + 1 is uploaded and plane i - 1 downloaded while plane i is filtered on
 * `stream` (two copy streams and two device slots owned by the context).
 * Results equal per-plane bm3d_full bit for bit. With `async` = 0 the call
 * returns when every result is in dst. With `async` != 0 it returns once the
 * work is enqueued: `stream` completes after the last download, so the caller
 * synchronises it (or records an event on it) before reading dst or reusing
 * src; consecutive async calls overlap one another's copies too. Overlap
 * needs page-locked host planes; pageable planes still work, with the copies
 * serialised. Replaces looping BM3D::process over host images
 * (source/BM3D.cpp:464-472), which has no overlap. */
int bm3d_full_many(bm3d_ctx *ctx, int count, const bm3d_stage_params *basic,
                   const bm3d_stage_params *final_, float *const dst[], const float *const src[],
                   const int width[], const int height[], const size_t stride[],
                   float value_range, int async, void *stream);

/* ---- Integer planes and RGB frames ------------------------------------
 * Planes of the reference's integer pixel type (DType = int32,
 * include/Type.h:25) with its quantisation: Floor, Neutral and Ceil of the plane
 * (include/Image_Type.h:77-79); Neutral > Floor marks a chroma plane. RGB
 * planes have Neutral = Floor. `stride` is in pixels. The float working
 * planes have the reference's default Plane_FL ranges (luma [0, 1], chroma
 * [-0.5, 0.5]) and live in context scratch; the filtering itself is
 * bm3d_stage / bm3d_stage3 / bm3d_full / bm3d_full3 on them. Returns the
 * status codes of those calls; BM3D_ERR_INVALID also for ceil <= floor. */

/* Basic then final on one integer plane: RangeConvert to float, the two
 * stages, RangeConvert back clipped to [floor, ceil] (+0.5, or +0.499999 for
 * full-range chroma, then truncation). Replaces BM3D::process_Plane
 * (reference source/BM3D.cpp:475-497) through FilterIF2::operator()(Plane)
 * (include/Filter.h:210-215), with the basic estimate sized from src (the
 * reference's process_Plane_FL passes an empty plane there). `ref` may be
 * NULL (ref = src); the basic stage matches on it. */
int bm3d_plane_int(bm3d_ctx *ctx, const bm3d_stage_params *basic,
                   const bm3d_stage_params *final_, int32_t *dst, const int32_t *src,
                   const int32_t *ref, int width, int height, size_t stride, int floor_,
                   int neutral, int ceil_, int mem, void *stream);

/* One stage on one integer plane (ref may be NULL: ref = src). Replaces
 * BM3D_Basic / BM3D_Final used as a filter on a Plane,
 * BM3D_Base::process_Plane (reference source/BM3D.cpp:248-281), including
 * its guard: sigma[0] <= 0, GroupSize == 1, BlockSize <= 0, BMrange <= 0,
 * BMrange < BMstep or thMSE <= 0 copy src (BM3D_COPIED). */
int bm3d_stage_int(bm3d_ctx *ctx, const bm3d_stage_params *params, int wiener, int32_t *dst,
                   const int32_t *src, const int32_t *ref, int width, int height, size_t stride,
                   int floor_, int neutral, int ceil_, int mem, void *stream);

/* Basic then final on an RGB frame (R, G, B planes with Floor floor_ and
 * Ceil ceil_): OPP RGB->YUV (MatrixConvert_RGB2YUV, include/Conversion.hpp:
 * 518-575), three-plane basic and final with groups matched on Y,
 * YUV->RGB clipped to [floor_, ceil_] (MatrixConvert_YUV2RGB,
 * include/Conversion.hpp:661-748). `ref` may be NULL (ref = src); a
 * distinct ref frame contributes only its Y, on which the basic stage matches
 * (BM3D_Basic::RGB2YUV, source/BM3D.cpp:320-336). Replaces BM3D::process_Frame
 * (reference source/BM3D.cpp:501-527) through FilterIF2::operator()(Frame[, ref]). */
int bm3d_frame(bm3d_ctx *ctx, const bm3d_stage_params *basic, const bm3d_stage_params *final_,
               int32_t *const dst[3], const int32_t *const src[3], const int32_t *const ref[3],
               int width, int height, size_t stride, int floor_, int ceil_, int mem,
               void *stream);

/* One stage on an RGB frame (ref may be NULL: ref = src); the basic stage
 * converts only Y of a distinct ref, the final stage all of it. Replaces
 * BM3D_Basic / BM3D_Final used as a filter on a Frame,
 * BM3D_Base::process_Frame (reference source/BM3D.cpp:284-313) with
 * RGB2YUV (320-336, 392-408), including its guard (all sigma <= 0,
 * GroupSize == 1, ... copy src: BM3D_COPIED). */
int bm3d_stage_frame(bm3d_ctx *ctx, const bm3d_stage_params *params, int wiener,
                     int32_t *const dst[3], const int32_t *const src[3],
                     const int32_t *const ref[3], int width, int height, size_t stride,
                     int floor_, int ceil_, int mem, void *stream);

/* FP64 forms of bm3d_stage / bm3d_full: the same kernels instantiated for
 * double (the reference's FLType without _CUDA_, include/Type.h:26-30). */
int bm3d_stage_f64(bm3d_ctx *ctx, const bm3d_stage_params *params, int wiener, double *dst,
                   const double *src, const double *ref, int width, int height, size_t stride,
                   double value_range, int mem, void *stream);

/* Number of reference blocks a stage visits on a width x height plane
 * (the scan of reference source/BM3D.cpp:98-121), or -1 for bad arguments. */
long long bm3d_ref_block_count(const bm3d_stage_params *params, int width, int height);

/* Group of every reference block, in scan order (ref-block index = row-major
 * over the scan): counts[r], pos_yx[(r * 32 + k) * 2 + {0, 1}] = (y, x) and
 * keys[r * 32 + k] of member k. Arrays are host memory sized from
 * bm3d_ref_block_count. Replaces BM3D_Base::BlockMatching
 * (reference source/BM3D.cpp:221-236) for parity checks. */
int bm3d_debug_groups(bm3d_ctx *ctx, const bm3d_stage_params *params, int wiener, const float *ref,
                      int width, int height, size_t stride, float value_range, int *counts,
                      int *pos_yx, float *keys);

/* Counters of the last stage run on this context: out[0] = sum of group
 * sizes, out[1] = sum of squared group sizes, out[2] = candidate blocks
 * evaluated, out[3] = groups re-ordered to follow std::partial_sort's tie
 * placement. Synchronises the context's last stream. */
int bm3d_last_stats(bm3d_ctx *ctx, unsigned long long out[4]);

/* Device-memory calls return once their work is enqueued, so the kernels'
 * internal consistency counter (group blocks found outside their tile's
 * staged window, tiles launched with less shared memory than their layout
 * needs; both skipped, never touched) is checked only by host-memory calls.
 * bm3d_check waits for the context's last stream and returns BM3D_ERR_CUDA,
 * with the counts in bm3d_last_error, if the counter has moved since the
 * context was made; BM3D_OK otherwise. It covers the stage and combined
 * entries (batches keep no counter). No counterpart in the reference, which
 * has no asynchronous calls. */
int bm3d_check(bm3d_ctx *ctx);

/* One stage on one plane of DEVICE memory, like bm3d_stage with
 * BM3D_MEM_DEVICE, but without a context and without allocating anything:
 * no cudaMalloc / cudaFree / allocating library routine is called. It is for
 * callers that cannot allocate device memory once running -- e.g. a filter
 * plugin whose host application owns every device allocation, or a real-time
 * frame loop that may not risk a device-synchronising, possibly failing
 * cudaMalloc per frame. No counterpart in the reference (whose CPU filter
 * allocates its accumulators per call, source/BM3D.cpp:89-90).
 *
 * Scratch is a file-scope static device array of this library: 32 MiB + 512
 * bytes (fixed-point numerator and weight sums for up to 2,097,152 pixels,
 * e.g. 1920x1080, plus a small header). Every GPU that loads the library holds
 * it until the process exits. Planes larger than that are rejected with
 * BM3D_ERR_TOO_LARGE (use bm3d_stage instead).
 *
 * The first call on a device, with that device current, sets up that device
 * (looks up the scratch array's device address, uploads the cosine tables);
 * make that first call before any stream capture. Work is enqueued on
 * `stream` (NULL = legacy default stream) and the call returns without
 * waiting. All calls share the one scratch array and every call clears the
 * parts it needs before use, but two calls whose work overlaps on the GPU
 * (e.g. on two streams of the same device) race on it: serialise them.
 * Returns the status codes of bm3d_stage, plus BM3D_ERR_TOO_LARGE; the
 * message of a failed call is bm3d_last_error(NULL) on the calling thread.
 * Like a device-memory bm3d_stage, the call returns before the kernels run,
 * so their consistency counter is read by bm3d_noalloc_check. */
int bm3d_stage_noalloc(const bm3d_stage_params *params, int wiener, float *dst, const float *src,
                       const float *ref, int width, int height, size_t stride, float value_range,
                       void *stream);

/* The consistency check of bm3d_stage_noalloc (as bm3d_check is for a
 * context): waits for `stream`, then reads the kernels' consistency counter
 * of the current device's static scratch -- group blocks found outside their
 * tile's staged window, tiles launched with less shared memory than their
 * layout needs, both skipped -- which covers every bm3d_stage_noalloc call on
 * the device since the library loaded or since the last check. Returns BM3D_OK
 * if it is zero; otherwise clears it and returns BM3D_ERR_CUDA with the counts
 * in bm3d_last_error(NULL). Allocates nothing. No counterpart in the
 * reference. */
int bm3d_noalloc_check(void *stream);

/* Batched basic + final over `count` device planes of any sizes and noise
 * levels: one persistent launch per stage walks a device work queue of
 * (plane, tile) items, and the whole pipeline (accumulator set-up, basic
 * stage, normalisation, final stage, normalisation) is captured once in a
 * CUDA graph that bm3d_batch_run replays. Per plane i: basic[i] / final_[i]
 * (planes in one batch share BlockSize, BlockStep, GroupSize, BMrange and
 * BMstep per stage; sigma, thMSE and lambda may differ), src[i] / dst[i]
 * with width[i] x height[i] and row pitch stride[i]. With `autotune` the
 * tile shape and warps per CTA of each stage are picked by timing candidate
 * configurations on this batch. Results equal per-plane bm3d_full bit for bit.
 * The batch keeps its own device buffers (16 B per pixel of accumulators and
 * the basic estimates) until bm3d_batch_destroy. Replaces looping the
 * reference's BM3D over images (no batched form exists there). */
typedef struct bm3d_batch bm3d_batch;
int bm3d_batch_create(bm3d_ctx *ctx, int count, const bm3d_stage_params *basic,
                      const bm3d_stage_params *final_, float *const dst[],
                      const float *const src[], const int width[], const int height[],
                      const size_t stride[], int autotune, bm3d_batch **out);
/* The same over `count` images of three planes (Y, U, V) each, sharing the
 * groups matched on Y (as bm3d_full3): plane c of image i is dst[3 * i + c] /
 * src[3 * i + c], all three of width[i] x height[i] with row pitch stride[i].
 * Results equal per-image bm3d_full3 bit for bit. Replaces looping the
 * reference's 9-plane BM3D_Base::Kernel (source/BM3D.cpp:139-218) over
 * frames. */
int bm3d_batch3_create(bm3d_ctx *ctx, int count, const bm3d_stage_params *basic,
                       const bm3d_stage_params *final_, float *const dst[],
                       const float *const src[], const int width[], const int height[],
                       const size_t stride[], int autotune, bm3d_batch **out);
/* Final (Wiener) stage only, over `count` device planes (or, for the "3" form,
 * images of three planes sharing the groups matched on ref[3 * i]) with the
 * caller's reference planes ref[] in place of the basic estimates -- e.g. the
 * learned pilot's estimates (bm3d_pilot_estimate). ref planes have the same
 * size and row pitch as src. Otherwise as bm3d_batch_create /
 * bm3d_batch3_create; results equal per-plane bm3d_stage (wiener = 1) /
 * bm3d_stage3 with the same ref, bit for bit. Replaces looping the reference's
 * BM3D_Final over images (source/BM3D.cpp:411-457). */
int bm3d_batch_final_create(bm3d_ctx *ctx, int count, const bm3d_stage_params *final_,
                            float *const dst[], const float *const src[],
                            const float *const ref[], const int width[], const int height[],
                            const size_t stride[], int autotune, bm3d_batch **out);
int bm3d_batch3_final_create(bm3d_ctx *ctx, int count, const bm3d_stage_params *final_,
                             float *const dst[], const float *const src[],
                             const float *const ref[], const int width[], const int height[],
                             const size_t stride[], int autotune, bm3d_batch **out);
int bm3d_batch_run(bm3d_batch *batch, void *stream);
/* Waits for `stream` and returns BM3D_ERR_CUDA (counts in bm3d_last_error of
 * the batch's context) if the batch kernels' consistency counter has moved
 * since creation -- group blocks outside their tile's staged window, or tiles
 * launched with too little shared memory, both skipped -- else BM3D_OK (as
 * bm3d_check does for the single-call entries). No counterpart in the
 * reference. */
int bm3d_batch_check(bm3d_batch *batch, void *stream);
/* Batches fed from HOST memory: `count` planes (sizes and parameters fixed
 * at creation; device buffers owned by the batch). Each bm3d_host_batch_run
 * uploads src, runs the batch graph on `stream` and downloads dst; the batch
 * keeps two device slots, so with page-locked host planes one run's uploads
 * and downloads overlap the neighbouring runs' filtering.
 *   async = 0: returns with dst written.
 *   async = 1: returns once enqueued; `stream` completes after this run's
 *              download (which also holds the next run's filtering behind it).
 *   async = 2: returns once enqueued without tying `stream` to the download,
 *              so consecutive runs overlap fully; bm3d_host_batch_join then
 *              makes `stream` wait for every download issued so far.
 * Synchronise (after joining) before reading dst or reusing src. The first
 * run on each slot builds its graph (the autotuner times that run's data)
 * and waits for it. Results equal per-plane bm3d_full bit for bit. No
 * counterpart in the reference. */
typedef struct bm3d_host_batch bm3d_host_batch;
int bm3d_host_batch_create(bm3d_ctx *ctx, int count, const bm3d_stage_params *basic,
                           const bm3d_stage_params *final_, const int width[], const int height[],
                           int autotune, bm3d_host_batch **out);
/* The same over `count` images of three planes (Y, U, V) each, sharing the
 * groups matched on Y (as bm3d_batch3_create): bm3d_host_batch_run then takes
 * plane c of image i as dst[3 * i + c] / src[3 * i + c], with row pitch
 * stride[i] for all three. Results equal per-image bm3d_full3 bit for bit. */
int bm3d_host_batch3_create(bm3d_ctx *ctx, int count, const bm3d_stage_params *basic,
                            const bm3d_stage_params *final_, const int width[],
                            const int height[], int autotune, bm3d_host_batch **out);
int bm3d_host_batch_run(bm3d_host_batch *batch, float *const dst[], const float *const src[],
                        const size_t stride[], int async, void *stream);
int bm3d_host_batch_join(bm3d_host_batch *batch, void *stream);
void bm3d_host_batch_destroy(bm3d_host_batch *batch);

/* Runs the batch's pipeline once outside its graph, on `stream`, with CUDA
 * events around the two persistent stage launches, and returns their device
 * times in ms[0] (basic; 0 for a final-stage-only batch) and ms[1] (final);
 * results as bm3d_batch_run. For measuring the kernels the graph replays. No
 * counterpart in the reference. */
int bm3d_batch_stage_times(bm3d_batch *batch, void *stream, float ms[2]);

/* tile_x, tile_y, warps of the basic stage, then of the final stage. */
int bm3d_batch_tuning(const bm3d_batch *batch, int out[6]);
void bm3d_batch_destroy(bm3d_batch *batch);

/* Per-launch timing of the stage kernels with CUDA events recorded on the
 * launch stream (off by default). Turning it on or off resets the totals.
 * No counterpart in the reference, which has no timing hooks beyond an
 * untimed loop (source/ISP_MW.cpp:38-107). */
int bm3d_set_kernel_timing(bm3d_ctx *ctx, int on);

/* Total device time (ms) and launch count of the basic (wiener = 0) or final
 * (wiener = 1) stage kernel since timing was turned on. Waits for the
 * recorded launches to finish. */
int bm3d_kernel_time(bm3d_ctx *ctx, int wiener, double *ms, long long *launches);

/* ---- Learned pilot ------------------------------------------------------
 * A small convolutional network that stands in for the basic estimate feeding
 * the final (Wiener) stage: 8 layers of 3 x 3 convolutions, 48 channels, ReLU,
 * BF16 weights and activations with FP32 accumulation (tensor cores for the
 * 48 -> 48 layers), inputs the noisy plane and a constant noise-level plane
 * (true noise std on the 0-1 scale), output noisy + predicted residual. It is
 * trained (bm3d_pilot_train_step, Adam on FP32 master weights) to regress the
 * basic estimate this library computes. No counterpart in the reference,
 * whose final stage takes the basic estimate as `ref`
 * (BM3D_Final::CollaborativeFilter, source/BM3D.cpp:411-457); the plain
 * basic estimate stays available and is what the pilot is compared with. */
typedef struct bm3d_pilot bm3d_pilot;

/* Number of FP32 parameters (weights and biases of the eight layers). */
int bm3d_pilot_param_count(void);

/* Which kernel runs the 48 -> 48 convolutions (process-wide): 0 (default) the
 * warp-specialised TMA pipelines when their tensor maps encode -- N = 144
 * (three column taps per MMA) for forward layers, N = 48 for data gradients
 * -- else the cp.async kernel; 1 the cp.async kernel; 2 the N = 48 TMA
 * pipeline only; 3 the N = 144 pipeline for forward layers (2 and 3 fail with
 * BM3D_ERR_CUDA when their maps do not encode). The cp.async kernel and the
 * N = 48 pipeline give identical results; the N = 144 pipeline adds the same
 * FP32 products in another order. */
int bm3d_pilot_set_conv_kernel(int which);

/* Per-layer timing of the pilot's forward passes (off by default): with it on,
 * every forward pass records CUDA events on its stream around each of the
 * eight layers. */
int bm3d_pilot_set_timing(bm3d_pilot *pilot, int on);

/* Device ms of each of the eight layers of the last timed forward pass
 * (ms[0] layer 1, ms[1..6] the 48 -> 48 layers, ms[7] layer 8); waits for it. */
int bm3d_pilot_layer_ms(bm3d_pilot *pilot, float *ms);

/* The kernel of the last 48 -> 48 convolution launched: 3 = N = 144 TMA
 * pipeline, 2 = N = 48 TMA pipeline, 1 = cp.async kernel, 0 = none yet. */
int bm3d_pilot_conv_kernel(void);

/* A pilot on the context's device, He-initialised from `seed`. */
int bm3d_pilot_create(bm3d_ctx *ctx, unsigned long long seed, bm3d_pilot **out);
void bm3d_pilot_destroy(bm3d_pilot *p);

/* Parameters as one host FP32 vector of bm3d_pilot_param_count() values:
 * W1 [48][2][3][3], b1 [48], then for layers 2..7 W [48][48][3][3] and b
 * [48], then W8 [1][48][3][3] and b8 (PyTorch Conv2d weight order). Setting
 * them resets the optimiser state. */
int bm3d_pilot_set_params(bm3d_pilot *p, const float *host, int count);
int bm3d_pilot_get_params(bm3d_pilot *p, float *host, int count);
/* The loss gradient of the last bm3d_pilot_train_step, same order. */
int bm3d_pilot_get_grad(bm3d_pilot *p, float *host, int count);

/* Checkpoint file: parameters, optimiser moments and step count. */
int bm3d_pilot_save(bm3d_pilot *p, const char *path);
int bm3d_pilot_load(bm3d_pilot *p, const char *path);

/* dst = pilot(src) for `count` planes of width x height, row pitch `stride`,
 * planes `img_stride` elements apart; sigma[i] = true noise std (0-1 scale)
 * of plane i (host memory for BM3D_MEM_HOST, device otherwise). */
int bm3d_pilot_estimate(bm3d_pilot *p, float *dst, const float *src, int count, int width,
                        int height, size_t stride, size_t img_stride, const float *sigma, int mem,
                        void *stream);

/* One Adam step on `count` crops of height x width in DEVICE memory, stored
 * back to back (pitch = width): noisy inputs, targets (the basic estimates)
 * and per-crop noise std `sigma` (device). Loss = mean over pixels of
 * (sigma_ref / sigma)^2 (output - target)^2 with sigma_ref = 25/255: the
 * squared error scaled to a common noise level, so every noise level weighs
 * alike. Written to *loss (after a synchronisation) when loss is not NULL. */
int bm3d_pilot_train_step(bm3d_pilot *p, int count, int height, int width, const float *noisy,
                          const float *target, const float *sigma, float lr, double *loss,
                          void *stream);

/* Pilot then final stage on one plane: the final (Wiener) stage takes the
 * pilot's estimate as its reference in place of the basic estimate. The
 * pilot's noise-level input is final_->sigma[0] with the reference's OPP
 * luma scaling applied (include/BM3D.h:246-253). Replaces, for this
 * pipeline, the basic -> final sequence of BM3D::process_Plane_FL
 * (source/BM3D.cpp:464-472). */
int bm3d_pilot_full(bm3d_ctx *ctx, bm3d_pilot *p, const bm3d_stage_params *final_, float *dst,
                    const float *src, int width, int height, size_t stride, float value_range,
                    int mem, void *stream);

/* Layer-level entry points of the pilot's tensor-core kernels, on DEVICE
 * memory (BF16 activations [n][h][w][48]): one 48 -> 48 3 x 3 convolution with
 * padding 1 and FP32 weights [48][48][3][3] (mode 0: + bias, ReLU; mode 1:
 * + bias; mode 2: the data gradient -- the transposed, flipped convolution --
 * kept where aux > 0), and the weight / bias gradients of such a layer from
 * its input x and the gradient g at its output. Both synchronise `stream`.
 * For tests and tools; no counterpart in the reference. */
int bm3d_pilot_conv48(bm3d_ctx *ctx, int n, int h, int w, const void *x, const float *weight,
                      const float *bias, const void *aux, int mode, void *y, void *stream);
int bm3d_pilot_wgrad48(bm3d_ctx *ctx, int n, int h, int w, const void *x, const void *g, float *dw,
                       float *db, void *stream);

/* Fault injection for callers' error paths: the next `count` device buffer
 * allocations of contexts and batches fail as if cudaMalloc had run out of
 * memory (the call returns BM3D_ERR_NOMEM, nothing is left half-built, and
 * later calls allocate normally); 0 turns it off. Process-wide. No
 * counterpart in the reference, which exits on allocation failure. */
int bm3d_inject_alloc_failures(int count);

/* Tile shape used by the stage kernels: reference blocks per CTA tile
 * (tile_x x tile_y) and warps per CTA. 0 keeps the current value. */
int bm3d_set_tiling(bm3d_ctx *ctx, int tile_x, int tile_y, int warps);

#ifdef __cplusplus
}
#endif

#endif
