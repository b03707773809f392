/* Oracle (test infrastructure only): a plain-C restatement of the reference's
 * BM3D basic (hard-threshold) and final (Wiener) stages, single plane and
 * three planes sharing luma groups. Tests and bench.py's CPU-baseline leg use
 * it as the checker; the product never links it.
 *
 * Every function cites the reference code it restates. With the same DCT
 * (dct_ref.c) and -ffp-contract=off it reproduces the compiled reference
 * (oracle/_ref) bit for bit, which tests/test_oracle.py checks. */
#ifndef ORACLE_BM3D_ORACLE_H_
#define ORACLE_BM3D_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

/* Numeric fields of BM3D_Para_Base (include/BM3D.h:15-45). */
typedef struct oracle_stage_params {
    int block_size;
    int block_step;
    int group_size;
    int bm_range;
    int bm_step;
    double thMSE;
    double lambda;
    double sigma[3];
} oracle_stage_params;

/* Status: 0 = filtered, 2 = parameters rejected by the reference's guard
 * (source/BM3D.cpp:82-87 / 143-151) and src copied to dst. */
int oracle_bm3d_stage_f32(int wiener, const oracle_stage_params *p, float *dst, const float *src,
                          const float *ref, int width, int height, double value_range);
int oracle_bm3d_stage_f64(int wiener, const oracle_stage_params *p, double *dst,
                          const double *src, const double *ref, int width, int height,
                          double value_range);
int oracle_bm3d_stage3_f32(int wiener, const oracle_stage_params *p, float *const dst[3],
                           const float *const src[3], const float *const ref[3], int width,
                           int height, double value_range);
int oracle_bm3d_stage3_f64(int wiener, const oracle_stage_params *p, double *const dst[3],
                           const double *const src[3], const double *const ref[3], int width,
                           int height, double value_range);
long long oracle_bm3d_groups_f32(int wiener, const oracle_stage_params *p, const float *ref,
                                 int width, int height, double value_range, int max_refs,
                                 int max_group, int *counts, int *pos_yx, float *keys);
long long oracle_bm3d_groups_f64(int wiener, const oracle_stage_params *p, const double *ref,
                                 int width, int height, double value_range, int max_refs,
                                 int max_group, int *counts, int *pos_yx, double *keys);

/* BM3D::process_Frame on int32 RGB planes with the given Floor / Ceil. */
int oracle_bm3d_frame_f32(const oracle_stage_params *pb, const oracle_stage_params *pf,
                          int *const dst[3], const int *const src[3], const int *const ref[3],
                          int width, int height, int floor_, int ceil_);
int oracle_bm3d_frame_f64(const oracle_stage_params *pb, const oracle_stage_params *pf,
                          int *const dst[3], const int *const src[3], const int *const ref[3],
                          int width, int height, int floor_, int ceil_);

/* BM3D::process_Plane on an int32 plane quantised as (floor, neutral, ceil). */
int oracle_bm3d_plane_int_f32(const oracle_stage_params *pb, const oracle_stage_params *pf,
                              int *dst, const int *src, const int *ref, int width, int height,
                              int floor_, int neutral, int ceil_);
int oracle_bm3d_plane_int_f64(const oracle_stage_params *pb, const oracle_stage_params *pf,
                              int *dst, const int *src, const int *ref, int width, int height,
                              int floor_, int neutral, int ceil_);

/* One stage on an RGB frame (ref may be null) / an integer plane. */
int oracle_bm3d_stage_frame_f32(int wiener, const oracle_stage_params *p, int *const dst[3],
                                const int *const src[3], const int *const ref[3], int width,
                                int height, int floor_, int ceil_);
int oracle_bm3d_stage_frame_f64(int wiener, const oracle_stage_params *p, int *const dst[3],
                                const int *const src[3], const int *const ref[3], int width,
                                int height, int floor_, int ceil_);
int oracle_bm3d_stage_int_f32(int wiener, const oracle_stage_params *p, int *dst, const int *src,
                              const int *ref, int width, int height, int floor_, int neutral,
                              int ceil_);
int oracle_bm3d_stage_int_f64(int wiener, const oracle_stage_params *p, int *dst, const int *src,
                              const int *ref, int width, int height, int floor_, int neutral,
                              int ceil_);

/* libstdc++'s std::partial_sort (heap select + sort_heap) on (key, payload)
 * pairs compared by key only, exposed so a test can pin it against the real
 * std::partial_sort. keys/payload have n entries; the first m become sorted. */
void oracle_partial_sort_f32(float *keys, int *payload, int m, int n);

#ifdef __cplusplus
}
#endif

#endif
