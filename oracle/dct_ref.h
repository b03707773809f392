/* Oracle (test infrastructure only): unnormalised separable 3-D DCT used in
 * place of FFTW's r2r plans. Shared by the compiled reference
 * (through oracle/fftw_shim.cpp) and by the C restatement (oracle/bm3d_oracle.c),
 * so both compute bit-identical transforms.
 *
 * Definitions (FFTW 3 manual, "1d Real-even DFTs (DCTs)"):
 *   REDFT10 (forward):  Y_k = 2 * sum_{j=0}^{n-1} X_j cos(pi (j + 1/2) k / n)
 *   REDFT01 (backward): Y_k = X_0 + 2 * sum_{j=1}^{n-1} X_j cos(pi j (k + 1/2) / n)
 * applied along every axis of an n0 x n1 x n2 row-major array (n2 fastest),
 * as fftw_plan_r2r_3d does (reference: source/BM3D.cpp:13-23, 358, 374).
 * A forward then backward transform scales the data by 2*n0 * 2*n1 * 2*n2.
 *
 * Rounding: the float transform accumulates all three axes in double and
 * rounds once at the end; the double transform accumulates in long double.
 * Both are therefore closer to the exact transform than FFTW's own codelets. */
#ifndef ORACLE_DCT_REF_H_
#define ORACLE_DCT_REF_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_dct_plan oracle_dct_plan;

/* kind: 0 = REDFT10 (forward), 1 = REDFT01 (backward). */
oracle_dct_plan *oracle_dct_plan_create(int n0, int n1, int n2, int kind);
void oracle_dct_plan_destroy(oracle_dct_plan *p);
void oracle_dct_exec_f32(const oracle_dct_plan *p, float *data);
void oracle_dct_exec_f64(const oracle_dct_plan *p, double *data);
void oracle_dct_exec_f80(const oracle_dct_plan *p, long double *data);

/* How oracle_dct_exec_f32 evaluates the transform (process-wide):
 *   0 (default): accumulate all three axes in double, round once;
 *   1: in float, each axis rounded to float, terms summed in index order;
 *   2: as 1 with the terms summed in reverse index order;
 *   3: as 1 with the terms summed pairwise (balanced tree).
 * Modes 1-3 are three more valid FP32 evaluations of the same transform;
 * the parity tests run the reference's chain under them to measure how far
 * the reference diverges from itself when only its transform rounding
 * changes. */
void oracle_dct_set_f32_mode(int mode);
int oracle_dct_get_f32_mode(void);

#ifdef __cplusplus
}
#endif

#endif
