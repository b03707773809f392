/* Oracle (test infrastructure only): implementations of the three FFTW entry
 * points the reference's BM3D path calls (declared in shim/fftw3.h), on top of
 * the separable DCT in dct_ref.c. Only REDFT10 and REDFT01 with the same kind
 * on all three axes are supported, which is all source/BM3D.cpp:13-23 plans. */
#include "shim/fftw3.h"
#include "dct_ref.h"

#include <cstdio>
#include <cstdlib>

struct oracle_r2r_plan {
    oracle_dct_plan *dct;
};

static oracle_r2r_plan *make_plan(int n0, int n1, int n2, oracle_fftw_r2r_kind k0,
                                  oracle_fftw_r2r_kind k1, oracle_fftw_r2r_kind k2)
{
    if (k0 != k1 || k1 != k2 || (k0 != FFTW_REDFT10 && k0 != FFTW_REDFT01)) {
        std::fprintf(stderr, "oracle fftw shim: unsupported r2r kinds %d %d %d\n", k0, k1, k2);
        std::abort();
    }
    oracle_r2r_plan *p = new oracle_r2r_plan;
    p->dct = oracle_dct_plan_create(n0, n1, n2, k0 == FFTW_REDFT10 ? 0 : 1);
    return p;
}

static void destroy(oracle_r2r_plan *p)
{
    if (!p) return;
    oracle_dct_plan_destroy(p->dct);
    delete p;
}

fftw_plan_s *fftw_plan_r2r_3d(int n0, int n1, int n2, double *, double *, fftw_r2r_kind k0,
                              fftw_r2r_kind k1, fftw_r2r_kind k2, unsigned)
{
    return make_plan(n0, n1, n2, k0, k1, k2);
}
void fftw_execute_r2r(const fftw_plan_s *p, double *in, double *out)
{
    if (in != out) std::abort();
    oracle_dct_exec_f64(p->dct, in);
}
void fftw_destroy_plan(fftw_plan_s *p) { destroy(p); }

fftwf_plan_s *fftwf_plan_r2r_3d(int n0, int n1, int n2, float *, float *, fftwf_r2r_kind k0,
                                fftwf_r2r_kind k1, fftwf_r2r_kind k2, unsigned)
{
    return make_plan(n0, n1, n2, k0, k1, k2);
}
void fftwf_execute_r2r(const fftwf_plan_s *p, float *in, float *out)
{
    if (in != out) std::abort();
    oracle_dct_exec_f32(p->dct, in);
}
void fftwf_destroy_plan(fftwf_plan_s *p) { destroy(p); }

fftwl_plan_s *fftwl_plan_r2r_3d(int n0, int n1, int n2, long double *, long double *,
                                fftwl_r2r_kind k0, fftwl_r2r_kind k1, fftwl_r2r_kind k2, unsigned)
{
    return make_plan(n0, n1, n2, k0, k1, k2);
}
void fftwl_execute_r2r(const fftwl_plan_s *p, long double *in, long double *out)
{
    if (in != out) std::abort();
    oracle_dct_exec_f80(p->dct, in);
}
void fftwl_destroy_plan(fftwl_plan_s *p) { destroy(p); }
