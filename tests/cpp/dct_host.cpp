// Host build of the kernels' register-resident DCTs (isp_mw_b200/csrc/dct.cuh)
// so tests/test_dct_host.py can check them against scipy without a GPU.
#include "dct.cuh"

extern "C" {

void host_redft10_8_f32(float *x) { float (&a)[8] = *reinterpret_cast<float(*)[8]>(x); bm3d::redft10_8(a); }
void host_redft01_8_f32(float *x) { float (&a)[8] = *reinterpret_cast<float(*)[8]>(x); bm3d::redft01_8(a); }
void host_redft10_16_f32(float *x) { float (&a)[16] = *reinterpret_cast<float(*)[16]>(x); bm3d::redft10_16(a); }
void host_redft01_16_f32(float *x) { float (&a)[16] = *reinterpret_cast<float(*)[16]>(x); bm3d::redft01_16(a); }
void host_redft10_8_f64(double *x) { double (&a)[8] = *reinterpret_cast<double(*)[8]>(x); bm3d::redft10_8(a); }
void host_redft01_8_f64(double *x) { double (&a)[8] = *reinterpret_cast<double(*)[8]>(x); bm3d::redft01_8(a); }
void host_redft10_16_f64(double *x) { double (&a)[16] = *reinterpret_cast<double(*)[16]>(x); bm3d::redft10_16(a); }
void host_redft01_16_f64(double *x) { double (&a)[16] = *reinterpret_cast<double(*)[16]>(x); bm3d::redft01_16(a); }
void host_dct_matrix_f64(double *x, int n, const double *mat)
{
    double (&a)[16] = *reinterpret_cast<double(*)[16]>(x);
    bm3d::dct_matrix<double, 16>(a, n, mat);
}
}
