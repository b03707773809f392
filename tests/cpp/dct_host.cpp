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
}

// Length-n symmetric matrix transforms (n in 1..16) of two pencils x and y,
// with the n x n matrix `mat`; inverse selects REDFT01.
template <int N>
static void pair(double *x, double *y, const double *mat, int inverse)
{
    double (&a)[16] = *reinterpret_cast<double(*)[16]>(x);
    double (&b)[16] = *reinterpret_cast<double(*)[16]>(y);
    if (inverse) bm3d::redft01_pair<double, N>(a, b, mat);
    else bm3d::redft10_pair<double, N>(a, b, mat);
}

template <int... Ns> struct PairTable {
    static void run(int n, double *x, double *y, const double *mat, int inverse)
    {
        ((n == Ns ? pair<Ns>(x, y, mat, inverse) : void()), ...);
    }
};

extern "C" void host_dct_pair_f64(double *x, double *y, int n, const double *mat, int inverse)
{
    PairTable<1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16>::run(n, x, y, mat, inverse);
}

// One line of length 32 through the symmetric forms, with the 32 x 32 matrix.
extern "C" void host_dct_line32_f64(double *x, const double *mat, int inverse)
{
    double (&a)[32] = *reinterpret_cast<double(*)[32]>(x);
    if (inverse) bm3d::redft01_line<double, 32>(a, mat);
    else bm3d::redft10_line<double, 32>(a, mat);
}

// Power-of-two lengths 16 and 32 through the recursive even/odd splits.
#define BM3D_HOST_POW2(N, T, SFX)                                                             \
    extern "C" void host_pow2_redft10_##N##_##SFX(T *x)                                       \
    {                                                                                         \
        bm3d::redft10_pow2<T, N>(*reinterpret_cast<T(*)[N]>(x));                              \
    }                                                                                         \
    extern "C" void host_pow2_redft01_##N##_##SFX(T *x)                                       \
    {                                                                                         \
        bm3d::redft01_pow2<T, N>(*reinterpret_cast<T(*)[N]>(x));                              \
    }
BM3D_HOST_POW2(16, float, f32)
BM3D_HOST_POW2(32, float, f32)
BM3D_HOST_POW2(16, double, f64)
BM3D_HOST_POW2(32, double, f64)
