// Register-resident unnormalised DCTs for the BM3D collaborative filter.
//
// They compute exactly the transforms the reference gets from FFTW r2r plans
// (source/BM3D.cpp:13-23): REDFT10 forward and REDFT01 backward,
//   REDFT10: Y_k = 2 sum_{j=0}^{n-1} x_j cos(pi (2j+1) k / (2n))
//   REDFT01: Y_k = x_0 + 2 sum_{j=1}^{n-1} x_j cos(pi j (2k+1) / (2n))
// so REDFT01(REDFT10(x)) = 2n x, which the reference undoes with finalAMP.
//
// Lengths 8 and 16 use an even/odd split (the 8-point even half is split once
// more); other lengths multiply by a small cosine matrix, halved by its
// symmetry. All functions are __host__ __device__ so the CPU unit tests can
// check them against scipy.
#pragma once

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace bm3d {

// 2 cos(k pi / 16), k = 1..7
#define BM3D_C16_1 1.9615705608064609
#define BM3D_C16_2 1.8477590650225735
#define BM3D_C16_3 1.6629392246050905
#define BM3D_C16_4 1.4142135623730951
#define BM3D_C16_5 1.1111404660392046
#define BM3D_C16_6 0.7653668647301797
#define BM3D_C16_7 0.39018064403225666

// REDFT10 of length 8, in place.
template <typename T>
__host__ __device__ __forceinline__ void redft10_8(T (&x)[8])
{
    const T C1 = T(BM3D_C16_1), C2 = T(BM3D_C16_2), C3 = T(BM3D_C16_3), C4 = T(BM3D_C16_4);
    const T C5 = T(BM3D_C16_5), C6 = T(BM3D_C16_6), C7 = T(BM3D_C16_7);
    const T u0 = x[0] + x[7], u1 = x[1] + x[6], u2 = x[2] + x[5], u3 = x[3] + x[4];
    const T v0 = x[0] - x[7], v1 = x[1] - x[6], v2 = x[2] - x[5], v3 = x[3] - x[4];
    const T a = u0 + u3, b = u1 + u2, c = u0 - u3, d = u1 - u2;
    x[0] = T(2) * (a + b);
    x[4] = C4 * (a - b);
    x[2] = C2 * c + C6 * d;
    x[6] = C6 * c - C2 * d;
    x[1] = C1 * v0 + C3 * v1 + C5 * v2 + C7 * v3;
    x[3] = C3 * v0 - C7 * v1 - C1 * v2 - C5 * v3;
    x[5] = C5 * v0 - C1 * v1 + C7 * v2 + C3 * v3;
    x[7] = C7 * v0 - C5 * v1 + C3 * v2 - C1 * v3;
}

// REDFT01 of length 8, in place.
template <typename T>
__host__ __device__ __forceinline__ void redft01_8(T (&x)[8])
{
    const T C1 = T(BM3D_C16_1), C2 = T(BM3D_C16_2), C3 = T(BM3D_C16_3), C4 = T(BM3D_C16_4);
    const T C5 = T(BM3D_C16_5), C6 = T(BM3D_C16_6), C7 = T(BM3D_C16_7);
    const T p = x[0] + C4 * x[4], q = x[0] - C4 * x[4];
    const T s = C2 * x[2] + C6 * x[6], t = C6 * x[2] - C2 * x[6];
    const T e0 = p + s, e3 = p - s, e1 = q + t, e2 = q - t;
    const T o0 = C1 * x[1] + C3 * x[3] + C5 * x[5] + C7 * x[7];
    const T o1 = C3 * x[1] - C7 * x[3] - C1 * x[5] - C5 * x[7];
    const T o2 = C5 * x[1] - C1 * x[3] + C7 * x[5] + C3 * x[7];
    const T o3 = C7 * x[1] - C5 * x[3] + C3 * x[5] - C1 * x[7];
    x[0] = e0 + o0;
    x[7] = e0 - o0;
    x[1] = e1 + o1;
    x[6] = e1 - o1;
    x[2] = e2 + o2;
    x[5] = e2 - o2;
    x[3] = e3 + o3;
    x[4] = e3 - o3;
}

// D16[m][j] = 2 cos(pi (2j+1)(2m+1) / 32): odd half of the 16-point transforms.
#define BM3D_D16 \
    {{1.9903694533443939, 1.9138806714644176, 1.76384252869671, 1.546020906725474, 1.268786568327291, 0.9427934736519956, 0.5805693545089247, 0.19603428065912154},\
     {1.9138806714644176, 1.268786568327291, 0.19603428065912154, -0.9427934736519954, -1.7638425286967099, -1.9903694533443939, -1.5460209067254738, -0.5805693545089265},\
     {1.76384252869671, 0.19603428065912154, -1.546020906725474, -1.9138806714644179, -0.5805693545089249, 1.2687865683272899, 1.9903694533443936, 0.942793473651996},\
     {1.546020906725474, -0.9427934736519954, -1.9138806714644179, 0.19603428065912018, 1.9903694533443939, 0.5805693545089268, -1.7638425286967112, -1.2687865683272934},\
     {1.268786568327291, -1.7638425286967099, -0.5805693545089249, 1.9903694533443939, -0.19603428065911993, -1.9138806714644185, 0.9427934736519947, 1.5460209067254753},\
     {0.9427934736519956, -1.9903694533443939, 1.2687865683272912, 0.5805693545089251, -1.9138806714644174, 1.5460209067254718, 0.1960342806591181, -1.7638425286967123},\
     {0.5805693545089247, -1.5460209067254742, 1.9903694533443939, -1.7638425286967097, 0.9427934736519947, 0.19603428065912518, -1.2687865683272912, 1.9138806714644188},\
     {0.19603428065912154, -0.5805693545089249, 0.942793473651996, -1.2687865683272908, 1.5460209067254753, -1.7638425286967123, 1.9138806714644168, -1.990369453344394}}

// REDFT10 of length 16, in place.
template <typename T>
__host__ __device__ __forceinline__ void redft10_16(T (&x)[16])
{
    constexpr double D[8][8] = BM3D_D16;
    T u[8], v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        u[j] = x[j] + x[15 - j];
        v[j] = x[j] - x[15 - j];
    }
    redft10_8(u);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        T acc = T(D[m][0]) * v[0];
#pragma unroll
        for (int j = 1; j < 8; ++j) acc += T(D[m][j]) * v[j];
        x[2 * m + 1] = acc;
        x[2 * m] = u[m];
    }
}

// REDFT01 of length 16, in place.
template <typename T>
__host__ __device__ __forceinline__ void redft01_16(T (&x)[16])
{
    constexpr double D[8][8] = BM3D_D16;
    T e[8], o[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) e[m] = x[2 * m];
    redft01_8(e);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        T acc = T(D[0][k]) * x[1];
#pragma unroll
        for (int m = 1; m < 8; ++m) acc += T(D[m][k]) * x[2 * m + 1];
        o[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        x[k] = e[k] + o[k];
        x[15 - k] = e[k] - o[k];
    }
}

// Power-of-two lengths 16 and 32 by recursive even/odd splits, in place.
//   REDFT10 (n = 2h): even outputs are REDFT10_h of x_j + x_{n-1-j}; odd
//     outputs are REDFT11_h (DCT-IV) of x_j - x_{n-1-j}.
//   REDFT01 (n = 2h): y_j = e_j + o_j and y_{n-1-j} = e_j - o_j, with e the
//     REDFT01_h of the even inputs and o the REDFT11_h of the odd ones.
//   REDFT11_h(v)_k = 2 sum_j v_j cos(pi (2j+1)(2k+1) / (4h)) equals
//     W_k + W_{k+1} (W_h = 0) with W = REDFT10_h of w_j = v_j / (2 cos th_j),
//     th_j = pi (2j+1) / (4h), because 2 cos(th) cos((2k+1) th) =
//     cos(2k th) + cos((2k+2) th). (The REDFT11 matrix is symmetric, so the
//     same routine serves the inverse.)
// Length 8 is redft10_8 / redft01_8. A length-32 transform takes 269 adds and
// multiplies against 544 for the mirrored 32 x 32 matrix form.

// 1 / (2 cos(pi (2j + 1) / (4 h))), j < h: the DCT-IV pre-scales.
#define BM3D_S11_8 \
    {0.5024192861881557, 0.5224986149396889, 0.5669440348163577, 0.6468217833599901, \
     0.7881546234512502, 1.060677685990347, 1.7224470982383342, 5.101148618689155}
#define BM3D_S11_16 \
    {0.5006029982351963, 0.5054709598975436, 0.5154473099226246, 0.5310425910897841, \
     0.5531038960344445, 0.5829349682061339, 0.6225041230356648, 0.6748083414550057, \
     0.7445362710022986, 0.8393496454155268, 0.9725682378619608, 1.1694399334328847, \
     1.4841646163141662, 2.057781009953411, 3.407608418468719, 10.190008123548033}

template <typename T, int N> __host__ __device__ __forceinline__ void redft10_pow2(T (&x)[N]);

// REDFT11 (DCT-IV) of length H = 8 or 16, in place.
template <typename T, int H>
__host__ __device__ __forceinline__ void redft11_pow2(T (&v)[H])
{
    static_assert(H == 8 || H == 16, "DCT-IV lengths 8 and 16");
    constexpr double S8[8] = BM3D_S11_8;
    constexpr double S16[16] = BM3D_S11_16;
#pragma unroll
    for (int j = 0; j < H; ++j) v[j] *= T(H == 8 ? S8[j] : S16[j]);
    redft10_pow2<T, H>(v);
#pragma unroll
    for (int k = 0; k < H - 1; ++k) v[k] += v[k + 1];
}

// REDFT10 of length N = 8, 16 or 32, in place.
template <typename T, int N>
__host__ __device__ __forceinline__ void redft10_pow2(T (&x)[N])
{
    if constexpr (N == 8) {
        redft10_8(x);
    } else {
        constexpr int H = N / 2;
        T u[H], v[H];
#pragma unroll
        for (int j = 0; j < H; ++j) {
            u[j] = x[j] + x[N - 1 - j];
            v[j] = x[j] - x[N - 1 - j];
        }
        redft10_pow2<T, H>(u);
        redft11_pow2<T, H>(v);
#pragma unroll
        for (int m = 0; m < H; ++m) {
            x[2 * m] = u[m];
            x[2 * m + 1] = v[m];
        }
    }
}

// REDFT01 of length N = 8, 16 or 32, in place.
template <typename T, int N>
__host__ __device__ __forceinline__ void redft01_pow2(T (&x)[N])
{
    if constexpr (N == 8) {
        redft01_8(x);
    } else {
        constexpr int H = N / 2;
        T e[H], o[H];
#pragma unroll
        for (int m = 0; m < H; ++m) {
            e[m] = x[2 * m];
            o[m] = x[2 * m + 1];
        }
        redft01_pow2<T, H>(e);
        redft11_pow2<T, H>(o);
#pragma unroll
        for (int j = 0; j < H; ++j) {
            x[j] = e[j] + o[j];
            x[N - 1 - j] = e[j] - o[j];
        }
    }
}

// Length-N transforms of two pencils at once with an explicit N x N cosine
// matrix `m` (row k = output k), using the matrices' symmetries to halve the
// multiplies:
//   REDFT10: C[k][N-1-j] = (-1)^k C[k][j] -> sums (even k) and differences
//            (odd k) of mirrored inputs;
//   REDFT01: C[N-1-k][j] = (-1)^j C[k][j] -> even and odd input halves give
//            outputs k and N-1-k together.
// Entries N..15 of the pencils are left alone. On the device `m` is a
// constant-bank table at a compile-time offset, so every coefficient is an
// instruction operand.
template <typename T, int N, typename Mat>
__host__ __device__ __forceinline__ void redft10_pair(T (&a)[16], T (&b)[16], const Mat *m)
{
    constexpr int H = N / 2;
    T ua[H + 1], va[H + 1], ub[H + 1], vb[H + 1];
#pragma unroll
    for (int j = 0; j < H; ++j) {
        ua[j] = a[j] + a[N - 1 - j];
        va[j] = a[j] - a[N - 1 - j];
        ub[j] = b[j] + b[N - 1 - j];
        vb[j] = b[j] - b[N - 1 - j];
    }
    ua[H] = (N & 1) ? a[H] : T(0);
    ub[H] = (N & 1) ? b[H] : T(0);
    T ya[N], yb[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
        T sa = T(0), sb = T(0);
        if ((k & 1) == 0) {
#pragma unroll
            for (int j = 0; j < H + (N & 1); ++j) {
                sa += T(m[k * N + j]) * ua[j];
                sb += T(m[k * N + j]) * ub[j];
            }
        } else {
#pragma unroll
            for (int j = 0; j < H; ++j) {
                sa += T(m[k * N + j]) * va[j];
                sb += T(m[k * N + j]) * vb[j];
            }
        }
        ya[k] = sa;
        yb[k] = sb;
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
        a[k] = ya[k];
        b[k] = yb[k];
    }
}

template <typename T, int N, typename Mat>
__host__ __device__ __forceinline__ void redft01_pair(T (&a)[16], T (&b)[16], const Mat *m)
{
    T ya[N], yb[N];
#pragma unroll
    for (int k = 0; k < (N + 1) / 2; ++k) {
        T ea = T(0), oa = T(0), eb = T(0), ob = T(0);
#pragma unroll
        for (int j = 0; j < N; j += 2) {
            ea += T(m[k * N + j]) * a[j];
            eb += T(m[k * N + j]) * b[j];
        }
#pragma unroll
        for (int j = 1; j < N; j += 2) {
            oa += T(m[k * N + j]) * a[j];
            ob += T(m[k * N + j]) * b[j];
        }
        ya[k] = ea + oa;
        yb[k] = eb + ob;
        if (N - 1 - k != k) {
            ya[N - 1 - k] = ea - oa;
            yb[N - 1 - k] = eb - ob;
        }
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
        a[k] = ya[k];
        b[k] = yb[k];
    }
}

// The same symmetric forms for one line of N values (N up to the group
// size limit, 32), in place.
template <typename T, int N, typename Mat>
__host__ __device__ __forceinline__ void redft10_line(T (&a)[N], const Mat *m)
{
    constexpr int H = N / 2;
    T u[H + 1], v[H + 1];
#pragma unroll
    for (int j = 0; j < H; ++j) {
        u[j] = a[j] + a[N - 1 - j];
        v[j] = a[j] - a[N - 1 - j];
    }
    u[H] = (N & 1) ? a[H] : T(0);
    T y[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
        T s = T(0);
        if ((k & 1) == 0) {
#pragma unroll
            for (int j = 0; j < H + (N & 1); ++j) s += T(m[k * N + j]) * u[j];
        } else {
#pragma unroll
            for (int j = 0; j < H; ++j) s += T(m[k * N + j]) * v[j];
        }
        y[k] = s;
    }
#pragma unroll
    for (int k = 0; k < N; ++k) a[k] = y[k];
}

template <typename T, int N, typename Mat>
__host__ __device__ __forceinline__ void redft01_line(T (&a)[N], const Mat *m)
{
    T y[N];
#pragma unroll
    for (int k = 0; k < (N + 1) / 2; ++k) {
        T e = T(0), o = T(0);
#pragma unroll
        for (int j = 0; j < N; j += 2) e += T(m[k * N + j]) * a[j];
#pragma unroll
        for (int j = 1; j < N; j += 2) o += T(m[k * N + j]) * a[j];
        y[k] = e + o;
        if (N - 1 - k != k) y[N - 1 - k] = e - o;
    }
#pragma unroll
    for (int k = 0; k < N; ++k) a[k] = y[k];
}

}  // namespace bm3d
