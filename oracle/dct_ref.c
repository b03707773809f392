/* Oracle (test infrastructure only): see dct_ref.h for the definitions and
 * the rounding contract. */
#include "dct_ref.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct oracle_dct_plan {
    int n[3];
    int kind;
    long double *tab[3]; /* tab[a][k * n + j]: coefficient of input j in output k */
};

static long double *make_table(int n, int kind)
{
    long double *t = (long double *)malloc(sizeof(long double) * (size_t)n * (size_t)n);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < n; ++k) {
        for (int j = 0; j < n; ++j) {
            long double c;
            if (kind == 0) {
                c = 2.0L * cosl(pi * ((long double)j + 0.5L) * (long double)k / (long double)n);
            } else {
                c = (j == 0) ? 1.0L
                             : 2.0L * cosl(pi * (long double)j * ((long double)k + 0.5L) / (long double)n);
            }
            t[k * n + j] = c;
        }
    }
    return t;
}

oracle_dct_plan *oracle_dct_plan_create(int n0, int n1, int n2, int kind)
{
    oracle_dct_plan *p = (oracle_dct_plan *)calloc(1, sizeof(*p));
    p->n[0] = n0;
    p->n[1] = n1;
    p->n[2] = n2;
    p->kind = kind;
    for (int a = 0; a < 3; ++a) p->tab[a] = make_table(p->n[a], kind);
    return p;
}

void oracle_dct_plan_destroy(oracle_dct_plan *p)
{
    if (!p) return;
    for (int a = 0; a < 3; ++a) free(p->tab[a]);
    free(p);
}

/* Transform one axis of a long-double buffer. `stride` is the distance
 * between consecutive elements along the axis, `count`/`outer` enumerate the
 * lines. ACC is the accumulation type. */
#define DEFINE_AXIS(NAME, ACC)                                                        \
    static void NAME(ACC *buf, const long double *tab, int n, int stride, int inner,  \
                     int outer)                                                       \
    {                                                                                 \
        ACC line[64];                                                                 \
        ACC *tmp = n <= 64 ? line : (ACC *)malloc(sizeof(ACC) * (size_t)n);           \
        for (int o = 0; o < outer; ++o) {                                             \
            for (int in = 0; in < inner; ++in) {                                      \
                ACC *base = buf + (size_t)o * (size_t)n * (size_t)stride + in;        \
                for (int k = 0; k < n; ++k) {                                         \
                    ACC s = 0;                                                        \
                    const long double *row = tab + (size_t)k * (size_t)n;             \
                    for (int j = 0; j < n; ++j) s += (ACC)row[j] * base[(size_t)j * stride]; \
                    tmp[k] = s;                                                       \
                }                                                                     \
                for (int k = 0; k < n; ++k) base[(size_t)k * stride] = tmp[k];        \
            }                                                                         \
        }                                                                             \
        if (tmp != line) free(tmp);                                                   \
    }

DEFINE_AXIS(axis_f64acc, double)
DEFINE_AXIS(axis_f80acc, long double)

/* FP32 variants for the self-divergence envelope: the same definitions
 * evaluated in float, each axis rounded to float before the next, with the
 * cosines rounded to float -- as an FP32 FFT library's codelets compute.
 * order 0 sums the terms of each output from the first input up, order 1
 * from the last input down, order 2 pairwise (a balanced tree, the way
 * butterfly stages combine partial sums). */
static float pairwise_f32(const float *t, int n)
{
    if (n == 1) return t[0];
    const int h = n / 2;
    return pairwise_f32(t, h) + pairwise_f32(t + h, n - h);
}

static void axis_f32acc(float *buf, const long double *tab, int n, int stride, int inner,
                        int outer, int order)
{
    float line[64];
    float *tmp = n <= 64 ? line : (float *)malloc(sizeof(float) * (size_t)n);
    for (int o = 0; o < outer; ++o) {
        for (int in = 0; in < inner; ++in) {
            float *base = buf + (size_t)o * (size_t)n * (size_t)stride + in;
            for (int k = 0; k < n; ++k) {
                float s = 0.0f;
                const long double *row = tab + (size_t)k * (size_t)n;
                if (order == 2) {
                    float terms[64];
                    for (int j = 0; j < n && j < 64; ++j) terms[j] = (float)row[j] * base[(size_t)j * stride];
                    s = pairwise_f32(terms, n < 64 ? n : 64);
                } else if (order == 1) {
                    for (int j = n - 1; j >= 0; --j) s += (float)row[j] * base[(size_t)j * stride];
                } else {
                    for (int j = 0; j < n; ++j) s += (float)row[j] * base[(size_t)j * stride];
                }
                tmp[k] = s;
            }
            for (int k = 0; k < n; ++k) base[(size_t)k * stride] = tmp[k];
        }
    }
    if (tmp != line) free(tmp);
}

static int g_f32_mode = 0;

void oracle_dct_set_f32_mode(int mode) { g_f32_mode = (mode >= 0 && mode <= 3) ? mode : 0; }
int oracle_dct_get_f32_mode(void) { return g_f32_mode; }

static void exec_f32_float(const oracle_dct_plan *p, float *data, int order)
{
    const int n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
    axis_f32acc(data, p->tab[2], n2, 1, 1, n0 * n1, order);
    axis_f32acc(data, p->tab[1], n1, n2, n2, n0, order);
    axis_f32acc(data, p->tab[0], n0, n1 * n2, n1 * n2, 1, order);
}

#define DEFINE_EXEC(NAME, T, ACC, AXIS)                                         \
    void NAME(const oracle_dct_plan *p, T *data)                                \
    {                                                                           \
        const int n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];                     \
        const size_t total = (size_t)n0 * (size_t)n1 * (size_t)n2;              \
        ACC stackbuf[4096];                                                     \
        ACC *buf = total <= 4096 ? stackbuf : (ACC *)malloc(sizeof(ACC) * total); \
        for (size_t i = 0; i < total; ++i) buf[i] = (ACC)data[i];               \
        AXIS(buf, p->tab[2], n2, 1, 1, n0 * n1);   /* along x (n2) */           \
        AXIS(buf, p->tab[1], n1, n2, n2, n0);      /* along y (n1) */           \
        AXIS(buf, p->tab[0], n0, n1 * n2, n1 * n2, 1); /* along z (n0) */       \
        for (size_t i = 0; i < total; ++i) data[i] = (T)buf[i];                 \
        if (buf != stackbuf) free(buf);                                         \
    }

DEFINE_EXEC(exec_f32_double, float, double, axis_f64acc)

void oracle_dct_exec_f32(const oracle_dct_plan *p, float *data)
{
    if (g_f32_mode == 0) exec_f32_double(p, data);
    else exec_f32_float(p, data, g_f32_mode - 1);
}
DEFINE_EXEC(oracle_dct_exec_f64, double, long double, axis_f80acc)
DEFINE_EXEC(oracle_dct_exec_f80, long double, long double, axis_f80acc)
