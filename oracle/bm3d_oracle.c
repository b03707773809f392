/* Oracle (test infrastructure only): C restatement of the reference's BM3D
 * path; the body lives in bm3d_oracle_impl.h and is instantiated for the
 * reference's two FLType builds (float under _CUDA_, double otherwise). */
#include "bm3d_oracle.h"
#include "dct_ref.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define FLT float
#define SFX f32
#define DCT_EXEC oracle_dct_exec_f32
#include "bm3d_oracle_impl.h"
#undef FLT
#undef SFX
#undef DCT_EXEC

#define FLT double
#define SFX f64
#define DCT_EXEC oracle_dct_exec_f64
#include "bm3d_oracle_impl.h"
#undef FLT
#undef SFX
#undef DCT_EXEC

void oracle_partial_sort_f32(float *keys, int *payload, int m, int n)
{
    match_t_f32 *a = (match_t_f32 *)malloc(sizeof(match_t_f32) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) {
        a[i].key = keys[i];
        a[i].y = payload[i];
        a[i].x = 0;
    }
    partial_sort_f32(a, m, n);
    for (int i = 0; i < n; ++i) {
        keys[i] = a[i].key;
        payload[i] = a[i].y;
    }
    free(a);
}
