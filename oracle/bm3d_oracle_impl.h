/* Oracle (test infrastructure only): body of the C restatement, included by
 * bm3d_oracle.c once per floating-point type with FLT (the reference's FLType,
 * include/Type.h:26-30), SFX (name suffix) and DCT_EXEC (the matching
 * oracle_dct_exec_*) defined. */

#define CAT_(a, b) a##_##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SFX)

typedef struct {
    FLT key;
    int y, x;
} FN(match_t);

/* KeyPair ordering (include/Type.h:449-452): key only. */
static int FN(key_less)(const FN(match_t) *a, const FN(match_t) *b) { return a->key < b->key; }

/* libstdc++ std::__adjust_heap / std::__push_heap with a key-only "<". */
static void FN(push_heap)(FN(match_t) *a, long hole, long top, FN(match_t) value)
{
    long parent = (hole - 1) / 2;
    while (hole > top && FN(key_less)(&a[parent], &value)) {
        a[hole] = a[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a[hole] = value;
}

static void FN(adjust_heap)(FN(match_t) *a, long hole, long len, FN(match_t) value)
{
    const long top = hole;
    long child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (FN(key_less)(&a[child], &a[child - 1])) child--;
        a[hole] = a[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        a[hole] = a[child - 1];
        hole = child - 1;
    }
    FN(push_heap)(a, hole, top, value);
}

/* std::partial_sort(first, first + m, first + n) as libstdc++ implements it:
 * __heap_select (make_heap on [0,m), then pop the top for every later element
 * that compares less than it) followed by __sort_heap. The reference calls it
 * at include/Block.h:694 when more than GroupSize blocks match. */
static void FN(partial_sort)(FN(match_t) *a, long m, long n)
{
    if (m > 1) { /* __make_heap */
        long parent = (m - 2) / 2;
        for (;;) {
            FN(adjust_heap)(a, parent, m, a[parent]);
            if (parent == 0) break;
            parent--;
        }
    }
    for (long i = m; i < n; ++i) {
        if (FN(key_less)(&a[i], &a[0])) { /* __pop_heap(first, middle, i) */
            FN(match_t) v = a[i];
            a[i] = a[0];
            FN(adjust_heap)(a, 0, m, v);
        }
    }
    for (long last = m; last > 1;) { /* __sort_heap */
        --last;
        FN(match_t) v = a[last];
        a[last] = a[0];
        FN(adjust_heap)(a, 0, last, v);
    }
}

/* std::stable_sort by key (include/Block.h:699): any stable sort gives the
 * same order; insertion sort keeps ties in input (raster) order. */
static void FN(stable_sort)(FN(match_t) *a, long n)
{
    for (long i = 1; i < n; ++i) {
        FN(match_t) v = a[i];
        long j = i;
        while (j > 0 && FN(key_less)(&v, &a[j - 1])) {
            a[j] = a[j - 1];
            --j;
        }
        a[j] = v;
    }
}

/* Block::_SearchBoundary (include/Block.h:716-746). */
static int FN(search_boundary)(int pos, int plane_boundary, int search_range, int search_step)
{
    int b;
    search_range = search_range / search_step * search_step;
    if (pos == plane_boundary) {
        b = plane_boundary;
    } else if (pos > plane_boundary) {
        b = pos - search_range;
        while (b < plane_boundary) b += search_step;
    } else {
        b = pos + search_range;
        while (b > plane_boundary) b -= search_step;
    }
    return b;
}

typedef struct {
    int block_size, block_step, group_size, bm_range, bm_step;
    double thMSE;          /* already scaled by normY (include/BM3D.h:250) */
    double sigma[3];       /* raw 0-255 sigmas, for the per-plane guards */
    double finalAMP[64];   /* indexed by group size - 1 */
    FLT *thr[3][64];       /* basic: hard-threshold table per plane and group size */
    FLT wss[3][64];        /* final: wienerSigmaSqr per plane and group size */
    oracle_dct_plan *fwd[64], *bwd[64];
    int wiener;
} FN(stage_t);

/* OPP colour-matrix norms: BM3D_Base ctor (include/BM3D.h:241-248) with the
 * coefficients of ColorMatrix_RGB2YUV_Parameter(OPP) (include/Specification.h:391-406). */
static void FN(opp_norms)(double norm[3])
{
    const double Yr = (double)(1.0L / 3.0L), Yg = (double)(1.0L / 3.0L), Yb = (double)(1.0L / 3.0L);
    const double Ur = (double)(1.0L / 2.0L), Ug = (double)(0.0L), Ub = (double)(-1.0L / 2.0L);
    const double Vr = (double)(1.0L / 4.0L), Vg = (double)(-1.0L / 2.0L), Vb = (double)(1.0L / 4.0L);
    norm[0] = sqrt(Yr * Yr + Yg * Yg + Yb * Yb);
    norm[1] = sqrt(Ur * Ur + Ug * Ug + Ub * Ub);
    norm[2] = sqrt(Vr * Vr + Vg * Vg + Vb * Vb);
}

/* BM3D_Base ctor (include/BM3D.h:237-259) + BM3D_FilterData ctor
 * (source/BM3D.cpp:9-73). */
static void FN(stage_init)(FN(stage_t) *s, int wiener, const oracle_stage_params *p)
{
    double norm[3];
    memset(s, 0, sizeof(*s));
    FN(opp_norms)(norm);
    s->wiener = wiener;
    s->block_size = p->block_size;
    s->block_step = p->block_step;
    s->group_size = p->group_size;
    s->bm_range = p->bm_range;
    s->bm_step = p->bm_step;
    s->thMSE = p->thMSE * norm[0];
    for (int c = 0; c < 3; ++c) s->sigma[c] = p->sigma[c];
    const int GS = p->group_size, BS = p->block_size;
    if (GS < 1 || GS > 64 || BS < 1) return;
    for (int i = 1; i <= GS; ++i) {
        s->fwd[i - 1] = oracle_dct_plan_create(i, BS, BS, 0);
        s->bwd[i - 1] = oracle_dct_plan_create(i, BS, BS, 1);
        s->finalAMP[i - 1] = 2 * i * 2 * BS * 2 * BS;
    }
    for (int c = 0; c < 3; ++c) {
        if (!(p->sigma[c] > 0)) continue;
        const double sigma = p->sigma[c] / (double)255 * norm[c];
        for (int i = 1; i <= GS; ++i) {
            const double forwardAMP = sqrt(s->finalAMP[i - 1]);
            if (wiener) {
                s->wss[c][i - 1] = (FLT)(sigma * forwardAMP * sigma * forwardAMP);
            } else {
                const double thrBase = sigma * p->lambda * forwardAMP;
                double thr[4];
                thr[0] = thrBase;
                thr[1] = thrBase * sqrt((double)2);
                thr[2] = thrBase * (double)2;
                thr[3] = thrBase * sqrt((double)8);
                FLT *t = (FLT *)malloc(sizeof(FLT) * (size_t)i * (size_t)BS * (size_t)BS);
                s->thr[c][i - 1] = t;
                for (int z = 0; z < i; ++z)
                    for (int y = 0; y < BS; ++y)
                        for (int x = 0; x < BS; ++x) {
                            int flag = (x == 0) + (y == 0) + (z == 0);
                            *t++ = (FLT)thr[flag];
                        }
            }
        }
    }
}

static void FN(stage_free)(FN(stage_t) *s)
{
    for (int i = 0; i < 64; ++i) {
        oracle_dct_plan_destroy(s->fwd[i]);
        oracle_dct_plan_destroy(s->bwd[i]);
        for (int c = 0; c < 3; ++c) free(s->thr[c][i]);
    }
}

/* One candidate of the per-candidate Block::BlockMatchingMulti
 * (include/Block.h:589-611): sequential row-major sum of squared differences
 * in FLType, kept iff dist <= thSSE && dist != 0, key = FLType(dist * distMul). */
static int FN(match_one)(const FLT *refb, const FLT *plane, int width, int BS, FLT thSSE,
                         double distMul, int j, int i, FN(match_t) *out)
{
    const FLT *cand = plane + (size_t)j * width + i;
    FLT dist = 0;
    for (int y = 0; y < BS; ++y)
        for (int x = 0; x < BS; ++x) {
            FLT temp = refb[(size_t)y * width + x] - cand[(size_t)y * width + x];
            dist += temp * temp;
        }
    if (dist <= thSSE && dist != 0) {
        out->key = (FLT)(dist * distMul);
        out->y = j;
        out->x = i;
        return 1;
    }
    return 0;
}

/* BM3D_Base::BlockMatching (source/BM3D.cpp:221-236) and the positional
 * Block::BlockMatchingMulti (include/Block.h:578-615, 658-703).
 * Writes the group into out (capacity >= group_size) and returns its size. */
static int FN(block_matching)(const FN(stage_t) *s, const FLT *ref, int width, int height,
                              FLT range, int j0, int i0, FN(match_t) *work, FN(match_t) *out)
{
    const int BS = s->block_size, GS = s->group_size;
    if (GS == 1 || s->thMSE <= 0) {
        out[0].key = 0;
        out[0].y = j0;
        out[0].x = i0;
        return 1;
    }
    const int step = s->bm_step;
    const int R = s->bm_range / step * step;
    const int l = FN(search_boundary)(i0, 0, R, step);
    const int r = FN(search_boundary)(i0, width - BS, R, step);
    const int t = FN(search_boundary)(j0, 0, R, step);
    const int b = FN(search_boundary)(j0, height - BS, R, step);

    const double MSE2SSE = (double)(BS * BS) * range * range / (double)(255 * 255);
    const double distMul = (double)1 / MSE2SSE;
    const FLT thSSE = (FLT)(s->thMSE * MSE2SSE);

    long n = 0;
    work[n].key = 0; /* excludeCurPos == 1: the reference block leads */
    work[n].y = j0;
    work[n].x = i0;
    ++n;
    const FLT *refb = ref + (size_t)j0 * width + i0;
    for (int j = t; j <= b; j += step) {
        for (int i = l; i <= r; i += step) {
            if (j == j0 && i == i0) continue;
            n += FN(match_one)(refb, ref, width, BS, thSSE, distMul, j, i, &work[n]);
        }
    }
    /* include/Block.h:668-682 sizes search_pos for the whole grid, the
     * reference block included, but skips the reference block while filling
     * it; the last slot keeps its value-initialised Pos(0, 0), and
     * include/Block.h:589 then matches that slot like any other candidate.
     * So the block at (0, 0) is always evaluated once more, last. */
    n += FN(match_one)(refb, ref, width, BS, thSSE, distMul, 0, 0, &work[n]);
    if (GS > 0 && n > GS) {
        FN(partial_sort)(work, GS, n);
        n = GS;
    } else {
        FN(stable_sort)(work, n);
    }
    for (long k = 0; k < n; ++k) out[k] = work[k];
    return (int)n;
}

/* BM3D_Basic::CollaborativeFilter (source/BM3D.cpp:339-385) and
 * BM3D_Final::CollaborativeFilter (source/BM3D.cpp:411-457), with
 * BlockGroup::From / AddTo / CountTo (include/Block.h:1114-1133, 1240-1265,
 * 1334-1357). */
static void FN(collaborative_filter)(const FN(stage_t) *s, int plane, FLT *num, FLT *den,
                                     const FLT *src, const FLT *ref, int width,
                                     const FN(match_t) *code, int code_size, FLT *gs, FLT *gr)
{
    const int BS = s->block_size;
    int n = code_size;
    if (s->group_size > 0 && n > s->group_size) n = s->group_size;
    const size_t bsz = (size_t)BS * BS;
    for (int z = 0; z < n; ++z) {
        const FLT *ps = src + (size_t)code[z].y * width + code[z].x;
        const FLT *pr = ref + (size_t)code[z].y * width + code[z].x;
        for (int y = 0; y < BS; ++y)
            for (int x = 0; x < BS; ++x) {
                gs[z * bsz + y * BS + x] = ps[(size_t)y * width + x];
                if (s->wiener) gr[z * bsz + y * BS + x] = pr[(size_t)y * width + x];
            }
    }
    const size_t total = (size_t)n * bsz;
    FLT denWeight;
    DCT_EXEC(s->fwd[n - 1], gs);
    if (!s->wiener) {
        int retained = 0;
        const FLT *thr = s->thr[plane][n - 1];
        for (size_t k = 0; k < total; ++k) {
            FLT x = gs[k];
            FLT ax = x < 0 ? -x : x;
            if (ax <= thr[k]) gs[k] = 0;
            else ++retained;
        }
        DCT_EXEC(s->bwd[n - 1], gs);
        denWeight = retained < 1 ? 1 : (FLT)1 / (FLT)retained;
    } else {
        DCT_EXEC(s->fwd[n - 1], gr);
        const FLT sigmaSquare = s->wss[plane][n - 1];
        FLT L2 = 0;
        for (size_t k = 0; k < total; ++k) {
            FLT ySquare = gr[k] * gr[k];
            FLT w = ySquare / (ySquare + sigmaSquare);
            gs[k] *= w;
            L2 += w * w;
        }
        DCT_EXEC(s->bwd[n - 1], gs);
        denWeight = L2 <= 0 ? 1 : (FLT)1 / L2;
    }
    const FLT numWeight = (FLT)(denWeight / s->finalAMP[n - 1]);
    for (int z = 0; z < n; ++z) {
        FLT *pn = num + (size_t)code[z].y * width + code[z].x;
        FLT *pd = den + (size_t)code[z].y * width + code[z].x;
        for (int y = 0; y < BS; ++y)
            for (int x = 0; x < BS; ++x) {
                pn[(size_t)y * width + x] += (FLT)(gs[z * bsz + y * BS + x] * numWeight);
                pd[(size_t)y * width + x] += denWeight;
            }
    }
}

static int FN(params_rejected)(const FN(stage_t) *s, int three)
{
    int sig = three ? (s->sigma[0] <= 0 && s->sigma[1] <= 0 && s->sigma[2] <= 0) : (s->sigma[0] <= 0);
    return sig || s->group_size == 0 || s->block_size <= 0 || s->bm_range <= 0 ||
           s->bm_range < s->bm_step || s->thMSE <= 0;
}

/* BM3D_Base::Kernel, single plane (source/BM3D.cpp:80-136) and the 9-plane
 * overload (source/BM3D.cpp:139-218): the reference-block scan, block
 * matching on plane 0 of ref, collaborative filtering per plane with
 * sigma > 0, then dst = num / den. */
static int FN(run)(int wiener, const oracle_stage_params *p, int nplanes, FLT *const dst[3],
                   const FLT *const src[3], const FLT *const ref[3], int width, int height,
                   double value_range)
{
    FN(stage_t) s;
    FN(stage_init)(&s, wiener, p);
    const size_t npx = (size_t)width * height;
    if (FN(params_rejected)(&s, nplanes == 3)) {
        for (int c = 0; c < nplanes; ++c) memcpy(dst[c], src[c], sizeof(FLT) * npx);
        FN(stage_free)(&s);
        return 2;
    }
    const int BS = s.block_size, GS = s.group_size;
    FLT *num[3] = {0}, *den[3] = {0};
    int active[3];
    for (int c = 0; c < nplanes; ++c) {
        active[c] = nplanes == 1 ? 1 : (s.sigma[c] > 0);
        num[c] = (FLT *)calloc(npx, sizeof(FLT));
        den[c] = (FLT *)calloc(npx, sizeof(FLT));
    }
    const long cap = 4L * (s.bm_range + 1) * (s.bm_range + 1) + 2;
    FN(match_t) *work = (FN(match_t) *)malloc(sizeof(FN(match_t)) * (size_t)cap);
    FN(match_t) *code = (FN(match_t) *)malloc(sizeof(FN(match_t)) * (size_t)(GS > 0 ? GS : 1));
    FLT *gs = (FLT *)malloc(sizeof(FLT) * (size_t)(GS > 0 ? GS : 1) * BS * BS);
    FLT *gr = (FLT *)malloc(sizeof(FLT) * (size_t)(GS > 0 ? GS : 1) * BS * BS);
    const FLT range = (FLT)value_range;
    const int right = width - BS, bottom = height - BS;
    for (int j = 0;; j += s.block_step) {
        if (j >= bottom + s.block_step) break;
        if (j > bottom) j = bottom;
        for (int i = 0;; i += s.block_step) {
            if (i >= right + s.block_step) break;
            if (i > right) i = right;
            int n = FN(block_matching)(&s, ref[0], width, height, range, j, i, work, code);
            for (int c = 0; c < nplanes; ++c)
                if (active[c])
                    FN(collaborative_filter)(&s, c, num[c], den[c], src[c], ref[c], width, code, n,
                                             gs, gr);
        }
    }
    for (int c = 0; c < nplanes; ++c) {
        if (active[c])
            for (size_t k = 0; k < npx; ++k) dst[c][k] = num[c][k] / den[c][k];
        free(num[c]);
        free(den[c]);
    }
    free(work);
    free(code);
    free(gs);
    free(gr);
    FN(stage_free)(&s);
    return 0;
}

int FN(oracle_bm3d_stage)(int wiener, const oracle_stage_params *p, FLT *dst, const FLT *src,
                          const FLT *ref, int width, int height, double value_range)
{
    FLT *d[3] = {dst, 0, 0};
    const FLT *sp[3] = {src, 0, 0};
    const FLT *rp[3] = {ref, 0, 0};
    return FN(run)(wiener, p, 1, d, sp, rp, width, height, value_range);
}

int FN(oracle_bm3d_stage3)(int wiener, const oracle_stage_params *p, FLT *const dst[3],
                           const FLT *const src[3], const FLT *const ref[3], int width, int height,
                           double value_range)
{
    return FN(run)(wiener, p, 3, dst, src, ref, width, height, value_range);
}

long long FN(oracle_bm3d_groups)(int wiener, const oracle_stage_params *p, const FLT *ref,
                                 int width, int height, double value_range, int max_refs,
                                 int max_group, int *counts, int *pos_yx, FLT *keys)
{
    FN(stage_t) s;
    FN(stage_init)(&s, wiener, p);
    const int BS = s.block_size, GS = s.group_size;
    const long cap = 4L * (s.bm_range + 1) * (s.bm_range + 1) + 2;
    FN(match_t) *work = (FN(match_t) *)malloc(sizeof(FN(match_t)) * (size_t)cap);
    FN(match_t) *code = (FN(match_t) *)malloc(sizeof(FN(match_t)) * (size_t)(GS > 0 ? GS : 1));
    const FLT range = (FLT)value_range;
    const int right = width - BS, bottom = height - BS;
    long long r = 0;
    for (int j = 0;; j += s.block_step) {
        if (j >= bottom + s.block_step) break;
        if (j > bottom) j = bottom;
        for (int i = 0;; i += s.block_step) {
            if (i >= right + s.block_step) break;
            if (i > right) i = right;
            int n = FN(block_matching)(&s, ref, width, height, range, j, i, work, code);
            if (r < max_refs) {
                counts[r] = n;
                for (int z = 0; z < n && z < max_group; ++z) {
                    pos_yx[(r * max_group + z) * 2 + 0] = code[z].y;
                    pos_yx[(r * max_group + z) * 2 + 1] = code[z].x;
                    keys[r * max_group + z] = code[z].key;
                }
            }
            ++r;
        }
    }
    free(work);
    free(code);
    FN(stage_free)(&s);
    return r;
}

/* ---- integer planes and RGB frames ---------------------------------------
 * The float planes are the reference's default Plane_FL ranges: luma [0, 1],
 * chroma [-0.5, 0.5] (include/Image_Type.cpp:407-421, Image_Type.hpp:184-202).
 */

/* MatrixConvert_RGB2YUV with ColorMatrix::OPP to a float destination, no
 * clipping (include/Conversion.hpp:518-575); `only_y` is ConvertToY
 * (include/Conversion.hpp:398-430), whose Y formula is the same. RGB planes
 * have Floor = Neutral = floor_. */
static void FN(rgb_to_opp)(FLT *const yuv[3], const int *const rgb[3], size_t npx, int floor_,
                           int ceil_, int only_y)
{
    const int sRange = ceil_ - floor_;
    const FLT dRangeY = (FLT)1, dRangeC = (FLT)0.5 - (FLT)-0.5, dFloorY = 0, dNeutralC = 0;
    const FLT gainY = dRangeY / ((FLT)sRange * (FLT)3);
    const FLT offsetY = -(FLT)floor_ * (FLT)3 * gainY + dFloorY;
    const FLT gainU = dRangeC / ((FLT)sRange * (FLT)2);
    const FLT gainV = dRangeC / ((FLT)sRange * (FLT)4);
    const FLT offsetC = dNeutralC;
    for (size_t i = 0; i < npx; ++i) {
        const FLT r = (FLT)rgb[0][i], g = (FLT)rgb[1][i], b = (FLT)rgb[2][i];
        yuv[0][i] = (r + g + b) * gainY + offsetY;
        if (only_y) continue;
        yuv[1][i] = (r - b) * gainU + offsetC;
        yuv[2][i] = (r - g * (FLT)2 + b) * gainV + offsetC;
    }
}

/* MatrixConvert_YUV2RGB with ColorMatrix::OPP from the float planes to
 * integers in [floor_, ceil_], clipped, +0.5 and truncated
 * (include/Conversion.hpp:661-748; coefficients include/Specification.h:
 * 468-484). */
static void FN(opp_to_rgb)(int *const rgb[3], const FLT *const yuv[3], size_t npx, int floor_,
                           int ceil_)
{
    const int dRange = ceil_ - floor_;
    const FLT sRangeY = (FLT)1 - (FLT)0, sRangeC = (FLT)0.5 - (FLT)-0.5;
    const FLT gY = (FLT)dRange / sRangeY, gC = (FLT)dRange / sRangeC;
    const FLT Ry = (FLT)(1.0L) * gY, Ru = (FLT)(1.0L) * gC, Rv = (FLT)(2.0L / 3.0L) * gC;
    const FLT Gy = (FLT)(1.0L) * gY, Gu = (FLT)(0.0L) * gC, Gv = (FLT)(-4.0L / 3.0L) * gC;
    const FLT By = (FLT)(1.0L) * gY, Bu = (FLT)(-1.0L) * gC, Bv = (FLT)(2.0L / 3.0L) * gC;
    const FLT sFloorY = 0, sNeutralC = 0;
    const FLT offR = -sFloorY * Ry - sNeutralC * (Ru + Rv) + (FLT)floor_ + (FLT)0.5;
    const FLT offG = -sFloorY * Gy - sNeutralC * (Gu + Gv) + (FLT)floor_ + (FLT)0.5;
    const FLT offB = -sFloorY * By - sNeutralC * (Bu + Bv) + (FLT)floor_ + (FLT)0.5;
    const FLT lo = (FLT)floor_, hi = (FLT)ceil_;
    for (size_t i = 0; i < npx; ++i) {
        const FLT y = yuv[0][i], u = yuv[1][i], v = yuv[2][i];
        FLT t;
        t = Ry * y + Ru * u + Rv * v + offR;
        rgb[0][i] = (int)(t <= lo ? lo : t >= hi ? hi : t);
        t = Gy * y + Gv * v + offG;
        rgb[1][i] = (int)(t <= lo ? lo : t >= hi ? hi : t);
        t = By * y + Bu * u + Bv * v + offB;
        rgb[2][i] = (int)(t <= lo ? lo : t >= hi ? hi : t);
    }
}

/* RangeConvert from an integer plane (floor_, neutral, ceil_) to the float
 * plane of range 1, no clipping except for full-range chroma
 * (include/Conversion.hpp:134-254, different-range branch). */
static void FN(int_to_fl)(FLT *dst, const int *src, size_t npx, int floor_, int neutral, int ceil_)
{
    const int chroma = floor_ < neutral;
    const int pc_chroma = chroma && (floor_ + ceil_) % 2 == 1;
    const FLT fFloor = chroma ? (FLT)-0.5 : (FLT)0, fCeil = chroma ? (FLT)0.5 : (FLT)1;
    const FLT fNeutral = 0;
    const int sRange = ceil_ - floor_;
    const FLT dRange = fCeil - fFloor;
    const FLT gain = dRange / (FLT)sRange;
    const FLT offset = -(FLT)neutral * gain + fNeutral;
    for (size_t i = 0; i < npx; ++i) {
        const FLT t = (FLT)src[i] * gain + offset;
        dst[i] = pc_chroma ? (t <= fFloor ? fFloor : t >= fCeil ? fCeil : t) : t;
    }
}

/* RangeConvert back: clipped to [floor_, ceil_] after +0.5 (+0.499999 for
 * full-range chroma), truncated. */
static void FN(fl_to_int)(int *dst, const FLT *src, size_t npx, int floor_, int neutral, int ceil_)
{
    const int chroma = floor_ < neutral;
    const int pc_chroma = chroma && (floor_ + ceil_) % 2 == 1;
    const FLT fFloor = chroma ? (FLT)-0.5 : (FLT)0, fCeil = chroma ? (FLT)0.5 : (FLT)1;
    const FLT fNeutral = 0;
    const FLT sRange = fCeil - fFloor;
    const int dRange = ceil_ - floor_;
    const FLT gain = (FLT)dRange / sRange;
    const FLT offset = -fNeutral * gain + (FLT)neutral + (pc_chroma ? (FLT)0.499999 : (FLT)0.5);
    const FLT lo = (FLT)floor_, hi = (FLT)ceil_;
    for (size_t i = 0; i < npx; ++i) {
        const FLT t = src[i] * gain + offset;
        dst[i] = (int)(t <= lo ? lo : t >= hi ? hi : t);
    }
}

/* The guard of the stage-level integer and Frame paths
 * (source/BM3D.cpp:250-256, 286-293): GroupSize == 1 (not 0) copies. */
static int FN(int_path_rejected)(const oracle_stage_params *p, int nplanes)
{
    const int sig = nplanes == 1 ? p->sigma[0] > 0
                                 : (p->sigma[0] > 0 || p->sigma[1] > 0 || p->sigma[2] > 0);
    return !sig || p->group_size == 1 || p->block_size <= 0 || p->bm_range <= 0 ||
           p->bm_range < p->bm_step || p->thMSE <= 0;
}

static FLT *FN(alloc)(size_t npx) { return (FLT *)malloc(sizeof(FLT) * (npx ? npx : 1)); }

/* BM3D::process_Frame (source/BM3D.cpp:501-527): OPP RGB->YUV, three-plane
 * basic then final (final in place on the YUV source), YUV->RGB; a ref frame
 * (may be null) gives the basic stage its Y to match on. */
int FN(oracle_bm3d_frame)(const oracle_stage_params *pb, const oracle_stage_params *pf,
                          int *const dst[3], const int *const src[3], const int *const ref[3],
                          int width, int height, int floor_, int ceil_)
{
    const size_t npx = (size_t)width * height;
    FLT *yuv[3], *tmp[3], *out[3], *ry[1] = {0};
    for (int c = 0; c < 3; ++c) {
        yuv[c] = FN(alloc)(npx);
        tmp[c] = FN(alloc)(npx);
        out[c] = FN(alloc)(npx);
    }
    FN(rgb_to_opp)(yuv, src, npx, floor_, ceil_, 0);
    for (int c = 0; c < 3; ++c) {
        memcpy(tmp[c], yuv[c], sizeof(FLT) * npx);
        memcpy(out[c], yuv[c], sizeof(FLT) * npx);
    }
    const FLT *const yc[3] = {yuv[0], yuv[1], yuv[2]};
    const FLT *rc3[3] = {yuv[0], yuv[1], yuv[2]};
    if (ref) {  /* BM3D_Basic::RGB2YUV: only Y of ref (source/BM3D.cpp:333) */
        ry[0] = FN(alloc)(npx);
        FN(rgb_to_opp)(ry, ref, npx, floor_, ceil_, 1);
        rc3[0] = ry[0];
    }
    FN(oracle_bm3d_stage3)(0, pb, tmp, yc, rc3, width, height, 1.0);
    const FLT *const tc[3] = {tmp[0], tmp[1], tmp[2]};
    FN(oracle_bm3d_stage3)(1, pf, out, yc, tc, width, height, 1.0);
    FN(opp_to_rgb)(dst, (const FLT *const *)out, npx, floor_, ceil_);
    for (int c = 0; c < 3; ++c) {
        free(yuv[c]);
        free(tmp[c]);
        free(out[c]);
    }
    free(ry[0]);
    return 0;
}

/* BM3D_Base::process_Frame (source/BM3D.cpp:284-313): one stage on an RGB
 * frame, in place on the YUV source; ref (or src when null) converted by
 * the stage's RGB2YUV: Y only for the basic stage (320-336), all three
 * planes for the final stage (392-408). */
int FN(oracle_bm3d_stage_frame)(int wiener, const oracle_stage_params *p, int *const dst[3],
                                const int *const src[3], const int *const ref[3], int width,
                                int height, int floor_, int ceil_)
{
    const size_t npx = (size_t)width * height;
    if (FN(int_path_rejected)(p, 3)) {
        for (int c = 0; c < 3; ++c) memcpy(dst[c], src[c], sizeof(int) * npx);
        return 2;
    }
    FLT *yuv[3], *ryuv[3] = {0, 0, 0}, *out[3];
    for (int c = 0; c < 3; ++c) {
        yuv[c] = FN(alloc)(npx);
        out[c] = FN(alloc)(npx);
    }
    FN(rgb_to_opp)(yuv, src, npx, floor_, ceil_, 0);
    const FLT *rc3[3] = {yuv[0], yuv[1], yuv[2]};
    if (ref) {
        for (int c = 0; c < (wiener ? 3 : 1); ++c) ryuv[c] = FN(alloc)(npx);
        FN(rgb_to_opp)(ryuv, ref, npx, floor_, ceil_, !wiener);
        for (int c = 0; c < 3; ++c) rc3[c] = ryuv[wiener ? c : 0];
    }
    for (int c = 0; c < 3; ++c) memcpy(out[c], yuv[c], sizeof(FLT) * npx);
    const FLT *const yc[3] = {yuv[0], yuv[1], yuv[2]};
    FN(oracle_bm3d_stage3)(wiener, p, out, yc, rc3, width, height, 1.0);
    FN(opp_to_rgb)(dst, (const FLT *const *)out, npx, floor_, ceil_);
    for (int c = 0; c < 3; ++c) {
        free(yuv[c]);
        free(out[c]);
        free(ryuv[c]);
    }
    return 0;
}

/* Basic then final on an integer plane: BM3D::process_Plane
 * (source/BM3D.cpp:475-497) with the basic estimate sized like the source
 * (the reference's own process_Plane_FL passes a 0x0 one); the basic stage
 * matches on ref when given. */
int FN(oracle_bm3d_plane_int)(const oracle_stage_params *pb, const oracle_stage_params *pf,
                              int *dst, const int *src, const int *ref, int width, int height,
                              int floor_, int neutral, int ceil_)
{
    const size_t npx = (size_t)width * height;
    FLT *fsrc = FN(alloc)(npx), *ftmp = FN(alloc)(npx), *fdst = FN(alloc)(npx), *fref = fsrc;
    FN(int_to_fl)(fsrc, src, npx, floor_, neutral, ceil_);
    if (ref) {
        fref = FN(alloc)(npx);
        FN(int_to_fl)(fref, ref, npx, floor_, neutral, ceil_);
    }
    FN(oracle_bm3d_stage)(0, pb, ftmp, fsrc, fref, width, height, 1.0);
    if (fref != fsrc) free(fref);
    FN(oracle_bm3d_stage)(1, pf, fdst, fsrc, ftmp, width, height, 1.0);
    FN(fl_to_int)(dst, fdst, npx, floor_, neutral, ceil_);
    free(fsrc);
    free(ftmp);
    free(fdst);
    return 0;
}

/* BM3D_Base::process_Plane (source/BM3D.cpp:248-281): one stage on an
 * integer plane; ref (or src when null) converted the same way. */
int FN(oracle_bm3d_stage_int)(int wiener, const oracle_stage_params *p, int *dst, const int *src,
                              const int *ref, int width, int height, int floor_, int neutral,
                              int ceil_)
{
    const size_t npx = (size_t)width * height;
    if (FN(int_path_rejected)(p, 1)) {
        memcpy(dst, src, sizeof(int) * npx);
        return 2;
    }
    FLT *fsrc = FN(alloc)(npx), *fref = fsrc, *fdst = FN(alloc)(npx);
    FN(int_to_fl)(fsrc, src, npx, floor_, neutral, ceil_);
    if (ref) {
        fref = FN(alloc)(npx);
        FN(int_to_fl)(fref, ref, npx, floor_, neutral, ceil_);
    }
    FN(oracle_bm3d_stage)(wiener, p, fdst, fsrc, fref, width, height, 1.0);
    FN(fl_to_int)(dst, fdst, npx, floor_, neutral, ceil_);
    if (fref != fsrc) free(fref);
    free(fsrc);
    free(fdst);
    return 0;
}

#undef FN
#undef CAT
#undef CAT_
