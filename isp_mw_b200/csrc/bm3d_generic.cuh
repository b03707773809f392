// Generic BM3D stage kernel: any BlockSize <= 16, GroupSize <= 32, BMrange,
// BMstep -- the reference's other profiles ("np", "high", "vn") and custom
// parameters. One warp per reference block; the group lives in shared memory
// and the separable 3-D transforms run one line per lane: 8-point butterflies
// for BlockSize 8, recursive even/odd splits for full GroupSize-32 groups,
// cosine matrices from global memory otherwise. Block matching keeps the
// reference's exact distance order (BlockSize 8 with step 1 uses the
// register-resident kernel's strips); selection, aggregation and the staged
// windows are shared with the register-resident kernel.
//
// Reference: as bm3d_stage.cuh (source/BM3D.cpp:80-457, include/Block.h:578-751).
#pragma once

#include "bm3d_stage.cuh"

namespace bm3d {

// FP32 cosine matrices of length 11 (row k = output k) for BlockSize 11 rows
// and columns (the "vn" final stage): every coefficient a constant-bank
// operand. Each translation unit has its own copy, filled by the host when a
// context is made.
static __constant__ float c_dct11_fwd[11 * 11];
static __constant__ float c_dct11_inv[11 * 11];

// In-place length-n transform of one strided line, by one lane: out[k] =
// sum_j mat[k n + j] in[j] (row k = output k), n <= kGSTab.
template <typename T>
__device__ __forceinline__ void dct_line(T *base, int stride, int n, const T *mat)
{
    T in[kGSTab];
#pragma unroll
    for (int j = 0; j < kGSTab; ++j) in[j] = j < n ? base[j * stride] : T(0);
    for (int k = 0; k < n; ++k) {
        const T *row = mat + k * n;
        T acc = T(0);
#pragma unroll
        for (int j = 0; j < kGSTab; ++j)
            if (j < n) acc += __ldg(row + j) * in[j];
        base[k * stride] = acc;
    }
}

// One 8-point line of an 8 x 8 block, in place, by the butterflies of dct.cuh.
template <typename T>
__device__ __forceinline__ void dct_line8(T *base, int stride, bool inverse)
{
    T v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = base[j * stride];
    if (inverse) redft01_8(v);
    else redft10_8(v);
#pragma unroll
    for (int j = 0; j < 8; ++j) base[j * stride] = v[j];
}

// One 11-point line (FP32), in place, by the symmetric form with
// constant-bank cosines; other precisions never reach it.
template <typename T>
__device__ __forceinline__ void dct_line11(T *base, int stride, bool inverse)
{
    if constexpr (sizeof(T) == 4) {
        T v[11];
#pragma unroll
        for (int j = 0; j < 11; ++j) v[j] = base[j * stride];
        if (inverse) redft01_line<T, 11>(v, c_dct11_inv);
        else redft10_line<T, 11>(v, c_dct11_fwd);
#pragma unroll
        for (int j = 0; j < 11; ++j) base[j * stride] = v[j];
    }
}

template <typename T>
__device__ void dct_z_generic(T *G, int n, int bs, int lane, const T *tab, bool inverse);

// Separable 3-D transform of an n x bs x bs group (row-major [z][y][x]) with
// the concatenated matrices `tab` (forward REDFT10 or backward REDFT01, as
// `inverse` says): rows, columns, then the group axis. The row-fused block
// sizes (rows_fused) do not come here: their rows are transformed as they are
// gathered or aggregated, their other passes in dct_cols_z_fwd /
// dct_z_cols_inv.
template <typename T>
__device__ void dct3_generic(T *G, int n, int bs, int lane, const T *tab, bool inverse)
{
    const int bsq = bs * bs;
    if (sizeof(T) == 4 && bs == 11) {
        for (int line = lane; line < n * 11; line += kWarp)  // along x
            dct_line11(G + line * 11, 1, inverse);
        __syncwarp();
        for (int line = lane; line < n * 11; line += kWarp) {  // along y
            const int z = line / 11, x = line - z * 11;
            dct_line11(G + z * 121 + x, 11, inverse);
        }
    } else {
        const T *mb = tab + dct_table_offset(bs);
        for (int line = lane; line < n * bs; line += kWarp)  // along x
            dct_line(G + line * bs, 1, bs, mb);
        __syncwarp();
        for (int line = lane; line < n * bs; line += kWarp) {  // along y
            const int z = line / bs, x = line - z * bs;
            dct_line(G + z * bsq + x, bs, bs, mb);
        }
    }
    __syncwarp();
    dct_z_generic(G, n, bs, lane, tab, inverse);
}

// Row-fused block sizes: 8 (both precisions) and 11 (FP32, the "vn" final
// stage). Rows are transformed in registers as they are gathered
// (gather_rows) or aggregated (aggregate_rows); these run the other passes.
template <typename T> __host__ __device__ constexpr bool rows_fused(int bs)
{
    return bs == 8 || (bs == 11 && sizeof(T) == 4);
}

// One line of BS points, in place, by the block size's butterflies or
// constant-bank symmetric form.
template <typename T, int BS>
__device__ __forceinline__ void dct_line_bs(T *base, int stride, bool inverse)
{
    if constexpr (BS == 8) dct_line8(base, stride, inverse);
    else dct_line11(base, stride, inverse);
}

// Forward, after gather_rows (which transformed the rows): the columns, then
// the group axis -- the passes and order of dct3_generic.
template <typename T, int BS>
__device__ void dct_cols_z_fwd(T *G, int n, int lane, const T *tab)
{
    constexpr int ZS = BS == 8 ? 72 : BS * BS, RS = BS == 8 ? 9 : BS;
    for (int line = lane; line < n * BS; line += kWarp) {  // along y
        const int z = line / BS, x = line - z * BS;
        dct_line_bs<T, BS>(G + z * ZS + x, RS, false);
    }
    __syncwarp();
    dct_z_generic(G, n, BS, lane, tab, false);
}

// Inverse: the group axis, then the columns; the rows are transformed by
// aggregate_rows as it adds them (the register-resident kernel's inverse
// order).
template <typename T, int BS>
__device__ void dct_z_cols_inv(T *G, int n, int lane, const T *tab)
{
    constexpr int ZS = BS == 8 ? 72 : BS * BS, RS = BS == 8 ? 9 : BS;
    dct_z_generic(G, n, BS, lane, tab, true);
    for (int line = lane; line < n * BS; line += kWarp) {  // along y
        const int z = line / BS, x = line - z * BS;
        dct_line_bs<T, BS>(G + z * ZS + x, RS, true);
    }
    __syncwarp();
}

// The group-axis pass of a separable 3-D transform (see dct3_generic).
template <typename T>
__device__ void dct_z_generic(T *G, int n, int bs, int lane, const T *tab, bool inverse)
{
    // along the group: pencil p = (y, x) of every block
    const int bsq = bs * bs;
    const int zs = generic_block_stride(bs), rs = generic_row_stride(bs);
    if constexpr (sizeof(T) == 4) {
        if (n == 32) {  // full GroupSize-32 groups: recursive even/odd splits (dct.cuh)
            for (int line = lane; line < bsq; line += kWarp) {
                const int py = line / bs;
                T *g = G + py * rs + (line - py * bs);
                T v[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] = g[j * zs];
                if (inverse) redft01_pow2<T, 32>(v);
                else redft10_pow2<T, 32>(v);
#pragma unroll
                for (int k = 0; k < 32; ++k) g[k * zs] = v[k];
            }
            __syncwarp();
            return;
        }
    }
    const T *mz = tab + dct_table_offset(n);
    for (int line = lane; line < bsq; line += kWarp) {
        const int py = line / bs;
        dct_line(G + py * rs + (line - py * bs), zs, n, mz);
    }
    __syncwarp();
}

// Block matching of (j0, i0) for any block size and search step: one lane per
// candidate, sequential row-major distances against a copy of the reference
// block (include/Block.h:589-611), then the shared ordered selection.
template <typename T>
__device__ int match_generic(const StageArgs<T> &a, const Tile<T> &t, int j0, int i0, int lane,
                             SortKey<T> *keys, T *refblk, SortKey<T> *heap, BlockPos *list,
                             T *lkeys, unsigned &n_cand, unsigned &n_fix)
{
    using K = SortKey<T>;
    if (!a.match) {
        if (lane == 0) {
            list[0] = BlockPos{j0, i0};
            lkeys[0] = T(0);
        }
        __syncwarp();
        return 1;
    }
    const int bs = t.bs, bsq = bs * bs;
    const int st = a.bm_step, R = a.range;
    const int right = a.width - bs, bottom = a.height - bs;
    const int l = search_boundary(i0, 0, R, st), r = search_boundary(i0, right, R, st);
    const int tp = search_boundary(j0, 0, R, st), b = search_boundary(j0, bottom, R, st);
    const int nr = (b - tp) / st + 1, nc = (r - l) / st + 1;
    const int ngrid = nr * nc;
    {
        const T *rb = t.refw[0] + (j0 - t.ry0) * t.pitch + (i0 - t.rx0);
        for (int e = lane; e < bsq; e += kWarp) {
            const int y = e / bs;
            refblk[e] = rb[y * t.pitch + (e - y * bs)];
        }
    }
    __syncwarp();
    for (int c = lane; c <= ngrid; c += kWarp) {
        const T *cand;
        int cp;
        bool self = false;
        if (c < ngrid) {
            const int rr = c / nc, cc = c - rr * nc;
            const int cy = tp + rr * st, cx = l + cc * st;
            self = (cy == j0 && cx == i0);
            cand = t.refw[0] + (cy - t.ry0) * t.pitch + (cx - t.rx0);
            cp = t.pitch;
        } else {
            cand = block_ptr(t, t.refw[0], t.ref0[0], 0, 0, cp);  // the trailing (0, 0) slot
        }
        T d = T(0);
        if (bs == 11) {  // the same order, unrolled
#pragma unroll
            for (int y = 0; y < 11; ++y)
#pragma unroll
                for (int x = 0; x < 11; ++x) {
                    const T df = sub_rn(refblk[y * 11 + x], cand[y * cp + x]);
                    d = add_rn(d, mul_rn(df, df));
                }
        } else {
            for (int y = 0; y < bs; ++y)
                for (int x = 0; x < bs; ++x) {
                    const T df = sub_rn(refblk[y * bs + x], cand[y * cp + x]);
                    d = add_rn(d, mul_rn(df, df));
                }
        }
        const bool ok = !self && d <= a.thSSE && d != T(0);
        keys[c] = ok ? K::make(key_from_dist(d, a.distMul), static_cast<unsigned>(c)) : K::invalid();
    }
    __syncwarp();
    n_cand += static_cast<unsigned>(ngrid);
    return select_group<T>(a, keys, ngrid, nc, tp, l, st, j0, i0, lane, heap, list, lkeys, n_fix);
}

// Element e of a group stored [z][y][x]: shifts for BlockSize 8, divisions
// otherwise.
__device__ __forceinline__ void group_index(int e, int bs, int bsq, int &z, int &y, int &x)
{
    if (bs == 8) {
        z = e >> 6;
        y = (e >> 3) & 7;
        x = e & 7;
    } else if (bs == 11) {  // constant divisors
        z = e / 121;
        const int rem = e - z * 121;
        y = rem / 11;
        x = rem - y * 11;
    } else {
        z = e / bsq;
        const int rem = e - z * bsq;
        y = rem / bs;
        x = rem - y * bs;
    }
}

// Gather the group's block rows and transform each along x in registers as
// it arrives (the rows pass of the forward transform), into G's layout (row
// stride RS, block stride ZS; row z * BS + y starts at its index times RS).
// Members outside the tile (never, by construction) read as zero blocks and
// are counted in n_bad.
template <typename T, int BS>
__device__ __forceinline__ void gather_rows(const Tile<T> &t, const T *win, const T *win0,
                                            const BlockPos *list, int n, int lane, T *G,
                                            unsigned *n_bad)
{
    constexpr int RS = BS == 8 ? 9 : BS;
    for (int line = lane; line < n * BS; line += kWarp) {  // line = z * BS + y
        const int z = line / BS, y = line - z * BS;
        const BlockPos q = list[z];
        const bool ok = block_in_tile(t, q.y, q.x);
        if (n_bad && !ok && y == 0) ++*n_bad;
        T v[BS];
        if (ok) {
            int pitch;
            const T *bp = block_ptr(t, win, win0, q.y, q.x, pitch);
            bp += y * pitch;
#pragma unroll
            for (int x = 0; x < BS; ++x) v[x] = bp[x];
        } else {
#pragma unroll
            for (int x = 0; x < BS; ++x) v[x] = T(0);
        }
        if constexpr (BS == 8) redft10_8(v);
        else redft10_line<T, BS>(v, c_dct11_fwd);
        T *g = G + line * RS;
#pragma unroll
        for (int x = 0; x < BS; ++x) g[x] = v[x];
    }
}

// The rows pass of the inverse transform, each row added to the tile's sums
// as soon as it is transformed (BlockGroup::AddTo / CountTo,
// include/Block.h:1240-1265, 1334-1357); the block weight once per block, at
// its origin. Members reaching block (0, 0)'s pixels, and planes with
// non-finite pixels, take the checking per-term form.
template <typename T, int BS>
__device__ __forceinline__ void aggregate_rows(const StageArgs<T> &a, const Tile<T> &t, int p,
                                               int pt, const BlockPos *list, int n, int lane,
                                               const T *G, T numW, T denW, float scale,
                                               bool check)
{
    constexpr int RS = BS == 8 ? 9 : BS;
    for (int line = lane; line < n * BS; line += kWarp) {  // line = z * BS + y
        const int z = line / BS, y = line - z * BS;
        const BlockPos q = list[z];
        if (!block_in_tile(t, q.y, q.x)) continue;
        T v[BS];
        const T *g = G + line * RS;
#pragma unroll
        for (int x = 0; x < BS; ++x) v[x] = g[x];
        if constexpr (BS == 8) redft01_8(v);
        else redft01_line<T, BS>(v, c_dct11_inv);
        int pitch;
        auto *dn = block_ptr(t, t.accN[p], t.accN0[p], q.y, q.x, pitch);
        dn += y * pitch;
        if (!check && (q.y >= BS || q.x >= BS)) {
#pragma unroll
            for (int x = 0; x < BS; ++x) acc_add(dn + x, v[x] * numW, scale);
            if (y == 0) acc_add(block_ptr(t, t.accD[p], t.accD0[p], q.y, q.x, pitch), denW, scale);
        } else {
            const float scale_c = fixed_scale(a.absmax[pt], a.log2_corner);
            unsigned char *const poison = poison_map(a, pt);
            unsigned char *mk =
                poison ? poison + static_cast<long long>(q.y + y) * a.width + q.x : nullptr;
            for (int x = 0; x < BS; ++x) {
                const bool corner = q.y + y < BS && q.x + x < BS;
                acc_add_checked(dn + x, v[x] * numW, corner ? scale_c : scale,
                                mk ? mk + x : nullptr);
            }
            if (y == 0) {
                const float sd = (q.y == 0 && q.x == 0) ? scale_c : scale;
                if (mk == nullptr || fabsf(static_cast<float>(denW) * sd) < kFixedLimit)
                    acc_add(block_ptr(t, t.accD[p], t.accD0[p], q.y, q.x, pitch), denW, sd);
                else  // the block's weight reaches all of its pixels
                    for (int i = 0; i < BS * BS; ++i)
                        mk[static_cast<long long>(i / BS) * a.width + i % BS] = 1;
            }
        }
    }
}

// Wiener shrinkage of a BlockSize-8 FP32 group with ONE group buffer: the
// basic estimate's group is transformed in G, each lane keeps the Wiener
// weights of its two pencils (lane and lane + 32: 2 x 32 registers), then
// the noisy group is transformed in the same buffer and scaled. Elements,
// weights and the lane's sum of squared weights come out in exactly the
// order of the two-buffer form (a lane's elements e = lane + 32 k are pencil
// lane + 32 (k % 2) at z = k / 2), so results are bit-identical; the warp
// needs half the shared memory. Returns the lane's sum of w^2.
template <typename T>
__device__ __forceinline__ T wiener_one_buffer(const StageArgs<T> &a, const Tile<T> &t, int p,
                                               int pt, const BlockPos *list, int n, int lane, T *G,
                                               unsigned &n_bad)
{
    gather_rows<T, 8>(t, t.refw[p], t.ref0[p], list, n, lane, G, static_cast<unsigned *>(nullptr));
    __syncwarp();
    dct_cols_z_fwd<T, 8>(G, n, lane, a.dct_fwd);
    const T s2 = a.wss[pt][n - 1];
    T *const p0 = G + (lane >> 3) * 9 + (lane & 7);  // pencil lane
    T *const p1 = p0 + 4 * 9;                        // pencil lane + 32
    T w0[kGSTab], w1[kGSTab];
    T l2 = T(0);
#pragma unroll
    for (int z = 0; z < kGSTab; ++z) {
        w0[z] = w1[z] = T(0);
        if (z < n) {
            const T y0 = p0[z * 72], y1 = p1[z * 72];
            w0[z] = wiener_weight(y0 * y0, s2);
            l2 += w0[z] * w0[z];
            w1[z] = wiener_weight(y1 * y1, s2);
            l2 += w1[z] * w1[z];
        }
    }
    __syncwarp();
    gather_rows<T, 8>(t, t.srcw[p], t.src0[p], list, n, lane, G, &n_bad);
    __syncwarp();
    dct_cols_z_fwd<T, 8>(G, n, lane, a.dct_fwd);
#pragma unroll
    for (int z = 0; z < kGSTab; ++z)
        if (z < n) {
            p0[z * 72] *= w0[z];
            p1[z * 72] *= w1[z];
        }
    __syncwarp();
    return l2;
}

// Collaborative filtering of one group on plane p (generic sizes).
template <typename T, bool WIENER>
__device__ void filter_generic(const StageArgs<T> &a, const Tile<T> &t, int p, const BlockPos *list,
                               int n, int lane, T *Gs, T *Gr, float scale,
                               unsigned &n_bad, int pt = -1, bool check = false)
{
    // p indexes the tile's windows; pt (default p) the plane's threshold /
    // Wiener tables, which differ when planes share one set of windows
    if (pt < 0) pt = p;
    const int bs = t.bs, bsq = bs * bs, total = n * bsq;
    const int zs = generic_block_stride(bs), rs = generic_row_stride(bs);
    T denW;
    if (WIENER && generic_one_buffer<T>(WIENER, bs)) {
        const T l2 = warp_sum(wiener_one_buffer(a, t, p, pt, list, n, lane, Gs, n_bad));
        denW = l2 <= T(0) ? T(1) : T(1) / l2;
    } else {
    if (bs == 8) {
        gather_rows<T, 8>(t, t.srcw[p], t.src0[p], list, n, lane, Gs, &n_bad);
        if (WIENER)
            gather_rows<T, 8>(t, t.refw[p], t.ref0[p], list, n, lane, Gr,
                              static_cast<unsigned *>(nullptr));
        __syncwarp();
        dct_cols_z_fwd<T, 8>(Gs, n, lane, a.dct_fwd);
    } else if (rows_fused<T>(bs)) {  // 11, FP32
        if constexpr (sizeof(T) == 4) {
            gather_rows<T, 11>(t, t.srcw[p], t.src0[p], list, n, lane, Gs, &n_bad);
            if (WIENER)
                gather_rows<T, 11>(t, t.refw[p], t.ref0[p], list, n, lane, Gr,
                                   static_cast<unsigned *>(nullptr));
            __syncwarp();
            dct_cols_z_fwd<T, 11>(Gs, n, lane, a.dct_fwd);
        }
    } else {
        for (int e = lane; e < total; e += kWarp) {
            int z, y, x;
            group_index(e, bs, bsq, z, y, x);
            const int g = z * zs + y * rs + x;
            const BlockPos q = list[z];
            const bool ok = block_in_tile(t, q.y, q.x);
            if (!ok && y == 0 && x == 0) ++n_bad;
            int pitch;
            const T *bp =
                block_ptr(t, t.srcw[p], t.src0[p], ok ? q.y : t.ry0, ok ? q.x : t.rx0, pitch);
            Gs[g] = ok ? bp[y * pitch + x] : T(0);
            if (WIENER) {
                const T *rp =
                    block_ptr(t, t.refw[p], t.ref0[p], ok ? q.y : t.ry0, ok ? q.x : t.rx0, pitch);
                Gr[g] = ok ? rp[y * pitch + x] : T(0);
            }
        }
        __syncwarp();
        dct3_generic(Gs, n, bs, lane, a.dct_fwd, false);
    }
    if (!WIENER) {
        // hard threshold (source/BM3D.cpp:361-371) with thr by #zero indices
        const T *thr = a.thr[pt][n - 1];
        int kept = 0;
        for (int e = lane; e < total; e += kWarp) {
            int z, y, x;
            group_index(e, bs, bsq, z, y, x);
            const int g = z * zs + y * rs + x;
            const T v = Gs[g];
            const T av = v < T(0) ? -v : v;
            if (av <= thr[(x == 0) + (y == 0) + (z == 0)]) Gs[g] = T(0);
            else ++kept;
        }
        const int retained = __reduce_add_sync(0xffffffffu, kept);
        denW = retained < 1 ? T(1) : T(1) / static_cast<T>(retained);
    } else {
        if (bs == 8) dct_cols_z_fwd<T, 8>(Gr, n, lane, a.dct_fwd);
        else if (rows_fused<T>(bs)) {
            if constexpr (sizeof(T) == 4) dct_cols_z_fwd<T, 11>(Gr, n, lane, a.dct_fwd);
        } else {
            dct3_generic(Gr, n, bs, lane, a.dct_fwd, false);
        }
        const T s2 = a.wss[pt][n - 1];
        T l2 = T(0);
        for (int e = lane; e < total; e += kWarp) {
            // any one-to-one order works here; the padded layout needs its address
            const int g = bs == 8 ? (e >> 6) * 72 + ((e >> 3) & 7) * 9 + (e & 7) : e;
            const T y2 = Gr[g] * Gr[g];
            const T w = wiener_weight(y2, s2);
            Gs[g] *= w;
            l2 += w * w;
        }
        l2 = warp_sum(l2);
        denW = l2 <= T(0) ? T(1) : T(1) / l2;
    }
    }
    const T numW = static_cast<T>(static_cast<double>(denW) / a.finalAMP[n - 1]);
    __syncwarp();
    if (bs == 8) {
        dct_z_cols_inv<T, 8>(Gs, n, lane, a.dct_inv);
        aggregate_rows<T, 8>(a, t, p, pt, list, n, lane, Gs, numW, denW, scale, check);
        __syncwarp();
        return;
    }
    if constexpr (sizeof(T) == 4) {
        if (bs == 11) {
            dct_z_cols_inv<T, 11>(Gs, n, lane, a.dct_inv);
            aggregate_rows<T, 11>(a, t, p, pt, list, n, lane, Gs, numW, denW, scale, check);
            __syncwarp();
            return;
        }
    }
    dct3_generic(Gs, n, bs, lane, a.dct_inv, true);
    // the block weight once per block, at its origin (as the register-resident kernel)
    for (int e = lane; e < total; e += kWarp) {
        int z, y, x;
        group_index(e, bs, bsq, z, y, x);
        const BlockPos q = list[z];
        if (!block_in_tile(t, q.y, q.x)) continue;
        int pitch;
        auto *dn = block_ptr(t, t.accN[p], t.accN0[p], q.y, q.x, pitch);
        if (!check && (q.y >= bs || q.x >= bs)) {
            acc_add(dn + y * pitch + x, Gs[z * zs + y * rs + x] * numW, scale);
            if (y == 0 && x == 0)
                acc_add(block_ptr(t, t.accD[p], t.accD0[p], q.y, q.x, pitch), denW, scale);
        } else {
            // a member reaching block (0, 0)'s pixels (their own scale), or a plane
            // with non-finite pixels (per-term check, marks into the poison map)
            const float scale_c = fixed_scale(a.absmax[pt], a.log2_corner);
            unsigned char *const poison = poison_map(a, pt);
            const bool corner = q.y + y < bs && q.x + x < bs;
            unsigned char *mk =
                poison ? poison + static_cast<long long>(q.y) * a.width + q.x : nullptr;
            acc_add_checked(dn + y * pitch + x, Gs[z * zs + y * rs + x] * numW,
                            corner ? scale_c : scale,
                            mk ? mk + static_cast<long long>(y) * a.width + x : nullptr);
            if (y == 0 && x == 0) {
                const float sd = (q.y == 0 && q.x == 0) ? scale_c : scale;
                if (mk == nullptr || fabsf(static_cast<float>(denW) * sd) < kFixedLimit)
                    acc_add(block_ptr(t, t.accD[p], t.accD0[p], q.y, q.x, pitch), denW, sd);
                else  // the block's weight reaches all of its pixels
                    for (int i = 0; i < bsq; ++i)
                        mk[static_cast<long long>(i / bs) * a.width + i % bs] = 1;
            }
        }
    }
    __syncwarp();
}

template <typename T, bool WIENER, int NPL>
__device__ __forceinline__ void generic_tile_body(const StageArgs<T> &a, int tile, unsigned char *smem,
                                                  unsigned avail)
{
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const int bs = a.block_size;
    const int right = a.width - bs, bottom = a.height - bs;

    Tile<T> t;
    int kx0, kx1, ky0, ky1;
    tile_window(a, tile, bs, t, kx0, kx1, ky0, ky1);
    const SmemPlan sp = plan_smem<T>(NPL, WIENER, a.ref_alias_src, a.region_h, a.region_pitch,
                                     a.key_slots, nwarps, true, bs, a.group_size);
    if (sp.total > avail) {  // launched with less shared memory than the layout needs
        smem_shortfall(a);
        return;
    }
    carve_tile<T, WIENER, NPL>(a, sp, smem, t);
    stage_tile<T, WIENER, NPL>(a, t);

    unsigned char *wbase = smem + sp.off_warps + sp.warp_bytes * warp;
    const size_t scratch = sp.scratch_bytes;
    const int gvals = a.group_size * generic_block_stride(bs);
    T *Gs = reinterpret_cast<T *>(wbase);
    T *Gr = Gs + gvals;
    SortKey<T> *keys = reinterpret_cast<SortKey<T> *>(wbase);
    T *refblk = reinterpret_cast<T *>(wbase + scratch);
    unsigned char *after = wbase + scratch + sp.refblk_bytes;
    SortKey<T> *heap = reinterpret_cast<SortKey<T> *>(after);
    BlockPos *list = reinterpret_cast<BlockPos *>(after + sizeof(SortKey<T>) * kCand);
    T *lkeys = reinterpret_cast<T *>(after + sizeof(SortKey<T>) * kCand + sizeof(BlockPos) * kGSTab);

    // per-tile counters (small: 32 bits suffice), flushed once per tile
    unsigned n_sum = 0, n_sq = 0, n_cand = 0, n_fix = 0, n_bad = 0;
    float scale[NPL];
    bool check[NPL];
#pragma unroll
    for (int p = 0; p < NPL; ++p) {
        scale[p] = fixed_scale(a.absmax[p], a.log2_bound);
        check[p] = poison_map(a, p) != nullptr;
    }
    const int tw = kx1 - kx0, nrefs = tw * (ky1 - ky0);
    for (int r = warp; r < nrefs; r += nwarps) {
        const int ky = ky0 + r / tw, kx = kx0 + r % tw;
        const int j0 = ref_pos(ky, a.step, bottom), i0 = ref_pos(kx, a.step, right);
        // BlockSize 8 with step 1: the register-resident kernel's strips of
        // four candidates; otherwise one lane per candidate
        const int n = (bs == kBS && a.bm_step == 1)
                          ? match_block<T, 4>(a, t, j0, i0, lane, keys, heap, list, lkeys, n_cand,
                                              n_fix)
                          : match_generic<T>(a, t, j0, i0, lane, keys, refblk, heap, list, lkeys,
                                             n_cand, n_fix);
        n_sum += n;
        n_sq += static_cast<unsigned>(n * n);
        dump_group(a, ky, kx, n, lane, list, lkeys);
        if (!a.bm_only) {
#pragma unroll
            for (int p = 0; p < NPL; ++p)
                if (a.active & (1 << p))
                    filter_generic<T, WIENER>(a, t, p, list, n, lane, Gs, Gr, scale[p], n_bad,
                                              -1, check[p]);
        }
        __syncwarp();
    }
    flush_stats(a, lane, n_sum, n_sq, n_cand, n_fix, n_bad);
    if (a.bm_only) return;
    __syncthreads();
    flush_tile<T, NPL>(a, t);
}

// Three planes sharing the groups matched on plane 0, one plane at a time
// through a single plane's windows (as stage_tile_body_seq3): plane 0 matches
// and keeps each reference block's group list in shared memory, planes 1 and
// 2 re-stage their windows and filter with those lists.
template <typename T, bool WIENER>
__device__ __forceinline__ void generic_tile_body_seq3(const StageArgs<T> &a, int tile,
                                                       unsigned char *smem, unsigned avail)
{
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const int bs = a.block_size, GS = a.group_size;
    const int right = a.width - bs, bottom = a.height - bs;

    Tile<T> t;
    int kx0, kx1, ky0, ky1;
    tile_window(a, tile, bs, t, kx0, kx1, ky0, ky1);
    const SmemPlan sp = plan_smem<T>(3, WIENER, a.ref_alias_src, a.region_h, a.region_pitch,
                                     a.key_slots, nwarps, true, bs, GS, a.tile_x * a.tile_y);
    if (sp.total > avail) {  // launched with less shared memory than the layout needs
        smem_shortfall(a);
        return;
    }
    carve_tile<T, WIENER, 1>(a, sp, smem, t);  // every plane goes through windows [0]
    // group lists: position (y - ry0) << 8 | (x - rx0), or 0xffff for a
    // (0, 0) block held outside the window; then one count byte per block
    unsigned short *gpos = reinterpret_cast<unsigned short *>(smem + sp.off_groups);
    unsigned char *gn = reinterpret_cast<unsigned char *>(gpos + a.tile_x * a.tile_y * GS);

    unsigned char *wbase = smem + sp.off_warps + sp.warp_bytes * warp;
    const size_t scratch = sp.scratch_bytes;
    T *Gs = reinterpret_cast<T *>(wbase);
    T *Gr = Gs + GS * generic_block_stride(bs);
    SortKey<T> *keys = reinterpret_cast<SortKey<T> *>(wbase);
    T *refblk = reinterpret_cast<T *>(wbase + scratch);
    unsigned char *after = wbase + scratch + sp.refblk_bytes;
    SortKey<T> *heap = reinterpret_cast<SortKey<T> *>(after);
    BlockPos *list = reinterpret_cast<BlockPos *>(after + sizeof(SortKey<T>) * kCand);
    T *lkeys = reinterpret_cast<T *>(after + sizeof(SortKey<T>) * kCand + sizeof(BlockPos) * kGSTab);

    // per-tile counters (small: 32 bits suffice), flushed once per tile
    unsigned n_sum = 0, n_sq = 0, n_cand = 0, n_fix = 0, n_bad = 0;
    const int tw = kx1 - kx0, nrefs = tw * (ky1 - ky0);
    for (int c = 0; c < 3; ++c) {
        const bool filt = !a.bm_only && (a.active & (1 << c));
        if (c > 0 && !filt) continue;
        stage_plane<T, WIENER>(a, t, c);
        const float scale = fixed_scale(a.absmax[c], a.log2_bound);
        const bool check = poison_map(a, c) != nullptr;
        for (int r = warp; r < nrefs; r += nwarps) {
            int n;
            if (c == 0) {
                const int ky = ky0 + r / tw, kx = kx0 + r % tw;
                const int j0 = ref_pos(ky, a.step, bottom), i0 = ref_pos(kx, a.step, right);
                n = (bs == kBS && a.bm_step == 1)
                        ? match_block<T, 4>(a, t, j0, i0, lane, keys, heap, list, lkeys, n_cand,
                                            n_fix)
                        : match_generic<T>(a, t, j0, i0, lane, keys, refblk, heap, list, lkeys,
                                           n_cand, n_fix);
                n_sum += n;
                n_sq += static_cast<unsigned>(n * n);
                dump_group(a, ky, kx, n, lane, list, lkeys);
                if (lane == 0) gn[r] = static_cast<unsigned char>(n);
                for (int k = lane; k < n; k += kWarp) {
                    const BlockPos q = list[k];
                    const bool outside = q.y == 0 && q.x == 0 && !t.origin_inside;
                    gpos[r * GS + k] = outside ? 0xffff
                                               : static_cast<unsigned short>(
                                                     ((q.y - t.ry0) << 8) | (q.x - t.rx0));
                }
            } else {
                n = gn[r];
                for (int k = lane; k < n; k += kWarp) {
                    const unsigned v = gpos[r * GS + k];
                    list[k] = v == 0xffffu ? BlockPos{0, 0}
                                           : BlockPos{t.ry0 + static_cast<int>(v >> 8),
                                                      t.rx0 + static_cast<int>(v & 0xffu)};
                }
            }
            __syncwarp();
            if (filt)
                filter_generic<T, WIENER>(a, t, 0, list, n, lane, Gs, Gr, scale, n_bad, c, check);
            __syncwarp();
        }
        __syncthreads();
        if (filt) flush_plane<T>(a, t, c);
        __syncthreads();  // the windows are re-staged for the next plane
    }
    flush_stats(a, lane, n_sum, n_sq, n_cand, n_fix, n_bad);
}

template <typename T, bool WIENER, int NPL>
__global__ void __launch_bounds__(sizeof(T) == 4 ? 384 : 256, 1)
    generic_stage_kernel(const StageArgs<T> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    if constexpr (NPL == 3) generic_tile_body_seq3<T, WIENER>(a, blockIdx.x, smem, dynamic_smem_bytes());
    else generic_tile_body<T, WIENER, NPL>(a, blockIdx.x, smem, dynamic_smem_bytes());
}

}  // namespace bm3d
