// Fused BM3D stage kernel: block matching, 3-D transform, shrinkage, inverse
// transform and shared-memory aggregation for one tile of reference blocks per
// CTA, one reference block per warp at a time.
//
// Reference: BM3D_Base::Kernel (source/BM3D.cpp:80-136, 139-218),
// BM3D_Base::BlockMatching (source/BM3D.cpp:221-236),
// Block::BlockMatchingMulti (include/Block.h:578-615, 658-703),
// BM3D_Basic::CollaborativeFilter (source/BM3D.cpp:339-385),
// BM3D_Final::CollaborativeFilter (source/BM3D.cpp:411-457).
#pragma once

#include <type_traits>

#include "bm3d_device.cuh"
#include "dct.cuh"

namespace bm3d {

// Cosine matrices for group lengths 1..16 (row k = output k), concatenated;
// length n starts at (n-1) n (2n-1) / 6. Every translation unit that launches
// these kernels has its own copy, filled by the host when a context is made.
static __constant__ float c_dct_fwd_f[1496];
static __constant__ float c_dct_inv_f[1496];
static __constant__ double c_dct_fwd_d[1496];
static __constant__ double c_dct_inv_d[1496];
// FP32 cosine matrices of the lengths other than 8 and 16, column by column:
// length n starts at 16 * (sum of the lengths m < n, m != 8), and entry
// (row k, column j) sits at + 16 j + k, zero for k >= n.
static __constant__ float c_dct_pad_fwd[kPadTable];
static __constant__ float c_dct_pad_inv[kPadTable];

template <typename T> struct DctTab;
template <> struct DctTab<float> {
    static __device__ __forceinline__ const float *fwd() { return c_dct_fwd_f; }
    static __device__ __forceinline__ const float *inv() { return c_dct_inv_f; }
};
template <> struct DctTab<double> {
    static __device__ __forceinline__ const double *fwd() { return c_dct_fwd_d; }
    static __device__ __forceinline__ const double *inv() { return c_dct_inv_d; }
};

// Transforms along the group axis for two pencils at once. Lengths 8 and 16
// use the butterflies of dct.cuh. In FP64 every other length N has its own
// instantiation of the symmetric matrix form (dct.cuh), reading the
// constant-bank tables at compile-time offsets; FP32 runs those lengths
// through one compact loop instead (zgen, below).
template <typename T, int N>
__device__ __forceinline__ void zfwd_n(T (&a)[kGSMax], T (&b)[kGSMax])
{
    constexpr int O = (N - 1) * N * (2 * N - 1) / 6;  // start of length N: sum of m^2, m < N
    redft10_pair<T, N>(a, b, DctTab<T>::fwd() + O);
}

template <typename T, int N>
__device__ __forceinline__ void zinv_n(T (&a)[kGSMax], T (&b)[kGSMax])
{
    constexpr int O = (N - 1) * N * (2 * N - 1) / 6;
    redft01_pair<T, N>(a, b, DctTab<T>::inv() + O);
}

template <typename T>
__device__ __forceinline__ void zbfly8(T (&a)[kGSMax], bool inverse)
{
    T t[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) t[i] = a[i];
    if (inverse) redft01_8(t);
    else redft10_8(t);
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = t[i];
}

// Forward (REDFT10) transform of two pencils of length n <= 16.
template <typename T>
__device__ __forceinline__ void zdct_fwd2(T (&a)[kGSMax], T (&b)[kGSMax], int n)
{
    switch (n) {
    case 16: redft10_16(a); redft10_16(b); break;
    case 8: zbfly8(a, false); zbfly8(b, false); break;
    case 1: zfwd_n<T, 1>(a, b); break;
    case 2: zfwd_n<T, 2>(a, b); break;
    case 3: zfwd_n<T, 3>(a, b); break;
    case 4: zfwd_n<T, 4>(a, b); break;
    case 5: zfwd_n<T, 5>(a, b); break;
    case 6: zfwd_n<T, 6>(a, b); break;
    case 7: zfwd_n<T, 7>(a, b); break;
    case 9: zfwd_n<T, 9>(a, b); break;
    case 10: zfwd_n<T, 10>(a, b); break;
    case 11: zfwd_n<T, 11>(a, b); break;
    case 12: zfwd_n<T, 12>(a, b); break;
    case 13: zfwd_n<T, 13>(a, b); break;
    case 14: zfwd_n<T, 14>(a, b); break;
    default: zfwd_n<T, 15>(a, b); break;
    }
}

// Backward (REDFT01) transform of two pencils of length n <= 16.
template <typename T>
__device__ __forceinline__ void zdct_inv2(T (&a)[kGSMax], T (&b)[kGSMax], int n)
{
    switch (n) {
    case 16: redft01_16(a); redft01_16(b); break;
    case 8: zbfly8(a, true); zbfly8(b, true); break;
    case 1: zinv_n<T, 1>(a, b); break;
    case 2: zinv_n<T, 2>(a, b); break;
    case 3: zinv_n<T, 3>(a, b); break;
    case 4: zinv_n<T, 4>(a, b); break;
    case 5: zinv_n<T, 5>(a, b); break;
    case 6: zinv_n<T, 6>(a, b); break;
    case 7: zinv_n<T, 7>(a, b); break;
    case 9: zinv_n<T, 9>(a, b); break;
    case 10: zinv_n<T, 10>(a, b); break;
    case 11: zinv_n<T, 11>(a, b); break;
    case 12: zinv_n<T, 12>(a, b); break;
    case 13: zinv_n<T, 13>(a, b); break;
    case 14: zinv_n<T, 14>(a, b); break;
    default: zinv_n<T, 15>(a, b); break;
    }
}

// ---------------------------------------------------------------------------
// One CTA's view of its staged windows.
template <typename T> struct Tile {
    using Acc = typename AccOf<T>::type;
    int ry0, rx0, rh, rw;      // staged window origin / size in the plane
    int pitch;
    int bs;                    // block size
    bool origin_inside;        // block (0, 0) lies inside the staged window
    const T *srcw[kMaxPlanes]; // staged src windows
    const T *refw[kMaxPlanes]; // staged ref windows (refw[0] drives matching)
    const T *src0[kMaxPlanes]; // block (0, 0) of src when outside the window
    const T *ref0[kMaxPlanes];
    Acc *accN[kMaxPlanes], *accD[kMaxPlanes];
    Acc *accN0[kMaxPlanes], *accD0[kMaxPlanes];
};

// Adds q to the 64-bit two's-complement sum at p (shared memory). A 64-bit
// shared-memory atomic add has no native form (it runs as a compare-and-swap
// loop: a load, an add and a CAS round trip per attempt), so the sum is kept
// as two 32-bit words, low word at p, high word after it, each updated by a
// native 32-bit atomic. The low word's atomic returns the value it replaced,
// which tells whether this addition wrapped it; that carry goes into the high
// word with q's own high half. Every wrap of the low word is seen by exactly
// the addition that caused it, so once all additions are done the 8 bytes at
// p hold sum(q) mod 2^64 -- the value the 64-bit atomic add gave -- whatever
// the order. Nothing reads the slot until the tile's barrier.
__device__ __forceinline__ void acc_add_fixed(long long *p, long long q)
{
    unsigned *w = reinterpret_cast<unsigned *>(p);
    const unsigned lo = static_cast<unsigned>(q);
    const unsigned hi = static_cast<unsigned>(static_cast<unsigned long long>(q) >> 32);
    const unsigned old = atomicAdd(w, lo);
    atomicAdd(w + 1, hi + (old + lo < old ? 1u : 0u));
}

// One aggregation term: fixed point for FP32 stages, double for FP64.
__device__ __forceinline__ void acc_add(long long *p, float v, float scale)
{
    acc_add_fixed(p, __float2ll_rn(v * scale));
}
__device__ __forceinline__ void acc_add(double *p, double v, float) { atomicAdd(p, v); }

// The same for planes with non-finite pixels: a term that has no fixed-point
// value (NaN, +-Inf, or beyond the 2^62 range) marks its pixel instead, and
// the normalisation writes NaN there -- what the reference's float sums give
// once a NaN or an Inf of either sign reaches them (source/BM3D.cpp:130-135).
// Finite terms are converted exactly as acc_add does; with no mark they are
// always converted.
constexpr float kFixedLimit = 4.0e18f;
__device__ __forceinline__ void acc_add_checked(long long *p, float v, float scale,
                                                unsigned char *mark)
{
    const float x = v * scale;
    if (mark == nullptr || fabsf(x) < kFixedLimit)
        acc_add_fixed(p, __float2ll_rn(x));
    else
        *mark = 1;
}
__device__ __forceinline__ void acc_add_checked(double *p, double v, float, unsigned char *)
{
    atomicAdd(p, v);
}
__device__ __forceinline__ void acc_flush(long long *p, long long v)
{
    atomicAdd(reinterpret_cast<unsigned long long *>(p), static_cast<unsigned long long>(v));
}
__device__ __forceinline__ void acc_flush(double *p, double v) { atomicAdd(p, v); }

// Address of pixel (y, x) of the block at plane position (py, px) inside a
// staged window, or inside the (0, 0) copy when the block is (0, 0) and the
// window does not contain it.
template <typename T, typename P>
__device__ __forceinline__ P *block_ptr(const Tile<T> &t, P *win, P *origin, int py, int px,
                                        int &pitch)
{
    if (py == 0 && px == 0 && !t.origin_inside) {
        pitch = t.bs;
        return origin;
    }
    pitch = t.pitch;
    return win + (py - t.ry0) * t.pitch + (px - t.rx0);
}

// True when the block at (py, px) can be addressed: inside the staged window,
// or the (0, 0) block held in its own copy. Group members always are by
// construction; the check keeps a violated invariant from touching memory.
template <typename T>
__device__ __forceinline__ bool block_in_tile(const Tile<T> &t, int py, int px)
{
    if (py == 0 && px == 0 && !t.origin_inside) return true;
    return py >= t.ry0 && px >= t.rx0 && py + t.bs <= t.ry0 + t.rh && px + t.bs <= t.rx0 + t.rw;
}

// Ordered group of reference block (j0, i0) from its search list: keys[0,
// ngrid) are the window grid in raster order, keys[ngrid] the trailing (0, 0)
// slot (invalid keys = rejected or the block itself). Writes list/lkeys in the
// reference's group order and returns the group size.
template <typename T>
__device__ int select_group(const StageArgs<T> &a, const SortKey<T> *keys, int ngrid, int nc,
                            int tp, int l, int st, int j0, int i0, int lane, SortKey<T> *heap,
                            BlockPos *list, T *lkeys, unsigned &n_fix)
{
    using K = SortKey<T>;
    const int GS = a.group_size;
    // Ordered selection of the GS - 1 best candidates by (key, list index).
    // T = the (take)-th smallest of the lanes' minima bounds the take best
    // from above (those minima are take distinct candidates). All candidates
    // whose key value is <= T's -- ties with the cut-off included -- are
    // compacted and bitonic-sorted; typically 16-24 of ~360. Groups of more
    // than 17 blocks take T from the lanes' two smallest keys (64 distinct
    // candidates), which keeps the compacted set within the 64-wide sort.
    const int nkeys = ngrid + 1;
    const bool two = GS - 1 > kWarp / 2;
    K lmin = K::invalid(), lmin2 = K::invalid();
    int nvalid = 0;
    if (two) {
        for (int i = lane; i < nkeys; i += kWarp) {
            const K v = keys[i];
            nvalid += v.valid() ? 1 : 0;
            if (v < lmin) {
                lmin2 = lmin;
                lmin = v;
            } else if (v < lmin2) {
                lmin2 = v;
            }
        }
    } else {
        for (int i = lane; i < nkeys; i += kWarp) {
            const K v = keys[i];
            nvalid += v.valid() ? 1 : 0;
            if (v < lmin) lmin = v;
        }
    }
    const int accepted = __reduce_add_sync(0xffffffffu, nvalid);
    const int take = min(GS - 1, accepted);
    // list[0] is the reference block itself (key 0, include/Block.h:685)
    if (lane == 0) {
        list[0] = BlockPos{j0, i0};
        lkeys[0] = T(0);
    }
    auto put = [&](int rank, const K &m) {  // rank-th best candidate -> list[rank + 1]
        const int idx = static_cast<int>(m.idx());
        int y = 0, x = 0;
        if (idx < ngrid) {
            const int rr = idx / nc;
            y = tp + rr * st;
            x = l + (idx - rr * nc) * st;
        }
        list[rank + 1] = BlockPos{y, x};
        lkeys[rank + 1] = m.key();
    };
    bool tie = false;
    if (take > 0) {
        // The threshold depends on key values only, so the lanes' minima are
        // sorted by their key bits alone (the (take)-th smallest key value is
        // the same in (key, index) order).
        using KB = KeyBits<decltype(lmin.key_bits())>;
        decltype(lmin.key_bits()) tb;
        if (two) {  // element take - 1 (< 32) of the 64 sorted sits in lane take - 1's v0
            KB s0{lmin.key_bits()}, s1{lmin2.key_bits()};
            bitonic64(s0, s1, lane);
            tb = s0.shfl(take - 1).v;
        } else {
            tb = bitonic32(KB{lmin.key_bits()}, lane).shfl(take - 1).v;
        }
        // One pass counts the keys at or under the threshold (M) and packs the
        // first kCand of them into heap[] by warp ballot (their order there is
        // irrelevant: they are sorted next).
        int M = 0;
        const unsigned below = (1u << lane) - 1u;
        for (int first = 0; first < nkeys; first += kWarp) {
            const int i = first + lane;
            const K v = i < nkeys ? keys[i] : K::invalid();
            const bool in = v.valid() && v.key_bits() <= tb;
            const unsigned m = __ballot_sync(0xffffffffu, in);
            const int pos = M + __popc(m & below);
            if (in && pos < kCand) heap[pos] = v;
            M += __popc(m);
        }
        if (M <= kCand) {
            __syncwarp();
            K v0 = lane < M ? heap[lane] : K::invalid();
            K v1 = lane + kWarp < M ? heap[lane + kWarp] : K::invalid();
            if (M <= kWarp) v0 = bitonic32(v0, lane);
            else bitonic64(v0, v1, lane);
            if (lane < take) put(lane, v0);
            if (lane + kWarp < take) put(lane + kWarp, v1);
            // equal keys at adjacent ranks r, r + 1 with r < take
            // (every shuffle runs on all 32 lanes; only the selects below differ)
            const K n0 = v0.shfl((lane + 1) & (kWarp - 1));
            const K nx = v1.shfl((lane + 1) & (kWarp - 1));
            const K f1 = v1.shfl(0);
            const K next0 = lane < kWarp - 1 ? n0 : f1;
            const bool t0 = lane < take && lane + 1 < M && next0.key_bits() == v0.key_bits();
            const bool t1 = lane + kWarp < take && lane + kWarp + 1 < M && lane < kWarp - 1 &&
                            nx.key_bits() == v1.key_bits();
            tie = __any_sync(0xffffffffu, t0 || t1);
        } else {
            // Rare (many candidates share the cut-off): repeated warp minimum,
            // whose owner lane advances to the next key of its slice.
            K cur = lmin;
            T prev_key = T(-1);
            for (int k = 0; k < take; ++k) {
                const K m = warp_min(cur);
                tie |= (m.key() == prev_key);
                prev_key = m.key();
                if (lane == 0) put(k, m);
                if (cur == m) {
                    K nxt = K::invalid();
                    for (int i = lane; i < nkeys; i += kWarp) {
                        const K v = keys[i];
                        if (m < v && v < nxt) nxt = v;
                    }
                    cur = nxt;
                }
            }
            const K m = warp_min(cur);
            tie |= (m.valid() && m.key() == prev_key);
        }
    }
    __syncwarp();
    // More matches than the group holds: the reference keeps GroupSize of them
    // with std::partial_sort (include/Block.h:690-696), whose placement of
    // equal keys is libstdc++'s heap order, not list order. Redo such groups
    // with that exact algorithm when a tie touches the kept set.
    if (accepted + 1 > GS && GS > 1) {
        if (tie) {
            if (lane == 0) {
                ++n_fix;
                // heap[] holds the first GS entries of the reference's match list:
                // the reference block, then matches in list order.
                heap[0] = K::make(T(0), 0xffffffffu);
                int h = 1, i = 0;
                for (; i < nkeys && h < GS; ++i)
                    if (keys[i].valid()) heap[h++] = keys[i];
                auto less = [](const K &p, const K &q) { return p.key() < q.key(); };
                auto adjust = [&](int hole, int len, K value) {
                    const int top = hole;
                    int child = hole;
                    while (child < (len - 1) / 2) {
                        child = 2 * (child + 1);
                        if (less(heap[child], heap[child - 1])) child--;
                        heap[hole] = heap[child];
                        hole = child;
                    }
                    if ((len & 1) == 0 && child == (len - 2) / 2) {
                        child = 2 * (child + 1);
                        heap[hole] = heap[child - 1];
                        hole = child - 1;
                    }
                    int parent = (hole - 1) / 2;
                    while (hole > top && less(heap[parent], value)) {
                        heap[hole] = heap[parent];
                        hole = parent;
                        parent = (hole - 1) / 2;
                    }
                    heap[hole] = value;
                };
                for (int parent = (GS - 2) / 2;; --parent) {  // __make_heap
                    adjust(parent, GS, heap[parent]);
                    if (parent == 0) break;
                }
                for (; i < nkeys; ++i) {  // __heap_select
                    const K v = keys[i];
                    if (v.valid() && less(v, heap[0])) adjust(0, GS, v);
                }
                for (int last = GS; last > 1;) {  // __sort_heap
                    --last;
                    const K v = heap[last];
                    heap[last] = heap[0];
                    adjust(0, last, v);
                }
                for (int k = 0; k < GS; ++k) {
                    const unsigned idx = heap[k].idx();
                    int y = 0, x = 0;
                    if (idx == 0xffffffffu) {
                        y = j0;
                        x = i0;
                    } else if (static_cast<int>(idx) < ngrid) {
                        const int rr = static_cast<int>(idx) / nc;
                        y = tp + rr * st;
                        x = l + (static_cast<int>(idx) - rr * nc) * st;
                    }
                    list[k] = BlockPos{y, x};
                    lkeys[k] = heap[k].key();
                }
            }
        }
    }
    __syncwarp();
    return take + 1;
}

// ---------------------------------------------------------------------------
// Block matching for reference block (j0, i0) by one warp. Fills list[0..n)
// with (y, x) in the reference's group order and returns n.
template <typename T, int KS>
__device__ int match_block(const StageArgs<T> &a, const Tile<T> &t, int j0, int i0, int lane,
                           SortKey<T> *keys, SortKey<T> *heap, BlockPos *list, T *lkeys,
                           unsigned &n_cand, unsigned &n_fix)
{
    using K = SortKey<T>;
    const int GS = a.group_size;
    if (!a.match) {
        if (lane == 0) {
            list[0] = BlockPos{j0, i0};
            lkeys[0] = T(0);
        }
        __syncwarp();
        return 1;
    }
    const int st = a.bm_step, R = a.range;
    const int right = a.width - kBS, bottom = a.height - kBS;
    const int l = search_boundary(i0, 0, R, st), r = search_boundary(i0, right, R, st);
    const int tp = search_boundary(j0, 0, R, st), b = search_boundary(j0, bottom, R, st);
    const int nr = (b - tp) / st + 1, nc = (r - l) / st + 1;
    const int ngrid = nr * nc;

    // Reference block in registers.
    T refv[kBS][kBS];
    {
        const T *rb = t.refw[0] + (j0 - t.ry0) * t.pitch + (i0 - t.rx0);
#pragma unroll
        for (int y = 0; y < kBS; ++y)
#pragma unroll
            for (int x = 0; x < kBS; ++x) refv[y][x] = rb[y * t.pitch + x];
    }

    // Candidates: column strips of KS consecutive grid rows per task, plus one
    // task for the trailing (0, 0) slot of the reference's search list.
    const int nstrips = (nr + KS - 1) / KS;
    const int ntasks = nstrips * nc;
    constexpr int ROWS = (KS - 1) + kBS;  // KS > 1 only with BMstep == 1
    for (int task = lane; task <= ntasks; task += kWarp) {
        const T *base;
        int bp, nq, rr0 = 0, cc = 0;
        if (task < ntasks) {
            const int strip = task / nc;
            cc = task - strip * nc;
            rr0 = strip * KS;
            nq = min(KS, nr - rr0);
            bp = t.pitch;
            base = t.refw[0] + (tp + rr0 * st - t.ry0) * t.pitch + (l + cc * st - t.rx0);
        } else {
            nq = 1;
            base = block_ptr(t, t.refw[0], t.ref0[0], 0, 0, bp);
        }
        T acc[KS];
#pragma unroll
        for (int q = 0; q < KS; ++q) acc[q] = T(0);
        if (KS == 1) {
#pragma unroll
            for (int y = 0; y < kBS; ++y) {
                T row[kBS];
#pragma unroll
                for (int x = 0; x < kBS; ++x) row[x] = base[y * bp + x];
                acc[0] = ssd_row8(acc[0], refv[y], row);
            }
        } else {
            // Every strip computes all KS candidates over all ROWS window rows,
            // with no data-dependent branch; candidates past the window's
            // last row (q >= nq) are discarded below. Their rows lie at most
            // KS - 1 rows past a staged window or the (0, 0) copy, which are
            // always followed by other parts of the CTA's shared memory.
#pragma unroll
            for (int w = 0; w < ROWS; ++w) {
                T row[kBS];
#pragma unroll
                for (int x = 0; x < kBS; ++x) row[x] = base[w * bp + x];
#pragma unroll
                for (int q = 0; q < KS; ++q) {
                    const int y = w - q;
                    if (y >= 0 && y < kBS) acc[q] = ssd_row8(acc[q], refv[y], row);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < KS; ++q) {
            if (q < nq) {
                int idx;
                bool self;
                if (task < ntasks) {
                    const int rr = rr0 + q;
                    idx = rr * nc + cc;
                    self = (tp + rr * st == j0) && (l + cc * st == i0);
                } else {
                    idx = ngrid;
                    self = false;
                }
                const T d = acc[q];
                const bool ok = !self && d <= a.thSSE && d != T(0);
                keys[idx] = ok ? K::make(key_from_dist(d, a.distMul), static_cast<unsigned>(idx))
                               : K::invalid();
            }
        }
    }
    __syncwarp();
    n_cand += static_cast<unsigned>(ngrid);  // grid minus self, plus (0, 0)

    return select_group<T>(a, keys, ngrid, nc, tp, l, st, j0, i0, lane, heap, list, lkeys, n_fix);
}

// ---------------------------------------------------------------------------
// A warp's group buffer G holds block z at G + z * kGroupStride, element
// (y, x) at y * 8 + x plus a 4-value gap after row 3. The gap puts the two
// lanes that share a block on different shared-memory banks, so the row,
// column and pencil accesses below are all conflict-free.
__device__ __forceinline__ int gidx(int y, int x) { return y * 8 + x + ((y >> 2) << 2); }

template <typename T> struct Vec4;
template <> struct Vec4<float> {
    static __device__ __forceinline__ void load(const float *p, float &a, float &b, float &c,
                                                float &d)
    {
        const float4 v = *reinterpret_cast<const float4 *>(p);
        a = v.x; b = v.y; c = v.z; d = v.w;
    }
    static __device__ __forceinline__ void store(float *p, float a, float b, float c, float d)
    {
        *reinterpret_cast<float4 *>(p) = make_float4(a, b, c, d);
    }
    static __device__ __forceinline__ void load2(const float *p, float &a, float &b)
    {
        const float2 v = *reinterpret_cast<const float2 *>(p);
        a = v.x; b = v.y;
    }
    static __device__ __forceinline__ void store2(float *p, float a, float b)
    {
        *reinterpret_cast<float2 *>(p) = make_float2(a, b);
    }
};
template <> struct Vec4<double> {
    static __device__ __forceinline__ void load(const double *p, double &a, double &b, double &c,
                                                double &d)
    {
        const double2 u = reinterpret_cast<const double2 *>(p)[0];
        const double2 v = reinterpret_cast<const double2 *>(p)[1];
        a = u.x; b = u.y; c = v.x; d = v.y;
    }
    static __device__ __forceinline__ void store(double *p, double a, double b, double c, double d)
    {
        reinterpret_cast<double2 *>(p)[0] = make_double2(a, b);
        reinterpret_cast<double2 *>(p)[1] = make_double2(c, d);
    }
    static __device__ __forceinline__ void load2(const double *p, double &a, double &b)
    {
        const double2 v = *reinterpret_cast<const double2 *>(p);
        a = v.x; b = v.y;
    }
    static __device__ __forceinline__ void store2(double *p, double a, double b)
    {
        *reinterpret_cast<double2 *>(p) = make_double2(a, b);
    }
};

// Forward 2-D transform (rows then columns) of the n blocks of a group, read
// from a staged window and left in the warp's group buffer. Lane (z, h) =
// (lane / 2, lane % 2) owns rows 4h..4h+3, then columns 4h..4h+3, of block z.
template <typename T>
__device__ __forceinline__ void gather_xy_forward(const Tile<T> &t, const T *win, const T *origin,
                                                  const BlockPos *list, int n, int lane, T *G,
                                                  unsigned &n_bad)
{
    const int z = lane >> 1, h = lane & 1;
    T *gz = G + z * kGroupStride;
    if (z < n) {
        const BlockPos p = list[z];
        const bool ok = block_in_tile(t, p.y, p.x);
        n_bad += ok ? 0 : 1;
        int pitch;
        const T *bp = block_ptr(t, win, origin, ok ? p.y : t.ry0, ok ? p.x : t.rx0, pitch);
#pragma unroll 1
        for (int r = 0; r < 4; ++r) {
            T row[8];
            const int y = 4 * h + r;
#pragma unroll
            for (int x = 0; x < 8; ++x) row[x] = ok ? bp[y * pitch + x] : T(0);
            redft10_8(row);
            Vec4<T>::store(gz + gidx(y, 0), row[0], row[1], row[2], row[3]);
            Vec4<T>::store(gz + gidx(y, 4), row[4], row[5], row[6], row[7]);
        }
    }
    __syncwarp();
    if (z < n) {
        T col[4][8];
#pragma unroll
        for (int y = 0; y < 8; ++y)
            Vec4<T>::load(gz + gidx(y, 4 * h), col[0][y], col[1][y], col[2][y], col[3][y]);
#pragma unroll
        for (int c = 0; c < 4; ++c) redft10_8(col[c]);
#pragma unroll
        for (int y = 0; y < 8; ++y)
            Vec4<T>::store(gz + gidx(y, 4 * h), col[0][y], col[1][y], col[2][y], col[3][y]);
    }
    __syncwarp();
}

// Columns of the inverse 2-D transform, in place in the group buffer.
template <typename T>
__device__ __forceinline__ void xy_inverse_cols(T *G, int n, int lane)
{
    const int z = lane >> 1, h = lane & 1;
    T *gz = G + z * kGroupStride;
    if (z < n) {
        T col[4][8];
#pragma unroll
        for (int y = 0; y < 8; ++y)
            Vec4<T>::load(gz + gidx(y, 4 * h), col[0][y], col[1][y], col[2][y], col[3][y]);
#pragma unroll
        for (int c = 0; c < 4; ++c) redft01_8(col[c]);
#pragma unroll
        for (int y = 0; y < 8; ++y)
            Vec4<T>::store(gz + gidx(y, 4 * h), col[0][y], col[1][y], col[2][y], col[3][y]);
    }
    __syncwarp();
}

// Pencils along the group axis: lane owns positions p = 2 lane and 2 lane + 1,
// i.e. (y, x) = (lane / 4, 2 (lane % 4) + {0, 1}).
__device__ __forceinline__ int pencil_off(int lane) { return gidx(lane >> 2, 2 * (lane & 3)); }

template <typename T>
__device__ __forceinline__ void load_pencils(const T *G, int n, int lane, T (&a)[kGSMax],
                                             T (&b)[kGSMax])
{
    const int o = pencil_off(lane);
#pragma unroll
    for (int z = 0; z < kGSMax; ++z) {
        a[z] = T(0);
        b[z] = T(0);
        if (z < n) Vec4<T>::load2(G + z * kGroupStride + o, a[z], b[z]);
    }
}

template <typename T>
__device__ __forceinline__ void store_pencils(T *G, int n, int lane, const T (&a)[kGSMax],
                                              const T (&b)[kGSMax])
{
    const int o = pencil_off(lane);
#pragma unroll
    for (int z = 0; z < kGSMax; ++z)
        if (z < n) Vec4<T>::store2(G + z * kGroupStride + o, a[z], b[z]);
}

// Group-axis transform of the lane's two pencils for the FP32 lengths other
// than 8 and 16: y_k = sum_j m[k][j] x_j, x read from the group buffer, j in
// order, one runtime loop for every such length (a compact body: groups of
// varied lengths would otherwise run many unrolled bodies at once).
__device__ __forceinline__ void zgen(const float *G, int n, int lane, const float *m,
                                     float (&a)[kGSMax], float (&b)[kGSMax])
{
    const int o = pencil_off(lane);
#pragma unroll
    for (int k = 0; k < kGSMax; ++k) {
        a[k] = 0.0f;
        b[k] = 0.0f;
    }
#pragma unroll 1
    for (int j = 0; j < n; ++j) {
        float xa, xb;
        Vec4<float>::load2(G + j * kGroupStride + o, xa, xb);
        const float *mj = m + 16 * j;
#pragma unroll
        for (int k = 0; k < kGSMax; ++k) {
            a[k] = fmaf(mj[k], xa, a[k]);
            b[k] = fmaf(mj[k], xb, b[k]);
        }
    }
}

// Forward group-axis transform of the pencils held in the group buffer.
template <typename T>
__device__ __forceinline__ void group_fwd(T *G, int n, int lane, T (&a)[kGSMax], T (&b)[kGSMax])
{
    if constexpr (sizeof(T) == 4) {
        if (n != 16 && n != 8) {
            zgen(G, n, lane, c_dct_pad_fwd + pad_table_offset(n), a, b);
            return;
        }
        load_pencils(G, n, lane, a, b);
        if (n == 16) {
            redft10_16(a);
            redft10_16(b);
        } else {
            zbfly8(a, false);
            zbfly8(b, false);
        }
    } else {
        load_pencils(G, n, lane, a, b);
        zdct_fwd2(a, b, n);
    }
}

// Inverse group-axis transform; the result is left in the group buffer.
template <typename T>
__device__ __forceinline__ void group_inv(T *G, int n, int lane, T (&a)[kGSMax], T (&b)[kGSMax])
{
    if constexpr (sizeof(T) == 4) {
        if (n != 16 && n != 8) {
            store_pencils(G, n, lane, a, b);
            __syncwarp();
            zgen(G, n, lane, c_dct_pad_inv + pad_table_offset(n), a, b);
            __syncwarp();
        } else if (n == 16) {
            redft01_16(a);
            redft01_16(b);
        } else {
            zbfly8(a, true);
            zbfly8(b, true);
        }
    } else {
        zdct_inv2(a, b, n);
    }
    __syncwarp();
    store_pencils(G, n, lane, a, b);
}

// Empirical Wiener weight y^2 / (y^2 + sigma^2) (source/BM3D.cpp:440); the
// FP32 path uses the fast division (within 2 ulp), FP64 the exact one.
__device__ __forceinline__ float wiener_weight(float y2, float s2) { return __fdividef(y2, y2 + s2); }
__device__ __forceinline__ double wiener_weight(double y2, double s2) { return y2 / (y2 + s2); }

// The poison map of plane p when its inputs hold non-finite pixels, else null
// (the normal, unchecked aggregation).
template <typename T>
__device__ __forceinline__ unsigned char *poison_map(const StageArgs<T> &a, int p)
{
    if (a.nonfinite == nullptr || a.poison[p] == nullptr) return nullptr;
    return a.nonfinite[p] != 0 ? a.poison[p] : nullptr;
}

// One 8 x 8 group member whose footprint reaches block (0, 0)'s pixels, or any
// member on a plane with non-finite pixels: per pixel, the scale of its class
// (block (0, 0) or not) and, with a poison map, the check of acc_add_checked.
// gz is the member's transformed block in the group buffer; lane half h
// aggregates rows 4h .. 4h + 3 and h == 0 adds the block weight at the
// member's origin. `plane` indexes the plane's scale and poison map.
template <typename T>
__device__ __forceinline__ void aggregate_member_slow(const StageArgs<T> &a, const Tile<T> &t, int p,
                                                      int plane, BlockPos q, const T *gz, int h,
                                                      T numW, T denW, float scale)
{
    const float scale_c = fixed_scale(a.absmax[plane], a.log2_corner);
    unsigned char *const poison = poison_map(a, plane);
    int pitch;
    auto *dn = block_ptr(t, t.accN[p], t.accN0[p], q.y, q.x, pitch);
#pragma unroll 1
    for (int r = 0; r < 4; ++r) {
        const int y = 4 * h + r;
        T v[8];
        Vec4<T>::load(gz + gidx(y, 0), v[0], v[1], v[2], v[3]);
        Vec4<T>::load(gz + gidx(y, 4), v[4], v[5], v[6], v[7]);
        redft01_8(v);
#pragma unroll
        for (int x = 0; x < 8; ++x) {
            const bool corner = q.y + y < kBS && q.x + x < kBS;
            unsigned char *mk =
                poison ? poison + static_cast<long long>(q.y + y) * a.width + q.x + x : nullptr;
            acc_add_checked(dn + y * pitch + x, v[x] * numW, corner ? scale_c : scale, mk);
        }
    }
    if (h == 0) {
        const float sd = (q.y == 0 && q.x == 0) ? scale_c : scale;
        if (poison == nullptr || fabsf(static_cast<float>(denW) * sd) < kFixedLimit)
            acc_add(block_ptr(t, t.accD[p], t.accD0[p], q.y, q.x, pitch), denW, sd);
        else  // the block's weight reaches all of its pixels
            for (int i = 0; i < kBS * kBS; ++i)
                poison[static_cast<long long>(q.y + (i >> 3)) * a.width + q.x + (i & 7)] = 1;
    }
}

// Collaborative filtering of one group on plane p, aggregated into the CTA's
// accumulator windows.
// `check`: the plane holds non-finite pixels (poison_map is not null), so
// every member goes through the checking aggregation.
template <typename T, bool WIENER>
__device__ void filter_group(const StageArgs<T> &a, const Tile<T> &t, int p, const BlockPos *list,
                             int n, int lane, T *G, float scale, unsigned &n_bad, int pt = -1,
                             bool check = false)
{
    // p indexes the tile's windows; pt (default p) the plane's threshold /
    // Wiener tables, which differ when planes share one set of windows
    if (pt < 0) pt = p;
    T sa[kGSMax], sb[kGSMax];
    T ra[kGSMax], rb[kGSMax];
    if (WIENER) {
        gather_xy_forward(t, t.refw[p], t.ref0[p], list, n, lane, G, n_bad);
        group_fwd(G, n, lane, ra, rb);
        __syncwarp();
    }
    gather_xy_forward(t, t.srcw[p], t.src0[p], list, n, lane, G, n_bad);
    group_fwd(G, n, lane, sa, sb);

    T denW;
    if (!WIENER) {
        // Hard threshold: |x| <= thr -> 0, else retained (source/BM3D.cpp:361-371).
        // thr depends on how many of (x, y, z) are 0 (source/BM3D.cpp:52-67).
        // pencil a = (lane / 4, 2 (lane % 4)), pencil b = (lane / 4, 2 (lane % 4) + 1)
        const int fa = ((lane & 3) == 0) + (lane < 4), fb = (lane < 4);
        const T *thr = a.thr[pt][n - 1];
        int kept = 0;
#pragma unroll
        for (int z = 0; z < kGSMax; ++z) {
            if (z < n) {
                const T ta = thr[fa + (z == 0)], tb = thr[fb + (z == 0)];
                const T va = sa[z], vb = sb[z];
                const T aa = va < T(0) ? -va : va, ab = vb < T(0) ? -vb : vb;
                if (aa <= ta) sa[z] = T(0); else ++kept;
                if (ab <= tb) sb[z] = T(0); else ++kept;
            }
        }
        const int retained = __reduce_add_sync(0xffffffffu, kept);
        denW = retained < 1 ? T(1) : T(1) / static_cast<T>(retained);
    } else {
        // Empirical Wiener shrinkage guided by the basic estimate
        // (source/BM3D.cpp:435-443).
        const T s2 = a.wss[pt][n - 1];
        T l2 = T(0);
#pragma unroll
        for (int z = 0; z < kGSMax; ++z) {
            if (z < n) {
                const T ya2 = ra[z] * ra[z], yb2 = rb[z] * rb[z];
                const T wa = wiener_weight(ya2, s2), wb = wiener_weight(yb2, s2);
                sa[z] *= wa;
                sb[z] *= wb;
                l2 += wa * wa + wb * wb;
            }
        }
        l2 = warp_sum(l2);
        denW = l2 <= T(0) ? T(1) : T(1) / l2;
    }
    const T numW = static_cast<T>(static_cast<double>(denW) / a.finalAMP[n - 1]);

    group_inv(G, n, lane, sa, sb);
    __syncwarp();
    xy_inverse_cols(G, n, lane);

    // Rows of the inverse 2-D transform, each aggregated as soon as it is
    // ready: BlockGroup::AddTo / CountTo (include/Block.h:1240-1265,
    // 1334-1357). The weight is the same over the block, so it is added once,
    // at the block's origin; the normalisation sums origins over each pixel's
    // covering blocks. Integer sums make that exactly the per-pixel sum.
    const int z = lane >> 1, h = lane & 1;
    if (z < n && block_in_tile(t, list[z].y, list[z].x)) {
        const BlockPos q = list[z];
        const T *gz = G + z * kGroupStride;
        if (!check && (q.y >= kBS || q.x >= kBS)) {
            int pitch;
            auto *dn = block_ptr(t, t.accN[p], t.accN0[p], q.y, q.x, pitch);
#pragma unroll 1
            for (int r = 0; r < 4; ++r) {
                const int y = 4 * h + r;
                T v[8];
                Vec4<T>::load(gz + gidx(y, 0), v[0], v[1], v[2], v[3]);
                Vec4<T>::load(gz + gidx(y, 4), v[4], v[5], v[6], v[7]);
                redft01_8(v);
#pragma unroll
                for (int x = 0; x < 8; ++x) acc_add(dn + y * pitch + x, v[x] * numW, scale);
            }
            if (h == 0) acc_add(block_ptr(t, t.accD[p], t.accD0[p], q.y, q.x, pitch), denW, scale);
        } else {
            aggregate_member_slow<T>(a, t, p, pt, q, gz, h, numW, denW, scale);
        }
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// CTA-level pieces shared by the register-resident and the generic kernels.

// The CTA's tile of reference positions and its staged window: the union of
// the search windows of the tile's blocks (or the blocks themselves when no
// matching happens).
template <typename T>
__device__ __forceinline__ void tile_window(const StageArgs<T> &a, int tile, int bs, Tile<T> &t,
                                            int &kx0, int &kx1, int &ky0, int &ky1)
{
    const int tx = tile % a.tiles_x, ty = tile / a.tiles_x;
    kx0 = tx * a.tile_x;
    ky0 = ty * a.tile_y;
    kx1 = min(kx0 + a.tile_x, a.nx);
    ky1 = min(ky0 + a.tile_y, a.ny);
    const int right = a.width - bs, bottom = a.height - bs;
    int y0 = 1 << 30, y1 = -1, x0 = 1 << 30, x1 = -1;
    if (a.match) {
        for (int k = ky0; k < ky1; ++k) {
            const int j = ref_pos(k, a.step, bottom);
            y0 = min(y0, search_boundary(j, 0, a.range, a.bm_step));
            y1 = max(y1, search_boundary(j, bottom, a.range, a.bm_step));
        }
        for (int k = kx0; k < kx1; ++k) {
            const int i = ref_pos(k, a.step, right);
            x0 = min(x0, search_boundary(i, 0, a.range, a.bm_step));
            x1 = max(x1, search_boundary(i, right, a.range, a.bm_step));
        }
    } else {
        y0 = ref_pos(ky0, a.step, bottom);
        y1 = ref_pos(ky1 - 1, a.step, bottom);
        x0 = ref_pos(kx0, a.step, right);
        x1 = ref_pos(kx1 - 1, a.step, right);
    }
    t.ry0 = y0;
    t.rx0 = x0;
    t.rh = y1 + bs - y0;
    t.rw = x1 + bs - x0;
    t.pitch = a.region_pitch;
    t.bs = bs;
    t.origin_inside = (y0 == 0 && x0 == 0);
}

// Carve the CTA's shared memory into staged windows, accumulators and the
// (0, 0) copies, following plan_smem.
template <typename T, bool WIENER, int NPL>
__device__ __forceinline__ void carve_tile(const StageArgs<T> &a, const SmemPlan &sp,
                                           unsigned char *smem, Tile<T> &t)
{
    using Acc = typename AccOf<T>::type;
    const int bsq = t.bs * t.bs;
    int s = 0;
    T *origin = reinterpret_cast<T *>(smem + sp.off_origin);
    for (int p = 0; p < NPL; ++p) {
        t.srcw[p] = reinterpret_cast<const T *>(smem + sp.region_bytes * s);
        t.src0[p] = origin + bsq * s;
        ++s;
    }
    for (int p = 0; p < NPL; ++p) {
        const bool has_ref = WIENER || p == 0;
        if (!has_ref || (a.ref_alias_src & (1 << p))) {
            t.refw[p] = t.srcw[p];
            t.ref0[p] = t.src0[p];
        } else {
            t.refw[p] = reinterpret_cast<const T *>(smem + sp.region_bytes * s);
            t.ref0[p] = origin + bsq * s;
            ++s;
        }
    }
    Acc *origin_acc = reinterpret_cast<Acc *>(smem + sp.off_origin_acc);
    for (int p = 0; p < NPL; ++p) {
        t.accN[p] = reinterpret_cast<Acc *>(smem + sp.off_acc + sp.acc_bytes * (2 * p));
        t.accD[p] = reinterpret_cast<Acc *>(smem + sp.off_acc + sp.acc_bytes * (2 * p + 1));
        t.accN0[p] = origin_acc + bsq * (2 * p);
        t.accD0[p] = origin_acc + bsq * (2 * p + 1);
    }
}

// One element global -> shared without a register round trip (cp.async;
// element-sized, so no alignment beyond the element's own). Completed by
// cp_async_wait_all before the CTA barrier that publishes the windows.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src)
{
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src), "n"(sizeof(T))
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Load the staged windows (and block (0, 0) when outside) and zero the
// accumulators. Ends with __syncthreads().
template <typename T, bool WIENER, int NPL>
__device__ __forceinline__ void stage_tile(const StageArgs<T> &a, const Tile<T> &t)
{
    const int tid = threadIdx.x;
    const int npx = t.rh * t.rw;
    const int bs = t.bs, bsq = bs * bs;
    for (int p = 0; p < NPL; ++p) {
        const bool need_src = !a.bm_only && (a.active & (1 << p));
        const bool need_ref = (p == 0) || (WIENER && need_src);
        const bool ref_sep = need_ref && t.refw[p] != t.srcw[p];
        for (int i = tid; i < npx; i += blockDim.x) {
            const int y = i / t.rw, x = i - y * t.rw;
            const long long g = static_cast<long long>(t.ry0 + y) * a.stride + (t.rx0 + x);
            const int s = y * t.pitch + x;
            if (need_src || (p == 0 && !ref_sep)) cp_async_elem(const_cast<T *>(t.srcw[p]) + s, a.src[p] + g);
            if (ref_sep) cp_async_elem(const_cast<T *>(t.refw[p]) + s, a.ref[p] + g);
            if (need_src) {
                t.accN[p][s] = 0;
                t.accD[p][s] = 0;
            }
        }
        if (!t.origin_inside && (need_src || p == 0)) {
            for (int i = tid; i < bsq; i += blockDim.x) {
                const int y = i / bs, x = i - y * bs;
                const long long g = static_cast<long long>(y) * a.stride + x;
                const_cast<T *>(t.src0[p])[i] = __ldg(a.src[p] + g);
                if (ref_sep) const_cast<T *>(t.ref0[p])[i] = __ldg(a.ref[p] + g);
                t.accN0[p][i] = 0;
                t.accD0[p][i] = 0;
            }
        }
    }
    cp_async_wait_all();
    __syncthreads();
}

// Flush the accumulator windows into the plane-wide num / den sums.
template <typename T, int NPL>
__device__ __forceinline__ void flush_tile(const StageArgs<T> &a, const Tile<T> &t)
{
    const int tid = threadIdx.x;
    const int npx = t.rh * t.rw;
    const int bs = t.bs, bsq = bs * bs;
    for (int p = 0; p < NPL; ++p) {
        if (!(a.active & (1 << p))) continue;
        for (int i = tid; i < npx; i += blockDim.x) {
            const int y = i / t.rw, x = i - y * t.rw;
            const int s = y * t.pitch + x;
            const auto nv = t.accN[p][s], d = t.accD[p][s];
            const long long g = static_cast<long long>(t.ry0 + y) * a.width + (t.rx0 + x);
            if (nv != 0) acc_flush(a.num[p] + g, nv);
            if (d != 0) acc_flush(a.den[p] + g, d);
        }
        if (!t.origin_inside) {
            for (int i = tid; i < bsq; i += blockDim.x) {
                const auto nv = t.accN0[p][i], d = t.accD0[p][i];
                const int y = i / bs, x = i - y * bs;
                const long long g = static_cast<long long>(y) * a.width + x;
                if (nv != 0) acc_flush(a.num[p] + g, nv);
                if (d != 0) acc_flush(a.den[p] + g, d);
            }
        }
    }
}

template <typename T>
__device__ __forceinline__ void dump_group(const StageArgs<T> &a, int ky, int kx, int n, int lane,
                                           const BlockPos *list, const T *lkeys)
{
    if (a.group_count == nullptr) return;
    const long long ridx = static_cast<long long>(ky) * a.nx + kx;
    if (lane == 0) a.group_count[ridx] = n;
    for (int k = lane; k < n; k += kWarp) {
        a.group_pos[(ridx * kGSTab + k) * 2 + 0] = list[k].y;
        a.group_pos[(ridx * kGSTab + k) * 2 + 1] = list[k].x;
        a.group_key[ridx * kGSTab + k] = lkeys[k];
    }
}

// A CTA whose launch gave it less shared memory than its layout needs does
// no work and counts itself in the invariant counter (host-mode calls then
// fail with an internal error) instead of touching memory past its share.
template <typename T>
__device__ __forceinline__ void smem_shortfall(const StageArgs<T> &a)
{
    if (a.bad != nullptr && threadIdx.x == 0) atomicAdd(a.bad, 1ull << 32);
}

template <typename T>
__device__ __forceinline__ void flush_stats(const StageArgs<T> &a, int lane, unsigned n_sum,
                                            unsigned n_sq, unsigned n_cand, unsigned n_fix,
                                            unsigned n_bad)
{
    using U = unsigned long long;
    if (a.stats != nullptr && lane == 0) {
        atomicAdd(a.stats + 0, static_cast<U>(n_sum));
        atomicAdd(a.stats + 1, static_cast<U>(n_sq));
        atomicAdd(a.stats + 2, static_cast<U>(n_cand));
        atomicAdd(a.stats + 3, static_cast<U>(n_fix));
    }
    if (a.bad != nullptr && n_bad) atomicAdd(a.bad, static_cast<U>(n_bad));
}

// ---------------------------------------------------------------------------
// Register-resident stage: BlockSize 8, GroupSize <= 16. One tile per call.
template <typename T, bool WIENER, int NPL, int KS>
__device__ __forceinline__ void stage_tile_body(const StageArgs<T> &a, int tile, unsigned char *smem,
                                                unsigned avail)
{
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const int right = a.width - kBS, bottom = a.height - kBS;

    Tile<T> t;
    int kx0, kx1, ky0, ky1;
    tile_window(a, tile, kBS, t, kx0, kx1, ky0, ky1);
    const SmemPlan sp = plan_smem<T>(NPL, WIENER, a.ref_alias_src, a.region_h, a.region_pitch,
                                     a.key_slots, nwarps);
    if (sp.total > avail) {  // launched with less shared memory than the layout needs
        smem_shortfall(a);
        return;
    }
    carve_tile<T, WIENER, NPL>(a, sp, smem, t);
    stage_tile<T, WIENER, NPL>(a, t);

    // Per-warp scratch.
    unsigned char *wbase = smem + sp.off_warps + sp.warp_bytes * warp;
    const size_t scratch = sp.scratch_bytes;
    T *G = reinterpret_cast<T *>(wbase);
    SortKey<T> *keys = reinterpret_cast<SortKey<T> *>(wbase);
    SortKey<T> *heap = reinterpret_cast<SortKey<T> *>(wbase + scratch);
    BlockPos *list = reinterpret_cast<BlockPos *>(wbase + scratch + sizeof(SortKey<T>) * kCand);
    T *lkeys = reinterpret_cast<T *>(wbase + scratch + sizeof(SortKey<T>) * kCand +
                                     sizeof(BlockPos) * kGSTab);

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
        const int n = match_block<T, KS>(a, t, j0, i0, lane, keys, heap, list, lkeys, n_cand, n_fix);
        n_sum += n;
        n_sq += static_cast<unsigned>(n * n);
        dump_group(a, ky, kx, n, lane, list, lkeys);
        if (!a.bm_only) {
#pragma unroll
            for (int p = 0; p < NPL; ++p)
                if (a.active & (1 << p))
                    filter_group<T, WIENER>(a, t, p, list, n, lane, G, scale[p], n_bad, -1,
                                            check[p]);
        }
        __syncwarp();
    }
    flush_stats(a, lane, n_sum, n_sq, n_cand, n_fix, n_bad);
    if (a.bm_only) return;
    __syncthreads();
    flush_tile<T, NPL>(a, t);
}

// One plane c of a three-plane tile into the single-plane windows: src[c],
// ref[c] where a stage reads it (matching on plane 0; Wiener on every plane),
// zeroed sums. Ends with __syncthreads().
template <typename T, bool WIENER>
__device__ __forceinline__ void stage_plane(const StageArgs<T> &a, const Tile<T> &t, int c)
{
    const int tid = threadIdx.x;
    const int npx = t.rh * t.rw;
    const int bs = t.bs, bsq = bs * bs;
    const bool ref_sep = t.refw[0] != t.srcw[0];
    const bool need_ref = ref_sep && (WIENER || c == 0);
    const bool filt = !a.bm_only && (a.active & (1 << c));
    for (int i = tid; i < npx; i += blockDim.x) {
        const int y = i / t.rw, x = i - y * t.rw;
        const long long g = static_cast<long long>(t.ry0 + y) * a.stride + (t.rx0 + x);
        const int s = y * t.pitch + x;
        cp_async_elem(const_cast<T *>(t.srcw[0]) + s, a.src[c] + g);
        if (need_ref) cp_async_elem(const_cast<T *>(t.refw[0]) + s, a.ref[c] + g);
        if (filt) {
            t.accN[0][s] = 0;
            t.accD[0][s] = 0;
        }
    }
    if (!t.origin_inside) {
        for (int i = tid; i < bsq; i += blockDim.x) {
            const int y = i / bs, x = i - y * bs;
            const long long g = static_cast<long long>(y) * a.stride + x;
            const_cast<T *>(t.src0[0])[i] = __ldg(a.src[c] + g);
            if (need_ref) const_cast<T *>(t.ref0[0])[i] = __ldg(a.ref[c] + g);
            t.accN0[0][i] = 0;
            t.accD0[0][i] = 0;
        }
    }
    cp_async_wait_all();
    __syncthreads();
}

// Flush plane c's accumulator windows (the single-plane windows) into its sums.
template <typename T>
__device__ __forceinline__ void flush_plane(const StageArgs<T> &a, const Tile<T> &t, int c)
{
    const int tid = threadIdx.x;
    const int npx = t.rh * t.rw;
    const int bs = t.bs, bsq = bs * bs;
    for (int i = tid; i < npx; i += blockDim.x) {
        const int y = i / t.rw, x = i - y * t.rw;
        const int s = y * t.pitch + x;
        const auto nv = t.accN[0][s], d = t.accD[0][s];
        const long long g = static_cast<long long>(t.ry0 + y) * a.width + (t.rx0 + x);
        if (nv != 0) acc_flush(a.num[c] + g, nv);
        if (d != 0) acc_flush(a.den[c] + g, d);
    }
    if (!t.origin_inside) {
        for (int i = tid; i < bsq; i += blockDim.x) {
            const auto nv = t.accN0[0][i], d = t.accD0[0][i];
            const int y = i / bs, x = i - y * bs;
            const long long g = static_cast<long long>(y) * a.width + x;
            if (nv != 0) acc_flush(a.num[c] + g, nv);
            if (d != 0) acc_flush(a.den[c] + g, d);
        }
    }
}

// Three planes sharing the groups matched on plane 0 (BM3D_Base::Kernel's
// 9-plane form, source/BM3D.cpp:139-218), one plane at a time through a
// single plane's windows: plane 0 matches and keeps each reference block's
// group list in shared memory, planes 1 and 2 re-stage their windows and
// filter with those lists. Per plane the arithmetic is that of the
// one-plane tile, so results equal the all-planes-resident form bit for bit
// while the footprint stays that of one plane (full-size tiles).
template <typename T, bool WIENER, int KS>
__device__ __forceinline__ void stage_tile_body_seq3(const StageArgs<T> &a, int tile,
                                                     unsigned char *smem, unsigned avail)
{
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const int right = a.width - kBS, bottom = a.height - kBS;

    Tile<T> t;
    int kx0, kx1, ky0, ky1;
    tile_window(a, tile, kBS, t, kx0, kx1, ky0, ky1);
    const SmemPlan sp = plan_smem<T>(3, WIENER, a.ref_alias_src, a.region_h, a.region_pitch,
                                     a.key_slots, nwarps, false, kBS, kGSMax,
                                     a.tile_x * a.tile_y);
    if (sp.total > avail) {  // launched with less shared memory than the layout needs
        smem_shortfall(a);
        return;
    }
    carve_tile<T, WIENER, 1>(a, sp, smem, t);  // every plane goes through windows [0]
    // group lists: position (y - ry0) << 8 | (x - rx0), or 0xffff for a
    // (0, 0) block held outside the window; then one count byte per block
    unsigned short *gpos = reinterpret_cast<unsigned short *>(smem + sp.off_groups);
    unsigned char *gn = reinterpret_cast<unsigned char *>(gpos + a.tile_x * a.tile_y * kGSMax);

    unsigned char *wbase = smem + sp.off_warps + sp.warp_bytes * warp;
    const size_t scratch = sp.scratch_bytes;
    T *G = reinterpret_cast<T *>(wbase);
    SortKey<T> *keys = reinterpret_cast<SortKey<T> *>(wbase);
    SortKey<T> *heap = reinterpret_cast<SortKey<T> *>(wbase + scratch);
    BlockPos *list = reinterpret_cast<BlockPos *>(wbase + scratch + sizeof(SortKey<T>) * kCand);
    T *lkeys = reinterpret_cast<T *>(wbase + scratch + sizeof(SortKey<T>) * kCand +
                                     sizeof(BlockPos) * kGSTab);

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
                n = match_block<T, KS>(a, t, j0, i0, lane, keys, heap, list, lkeys, n_cand, n_fix);
                n_sum += n;
                n_sq += static_cast<unsigned>(n * n);
                dump_group(a, ky, kx, n, lane, list, lkeys);
                if (lane == 0) gn[r] = static_cast<unsigned char>(n);
                for (int k = lane; k < n; k += kWarp) {
                    const BlockPos q = list[k];
                    const bool outside = q.y == 0 && q.x == 0 && !t.origin_inside;
                    gpos[r * kGSMax + k] = outside ? 0xffff
                                                   : static_cast<unsigned short>(
                                                         ((q.y - t.ry0) << 8) | (q.x - t.rx0));
                }
            } else {
                n = gn[r];
                for (int k = lane; k < n; k += kWarp) {
                    const unsigned v = gpos[r * kGSMax + k];
                    list[k] = v == 0xffffu ? BlockPos{0, 0}
                                           : BlockPos{t.ry0 + static_cast<int>(v >> 8),
                                                      t.rx0 + static_cast<int>(v & 0xffu)};
                }
            }
            __syncwarp();
            if (filt) filter_group<T, WIENER>(a, t, 0, list, n, lane, G, scale, n_bad, c, check);
            __syncwarp();
        }
        __syncthreads();
        if (filt) flush_plane<T>(a, t, c);
        __syncthreads();  // the windows are re-staged for the next plane
    }
    flush_stats(a, lane, n_sum, n_sq, n_cand, n_fix, n_bad);
}

template <typename T, bool WIENER, int NPL, int KS>
__global__ void __launch_bounds__(512, 1) stage_kernel(const StageArgs<T> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const unsigned avail = dynamic_smem_bytes();
    if constexpr (NPL == 3) stage_tile_body_seq3<T, WIENER, KS>(a, blockIdx.x, smem, avail);
    else stage_tile_body<T, WIENER, NPL, KS>(a, blockIdx.x, smem, avail);
}

// dst = num / den (source/BM3D.cpp:130-135, include/Image_Type.hpp:319-332).
// Outside block (0, 0) both sums carry the same fixed-point scale, which
// cancels.
__device__ __forceinline__ float ratio(long long n, long long d)
{
    return static_cast<float>(static_cast<double>(n) / static_cast<double>(d));
}
__device__ __forceinline__ double ratio(double n, double d) { return n / d; }

// Tile of the normalisation: 32 x 32 pixels per CTA.
constexpr int kNormTile = 32;

// dst = num / den for the kNormTile^2 pixels at (y0, x0), with den(y, x) the
// sum of the block weights W at the bs x bs origins whose block covers
// (y, x): y - bs < oy <= y, x - bs < ox <= x. Separable sums over a
// shared-memory copy of W; exact for integer sums.
//
// FP32 (fixed point): block (0, 0)'s pixels and the weight at origin (0, 0)
// carry the scale of log2_corner, everything else that of log2_bound
// (fixed_scale); for those pixels den = (sum of the other weights) * ratio +
// W(0, 0), ratio = corner scale / general scale (a power of two, exact).
// On planes whose prep found non-finite inputs (*nonfinite != 0) the pixels
// marked in `poison` get NaN -- a non-finite term reached them
// (acc_add_checked) -- and the map is cleared as it is read, so it is all
// zero again for the next stage; other planes never touch it.
template <typename T>
__device__ __forceinline__ void normalize_tile(T *dst, long long dst_stride,
                                               const typename AccOf<T>::type *num,
                                               const typename AccOf<T>::type *wsum, int width,
                                               int height, int bs, int y0, int x0,
                                               unsigned char *poison = nullptr,
                                               const unsigned *nonfinite = nullptr,
                                               const float *absmax = nullptr, int log2_bound = 0,
                                               int log2_corner = 0)
{
    using Acc = typename AccOf<T>::type;
    constexpr bool kFixed = std::is_same<Acc, long long>::value;
    constexpr int N = kNormTile, E = N + kBSMax - 1;
    __shared__ Acc w[E][E];
    __shared__ Acc hs[E][N];
    const int ext = N + bs - 1;
    // origin (0, 0) is summed apart in fixed point (its own scale)
    const bool split = kFixed && y0 < bs && x0 < bs;
    for (int i = threadIdx.x; i < ext * ext; i += blockDim.x) {
        const int ly = i / ext, lx = i - ly * ext;
        const int gy = y0 - bs + 1 + ly, gx = x0 - bs + 1 + lx;
        w[ly][lx] = (gy >= 0 && gx >= 0 && gy < height && gx < width &&
                     !(split && gy == 0 && gx == 0))
                        ? wsum[static_cast<long long>(gy) * width + gx]
                        : Acc(0);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < ext * N; i += blockDim.x) {
        const int ly = i / N, lx = i - ly * N;
        Acc v = 0;
        for (int d = 0; d < bs; ++d) v += w[ly][lx + d];
        hs[ly][lx] = v;
    }
    __syncthreads();
    const bool marked = poison != nullptr && nonfinite != nullptr && *nonfinite != 0;
    double cratio = 1.0;
    if (split) {
        const float am = absmax != nullptr ? *absmax : 1.0f;
        cratio = static_cast<double>(fixed_scale(am, log2_corner)) /
                 static_cast<double>(fixed_scale(am, log2_bound));
    }
    for (int i = threadIdx.x; i < N * N; i += blockDim.x) {
        const int ly = i / N, lx = i - ly * N;
        const int gy = y0 + ly, gx = x0 + lx;
        if (gy >= height || gx >= width) continue;
        Acc d = 0;
        for (int k = 0; k < bs; ++k) d += hs[ly + k][lx];
        const long long g = static_cast<long long>(gy) * width + gx;
        T out;
        if (split && gy < bs && gx < bs)  // block (0, 0): covered by origin (0, 0)
            out = static_cast<T>(static_cast<double>(num[g]) /
                                 (static_cast<double>(d) * cratio + static_cast<double>(wsum[0])));
        else
            out = ratio(num[g], d);
        if (marked && poison[g]) {
            out = static_cast<T>(NAN);
            poison[g] = 0;
        }
        dst[gy * dst_stride + gx] = out;
    }
    __syncthreads();  // before the next tile overwrites w / hs
}

// Fixed-point normalisation by strips, one warp per strip of 32 columns x
// kStripRows rows, no shared tile and no CTA barrier. Lane l owns column
// x0 + l. For each row r (from bs - 1 rows above the strip, to prime the
// sums) the warp loads the block weights W of columns x0 - bs + 1 .. x0 + 31
// (one or two 64-bit words per lane, four rows ahead), stores them in a
// per-warp row buffer and each lane sums the bs of them left of and at its
// column: h(r). The vertical box sum is a running sum over the last bs rows'
// h, kept in a per-warp ring. The integer sums are exactly those of
// normalize_tile, so the output is the same; the block-(0, 0) handling and
// poison marks are as there. `ring` is this warp's ring_rows x 32 words
// (ring_rows a power of two >= bs, ring_mask = ring_rows - 1), `hrow` its
// 2 x 64-word row buffer.
constexpr int kStripRows = 32;

// Rows of the per-warp ring of horizontal sums: bs rounded up to a power of
// two (8 for the 8 x 8 blocks of most profiles, so eight 256-thread CTAs fit
// an SM), and the dynamic shared memory of a 256-thread normalisation CTA.
__host__ __device__ inline int strip_ring_rows(int bs) { return bs <= 8 ? 8 : 16; }
__host__ __device__ inline int strip_smem_bytes(int bs)
{
    return 8 * (strip_ring_rows(bs) * 32 + 128) * static_cast<int>(sizeof(long long));
}

__device__ __forceinline__ void normalize_strip(float *dst, long long dst_stride, const long long *num,
                                                const long long *wsum, int width, int height, int bs,
                                                int x0, int y0, unsigned char *poison, bool marked,
                                                double cratio, long long *ring, int ring_mask,
                                                long long *hrow)
{
    const int lane = threadIdx.x & 31;
    const bool split = x0 == 0 && y0 == 0;  // the only strip whose sums reach W(0, 0)
    const int xa = x0 - bs + 1 + lane, xb = xa + 32;
    const int rstart = y0 - bs + 1, rend = min(y0 + kStripRows, height);
    const int x = x0 + lane;
    long long V = 0;
    // four rows at a time: their loads are all issued before the first row's
    // sums, so a warp has four rows of DRAM latency in flight, not one
    for (int rb = rstart; rb < rend; rb += 4) {
        long long A0[4], A1[4], NUM[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = rb + j;
            A0[j] = A1[j] = NUM[j] = 0;
            if (r >= 0 && r < rend) {
                const long long *row = wsum + static_cast<long long>(r) * width;
                if (xa >= 0 && xa < width && !(split && r == 0 && xa == 0)) A0[j] = row[xa];
                if (lane < bs - 1 && xb < width) A1[j] = row[xb];
                if (r >= y0 && x < width) NUM[j] = num[static_cast<long long>(r) * width + x];
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = rb + j;
            if (r >= rend) break;  // warp-uniform
            // the row's bs - 1 + 32 window words into this row's buffer (two
            // alternate, so one __syncwarp per row separates writes and reads)
            long long *hb = hrow + ((r - rstart) & 1) * 64;
            hb[lane] = A0[j];
            hb[32 + lane] = A1[j];
            __syncwarp();
            long long h = 0;
#pragma unroll 4
            for (int d = 0; d < bs; ++d) h += hb[lane + d];
            const int k = r - rstart;
            if (k >= bs) V -= ring[((k - bs) & ring_mask) * 32 + lane];  // read before reuse
            V += h;
            ring[(k & ring_mask) * 32 + lane] = h;
            if (r >= y0 && x < width) {
                const long long g = static_cast<long long>(r) * width + x;
                float out;
                if (split && r < bs && x < bs)  // block (0, 0): covered by origin (0, 0)
                    out = static_cast<float>(static_cast<double>(NUM[j]) /
                                             (static_cast<double>(V) * cratio +
                                              static_cast<double>(wsum[0])));
                else
                    out = ratio(NUM[j], V);
                if (marked && poison[g]) {
                    out = NAN;
                    poison[g] = 0;
                }
                dst[r * dst_stride + x] = out;
            }
        }
    }
}

// Every strip of one fixed-point plane, warp w of the calling grid taking
// strips w, w + nwarps, ... (256-thread CTAs: 8 warps).
__device__ __forceinline__ void normalize_plane_strips(float *dst, long long dst_stride,
                                                       const long long *num, const long long *wsum,
                                                       int width, int height, int bs,
                                                       unsigned char *poison,
                                                       const unsigned *nonfinite,
                                                       const float *absmax, int log2_bound,
                                                       int log2_corner, long long first_warp,
                                                       long long nwarps)
{
    extern __shared__ long long strip_ring[];  // per warp: ring_rows(bs) x 32 words, 128-word row buffer
    const int rows = strip_ring_rows(bs);
    const int sx = (width + 31) / 32, sy = (height + kStripRows - 1) / kStripRows;
    const bool marked = poison != nullptr && nonfinite != nullptr && *nonfinite != 0;
    const float am = absmax != nullptr ? *absmax : 1.0f;
    const double cratio = static_cast<double>(fixed_scale(am, log2_corner)) /
                          static_cast<double>(fixed_scale(am, log2_bound));
    long long *r = strip_ring + ((threadIdx.x >> 5) & 7) * (rows * 32 + 128);
    for (long long t = first_warp; t < static_cast<long long>(sx) * sy; t += nwarps) {
        const int ty = static_cast<int>(t / sx), tx = static_cast<int>(t - static_cast<long long>(ty) * sx);
        normalize_strip(dst, dst_stride, num, wsum, width, height, bs, tx * 32, ty * kStripRows,
                        poison, marked, cratio, r, rows - 1, r + rows * 32);
    }
}

// Grid of the single-plane normalisation: 32 x 32 tiles (FP64 sums), or one
// warp per strip (fixed point).
template <typename T>
inline dim3 normalize_grid(int width, int height)
{
    if (std::is_same<T, float>::value) {
        const long long strips = static_cast<long long>((width + 31) / 32) *
                                 ((height + kStripRows - 1) / kStripRows);
        return dim3(static_cast<unsigned>((strips + 7) / 8));
    }
    return dim3((width + kNormTile - 1) / kNormTile, (height + kNormTile - 1) / kNormTile);
}

// One plane: grid = normalize_grid<T>(width, height), 256 threads.
template <typename T>
__global__ void __launch_bounds__(256)
    normalize_kernel(T *dst, long long dst_stride, const typename AccOf<T>::type *num,
                     const typename AccOf<T>::type *wsum, int width, int height, int bs,
                     unsigned char *poison = nullptr, const unsigned *nonfinite = nullptr,
                     const float *absmax = nullptr, int log2_bound = 0, int log2_corner = 0)
{
    if constexpr (std::is_same<T, float>::value) {
        normalize_plane_strips(dst, dst_stride, num, wsum, width, height, bs, poison, nonfinite,
                               absmax, log2_bound, log2_corner,
                               static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) +
                                   (threadIdx.x >> 5),
                               static_cast<long long>(gridDim.x) * (blockDim.x >> 5));
    } else {
        normalize_tile<T>(dst, dst_stride, num, wsum, width, height, bs, blockIdx.y * kNormTile,
                          blockIdx.x * kNormTile, poison, nonfinite, absmax, log2_bound, log2_corner);
    }
}

// Zero one plane's accumulators and fold the largest finite |src| into
// *absmax (which the caller zeroes first; non-negative floats order like their
// bit patterns). With `nonfinite` (FP32 only) it also counts the NaN / Inf
// pixels of src and of ref (when given) into *nonfinite, so that the stage
// kernel checks its terms only on such planes. Rows row0, row0 + row_step, ...
// of the plane, threads along each row.
template <typename T>
__device__ __forceinline__ void prep_plane(typename AccOf<T>::type *num,
                                           typename AccOf<T>::type *den, const T *src,
                                           const T *ref, long long stride, int width, int height,
                                           float *absmax, unsigned *nonfinite, int row0,
                                           int row_step)
{
    float m = 0.0f;
    unsigned bad = 0;
    for (int y = row0; y < height; y += row_step) {
        const long long o = static_cast<long long>(y) * width;
        const T *s = src + static_cast<long long>(y) * stride;
        const T *r = ref != nullptr ? ref + static_cast<long long>(y) * stride : nullptr;
        if constexpr (sizeof(T) == 4) {
            // two pixels per thread where the row allows 16-byte sum stores
            // and 8-byte source loads (uniform over the CTA)
            const bool vec = (width % 2 == 0) &&
                             ((reinterpret_cast<uintptr_t>(num + o) | reinterpret_cast<uintptr_t>(den + o)) & 15) == 0 &&
                             ((reinterpret_cast<uintptr_t>(s) | reinterpret_cast<uintptr_t>(r)) & 7) == 0;
            if (vec) {
                for (int x = 2 * threadIdx.x; x < width; x += 2 * blockDim.x) {
                    *reinterpret_cast<longlong2 *>(num + o + x) = make_longlong2(0, 0);
                    *reinterpret_cast<longlong2 *>(den + o + x) = make_longlong2(0, 0);
                    const float2 v2 = *reinterpret_cast<const float2 *>(s + x);
                    const float v0 = fabsf(v2.x), v1 = fabsf(v2.y);
                    if (v0 <= 3.4028235e38f) m = v0 > m ? v0 : m;  // NaN and Inf are skipped
                    else ++bad;
                    if (v1 <= 3.4028235e38f) m = v1 > m ? v1 : m;
                    else ++bad;
                    if (r != nullptr) {
                        const float2 r2 = *reinterpret_cast<const float2 *>(r + x);
                        if (!(fabsf(r2.x) <= 3.4028235e38f)) ++bad;
                        if (!(fabsf(r2.y) <= 3.4028235e38f)) ++bad;
                    }
                }
                continue;
            }
        }
        for (int x = threadIdx.x; x < width; x += blockDim.x) {
            num[o + x] = 0;
            den[o + x] = 0;
            const float v = fabsf(static_cast<float>(s[x]));
            if (v <= 3.4028235e38f) m = v > m ? v : m;  // NaN and Inf are skipped
            else ++bad;
            if (r != nullptr && !(fabsf(static_cast<float>(r[x])) <= 3.4028235e38f)) ++bad;
        }
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        const float q = __shfl_xor_sync(0xffffffffu, m, o);
        m = q > m ? q : m;
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (m > 0.0f) atomicMax(reinterpret_cast<int *>(absmax), __float_as_int(m));
        if (nonfinite != nullptr && bad) atomicAdd(nonfinite, bad);
    }
}

// One plane, one row per CTA at a time.
template <typename T>
__global__ void prep_kernel(typename AccOf<T>::type *num, typename AccOf<T>::type *den,
                            const T *src, long long stride, int width, int height, float *absmax,
                            const T *ref = nullptr, unsigned *nonfinite = nullptr)
{
    prep_plane<T>(num, den, src, ref, stride, width, height, absmax, nonfinite, blockIdx.x,
                  gridDim.x);
}

}  // namespace bm3d
