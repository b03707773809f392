// Device-side pieces shared by the BM3D stage kernels: exactly-rounded
// arithmetic helpers, the search-window geometry of the reference, sort keys
// and the shared-memory layout of one CTA.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bm3d {

constexpr int kWarp = 32;
constexpr int kBS = 8;           // block size handled by the register-resident path
constexpr int kGSMax = 16;       // largest group the register-resident path holds
constexpr int kGSTab = 32;       // largest GroupSize handled at all (generic path)
constexpr int kBSMax = 16;       // largest BlockSize handled at all (generic path)
constexpr int kGroupStride = 72; // floats per block in a warp's group buffer (64 + 8 pad)
constexpr int kCand = 64;
// FP32 group-axis matrices of lengths 1..15 except 8, 16 rows per column
constexpr int kPadTable = 16 * (15 * 16 / 2 - 8);
__host__ __device__ constexpr int pad_table_offset(int n)
{
    return 16 * ((n - 1) * n / 2 - (n > 8 ? 8 : 0));
}        // candidates a warp sorts after thresholding

// ---------------------------------------------------------------------------
// Arithmetic that must not be contracted into FMA: the reference accumulates
// block distances as dist += temp * temp with separate rounding of the product
// (include/Block.h:600-603; MSVC /fp:precise, msvc/ISP_MW.vcxproj:161,179).
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

// dist += sum_x (r[x] - c[x])^2 over one 8-pixel row, x ascending, as the
// reference accumulates it (include/Block.h:596-605). FP32: the subtractions
// and squares run as packed f32x2 pairs (each element rounded exactly like
// the scalar op, no fused multiply-add), the additions stay scalar and in
// order, so the result is bit-identical to the sequential form.
__device__ __forceinline__ float ssd_row8(float acc, const float (&r)[8], const float (&c)[8])
{
#pragma unroll
    for (int x = 0; x < 8; x += 2) {
        unsigned long long a, b, d, q;
        asm("mov.b64 %0, {%1, %2};" : "=l"(a) : "f"(r[x]), "f"(r[x + 1]));
        asm("mov.b64 %0, {%1, %2};" : "=l"(b) : "f"(c[x]), "f"(c[x + 1]));
        asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
        asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(q) : "l"(d), "l"(d));
        float q0, q1;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(q0), "=f"(q1) : "l"(q));
        acc = __fadd_rn(acc, q0);
        acc = __fadd_rn(acc, q1);
    }
    return acc;
}
__device__ __forceinline__ double ssd_row8(double acc, const double (&r)[8], const double (&c)[8])
{
#pragma unroll
    for (int x = 0; x < 8; ++x) {
        const double d = __dsub_rn(r[x], c[x]);
        acc = __dadd_rn(acc, __dmul_rn(d, d));
    }
    return acc;
}

// FLType(dist * distMul) with distMul a double (include/Block.h:610).
__device__ __forceinline__ float key_from_dist(float d, double mul)
{
    return __double2float_rn(__dmul_rn(static_cast<double>(d), mul));
}
__device__ __forceinline__ double key_from_dist(double d, double mul) { return __dmul_rn(d, mul); }

// ---------------------------------------------------------------------------
// Block::_SearchBoundary (include/Block.h:716-746) in closed form.
__host__ __device__ __forceinline__ int search_boundary(int pos, int plane_boundary, int range,
                                                        int step)
{
    range = range / step * step;
    if (pos == plane_boundary) return plane_boundary;
    if (pos > plane_boundary) {
        int b = pos - range;
        if (b < plane_boundary) b += (plane_boundary - b + step - 1) / step * step;
        return b;
    }
    int b = pos + range;
    if (b > plane_boundary) b -= (b - plane_boundary + step - 1) / step * step;
    return b;
}

// Reference-block position k along one axis: 0, step, 2 step, ... with the
// last one clamped to the plane border (source/BM3D.cpp:98-120).
__host__ __device__ __forceinline__ int ref_pos(int k, int step, int last)
{
    const int p = k * step;
    return p > last ? last : p;
}

__host__ __device__ __forceinline__ int ref_count(int last, int step)
{
    return last / step + 1 + (last % step != 0 ? 1 : 0);
}

// ---------------------------------------------------------------------------
// Sort keys: (key value, candidate index) compared lexicographically. Valid
// keys are finite and >= 0, so the IEEE bit pattern orders like the value.
// The candidate index is the candidate's place in the reference's search list
// (raster order of the window, then the trailing (0, 0) slot), so ties in the
// key fall back to that list order, which is std::stable_sort's order
// (include/Block.h:699).
template <typename T> struct SortKey;

template <> struct SortKey<float> {
    unsigned long long v;
    static __device__ __forceinline__ SortKey invalid() { return SortKey{~0ull}; }
    static __device__ __forceinline__ SortKey make(float key, unsigned idx)
    {
        return SortKey{(static_cast<unsigned long long>(__float_as_uint(key)) << 32) | idx};
    }
    __device__ __forceinline__ bool valid() const { return v != ~0ull; }
    __device__ __forceinline__ float key() const { return __uint_as_float(static_cast<unsigned>(v >> 32)); }
    __device__ __forceinline__ unsigned idx() const { return static_cast<unsigned>(v); }
    __device__ __forceinline__ bool operator<(const SortKey &o) const { return v < o.v; }
    __device__ __forceinline__ bool operator==(const SortKey &o) const { return v == o.v; }
    __device__ __forceinline__ unsigned key_bits() const { return static_cast<unsigned>(v >> 32); }
    __device__ __forceinline__ SortKey shfl_xor(int m) const
    {
        return SortKey{__shfl_xor_sync(0xffffffffu, v, m)};
    }
    __device__ __forceinline__ SortKey shfl(int src) const
    {
        return SortKey{__shfl_sync(0xffffffffu, v, src)};
    }
};

template <> struct SortKey<double> {
    unsigned long long k;
    unsigned long long i;
    static __device__ __forceinline__ SortKey invalid() { return SortKey{~0ull, ~0ull}; }
    static __device__ __forceinline__ SortKey make(double key, unsigned idx)
    {
        return SortKey{static_cast<unsigned long long>(__double_as_longlong(key)), idx};
    }
    __device__ __forceinline__ bool valid() const { return k != ~0ull; }
    __device__ __forceinline__ double key() const { return __longlong_as_double(static_cast<long long>(k)); }
    __device__ __forceinline__ unsigned idx() const { return static_cast<unsigned>(i); }
    __device__ __forceinline__ bool operator<(const SortKey &o) const
    {
        return k < o.k || (k == o.k && i < o.i);
    }
    __device__ __forceinline__ bool operator==(const SortKey &o) const { return k == o.k && i == o.i; }
    __device__ __forceinline__ unsigned long long key_bits() const { return k; }
    __device__ __forceinline__ SortKey shfl_xor(int m) const
    {
        return SortKey{__shfl_xor_sync(0xffffffffu, k, m), __shfl_xor_sync(0xffffffffu, i, m)};
    }
    __device__ __forceinline__ SortKey shfl(int src) const
    {
        return SortKey{__shfl_sync(0xffffffffu, k, src), __shfl_sync(0xffffffffu, i, src)};
    }
};

// The key part of a SortKey alone (its IEEE bits; an invalid key's are all
// ones), for the selection threshold, which depends on key values only.
template <typename B> struct KeyBits {
    B v;
    __device__ __forceinline__ bool operator<(const KeyBits &o) const { return v < o.v; }
    __device__ __forceinline__ KeyBits shfl_xor(int m) const
    {
        return KeyBits{__shfl_xor_sync(0xffffffffu, v, m)};
    }
    __device__ __forceinline__ KeyBits shfl(int src) const
    {
        return KeyBits{__shfl_sync(0xffffffffu, v, src)};
    }
};

template <typename K> __device__ __forceinline__ K warp_min(K v)
{
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) {
        K o = v.shfl_xor(m);
        if (o < v) v = o;
    }
    return v;
}

// Bitonic sort of one key per lane, ascending by lane.
template <typename K> __device__ __forceinline__ K bitonic32(K v, int lane)
{
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const K p = v.shfl_xor(j);
            const bool take_min = ((lane & k) == 0) == ((lane & j) == 0);
            v = (take_min == (p < v)) ? p : v;
        }
    }
    return v;
}

// Bitonic sort of two keys per lane (element e = lane + 32 s), ascending by e.
template <typename K> __device__ __forceinline__ void bitonic64(K &v0, K &v1, int lane)
{
#pragma unroll
    for (int k = 2; k <= 64; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j == 32) {
                if (v1 < v0) {
                    const K t = v0;
                    v0 = v1;
                    v1 = t;
                }
            } else {
                const K p0 = v0.shfl_xor(j), p1 = v1.shfl_xor(j);
                const bool lower = (lane & j) == 0;
                const bool up0 = (lane & k) == 0, up1 = ((lane + 32) & k) == 0;
                v0 = ((up0 == lower) == (p0 < v0)) ? p0 : v0;
                v1 = ((up1 == lower) == (p1 < v1)) ? p1 : v1;
            }
        }
    }
}

template <typename T> __device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    return v;
}

// Plane position (row, column) of one block of a group.
struct BlockPos {
    int y, x;
};

// ---------------------------------------------------------------------------
// Aggregation accumulators. FP32 stages accumulate numerator and weight sums
// in 64-bit fixed point (value * 2^scale rounded to an integer): integer
// atomics are associative, so the sums -- and everything downstream,
// including the final stage's block matching on the basic estimate -- are
// bit-reproducible and independent of tiling and scheduling. FP64 stages
// accumulate in double.
template <typename T> struct AccOf { using type = long long; };
template <> struct AccOf<double> { using type = double; };

// Fixed-point exponent for a plane whose |src| <= absmax when at most
// 2^log2_bound contributions reach one pixel: every contribution is bounded by
// 64 * absmax (a filtered block value is bounded by the group's L2 norm,
// <= 32 * absmax for a 1024-pixel group, times a weight <= 1), so a pixel's
// sum stays below 2^62.
//
// Two bounds are used per plane. A pixel outside block (0, 0) is reached only
// by group members within BMrange of their reference block, so by at most
// (ceil((BS + 2 BMrange) / step) + 1)^2 * GroupSize terms (the reference
// positions whose search window can hold a block covering it, the clamped
// last row / column included). Block (0, 0) is also the trailing candidate of
// every reference block's list (include/Block.h:668-687), so its pixels -- and
// its block weight, summed at origin (0, 0) -- may get up to two terms from
// every group. Each pixel and each weight origin keeps the scale of its class;
// the normalisation converts between them.
__device__ __forceinline__ float fixed_scale(float absmax, int log2_bound)
{
    if (!(absmax > 0.0f) || !(absmax <= 3.4028235e38f)) absmax = 1.0f;
    int e = 0;
    frexpf(absmax, &e);  // absmax < 2^e, so 64 * absmax < 2^(e + 6)
    int s = 62 - (e + 6) - log2_bound;
    s = s < -60 ? -60 : (s > 60 ? 60 : s);
    return ldexpf(1.0f, s);
}

// ---------------------------------------------------------------------------
// Per-stage launch arguments (one struct, passed by value).
constexpr int kMaxPlanes = 3;

template <typename T> struct StageArgs {
    const T *src[kMaxPlanes];   // noisy planes (collaborative filtering input)
    const T *ref[kMaxPlanes];   // basic: plane 0 drives matching; final: basic estimate
    typename AccOf<T>::type *num[kMaxPlanes];  // numerator sums, width x height, pitch = width
    typename AccOf<T>::type *den[kMaxPlanes];  // weight sums, same layout
    const float *absmax;        // per plane max finite |src| (device), sets the fixed-point scale
    int log2_bound;             // ceil(log2(max contributions to one pixel outside block (0, 0)))
    int log2_corner;            // the same for block (0, 0)'s pixels, which every group may reach
    // FP32 only (null for FP64, whose double sums carry NaN / Inf themselves):
    // per plane, the count of non-finite src / ref pixels found by the prep
    // kernel, and a byte per pixel (pitch = width) that marks pixels a
    // non-finite term reached. The kernels look at the count once per tile and
    // take the checking aggregation only when it is nonzero.
    const unsigned *nonfinite;
    unsigned char *poison[kMaxPlanes];
    int active;                 // bit p set: plane p is filtered (sigma[p] > 0)
    int width, height;
    long long stride;           // row pitch of src / ref, in elements
    int block_size;             // BlockSize (8 on the register-resident path, <= kBSMax)
    int step;                   // BlockStep
    int group_size;             // GroupSize (1..kGSMax fast path, 1..kGSTab generic)
    int range;                  // BMrange rounded down to a multiple of bm_step
    int bm_step;                // BMstep
    int match;                  // 0 when GroupSize == 1 or thMSE <= 0 (source/BM3D.cpp:226)
    int nx, ny;                 // reference positions per axis
    int tile_x, tile_y;         // reference positions per CTA tile
    int tiles_x;                // tiles per row of the tile grid
    int region_w, region_h;     // upper bounds of a tile's staged window
    int region_pitch;           // row pitch of staged windows in shared memory
    int key_slots;              // per-warp search list capacity
    int ref_alias_src;          // bit p set: ref[p] == src[p], stage once
    T thSSE;                    // FLType(thMSE * MSE2SSE)      (include/Block.h:582-584)
    double distMul;             // 1 / MSE2SSE
    T thr[kMaxPlanes][kGSTab][4];  // hard thresholds by (#zero indices) (source/BM3D.cpp:35-68)
    T wss[kMaxPlanes][kGSTab];     // wienerSigmaSqr                     (source/BM3D.cpp:31)
    double finalAMP[kGSTab];       // 2n * 2BS * 2BS                     (source/BM3D.cpp:26)
    const T *dct_fwd;           // generic path: cosine matrices of lengths 1..32 (device),
    const T *dct_inv;           //   length n at offset (n-1) n (2n-1) / 6
    // optional outputs
    int *group_count;           // per reference block: group size        (may be null)
    int *group_pos;             // per reference block: kGSTab x (y, x)   (may be null)
    T *group_key;               // per reference block: kGSTab keys       (may be null)
    unsigned long long *stats;  // [0] sum n, [1] sum n^2, [2] candidates, [3] tie fix-ups
                                // (may be null)
    unsigned long long *bad;    // consistency counter, must stay 0: low 32 bits group members
                                // outside the staged window, high 32 bits CTAs launched with
                                // too little shared memory (may be null)
    int bm_only;                // skip the collaborative filter (group dump)
};

// Offset of the length-n matrix in the concatenated cosine tables of the
// generic path: sum_{m < n} m^2.
__host__ __device__ __forceinline__ int dct_table_offset(int n) { return (n - 1) * n * (2 * n - 1) / 6; }
constexpr int kDctTableSize = 32 * 33 * 65 / 6;  // lengths 1..32

// Shared-memory carve-up of one CTA, identical on host and device.
// `generic` selects the layout of the generic-path kernel (group buffers of
// gs * bs^2 values, a reference-block copy per warp) instead of the
// register-resident one (kGSMax blocks of 8x8 in kGroupStride rows).
struct SmemPlan {
    int n_stage;                 // staged windows (src planes + separate ref planes)
    size_t region_bytes;         // one staged window
    size_t acc_bytes;            // one accumulator window
    size_t off_acc;              // 2 * planes accumulator windows
    size_t off_origin;           // block (0, 0) copies per staged window
    size_t off_origin_acc;       // block (0, 0) accumulators
    size_t off_warps;
    size_t warp_bytes;
    size_t scratch_bytes;        // group buffer(s) / search list union at the start of a warp's area
    size_t refblk_bytes;         // generic path: copy of the reference block
    size_t off_groups;           // three-plane register-resident path: the tile's group lists
    size_t total;
};

// Bytes of dynamic shared memory this launch was given.
__device__ __forceinline__ unsigned dynamic_smem_bytes()
{
    unsigned v;
    asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(v));
    return v;
}

// Generic kernel's group buffers, [z][y][x]: BlockSize 8 pads rows to 9 and
// blocks to 72 values, which keeps the row, column and group-axis passes of
// a warp on 32 distinct banks; other sizes are dense.
__host__ __device__ __forceinline__ int generic_block_stride(int bs) { return bs == 8 ? 72 : bs * bs; }
__host__ __device__ __forceinline__ int generic_row_stride(int bs) { return bs == 8 ? 9 : bs; }
// Whether the generic kernel's Wiener stage filters from one group buffer per
// warp, keeping the Wiener weights in registers (BlockSize 8, FP32), rather
// than from two.
template <typename T>
__host__ __device__ constexpr bool generic_one_buffer(bool wiener, int bs)
{
    return wiener && bs == 8 && sizeof(T) == 4;
}

// Shared-memory layout of one CTA. The register-resident kernel runs three
// planes one after another through a single plane's windows: it then also
// keeps the tile's group lists, per reference block kGSMax 16-bit positions
// relative to the window (windows under 255 x 255) and a count byte.
template <typename T>
__host__ __device__ inline SmemPlan plan_smem(int nplanes, bool wiener, int alias_mask,
                                              int region_h, int region_pitch, int key_slots,
                                              int nwarps, bool generic = false, int bs = kBS,
                                              int gs = kGSMax, int tile_refs = 0)
{
    SmemPlan s;
    const bool seq3 = nplanes == 3;
    if (seq3) {
        nplanes = 1;
        alias_mask &= 1;
    }
    int nref = 0;
    const int nref_planes = wiener ? nplanes : 1;
    for (int p = 0; p < nref_planes; ++p)
        if (!(alias_mask & (1 << p))) ++nref;
    s.n_stage = nplanes + nref;
    using Acc = typename AccOf<T>::type;
    const int bsq = bs * bs;
    s.region_bytes = (static_cast<size_t>(region_h) * region_pitch * sizeof(T) + 15) / 16 * 16;
    s.acc_bytes = (static_cast<size_t>(region_h) * region_pitch * sizeof(Acc) + 15) / 16 * 16;
    s.off_acc = s.region_bytes * s.n_stage;
    s.off_origin = s.off_acc + s.acc_bytes * 2 * nplanes;
    // block (0, 0) copies: T per staged window, then (16-byte aligned) Acc per accumulator
    s.off_origin_acc = s.off_origin + (sizeof(T) * bsq * s.n_stage + 15) / 16 * 16;
    s.off_warps = (s.off_origin_acc + sizeof(Acc) * bsq * 2 * nplanes + 15) / 16 * 16;
    const size_t group_bytes = generic
        ? sizeof(T) * static_cast<size_t>(gs) * generic_block_stride(bs) *
              (wiener && !generic_one_buffer<T>(wiener, bs) ? 2 : 1)
        : sizeof(T) * kGSMax * kGroupStride;
    const size_t key_bytes = sizeof(SortKey<T>) * key_slots;
    const size_t scratch = group_bytes > key_bytes ? group_bytes : key_bytes;
    s.scratch_bytes = (scratch + 15) / 16 * 16;
    s.refblk_bytes = generic ? (sizeof(T) * bsq + 15) / 16 * 16 : 0;
    // scratch | reference block (generic) | candidate/heap buffer (kCand sort keys) |
    // group list (kGSTab BlockPos) | group keys (kGSTab T)
    s.warp_bytes = (s.scratch_bytes + s.refblk_bytes + sizeof(SortKey<T>) * kCand +
                    sizeof(BlockPos) * kGSTab + sizeof(T) * kGSTab + 15) / 16 * 16;
    s.off_groups = (s.off_warps + s.warp_bytes * nwarps + 15) / 16 * 16;
    const int glist = generic ? gs : kGSMax;  // group-list entries per reference block
    s.total = seq3 ? s.off_groups + static_cast<size_t>(tile_refs) * (2 * glist + 1)
                   : s.off_warps + s.warp_bytes * nwarps;
    if (seq3 && (region_h > 255 || region_pitch > 255)) s.total = ~size_t(0) >> 1;  // too wide
    return s;
}

}  // namespace bm3d
