// Blackwell (sm_100a) tensor-core primitives for the learned pilot's
// convolutions: shared-memory matrix descriptors, the tcgen05 instruction
// descriptor, tensor-memory (TMEM) allocation, MMA issue / commit, TMEM
// loads and mbarrier waits with an iteration cap.
//
// Operand layouts are the canonical no-swizzle ("interleaved") forms, in
// 16-byte core-matrix rows:
//   K-major  : element (r, k) at (r % 8) * 16 + (r / 8) * SBO + (k / 8) * LBO + (k % 8) * 2
//   MN-major : element (m, k) at (m % 8) * 2 + (m / 8) * SBO + (k % 8) * 16 + (k / 8) * LBO
// (bf16 elements; r / m run along M or N, k along K).
#pragma once

#include <cstdint>

namespace pilot {

// Shared-memory matrix descriptor (64 bits): start address >> 4 in [0, 14),
// leading-dimension byte offset >> 4 in [16, 30), stride-dimension byte
// offset >> 4 in [32, 46), descriptor version 1 at [46, 48), base offset 0,
// layout type 0 (no swizzle) at [61, 64).
__device__ __forceinline__ uint64_t smem_desc(uint32_t smem_addr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= static_cast<uint64_t>((smem_addr >> 4) & 0x3fffu);
    d |= static_cast<uint64_t>((lbo >> 4) & 0x3fffu) << 16;
    d |= static_cast<uint64_t>((sbo >> 4) & 0x3fffu) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    return d;
}

// Instruction descriptor of tcgen05.mma.kind::f16 with BF16 A and B and an
// FP32 accumulator: D format F32 at [4, 6), A format BF16 at [7, 10), B format
// BF16 at [10, 13), A / B major at bits 15 / 16 (0 = K-major, 1 = MN-major),
// N >> 3 at [17, 23), M >> 4 at [24, 29).
__host__ __device__ constexpr uint32_t instr_desc_bf16(int m, int n, bool a_mn_major,
                                                       bool b_mn_major)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn_major ? 1u : 0u) << 15) |
           ((b_mn_major ? 1u : 0u) << 16) | (static_cast<uint32_t>(n >> 3) << 17) |
           (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// --- tensor memory ----------------------------------------------------------
// Allocation and release are warp-wide (.sync.aligned): call from one full
// warp. The allocated column base is written to *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Generic-proxy shared-memory writes (st.shared, cp.async) made visible to the
// tensor core's reads (async proxy). Every writing thread runs it before the
// barrier that precedes the MMA issue.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A[desc] * B[desc]^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                         uint32_t idesc, bool accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate ? 1u : 0u)
        : "memory");
}

// Arrive once on the mbarrier when every MMA this thread issued before has
// completed (and stopped reading its shared-memory operands).
__device__ __forceinline__ void mma_commit(uint64_t *mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(mbar))
                 : "memory");
}

// 16 consecutive FP32 accumulator columns of this warp's 32 TMEM lanes (one
// lane per thread). taddr carries the warp's lane base in bits [16, 32).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// --- mbarriers ----------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *mbar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(mbar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity to complete, at most `limit`
// polls (each try_wait itself blocks for a hardware-defined time slice).
// Returns false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, uint32_t limit)
{
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(mbar, parity)) return true;
    return false;
}

// --- asynchronous global -> shared copies --------------------------------------
// 16 bytes, or 16 zero bytes when `valid` is false (src-size 0; src must still
// be a mapped address).
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc, bool valid)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(smem_dst)),
                 "l"(gsrc), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// All but the most recently committed group have landed.
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// --- tensor memory access (TMA) ------------------------------------------------
// Tiled copies through a tensor map (a __grid_constant__ kernel parameter,
// addressed generically). Single-CTA forms only: no cluster multicast.

// One arrival that also announces `bytes` of asynchronous copies to come.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *mbar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *mbar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(mbar)) : "memory");
}

// Box of a 5-D tensor map at coordinates c0..c4 (c0, the innermost, in
// elements and a multiple of 16 bytes) into shared memory; completes on mbar.
__device__ __forceinline__ void tma_load_5d(void *smem_dst, const void *tmap, uint64_t *mbar, int c0,
                                            int c1, int c2, int c3, int c4)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_u32(mbar)), "r"(c0), "r"(c1), "r"(c2),
        "r"(c3), "r"(c4)
        : "memory");
}

// Box of a 4-D tensor map from shared memory to coordinates c0..c3 (c0 = 0
// here); elements outside the tensor are not written.
__device__ __forceinline__ void tma_store_4d(const void *tmap, const void *smem_src, int c0, int c1,
                                             int c2, int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4, %5}], [%1];" ::
            "l"(reinterpret_cast<uint64_t>(tmap)),
        "r"(smem_u32(smem_src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// This thread's bulk stores but the most recent one have finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read_1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
// This thread's bulk stores have completed.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

}  // namespace pilot
