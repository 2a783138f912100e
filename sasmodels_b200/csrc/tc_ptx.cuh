// Thin inline-PTX layer for the 5th-generation tensor cores (tcgen05) on
// sm_100a: TMEM allocation, single-thread MMA issue with shared-memory
// matrix descriptors, completion through an mbarrier, and TMEM loads for the
// epilogue.
//
// Operand layout.  Both operands are K-major and stored in shared memory in
// the canonical no-swizzle ("interleaved") form: 8-row x 16-byte core
// matrices, the 8-row groups of one 8-element K chunk contiguous (stride
// SBO = 128 B), successive K chunks ROWS*16 bytes apart (LBO).  For a tile of
// ROWS rows and element (r, k):
//
//     byte offset = (k/8)*ROWS*16 + (r/8)*128 + (r%8)*16 + (k%8)*2
//
// One kind::f16 MMA consumes K = 16 (two chunks), so the descriptor of MMA
// step s starts 2*s*ROWS*16 bytes into the tile.
//
// Waits on mbarriers are bounded: a wait that runs out sets an error flag in
// global memory and the kernel unwinds (still releasing its TMEM), so a
// fault in the pipeline cannot hang the GPU.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_bf16.h>

namespace tc {

constexpr uint32_t WAIT_LIMIT = 1u << 22;   // bounded polling, far above any tile

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- mbarrier -------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;"
                 :: "r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return done != 0;
}

// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    for (uint32_t i = 0; i < WAIT_LIMIT; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
    }
    return false;
}

// Arrive once and add `bytes` to the transaction count of the current phase
// (the phase completes when the bulk copies have delivered that many bytes).
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Arrive once (release at CTA scope).
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(bar)) : "memory");
}

// ---- release/acquire flags in shared memory ------------------------------
__device__ __forceinline__ uint32_t ld_acquire_shared(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.acquire.cta.shared::cta.u32 %0, [%1];" : "=r"(v) : "r"(smem_u32(p)) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_shared(uint32_t *p, uint32_t v)
{
    asm volatile("st.release.cta.shared::cta.u32 [%0], %1;" :: "r"(smem_u32(p)), "r"(v) : "memory");
}
// Bounded spin until *p >= target (acquire).
__device__ __forceinline__ bool spin_acquire_ge(const uint32_t *p, uint32_t target)
{
    for (uint32_t i = 0; i < WAIT_LIMIT; ++i)
        if (ld_acquire_shared(p) >= target) return true;
    return false;
}

// ---- bulk copy (TMA engine, untiled, no multicast) --------------------------
// global -> this CTA's shared memory, completion counted on *bar.  Both
// addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes,
                                          uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// ---- named barriers ----------------------------------------------------------
// Barrier `id` among `count` threads (a multiple of 32) of the CTA.
__device__ __forceinline__ void bar_sync(int id, int count)
{
    asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(count) : "memory");
}

// Barrier `id` among `count` threads that also ANDs `pred` over them.
__device__ __forceinline__ bool bar_and(int id, int count, bool pred)
{
    uint32_t r;
    asm volatile("{\n\t.reg .pred p, q;\n\t"
                 "setp.ne.u32 p, %1, 0;\n\t"
                 "bar.red.and.pred q, %2, %3, p;\n\t"
                 "selp.u32 %0, 1, 0, q;\n\t}"
                 : "=r"(r) : "r"((uint32_t)pred), "r"(id), "r"(count) : "memory");
    return r != 0;
}

// ---- fences ----------------------------------------------------------------
// generic-proxy shared-memory writes -> visible to the tensor-core (async) proxy
__device__ __forceinline__ void fence_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_before_sync()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// ---- TMEM ------------------------------------------------------------------
// Executed by one whole warp; the allocated base address is written to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(slot)), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :: "r"(taddr), "r"(ncols) : "memory");
}

// 32 TMEM lanes x 16 consecutive 32-bit columns into 16 registers (one row
// per thread of the warp); pair with tmem_wait_ld before use.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld()
{
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 32 TMEM lanes x 8 columns; tmem_wait_ld8 on the same registers completes
// it (the registers are operands of the wait, so no use of them can be
// scheduled before it).
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld8(uint32_t (&r)[8])
{
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                   "+r"(r[6]), "+r"(r[7])
                 :: "memory");
}

// ---- MMA -------------------------------------------------------------------
// Shared-memory matrix descriptor: start address, leading (K-chunk) and
// stride (8-row group) byte offsets, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu)
         | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16)
         | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32)
         | ((uint64_t)1 << 46);
}

// kind::f16 instruction descriptor: BF16 A and B (K-major), FP32 D, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n)
{
    return (1u << 4)                              // D format F32
         | (1u << 7)                              // A format BF16
         | (1u << 10)                             // B format BF16
         | ((uint32_t)(n >> 3) << 17)             // N / 8
         | ((uint32_t)(m >> 4) << 24);            // M / 16
}

// D[tmem] (+)= A * B^T, issued by a single thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                         uint32_t idesc, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
                 : "memory");
}

// Arrive on *bar once every MMA this thread issued so far has completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(bar)) : "memory");
}

// ---- canonical layout ------------------------------------------------------
template <int ROWS>
__device__ __forceinline__ uint32_t kmajor_offset(int r, int k)
{
    return (uint32_t)((k >> 3)*ROWS*16 + (r >> 3)*128 + (r & 7)*16 + (k & 7)*2);
}

// Descriptor of MMA step s (K = 16) of a ROWS-row K-major tile at smem addr.
template <int ROWS>
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t tile_addr, int s)
{
    return smem_desc(tile_addr + (uint32_t)(2*s*ROWS*16), ROWS*16, 128);
}

}  // namespace tc
