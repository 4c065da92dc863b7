// fsl_umma.cuh -- minimal sm_100a tensor-core (tcgen05) building blocks for
// the learned closure: BF16 x BF16 -> FP32 GEMM tiles of M = 128 rows with
// the accumulator in tensor memory (TMEM).
//
// Operand layout in shared memory ("K-major, no swizzle" canonical layout of
// the UMMA descriptors): an R x K bf16 tile is stored as 8-row x 16-byte core
// matrices, element (r, k) at byte
//     (r / 8) * (16 K) + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// i.e. the two core matrices an instruction's K = 16 slice spans are 128 bytes
// apart (leading byte offset) and consecutive 8-row groups are 16 K bytes
// apart (stride byte offset).  The product D[128 x N] (+)= A[128 x K] B[N x K]^T
// is issued as K/16 tcgen05.mma instructions by one thread; completion is
// signalled on an mbarrier through tcgen05.commit.  Every wait is bounded: on
// timeout the caller sets an error flag and returns after releasing TMEM.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace fsl {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (r, k) in a K-major core-matrix tile of width K
__host__ __device__ __forceinline__ uint32_t tile_off(int r, int k, int K)
{
    return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor, no swizzle, sm_100 version field = 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46; // descriptor version (sm_100)
    // base offset 0, legacy LBO mode, layout type 0 = no swizzle
    return d;
}

// instruction descriptor of kind::f16: A, B = BF16 (K-major), D = F32, M = 128
__host__ __device__ __forceinline__ uint32_t idesc_bf16_f32(int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile("{\n\t"
                 ".reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
                 "}\n" ::"r"(tmem_d),
                 "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// D[128 x N] (+)= A[128 x K] B[N x K]^T, issued by the calling thread.
__device__ __forceinline__ void gemm_issue(uint32_t tmem_d, uint32_t a_addr, uint32_t b_addr, int K, int N,
                                           bool accumulate)
{
    const uint32_t id = idesc_bf16_f32(N);
    const uint32_t sbo = (uint32_t)K * 16u;
    for (int s = 0; s < K / 16; s++) {
        const uint64_t da = smem_desc(a_addr + s * 256u, 128u, sbo);
        const uint64_t db = smem_desc(b_addr + s * 256u, 128u, sbo);
        mma_bf16(tmem_d, da, db, id, (accumulate || s > 0) ? 1u : 0u);
    }
}

// The same with operands of different stored widths: A stored with width Ka,
// B with width Kb, the product over the first K columns of both.
__device__ __forceinline__ void gemm_issue2(uint32_t tmem_d, uint32_t a_addr, int Ka, uint32_t b_addr, int Kb, int K,
                                            int N)
{
    const uint32_t id = idesc_bf16_f32(N);
    for (int s = 0; s < K / 16; s++) {
        const uint64_t da = smem_desc(a_addr + s * 256u, 128u, (uint32_t)Ka * 16u);
        const uint64_t db = smem_desc(b_addr + s * 256u, 128u, (uint32_t)Kb * 16u);
        mma_bf16(tmem_d, da, db, id, s > 0 ? 1u : 0u);
    }
}

__device__ __forceinline__ void commit(uint64_t *mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

// Wait for phase `parity` of the mbarrier; false after `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, uint32_t limit)
{
    const uint32_t a = smem_u32(mbar);
    for (uint32_t n = 0; n < limit; n++) {
        uint32_t done;
        asm volatile("{\n\t"
                     ".reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t"
                     "}\n"
                     : "=r"(done)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_before_sync()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

// TMEM allocation by one full warp; the address lands in *holder.
__device__ __forceinline__ void tmem_alloc(uint32_t *holder, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(holder)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes
// 32w .. 32w+31; the lane offset is part of taddr).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                   "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = __uint_as_float(r[q]);
}
__device__ __forceinline__ void tmem_wait_ld()
{
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

} // namespace umma
} // namespace fsl
