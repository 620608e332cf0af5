// qg_tc.cuh -- fifth-generation tensor-core (tcgen05) building blocks for
// sm_100a: tensor-memory (TMEM) allocation, shared-memory operand
// descriptors, the BF16 x BF16 -> FP32 MMA with its completion on an
// mbarrier, and the TMEM -> register load.  One CTA, no cluster, no
// multicast.
//
// Operands are K-major with no swizzle: an operand of R rows and K BF16
// columns is stored as core matrices of 8 rows x 16 bytes (8 BF16 along K),
// the 8 rows of a core matrix 16 bytes apart, the K-chunks of a row group
// 128 bytes apart (the leading byte offset) and the row groups K * 16 bytes
// apart (the stride byte offset).  kmajor_off() gives the byte offset of
// element (row, col) in that layout; one MMA of depth 16 at K-offset k0 starts
// at kmajor_off(0, k0).
//
// The descriptor and instruction-descriptor bit fields follow the sm100
// UMMA formats (PTX ISA "tcgen05 matrix descriptors" / "instruction
// descriptor"): start address, leading and stride byte offsets in 16-byte
// units, descriptor version 1; kind::f16 with F32 accumulation, BF16 A and
// B, both K-major, N / 8 and M / 16.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace qg {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__host__ __device__ constexpr uint32_t kmajor_off(int row, int col, int K)
{
    return (uint32_t)((row >> 3) * (K * 16) + (col >> 3) * 128 + (row & 7) * 16 + (col & 7) * 2);
}

__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// the operand of K columns (a multiple of 16) at K-offset k0
__device__ __forceinline__ uint64_t desc_operand(const void *base, int K, int k0)
{
    return desc_kmajor(smem_u32(base) + kmajor_off(0, k0, K), 128u, (uint32_t)K * 16u);
}

__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A B^T for one MMA of depth 16; issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                 ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
// arrive on the mbarrier once every MMA issued so far by this thread is done
__device__ __forceinline__ void mma_commit(uint64_t *mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// wait for completion of phase `parity`; gives up after `limit` polls and
// returns false (the caller reports the timeout and unwinds)
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, uint32_t limit)
{
    const uint32_t a = smem_u32(mbar);
    for (uint32_t i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P1;\n\t}"
                     : "=r"(done)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}

// generic-proxy shared-memory writes made visible to the tensor core
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM columns for this CTA (one warp executes it); the base address is
// written to *slot
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 consecutive FP32 columns of the warp's 32 TMEM lanes: thread i of warp
// w receives lane 32 w + i (row 32 w + i of an M = 128 accumulator); the
// load and its wait are one statement, so no use of the values precedes it
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                 "[%32];\n\ttcgen05.wait::ld.sync.aligned;"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                   "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                   "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr)
                 : "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace qg
