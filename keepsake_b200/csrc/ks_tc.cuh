// 5th-generation tensor core (tcgen05) helpers for sm_100a: TMEM allocation, UMMA shared-memory
// and instruction descriptors, BF16 MMA with FP32 accumulation in TMEM, commit to an mbarrier,
// bounded mbarrier waits, and TMEM -> register loads.
//
// Operands live in shared memory in the no-swizzle canonical layout: 8 x 8 "core matrices" of
// 128 contiguous bytes (8 rows of 16 bytes).  A K-major operand has its K elements contiguous
// inside a core matrix; an MN-major operand has its M/N elements contiguous.  In both cases the
// descriptor's stride byte offset (SBO) is the distance between core matrices along M/N and the
// leading byte offset (LBO) the distance between core matrices along K.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace ksb
{
namespace tc
{

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (SWIZZLE_NONE).  addr, lbo and sbo in bytes (multiples of 16).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46; // descriptor version for sm_100
    // base offset 0, lbo mode 0, layout type 0 (no swizzle)
    return d;
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 accumulator, dense.
// a_mn / b_mn: operand is MN-major (1) instead of K-major (0).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn)
{
    return (1u << 4)                          // D format F32
           | (1u << 7)                        // A format BF16
           | (1u << 10)                       // B format BF16
           | ((uint32_t)a_mn << 15)           // A major
           | ((uint32_t)b_mn << 16)           // B major
           | ((uint32_t)(N >> 3) << 17)       // N >> 3
           | ((uint32_t)(M >> 4) << 24);      // M >> 4
}

// Warp-collective TMEM allocation of ncols columns (power of two, >= 32); the TMEM address is
// written to *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// D (TMEM) = A * B (+ D if accumulate); issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate)
{
    uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
    asm volatile("{\n\t"
                 ".reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
                 "}\n" ::"r"(d_tmem),
                 "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2),
                 "r"(mask3));
}

// The mbarrier at `bar` completes one phase when all previously issued tcgen05.mma of this thread
// have completed.
__device__ __forceinline__ void commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t phase)
{
    uint32_t done;
    asm volatile("{\n\t"
                 ".reg .pred P1;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                 "selp.b32 %0, 1, 0, P1;\n\t"
                 "}"
                 : "=r"(done)
                 : "r"(smem_addr(bar)), "r"(phase)
                 : "memory");
    return done != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("{\n\t"
                 ".reg .b64 state;\n\t"
                 "mbarrier.arrive.shared::cta.b64 state, [%0];\n\t"
                 "}" ::"r"(smem_addr(bar))
                 : "memory");
}

// Waits for `phase` of the mbarrier with an iteration limit; returns false (and the caller sets
// its error flag and stops) if the limit is reached.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t phase, uint32_t max_iter = 1u << 22)
{
    for (uint32_t i = 0; i < max_iter; ++i)
        if (mbar_try_wait(bar, phase))
            return true;
    return false;
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes become visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Each thread of warp w loads 16 consecutive FP32 columns of TMEM lane (32 w + lane).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16])
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i)
        v[i] = __uint_as_float(r[i]);
}

// Byte offset of element (mn, k) of an operand tile stored as canonical core matrices with
// k-groups `kstride` bytes apart and mn-groups `mnstride` bytes apart, K contiguous inside a core
// matrix (K-major storage).
__host__ __device__ constexpr uint32_t kmajor_offset(uint32_t mn, uint32_t k, uint32_t mnstride, uint32_t kstride)
{
    return (mn >> 3) * mnstride + (k >> 3) * kstride + (mn & 7u) * 16u + (k & 7u) * 2u;
}

} // namespace tc
} // namespace ksb
