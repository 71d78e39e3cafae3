// umma.cuh — the 5th-generation tensor-core path of sm_100a (tcgen05 / UMMA) in inline PTX:
// shared-memory matrix descriptors, the instruction descriptor of kind::f16 (BF16 inputs, FP32
// accumulators), TMEM allocation, MMA issue, commit to an mbarrier, TMEM loads.  Field layouts
// follow the public PTX ISA (tcgen05 "Matrix Descriptors", "Instruction descriptor") as CUTLASS
// documents them in cute/arch/mma_sm100_desc.hpp (SmemDescriptor, InstrDescriptor).
//
// Operand layout used throughout: K-major, no swizzle.  A tile of R rows x K columns (bf16) is
// stored as 8-row x 16-byte core matrices; the core matrix of rows [8i, 8i+8) and columns
// [8j, 8j+8) sits at byte ((i * K/8) + j) * 128, row r of it at +16 (r mod 8).  In the
// descriptor's terms the leading byte offset (next 8 columns) is 128 and the stride byte offset
// (next 8 rows) is K/8 * 128; one MMA consumes K = 16 (two core matrices along K), so the
// k-th MMA of a tile starts 256 k bytes further.
#pragma once

#include <cstdint>

namespace sw2d {
namespace umma {

constexpr int kTileM = 128;  // rows of one MMA (cta_group::1, M = 128: row i is TMEM lane i)

// byte offset of element (r, k) in the K-major core-matrix layout of a tile with K columns
__host__ __device__ constexpr uint32_t core_offset(int r, int k, int K)
{
    return (uint32_t)(((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// SmemDescriptor: start address >> 4 in [0,14), leading byte offset >> 4 in [16,30), stride
// byte offset >> 4 in [32,46), version 1 (Blackwell) in [46,48), base offset 0, leading-offset
// mode 0, layout type 0 (no swizzle) in [61,64)
__host__ __device__ constexpr uint64_t smem_desc(uint32_t saddr, int K)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((128u >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)(((uint32_t)(K / 8) * 128u >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// InstrDescriptor of kind::f16: D format F32 (bits [4,6) = 1), A and B BF16 ([7,10) = 1,
// [10,13) = 1), both K-major (bits 15, 16 = 0), N >> 3 in [17,23), M >> 4 in [24,29)
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

#if defined(__CUDACC__)
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tmem_alloc(uint32_t* holder, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(holder)),
                 "r"(ncols));
}
__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy writes to shared memory made visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// waits for the phase `parity` of the barrier to complete, at most `limit` polls; false if the
// limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit)
{
    const uint32_t a = smem_u32(bar);
    for (long long i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// D[tmem] (+)= A[smem desc] * B[smem desc]^T, issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// arrives on the barrier once every MMA this thread issued before has completed
__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 16 consecutive 32-bit columns of this thread's TMEM lane (warp w reads lanes 32w .. 32w+31)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
#endif

}  // namespace umma
}  // namespace sw2d
