// Blackwell fifth-generation tensor-core helpers (tcgen05) for the proposal
// network's implicit-GEMM convolutions: shared-memory matrix descriptors,
// the BF16 instruction descriptor, TMEM allocation and loads, mbarriers.
//
// Operand tiles use the no-swizzle canonical layout built by the CTA's own
// threads.  A tile of R rows x 16 K elements (one MMA K-step) is a set of
// 8 x 16-byte core matrices: core (row group g, K half c) sits at
// g * 256 + c * 128 bytes, so both descriptor strides (128 and 256 bytes) are
// small and every address an MMA forms stays inside its own R x 32-byte
// K-step block.  K-major tiles hold 8 consecutive K values of one row in each
// 16-byte unit; MN-major tiles hold 8 consecutive rows of one K value.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace spk {
namespace umma {

__device__ __forceinline__ std::uint32_t smem_addr(const void* p)
{
    return static_cast<std::uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of the 16-byte unit (row group g, K half c, unit row i) inside
// one K-step block.  For K-major tiles i is the row within the group; for
// MN-major tiles i is the K index within the half.
__device__ __forceinline__ std::uint32_t unit_offset(int g, int c, int i)
{
    return static_cast<std::uint32_t>(g * 256 + c * 128 + i * 16);
}

// Shared-memory matrix descriptor, SWIZZLE_NONE, sm100 version field.
//   K-major : leading byte offset = distance between the two K halves (128),
//             stride byte offset  = distance between row groups (256).
//   MN-major: leading byte offset = distance between the two K groups (128),
//             stride byte offset  = distance between row groups (256).
__device__ __forceinline__ std::uint64_t desc(std::uint32_t addr)
{
    constexpr std::uint64_t lbo = 128, sbo = 256;
    std::uint64_t d = 0;
    d |= static_cast<std::uint64_t>((addr >> 4) & 0x3FFFu);
    d |= ((lbo >> 4) & 0x3FFFu) << 16;
    d |= ((sbo >> 4) & 0x3FFFu) << 32;
    d |= static_cast<std::uint64_t>(1) << 46;  // descriptor version 1 (sm100)
    return d;                                  // base offset 0, legacy LBO mode, no swizzle
}

// kind::f16 instruction descriptor: BF16 A and B, FP32 accumulator, M x N.
__host__ __device__ constexpr std::uint32_t idesc_bf16(int m, int n, bool a_mn_major, bool b_mn_major)
{
    return (1u << 4)                                        // D format F32
           | (1u << 7)                                      // A format BF16
           | (1u << 10)                                     // B format BF16
           | ((a_mn_major ? 1u : 0u) << 15)                 // A major
           | ((b_mn_major ? 1u : 0u) << 16)                 // B major
           | (static_cast<std::uint32_t>(n >> 3) << 17)     // N / 8
           | (static_cast<std::uint32_t>(m >> 4) << 24);    // M / 16
}

__device__ __forceinline__ void mma_bf16(std::uint32_t tmem_d, std::uint64_t a, std::uint64_t b, std::uint32_t idesc,
                                         std::uint32_t accumulate)
{
    const std::uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2),
          "r"(mask3)
        : "memory");
}

// Arrives on `bar` once every MMA this thread issued so far has completed.
__device__ __forceinline__ void commit(unsigned long long* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :
                 : "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes become visible to the tensor core.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void bar_init(unsigned long long* bar, std::uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ bool bar_try_wait(unsigned long long* bar, std::uint32_t parity)
{
    std::uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait for the phase with `parity` to complete; false when the limit
// ran out (the caller records an error and carries on without hanging).
__device__ __forceinline__ bool bar_wait(unsigned long long* bar, std::uint32_t parity,
                                         std::uint32_t limit = 1u << 22)
{
    for (std::uint32_t spin = 0; spin < limit; ++spin) {
        if (bar_try_wait(bar, parity)) {
            return true;
        }
    }
    return false;
}

// Whole-warp TMEM allocation; the base address is written to *dst (shared).
__device__ __forceinline__ void tmem_alloc(std::uint32_t* dst, std::uint32_t columns)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_addr(dst)), "r"(columns)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(std::uint32_t taddr, std::uint32_t columns)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(taddr), "r"(columns) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w of the CTA
// reads lanes 32w..32w+31).  Whole-warp instruction; the load and its wait
// sit in one asm statement so no use of the registers can move above the
// wait.
__device__ __forceinline__ void tmem_load16(std::uint32_t taddr, float (&v)[16])
{
    std::uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        v[i] = __uint_as_float(r[i]);
    }
}

}  // namespace umma
}  // namespace spk
