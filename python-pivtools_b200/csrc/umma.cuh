// umma.cuh -- thin inline-PTX layer over the sm_100a 5th-generation tensor core
// (tcgen05): tensor-memory allocation, BF16 MMAs with FP32 accumulators in
// tensor memory, commit to an mbarrier, tensor-memory loads.
//
// Shared-memory operands use the K-major, no-swizzle canonical layout: a core
// matrix is 8 rows x 16 bytes (8 bf16 along K) stored as 128 contiguous bytes.
// Operand element (r, k) of a tile with R rows lives at byte
//     (k / 8) * (R * 16) + r * 16 + (k % 8) * 2
// so the leading-dimension byte offset (next 8 K-elements) is R * 16 and the
// stride-dimension byte offset (next 8 rows) is 128.  One MMA consumes K = 16,
// i.e. two core-matrix columns; the next K-step starts 2 * R * 16 bytes later.
//
// The MN-major no-swizzle layout keeps 8 consecutive rows of one K-element in a
// 16-byte vector; a core matrix is 8 rows x 8 K-elements (K-element k at
// 16-byte slot k % 8):
//     (k / 8) * (R * 16) + (r / 8) * 128 + (k % 8) * 16 + (r % 8) * 2
// with the same leading (K-block) and stride (row-block) byte offsets as above.
//
// Accumulator D of an M = 128 MMA: row i in tensor-memory lane i, column j in
// column (base + j), FP32.  Warp w of the CTA reads lanes 32*(w%4) .. +31.
#pragma once

#include <stdint.h>

namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, k) in a K-major no-swizzle tile of R rows.
__host__ __device__ constexpr uint32_t kmajor_offset(uint32_t R, uint32_t r, uint32_t k)
{
    return (k >> 3) * (R * 16u) + r * 16u + (k & 7u) * 2u;
}

// Byte offset of element (r, k) in an MN-major no-swizzle tile of R rows.
__host__ __device__ constexpr uint32_t mnmajor_offset(uint32_t R, uint32_t r, uint32_t k)
{
    return (k >> 3) * (R * 16u) + (r >> 3) * 128u + (k & 7u) * 16u + (r & 7u) * 2u;
}

// Shared-memory matrix descriptor (sm_100 format: version 1 at bits 46-47,
// layout type 0 = no swizzle at bits 61-63).
__host__ __device__ constexpr uint64_t desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Descriptor of K-step s (16 elements) of a K-major tile of R rows at saddr.
__host__ __device__ constexpr uint64_t desc_tile(uint32_t saddr, uint32_t R, uint32_t s)
{
    return desc_kmajor(saddr + s * 2u * R * 16u, R * 16u, 128u);
}

// Instruction descriptor: kind::f16 with BF16 A and B, FP32 D; a_mn / b_mn
// select the MN-major layout for A / B (default K-major).
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N, bool a_mn = false, bool b_mn = false)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((N >> 3) << 17) | ((M >> 4) << 24);
}

// D[tmem] (+)= A * B^T, one elected thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}

// Arrive on the mbarrier once every MMA issued so far by this thread has completed.
__device__ __forceinline__ void commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes -> visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Tensor-memory allocation by one whole warp; the base address is written to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false if the phase did not complete within `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint32_t limit = 1u << 24)
{
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// 32 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}

// 16 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

}  // namespace umma
