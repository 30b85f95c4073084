// dftcorr.cu -- libpivb_dft: tensor-core (tcgen05) building blocks and the
// DFT-as-GEMM correlation path for sm_100a.
#include <stdint.h>
#include <stdio.h>

#include "piv_common.cuh"
#include "umma.cuh"

namespace {

// One CTA: D (128 x N, FP32) = A (128 x K, BF16) * B (N x K, BF16)^T through
// shared-memory descriptors and a tensor-memory accumulator.  Checks the
// operand layout, the descriptors and the accumulator read-back of the
// correlation kernels on a product with a known answer.
__global__ void __launch_bounds__(128) umma_selftest_kernel(const uint16_t *__restrict__ A,
                                                            const uint16_t *__restrict__ B, float *__restrict__ D,
                                                            int N, int K, int a_mn, uint32_t ncols, int *status)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char *sA = sm;
    unsigned char *sB = sm + 128 * K * 2;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sB + N * K * 2);
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 1);
    const int t = threadIdx.x, warp = t >> 5;
    for (int e = t; e < 128 * K; e += 128)
        *reinterpret_cast<uint16_t *>(sA + (a_mn ? umma::mnmajor_offset(128, e / K, e % K)
                                                 : umma::kmajor_offset(128, e / K, e % K))) = A[e];
    for (int e = t; e < N * K; e += 128)
        *reinterpret_cast<uint16_t *>(sB + umma::kmajor_offset(N, e / K, e % K)) = B[e];
    if (t == 0) umma::mbar_init(bar, 1);
    if (warp == 0) umma::tmem_alloc(slot, ncols);
    umma::fence_smem_to_async();
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    const uint32_t tbase = *slot;
    if (t == 0) {
        const uint32_t id = umma::idesc_bf16(128, N, a_mn != 0);
        for (int s = 0; s < K / 16; ++s)
            umma::mma_bf16(tbase, umma::desc_tile(umma::smem_u32(sA), 128, s),
                           umma::desc_tile(umma::smem_u32(sB), N, s), id, s > 0 ? 1u : 0u);
        umma::commit(umma::smem_u32(bar));
    }
    const bool ok = umma::mbar_wait(umma::smem_u32(bar), 0);
    umma::fence_after();
    if (ok) {
        for (int c0 = 0; c0 < N; c0 += 32) {
            float v[32];
            umma::tmem_ld32(tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if (c0 + j < N) D[(32 * warp + (t & 31)) * N + c0 + j] = v[j];
        }
    } else if ((t & 31) == 0) {
        atomicExch(status, 1);
    }
    umma::fence_before();
    __syncthreads();
    if (warp == 0) umma::tmem_free(tbase, ncols);
}

}  // namespace

// Self-test of the tensor-core path: D (128 x N) = A (128 x K) B (N x K)^T with
// BF16 operands (raw 16-bit patterns, row-major) and FP32 results.  K in
// {16, 32, 48, 64}, N a multiple of 16 in [16, 128]; a_mn stages A in the
// MN-major layout instead of K-major.  *d_status is set to 1 if
// the MMA completion was not observed within the wait limit.  Returns 0, or 1
// for bad arguments / launch failure.
PIV_EXPORT int pivb_umma_selftest(const void *d_A, const void *d_B, float *d_D, int N, int K, int a_mn,
                                  int *d_status, void *stream)
{
    if (!d_A || !d_B || !d_D || !d_status) return 1;
    if (K < 16 || K > 64 || K % 16) return 1;
    if (N < 16 || N > 128 || N % 16) return 1;
    const uint32_t ncols = N <= 32 ? 32u : (N <= 64 ? 64u : 128u);
    // operands take 128*K*2 + N*K*2 <= 32 KB; the allocation is sized so that every
    // address a descriptor of these tiles can form stays inside it
    const int smem = 96 * 1024;
    if (cudaFuncSetAttribute(umma_selftest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return 1;
    umma_selftest_kernel<<<1, 128, smem, (cudaStream_t)stream>>>(static_cast<const uint16_t *>(d_A),
                                                                  static_cast<const uint16_t *>(d_B), d_D, N, K,
                                                                  a_mn, ncols, d_status);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
