/* libpivb_dft -- tensor-core (tcgen05, sm_100a) building blocks and the
 * DFT-as-GEMM correlation path.  No counterpart in the reference: the
 * reference correlates with FFT codelets only (pivtools_cli/lib/codelet_fft.c). */
#ifndef LIBPIVB_DFT_H
#define LIBPIVB_DFT_H

#ifdef __cplusplus
extern "C" {
#endif

/* D (128 x N, float32, row-major) = A (128 x K) * B (N x K)^T with bfloat16
 * operands given as raw 16-bit patterns, row-major.  K in {16, 32, 48, 64}; N a
 * multiple of 16 in [16, 128].  *d_status (device int) is set to 1 if the MMA
 * completion was not observed.  Returns 0, or 1 for bad arguments. */
int pivb_umma_selftest(const void *d_A, const void *d_B, float *d_D, int N, int K, int a_mn, int *d_status,
                       void *stream);

#ifdef __cplusplus
}
#endif
#endif
