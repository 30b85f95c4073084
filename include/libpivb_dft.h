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

/* The timeout path of the kernels' bounded mbarrier waits: one CTA allocates
 * tensor memory, waits `limit` polls on a phase that nothing completes, adds 1
 * per warp to *d_status (device int), frees the tensor memory and returns.  No
 * counterpart in the reference. */
int pivb_wait_timeout_selftest(int *d_status, int limit, void *stream);

/* Instantaneous correlation of 32 x 32 windows as DFT-as-GEMM on the tensor core:
 * four chained GEMMs (real row DFT, complex column DFT, inverse column DFT,
 * Hermitian inverse row DFT) with every operand split into BF16 hi + lo and three
 * products accumulated in FP32; then the same peak search, fit and outputs as
 * pivb_xcorr_dev (libbulkxcorr2d.h), whose arguments it takes, plus d_status.
 * Supported: win_h = win_w = 32, ensemble 0, n_peaks 1, peak_finder 3-6 (4-6 need
 * pivb_xcorr_scratch_bytes of scratch).  Replaces the FFT codelet correlation of
 * the reference (pivtools_cli/lib/codelet_fft.c:246-366) for that case; no
 * counterpart entry point in the reference.  Returns the reference's error codes
 * (1 NOMEM, 8 no plan for the size, 9 bad arguments) or 16 (CUDA); *d_status = 1 if an MMA
 * completion was not observed. */
int pivb_dft_xcorr_dev(const float *d_A, const float *d_B, long long img_stride, const float *d_mask, int H,
                       int W, int n_images, const float *d_ctr_x, const float *d_ctr_y, int n_win_y, int n_win_x,
                       const float *d_wA, const float *d_wB, const float *d_cw, int win_h, int win_w, int ensemble,
                       int n_peaks, int peak_finder, int peakfit_impl, float *d_pk_x, float *d_pk_y, float *d_pk_h,
                       float *d_sx, float *d_sy, float *d_sxy, float *d_pk_ratio, float *d_planes, void *d_scratch,
                       size_t scratch_bytes, int *d_status, void *stream);

#ifdef __cplusplus
}
#endif
#endif
