/*
 * pivoracle.h -- CPU restatement of the PIVtools correlation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the tests, the
 * smoke check and the CPU-baseline leg of bench.py compare the CUDA product
 * against.  It is never linked into, loaded by, or called from the product.
 *
 * Each entry point restates one reference routine (cited below by the file and
 * line of the reference project, pivtools_cli/lib/...).  Arithmetic follows the
 * reference's float semantics where the reference is float, with two documented
 * exceptions that make the oracle an FP64 oracle for the correlation itself:
 *   - correlation planes are formed from the float-weighted windows by an FP64
 *     FFT and rounded to float once (the reference uses float codelets);
 *   - the loss-of-correlation weight autocorrelation is FP64 (float in the
 *     reference's 2N codelet transform).
 * Parity of the peak fitter and of the warp against the reference itself is
 * pinned by compiling the reference's own peak_locate_lm*.c and fused_warp.c
 * from source (oracle/Makefile `ref` target) and comparing bit for bit.
 */
#ifndef PIVORACLE_H
#define PIVORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* 1 if n is one of the window axis lengths the reference supports. */
int orc_size_ok(int n);

/* Circular cross-correlation of two float windows, FP64 arithmetic:
 *   out[r][c] = sum_x a[x + s] * b[x],  s = (r - h/2, c - w/2) mod (h, w)
 * i.e. fftshift(IFFT(FFT(a) .* conj(FFT(b)))) / (h*w).
 * (codelet_fft.c:153-192; xcorr.c:175-185).  Returns 0, or 2 if a size is not built. */
int orc_xcorr_plane(const float *a, const float *b, int h, int w, double *out);

/* Loss-of-correlation weight numel / (W (*) W) for an h x w window weight
 * (PIV_2d_cross_correlate.c:216-222 via xcorr.c:55-122), FP64 autocorrelation,
 * float result.  Returns 0 or an error code. */
int orc_correl_weight(const float *weight, int h, int w, float *out);

/* Peak fit of one plane (peak_locate_lm.c:757-918).
 * exp_mode 0: libm expf and the scalar trust-rule arithmetic (scalar fitter);
 * exp_mode 1: the batch fitter's Cephes-style exp and trust-rule arithmetic
 *             (peak_locate_lm_batch.c:362-732, peak_simd.h vexpf). */
void orc_lsqpeaklocate_lm(const float *plane, const int *N, float *peak_loc, int nPeaks,
                          int iFitType, float *std_dev, const float *plane_weight,
                          int exp_mode);

/* peak_locate_lm.c:727-744 */
float orc_peak_detectability(const float *plane, const int *N);

/* bulkxcorr2d (PIV_2d_cross_correlate.c:203-397), same argument meaning.
 * peakfit_impl selects exp_mode for nPeaks==1 LM fits (the reference's
 * bulkxcorr2d_set_peakfit_impl).  planes_f64 (nullable) receives the FP64 planes
 * in the fCorrelPlane_Out layout.  n_threads <= 0: OpenMP default. */
unsigned char orc_bulkxcorr2d(const float *A, const float *B, const float *mask,
                              const int *img_size, int n_images, const float *ctr_x,
                              const float *ctr_y, const int *n_win, const float *wA,
                              int ensemble, const float *wB, const int *win_size,
                              int n_peaks, int peak_finder, float *pk_x, float *pk_y,
                              float *pk_h, float *sx, float *sy, float *sxy,
                              float *pk_ratio, float *plane_out, double *planes_f64,
                              int peakfit_impl, int n_threads);

/* bulkxcorr2d_accumulate_triple (PIV_2d_cross_correlate.c:627-833).  FP64 planes and
 * FP64 sums; the float output arrays are += (caller-zeroed), like the reference. */
unsigned char orc_accumulate_triple(const float *A, const float *B, const float *mask,
                                    const int *img_size, int n_images, const float *ctr_x,
                                    const float *ctr_y, const int *n_win,
                                    const float *wA_ab, const float *wB_ab,
                                    const float *w_auto_a, const float *w_auto_b,
                                    const int *win_size, const int *fit_size,
                                    int mean_subtract, int per_pair_norm, float *ab,
                                    float *aa, float *bb, int n_threads);

/* bulkxcorr2d_accumulate (PIV_2d_cross_correlate.c:502-607). */
unsigned char orc_accumulate(const float *A, const float *B, const float *mask,
                             const int *img_size, int n_images, const float *ctr_x,
                             const float *ctr_y, const int *n_win, const float *wA,
                             const float *wB, const int *win_size, const int *fit_size,
                             float *sum, int n_threads);

/* fused_symmetric_warp_batch, scalar route (fused_warp.c:52-307, 317-382, 479-582). */
int orc_fused_warp_batch(const float *imgs_a, const float *imgs_b, float *outs_a,
                         float *outs_b, const float *pred_dy, const float *pred_dx, int N,
                         int H, int W, int nPY, int nPX, const float *ctrs_y,
                         const float *ctrs_x, int interp_mode, int shared_predictor,
                         int round_shifts, int n_threads);

/* kspace_lm_fit_batch (kspace_lm_fit.c:669-884), FP64. */
int orc_kspace_lm_fit_batch(const double *R_AA, const double *R_BB, const double *R_AB,
                            const unsigned char *mask, const double *P_win, int n_windows,
                            int h, int w, int use_kx4, int use_ky4, double *gauss_flat,
                            int *status, double *initial_guess, double *diag_gain,
                            double *diag_N0, double *diag_b4x, double *diag_b4y,
                            double *diag_cost_per_pt, int *diag_n_valid, int *diag_iter,
                            unsigned char *diag_conv, int n_threads);

/* kspace_fft2_centered (kspace_lm_fit.c:934-947). */
int orc_kspace_fft2_centered(const double *plane, int h, int w, double *re, double *im);

/* fminvec / fmaxvec (PIV_2d_cross_correlate.c:836-860). */
float orc_fminvec(const float *v, int n);
float orc_fmaxvec(const float *v, int n);

#ifdef __cplusplus
}
#endif
#endif
