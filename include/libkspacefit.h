/*
 * libkspacefit.h -- C-ABI of the sm_100a libkspacefit.so.
 *
 * Drop-in for the reference library of the same name
 * (pivtools_cli/lib/kspace_lm_fit.h): same symbols, argument meaning, array
 * layouts, output contract and return codes (0 ok, -1 size outside the built
 * FFT sizes, -2 allocation / GPU failure, -3 coloured floor without tail bins).
 * The per-window FP64 fit runs on the GPU, one warp per window.
 */
#ifndef PIVB_LIBKSPACEFIT_H
#define PIVB_LIBKSPACEFIT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* kspace_lm_fit.h:54-61 (n_threads accepted, unused: the GPU sets its parallelism) */
int kspace_lm_fit_batch(const double *R_AA, const double *R_BB, const double *R_AB,
                        const unsigned char *mask_flat, const double *P_win, int n_windows,
                        int corr_h, int corr_w, int use_kx4, int use_ky4, int n_threads,
                        double *gauss_flat, int *status_flat, double *initial_guess_flat,
                        double *diag_gain, double *diag_N0, double *diag_b4x, double *diag_b4y,
                        double *diag_cost_per_pt, int *diag_n_valid, int *diag_iter,
                        unsigned char *diag_conv);

/* kspace_lm_fit.h:65 -- liveness probe; returns the GPU's multiprocessor count. */
int kspace_lm_fit_max_threads(void);

/* kspace_lm_fit.h:79-87 */
int kspace_debug_prep(const double *R_AA, const double *R_BB, const double *R_AB,
                      const double *P_centred, int H, int W, double *out_Dv, double *out_n0_seed);
int kspace_fft2_centered(const double *plane, int H, int W, double *out_re, double *out_im);

/* ---- device-pointer API (no counterpart in the reference; resident callers) ---- */
size_t pivb_kspace_scratch_bytes(int n_windows, int h, int w);
int pivb_kspace_fit_dev(const double *d_RAA, const double *d_RBB, const double *d_RAB,
                        const unsigned char *d_mask, const double *d_Pwin, int n_windows, int h,
                        int w, int use_kx4, int use_ky4, double *d_gauss, int *d_status,
                        double *d_init, double *d_gain, double *d_N0, double *d_b4x,
                        double *d_b4y, double *d_cpp, int *d_nvalid, int *d_iter,
                        unsigned char *d_conv, void *d_scratch, size_t scratch_bytes, void *stream);

#ifdef __cplusplus
}
#endif
#endif
