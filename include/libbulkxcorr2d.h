/*
 * libbulkxcorr2d.h -- C-ABI of the sm_100a libbulkxcorr2d.so.
 *
 * Drop-in for the reference library of the same name: every symbol below keeps
 * the reference declaration's name, argument meaning, array layout and error
 * codes.  The reference declaration each one replaces is cited as
 * file:line within the reference project (pivtools_cli/lib/...).
 *
 * Host-pointer entry points copy their arrays to the GPU, compute there and copy
 * the results back; they serialise on an internal lock.  The pivb_*_dev entry
 * points take device pointers and a cudaStream_t (passed as void*) for callers
 * that keep data resident on the GPU.
 *
 * Error codes (unsigned char / int): 0 none, 1 NOMEM, 2 NOPLAN_FWD, 4 NOPLAN_BWD,
 * 8 NOPLAN, 9 OUT_OF_BOUNDS (pivtools_cli/lib/common.h:31-36), and 16 when a
 * CUDA runtime call fails (no usable GPU).  Window sides must be one of
 * 8 12 16 24 32 48 64 96 128 (pivtools_core/fft_sizes.py:16) and, in this
 * library, square (h == w); other sizes return NOPLAN_BWD / NOPLAN.
 */
#ifndef PIVB_LIBBULKXCORR2D_H
#define PIVB_LIBBULKXCORR2D_H

#include <stdbool.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* PIV_2d_cross_correlate.h:18-20 (bulkxcorr2d).  Outputs [N][nPeaks][nWinY][nWinX];
 * fPkRatio [N][nWinY*nWinX]; fCorrelPlane_Out nullable [N*nWin*h*w].  Windows that
 * are masked or do not fit the image leave their outputs untouched. */
unsigned char bulkxcorr2d(const float *fImageA, const float *fImageB, const float *fMask,
                          const int *nImageSize, int N_images, const float *fWinCtrsX,
                          const float *fWinCtrsY, const int *nWindows, float *fWindowWeightA,
                          bool bEnsemble, const float *fWindowWeightB, const int *nWindowSize,
                          int nPeaks, int iPeakFinder, float *fPkLocX, float *fPkLocY,
                          float *fPkHeight, float *fSx, float *fSy, float *fSxy, float *fPkRatio,
                          float *fCorrelPlane_Out);

/* PIV_2d_cross_correlate.h:37-51 (bulkxcorr2d_accumulate): += the centre crop of
 * every pair's correlation plane into the caller-zeroed sums. */
unsigned char bulkxcorr2d_accumulate(const float *fImageA_stack, const float *fImageB_stack,
                                     const float *fMask, const int *nImageSize, int N_images,
                                     const float *fWinCtrsX, const float *fWinCtrsY,
                                     const int *nWindows, const float *fWindowWeightA,
                                     const float *fWindowWeightB, const int *nWindowSize,
                                     const int *nFitWindowSize, float *fCorrelPlane_Sum);

/* PIV_2d_cross_correlate.h:66-86 (bulkxcorr2d_accumulate_triple). */
unsigned char bulkxcorr2d_accumulate_triple(const float *fImageA_stack, const float *fImageB_stack,
                                            const float *fMask, const int *nImageSize, int N_images,
                                            const float *fWinCtrsX, const float *fWinCtrsY,
                                            const int *nWindows, const float *fWindowWeightA_AB,
                                            const float *fWindowWeightB_AB,
                                            const float *fAutoWeightA, const float *fAutoWeightB,
                                            const int *nWindowSize, const int *nFitWindowSize,
                                            int bMeanSubtract, int bPerPairNorm, float *fCorrAB_Sum,
                                            float *fCorrAA_Sum, float *fCorrBB_Sum);

/* PIV_2d_cross_correlate.h:88-89 */
float fminvec(const float *fVec, int n);
float fmaxvec(const float *fVec, int n);

/* PIV_2d_cross_correlate.h:97-99: GPU time of the correlation kernel (fft_s) and
 * of the deferred LM fit kernel (fit_s), seconds, summed over calls. */
void bulkxcorr2d_set_timing_enabled(int on);
void bulkxcorr2d_reset_timing(void);
void bulkxcorr2d_get_timing(double *fft_s, double *fit_s);

/* PIV_2d_cross_correlate.h:107-109: 0 = scalar-fitter semantics, 1 = batch-fitter
 * semantics (its exponential and trust-rule arithmetic). */
int bulkxcorr2d_set_peakfit_impl(int impl);
int bulkxcorr2d_get_peakfit_impl(void);
int bulkxcorr2d_peakfit_batch_available(void);

/* peak_locate_lm.h:39, 46, 51 */
void lsqpeaklocate_lm(const float *xcorr, const int *N, float *peak_loc, int nPeaks, int iFitType,
                      float *std_dev, const float *fPlaneWeight);
float peak_detectability(const float *xcorr, const int *N);
int pivtools_cpu_supported(void);

/* peak_locate_lm_batch.h:39-51 (component-major [3][peakfit_batch_lanes()]) */
void lsqpeaklocate_lm_batch(const float *planes, int L_real, const int *N, int iFitType,
                            float *peak_loc, float *std_dev, const float *fPlaneWeight);
int peakfit_batch_available(void);
int peakfit_batch_lanes(void);

/* xcorr.h:26-27 and codelet_fft.h:74 */
unsigned convolve(const float *w1, const float *w2, float *conv, const int *N);
unsigned xcorr(const float *w1, const float *w2, float *corr, const int *N);
int codelet_lanes(void);

/* ---- device-pointer API (no counterpart in the reference; resident callers) ---- */

/* Scratch bytes pivb_xcorr_dev needs (deferred LM fit records). */
size_t pivb_xcorr_scratch_bytes(long long n_windows_total, int n_peaks, int peak_finder);

/* Bytes of per-window records (128 B each) with which pivb_xcorr_dev defers every
 * single-peak fit, the 3-point Gaussian included, to a thread-per-window kernel.
 * Optional for peak finder 3 (passing less scratch keeps the fit in the
 * correlation kernel, with identical results); no counterpart in the reference. */
size_t pivb_xcorr_record_bytes(long long n_windows_total);

/* Scratch bytes pivb_xcorr_dev needs for h x w windows: pivb_xcorr_scratch_bytes
 * for square windows; for rectangular windows (h != w, both in 8..128) the
 * planes of the staged rectangular path, processed in chunks of at most 256 MiB
 * of windows.  No counterpart in the reference. */
size_t pivb_xcorr_scratch_bytes_hw(long long n_windows_total, int win_h, int win_w, int n_peaks,
                                   int peak_finder);

/* numel / (wB (*) wB) into d_out [h*w] (the fit patch's loss-of-correlation weight). */
int pivb_correl_weight_dev(const float *d_wB, int h, int w, float *d_out, void *stream);

/* bulkxcorr2d on device pointers; img_stride = elements between frames.
 * Rectangular windows (win_h != win_w) take the staged path and need
 * pivb_xcorr_scratch_bytes_hw bytes of scratch (else 1, NOMEM). */
int pivb_xcorr_dev(const float *d_A, const float *d_B, long long img_stride, const float *d_mask,
                   int H, int W, int n_images, const float *d_ctr_x, const float *d_ctr_y,
                   int n_win_y, int n_win_x, const float *d_wA, const float *d_wB,
                   const float *d_cw, int win_h, int win_w, int ensemble, int n_peaks,
                   int peak_finder, int peakfit_impl, float *d_pk_x, float *d_pk_y,
                   float *d_pk_h, float *d_sx, float *d_sy, float *d_sxy, float *d_pk_ratio,
                   float *d_planes, void *d_scratch, size_t scratch_bytes, void *stream);

/* Scratch bytes of the device accumulation entry points for one call. */
size_t pivb_accumulate_scratch_bytes(int win, long long n_windows);

/* bulkxcorr2d_accumulate_triple on device pointers.  Per window the spectra of up
 * to 64 pairs are summed in FP32 and transformed back once; each such block is
 * added to the sums with Kahan compensation in FP32; d_comp (nullable, 3 arrays of
 * the sums' size) carries the compensation terms across blocks and calls. */
int pivb_accumulate_triple_dev(const float *d_A, const float *d_B, long long img_stride,
                               const float *d_mask, int H, int W, int n_images,
                               const float *d_ctr_x, const float *d_ctr_y, int n_win_y,
                               int n_win_x, const float *d_w_ab_a, const float *d_w_ab_b,
                               const float *d_w_auto_a, const float *d_w_auto_b, int win_h,
                               int win_w, int out_h, int out_w, int mean_subtract,
                               int per_pair_norm, float *d_ab, float *d_aa, float *d_bb,
                               float *d_comp, void *d_scratch, size_t scratch_bytes, void *stream);

/* bulkxcorr2d_accumulate on device pointers (cross plane only). */
int pivb_accumulate_dev(const float *d_A, const float *d_B, long long img_stride,
                        const float *d_mask, int H, int W, int n_images, const float *d_ctr_x,
                        const float *d_ctr_y, int n_win_y, int n_win_x, const float *d_wA,
                        const float *d_wB, int win_h, int win_w, int out_h, int out_w,
                        float *d_sum, float *d_comp, void *d_scratch, size_t scratch_bytes,
                        void *stream);

/* Packed correlation launches (no counterpart in the reference; the serving
 * loop's work queue).  One job = the arguments of one single-peak pivb_xcorr_dev
 * call on device pointers.  pivb_xcorr_jobs_dev correlates and fits up to
 * pivb_xcorr_jobs_max() jobs of one square window size in one launch of the
 * correlation kernel and one of the fit kernel; jobs may differ in frames,
 * frame size, window grid, mask, weights and outputs, and each job's results
 * equal its own pivb_xcorr_dev call's.  d_records holds
 * pivb_xcorr_jobs_record_bytes bytes.  The job table is passed as the kernels'
 * parameter: no copy is issued.  Returns the codes of pivb_xcorr_dev. */
typedef struct {
    const float *A, *B;
    long long img_stride;
    const float *mask;
    int H, W, n_images;
    const float *ctr_x, *ctr_y;
    int n_win_y, n_win_x;
    const float *wA, *wB, *cw;
    float *pk_x, *pk_y, *pk_h, *sx, *sy, *sxy, *pk_ratio;
} PivbXcorrJob;

int pivb_xcorr_jobs_max(void);
size_t pivb_xcorr_jobs_record_bytes(const PivbXcorrJob *jobs, int n_jobs, int win);
int pivb_xcorr_jobs_dev(const PivbXcorrJob *jobs, int n_jobs, int win, int peak_finder,
                        int peakfit_impl, void *d_records, size_t record_bytes, void *stream);

/* Allocation-free variant of pivb_xcorr_dev (no counterpart in the reference),
 * for callers that cannot allocate device memory: a host whose GPU memory is
 * owned by another allocator, a stream being captured into a CUDA graph, or a
 * pipeline that cannot take the device synchronisation cudaFree implies.  The
 * deferred-LM scratch is a fixed 16 MiB file-scope device array: at most 131072
 * windows per call when LM records are needed (nPeaks 1, finder 4-6); larger calls
 * return 1 (NOMEM) with a message on stderr.  The first call on a device, of any
 * window size, resolves the array's address (cudaGetSymbolAddress) and sets up
 * the correlation kernels of every built window size on that device; make it
 * before any stream capture.  All calls share the array; calls overlapping on
 * the GPU race. */
int pivb_xcorr_dev_noalloc(const float *d_A, const float *d_B, long long img_stride,
                           const float *d_mask, int H, int W, int n_images, const float *d_ctr_x,
                           const float *d_ctr_y, int n_win_y, int n_win_x, const float *d_wA,
                           const float *d_wB, const float *d_cw, int win_h, int win_w, int ensemble,
                           int n_peaks, int peak_finder, int peakfit_impl, float *d_pk_x,
                           float *d_pk_y, float *d_pk_h, float *d_sx, float *d_sy, float *d_sxy,
                           float *d_pk_ratio, float *d_planes, void *stream);

/* Device ordinal (return) and name of the GPU in use; -1 if none. */
int pivb_device_info(char *name, int len);

#ifdef __cplusplus
}
#endif
#endif
