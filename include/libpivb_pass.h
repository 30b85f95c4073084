/*
 * libpivb_pass.h -- C-ABI of libpivb_pass.so: the steps between multipass
 * passes, on the GPU.  No counterpart in the reference's C libraries: the
 * reference runs these steps in Python between its C calls
 * (pivtools_cli/piv/piv_backend/cpu_instantaneous.py:559-870, :1040-1071).
 * All pointers are device pointers; stream is a cudaStream_t.  Return 0 on
 * success, 1 on bad arguments or a launch failure.
 */
#ifndef PIVB_LIBPIVB_PASS_H
#define PIVB_LIBPIVB_PASS_H

#ifdef __cplusplus
extern "C" {
#endif

/* Gate (|d| > thresh), add the window-grid predictor (nullable), peak-magnitude
 * (peak_thr < 0 disables) and normalised-median (med_thr <= 0 disables;
 * med_size 3 or 5) tests (cpu_instantaneous.py:575-760 with one peak,
 * outlier_detection.py:56-243).  ux/uy: NaN where invalid, 0 at masked windows;
 * invalid: 1 where the vector is to be infilled; nan_reason (nullable): int8
 * codes of nan_reason_codes.py:18-25 (-1 masked, 0 valid, 1 fit failure,
 * 6 large displacement, 9 unclassified, 10 outlier, 13 NaN peak height).
 * work: 2*N*ny*nx floats. */
int pivb_validate_dev(const float *pk_x, const float *pk_y, const float *pk_h, const float *pred_dy,
                      const float *pred_dx, const float *mask, int N, int ny, int nx, float thresh_x,
                      float thresh_y, float peak_thr, float med_eps, float med_thr, int med_size,
                      float *ux, float *uy, unsigned char *invalid, signed char *nan_reason,
                      float *work, void *stream);

/* Least-squares inpainting of the invalid vectors in place: the reference's
 * infill_harmonic (order 1) / infill_biharmonic (order 2) (infilling.py:150-283,
 * 336-421): squared first / second differences along y and x in physical units
 * (pitch spacing_y, spacing_x) minimised over the invalid cells, valid cells
 * fixed, rows touching a masked window (mask, (ny, nx), nullable) dropped; the
 * normal equations solved in FP64 by conjugate gradients to relative residual
 * tol (at most max_iter iterations).  One CTA per pair; deterministic.
 * work: pivb_infill_work_bytes(N, ny, nx) bytes. */
size_t pivb_infill_work_bytes(int N, int ny, int nx);
int pivb_infill_dev(float *ux, float *uy, const unsigned char *invalid, const float *mask, int N,
                    int ny, int nx, float spacing_y, float spacing_x, int order, int max_iter,
                    double tol, void *work, size_t work_bytes, void *stream);

/* Edge padding onto the predictor grid + Gaussian smoothing (taps: 2*radius+1
 * normalised weights on the device; radius 0 = none).  work: N*nyp*nxp floats. */
int pivb_pad_smooth_dev(const float *ux, const float *uy, int N, int ny, int nx, int nyp, int nxp,
                        int pre_y, int pre_x, const float *taps, int radius, float *pdy, float *pdx,
                        float *work, void *stream);

/* Keys-cubic remap of the padded predictor at fractional grid coordinates. */
int pivb_remap_dev(const float *pdy, const float *pdx, int N, int nyp, int nxp, const float *map_y,
                   const float *map_x, int ny, int nx, float *out_dy, float *out_dx, void *stream);

/* uint16 frames -> float32 (the reference's readers convert on the host,
 * pivtools_core/image_handling/load_images.py:594,625).  in 8-byte, out 16-byte aligned. */
int pivb_u16_to_f32_dev(const unsigned short *in, float *out, long long n, void *stream);

/* Ensemble pass on the GPU (the reference does these steps in NumPy:
 * pivtools_cli/piv/piv_backend/single_pass_accumulator.py:292-320, 508-800). */

/* sum (+)= the n_frames frames (stride elements apart, npix pixels each), Kahan-
 * compensated through comp (zero both before the first call). */
int pivb_frame_sum_dev(const float *frames, long long stride, int n_frames, long long npix, float *sum,
                       float *comp, void *stream);

/* out = sum / n: the mean frame of n accumulated pairs. */
int pivb_frame_mean_dev(const float *sum, long long npix, int n, float *out, void *stream);

/* The two-sweep 'image' background methods ('image', 'image+window_mean',
 * 'image+dc_zero'): dst frame k = src frame k - mean for n_frames frames of npix
 * pixels (strides src_stride / dst_stride elements), one float32 subtraction per
 * pixel as the reference's `images -= A_mean` before correlating
 * (pivtools_cli/piv/piv_backend/cpu_ensemble.py:1290-1291).  In place when
 * dst == src (equal strides); returns 1 on bad arguments. */
int pivb_center_frames_dev(const float *src, long long src_stride, int n_frames, long long npix, const float *mean,
                           float *dst, long long dst_stride, void *stream);

/* Finalise of one ensemble pass: average the accumulated AB/AA/BB sums of n_win
 * windows of h x w over n_pairs, subtract the background planes (all three or
 * none), optionally zero each plane's mean (the '+dc_zero' methods), divide by the
 * pair-count envelopes (nullable; env_ab defaults to env_auto), scale the AB plane
 * by ab_scale (single mode: sum-window area / particle-window area,
 * single_pass_accumulator.py:760-780; 1 in std mode), normalise by
 * sqrt(max(AA_c BB_c, 1e-12)) at the centre bin and write FP64 planes for
 * pivb_kspace_fit_dev.  norm (nullable) receives the per-window factors. */
int pivb_ensemble_finalize_dev(const float *sum_ab, const float *sum_aa, const float *sum_bb, const float *bg_ab,
                               const float *bg_aa, const float *bg_bb, int n_pairs, int n_win, int h, int w,
                               int dc_zero, const float *env_auto, const float *env_ab, double *out_ab,
                               double *out_aa, double *out_bb, float *norm, float ab_scale, void *stream);

/* Ensemble single mode: zero-padded copies of n_frames frames (H x W at
 * src_stride elements) into Hp x Wp frames at dst_stride, the source placed at
 * (pad_top, pad_left); with a mean frame (nullable) each source pixel has it
 * subtracted first, the 'image' methods' order (cpu_ensemble.py:1290-1324,
 * pivtools_core/window_utils.py:466-525). */
int pivb_pad_frames_dev(const float *src, long long src_stride, int n_frames, int H, int W, const float *mean,
                        int pad_top, int pad_left, float *dst, int Hp, int Wp, long long dst_stride, void *stream);

/* Decode n_frames camera payloads (frame k at raw + k * stride bytes) into float32
 * frames, as the reference's PIVTOOLs Acquisition reader does on the host
 * (pivtools_core/image_handling/readers/pivraw_reader.py:896-960,
 * set_reader.py:1296-1345): format 0 Mono12p (two pixels in three bytes, LSB
 * first), 1 BayerRG8 (2x2 superpixel sum R+G+G+B at half resolution); optional
 * in-run dark (same format, dark_frames 1 or 2: odd 1-based file indices, counted
 * from first_index, take dark frame A) subtracted as max(frame, dark) - dark per
 * photosite before the sum; view rotation as rot = np.rot90 turns (0..3; the
 * reader's cw90 is 3).  out_stride: floats between output frames.  Returns 0, or
 * 1 for bad arguments. */
int pivb_decode_frames_dev(const unsigned char *raw, long long stride, int n_frames, int first_index, int width,
                           int height, int format, const unsigned char *dark, long long dark_stride, int dark_frames,
                           int rot, float *out, long long out_stride, void *stream);

/* Nearest-donor infill of the invalid vectors in place (the reference's
 * infilling method 'nearest', infilling.py:114-141, 290-333): each invalid
 * vector takes both components of the nearest donor -- a vector neither invalid
 * nor masked (mask nullable, 1 = masked) and finite -- in physical distance
 * (pitch_y, pitch_x in pixels); among equidistant donors the one of smallest
 * column, then smallest row (the choice of the reference's scipy Euclidean
 * feature transform).  A pair without any donor keeps 0 there.  Returns 0, or 1
 * for bad arguments. */
int pivb_nearest_infill_dev(float *ux, float *uy, const unsigned char *invalid, const float *mask, int N, int ny,
                            int nx, double pitch_y, double pitch_x, void *stream);

/* The 'nearest' fill of a predictor's masked windows (config
 * masking.predictor_fill: nearest; infilling.py:808-874, 114-141): out[n][w] =
 * in[n][idx[w]] for N fields of `plane` windows (ux and uy alike), idx the
 * donor map of the mask (pivtools_b200.geometry.nearest_donor_map: the nearest
 * unmasked window in physical distance; each unmasked window its own donor).
 * Returns 0, or 1 for bad arguments. */
int pivb_gather_fill_dev(const float *ux, const float *uy, const int *idx, int N, long long plane, float *out_x,
                         float *out_y, void *stream);

/* Validation of one pass whose correlation returned n_peaks >= 1 peaks per
 * window (pk_* in the correlator's layout (N, n_peaks, ny, nx)), with the
 * reference's further outlier tests and its secondary-peak substitution
 * (cpu_instantaneous.py:589-760, outlier_detection.py:246-381): the primary peak
 * is gated, predicted and tested as by pivb_validate_dev, plus the local sigma
 * test on the vector norm when sigma_thr > 0 (the reference's `sigma` method)
 * and the divergence/vorticity test when divvort != 0 (`div_vort`; div_thr /
 * vort_thr < 0: 6 x 1.4826 x MAD of each pair's field), all reported as
 * outliers (reason 10); with `secondary` (config secondary_peak) and
 * n_peaks > 1, n_peaks - 1 rounds in which every invalid vector with peaks left
 * takes its next peak, is judged afresh (NaN: reason 13) and is tested by every
 * enabled test on the field of the current choices (reason 12 if it fails); at
 * the end a NaN height of the chosen peak invalidates (13).  Outputs as
 * pivb_validate_dev plus choice (N, ny, nx) uint8: the 1-based peak each valid
 * vector took, 0 for invalid and masked vectors.  work:
 * pivb_validate_peaks_work_floats(N, ny, nx) floats.  Returns 0, or 1 for bad
 * arguments. */
long long pivb_validate_peaks_work_floats(int N, int ny, int nx);
int pivb_validate_peaks_dev(const float *pk_x, const float *pk_y, const float *pk_h, int n_peaks, int secondary,
                            const float *pred_dy, const float *pred_dx, const float *mask, int N, int ny, int nx,
                            float thresh_x, float thresh_y, float peak_thr, float med_eps, float med_thr,
                            int med_size, float sigma_thr, int divvort, float div_thr, float vort_thr, float *ux,
                            float *uy, unsigned char *invalid, signed char *nan_reason, unsigned char *choice,
                            float *work, void *stream);

/* Bytes of one LaVision pixel payload of npix pixels in `encoding` (below), or -1
 * for an unknown encoding or a pixel count the packing cannot hold. */
long long pivb_payload_bytes(long long npix, int encoding);

/* Unpack n_frames LaVision pixel payloads (device memory, payload_stride bytes
 * apart) into float32 frames of npix pixels (out_stride floats apart), applying
 * the intensity scale in float32 as the reference's readers do (v * slope if
 * use_slope, then + offset if use_offset; im7_reader.py:1148-1152,
 * set_reader.py:2003-2008).  encoding: 0 raw-16-bit and the .im7 WORD buffer
 * (little-endian uint16), 1 raw-8-bit (widened, not rescaled), 2 mono-12p,
 * 3 mono-12pmsb, 4 mono-12packed, 5 mono-10p, 6 mono-10pmsb (the .set decoders of
 * set_reader.py:1196-1447), 7 the .im7 FLOAT buffer (little-endian float32).
 * Replaces the host decode of set_reader.py:1516-1549 and the float conversion of
 * im7_reader.py:1044-1053.  Returns 0, or 1 for bad arguments. */
int pivb_unpack_pixels_dev(const unsigned char *payload, long long payload_stride, int n_frames, long long npix,
                           int encoding, int use_slope, float slope, int use_offset, float offset, float *out,
                           long long out_stride, void *stream);

/* Coloured-floor regressor for the k-space fit (kspace_floor_psd.py:241-275 and
 * single_pass_accumulator.py:836-880): P_win (n_win, hw) FP64 from the fraction
 * grid P_grid (n_fracs, n_fracs, hw) FP64 indexed [fy][fx], fs (n_fracs) the
 * ascending grid fractions, pred_dy / pred_dx (nullable together) the pass
 * predictor on the window grid (float32; fractions |x - rint(x)| of x = pred / 2);
 * bilinear, rounded through float32.  The caller rejects non-finite predictors. */
int pivb_floor_interp_dev(const double *fs, int n_fracs, const double *P_grid, int hw,
                          const float *pred_dy, const float *pred_dx, int n_win, double *P_win,
                          void *stream);

#ifdef __cplusplus
}
#endif
#endif
