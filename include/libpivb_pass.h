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
 * med_size 3 or 5) tests.  ux/uy: NaN where invalid, 0 at masked windows.
 * work: 2*N*ny*nx floats. */
int pivb_validate_dev(const float *pk_x, const float *pk_y, const float *pk_h, const float *pred_dy,
                      const float *pred_dx, const float *mask, int N, int ny, int nx, float thresh_x,
                      float thresh_y, float peak_thr, float med_eps, float med_thr, int med_size,
                      float *ux, float *uy, unsigned char *invalid, float *work, void *stream);

/* Harmonic inpainting of the invalid vectors in place (infilling.py:336-376).
 * work: 2*N*ny*nx floats. */
int pivb_infill_dev(float *ux, float *uy, const unsigned char *invalid, const float *mask, int N,
                    int ny, int nx, float spacing_y, float spacing_x, int max_iter, float tol,
                    float *work, void *stream);

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

#ifdef __cplusplus
}
#endif
#endif
