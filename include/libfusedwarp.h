/*
 * libfusedwarp.h -- C-ABI of the sm_100a libfusedwarp.so.
 *
 * Drop-in for the reference library of the same name (pivtools_cli/lib/fused_warp.h):
 * same symbols, argument meaning, layouts and return codes (0 success, 1 bad
 * arguments / failure).  The warp runs on the GPU; host-pointer entry points
 * stage their arrays through a device workspace.
 *
 * impl 0 reproduces the reference's scalar route bit for bit; impl 1 (default)
 * its SIMD route's interior association (fused multiply-add column accumulator).
 */
#ifndef PIVB_LIBFUSEDWARP_H
#define PIVB_LIBFUSEDWARP_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* fused_warp.h:21-22 */
void fused_warp_set_impl(int impl);
int fused_warp_get_impl(void);

/* fused_warp.h:55-64 (single pair, shared predictor) */
int fused_symmetric_warp(const float *img_a, const float *img_b, float *out_a, float *out_b,
                         const float *pred_dy, const float *pred_dx, int H, int W, int nPY, int nPX,
                         const float *ctrs_y, const float *ctrs_x, int interp_mode, int round_shifts);

/* fused_warp.h:78-93 */
int fused_symmetric_warp_batch(const float *imgs_a, const float *imgs_b, float *outs_a,
                               float *outs_b, const float *pred_dy, const float *pred_dx, int N,
                               int H, int W, int nPY, int nPX, const float *ctrs_y,
                               const float *ctrs_x, int interp_mode, int shared_predictor,
                               int round_shifts);

/* ---- device-pointer API (no counterpart in the reference; resident callers) ---- */

/* Bytes of the per-geometry tables (pixel -> predictor index maps, Lanczos weights,
   per-row predictor weights). */
size_t pivb_warp_table_bytes(int H, int W);

/* Build the tables for predictor centres d_ctrs_y [nPY], d_ctrs_x [nPX] (ascending). */
int pivb_warp_setup_dev(const float *d_ctrs_y, int nPY, const float *d_ctrs_x, int nPX, int H,
                        int W, void *d_tables, void *stream);

/* Warp N pairs held on the device; img_stride = elements between frames. */
int pivb_warp_dev(const float *d_ia, const float *d_ib, float *d_oa, float *d_ob,
                  const float *d_pdy, const float *d_pdx, int N, int H, int W, int nPY, int nPX,
                  long long img_stride, const void *d_tables, int interp_mode,
                  int shared_predictor, int round_shifts, int impl, void *stream);

#ifdef __cplusplus
}
#endif
#endif
