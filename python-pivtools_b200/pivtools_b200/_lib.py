"""ctypes loading of the in-tree sm_100a libraries.

The libraries are loaded from pivtools_b200/lib/ only.  A missing library is an
error (FileNotFoundError), never a reason to compute elsewhere: this package has
no CPU implementation of the path.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

LIBDIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")

f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
vp = ctypes.c_void_p
ci = ctypes.c_int
cll = ctypes.c_longlong
csz = ctypes.c_size_t

_cache: dict[str, ctypes.CDLL] = {}


def lib_path(name: str) -> str:
    return os.path.join(LIBDIR, name)


def _load(name: str) -> ctypes.CDLL:
    if name in _cache:
        return _cache[name]
    path = lib_path(name)
    if not os.path.isfile(path):
        raise FileNotFoundError(
            f"{path} is not built; run `python -m pivtools_b200.build` (or __graft_entry__.build())")
    L = ctypes.CDLL(path)
    _cache[name] = L
    return L


class XcorrJob(ctypes.Structure):
    """One job of a packed correlation launch (PivbXcorrJob in libbulkxcorr2d.h)."""
    _fields_ = [("A", ctypes.c_void_p), ("B", ctypes.c_void_p), ("img_stride", ctypes.c_longlong),
                ("mask", ctypes.c_void_p), ("H", ctypes.c_int), ("W", ctypes.c_int), ("n_images", ctypes.c_int),
                ("ctr_x", ctypes.c_void_p), ("ctr_y", ctypes.c_void_p), ("n_win_y", ctypes.c_int),
                ("n_win_x", ctypes.c_int), ("wA", ctypes.c_void_p), ("wB", ctypes.c_void_p), ("cw", ctypes.c_void_p),
                ("pk_x", ctypes.c_void_p), ("pk_y", ctypes.c_void_p), ("pk_h", ctypes.c_void_p),
                ("sx", ctypes.c_void_p), ("sy", ctypes.c_void_p), ("sxy", ctypes.c_void_p),
                ("pk_ratio", ctypes.c_void_p)]


def bulkxcorr2d_lib() -> ctypes.CDLL:
    L = _load("libbulkxcorr2d.so")
    if getattr(L, "_pivb_bound", False):
        return L
    L.bulkxcorr2d.argtypes = [f32p, f32p, f32p, i32p, ci, f32p, f32p, i32p, f32p, ctypes.c_bool,
                              f32p, i32p, ci, ci, f32p, f32p, f32p, f32p, f32p, f32p, f32p, vp]
    L.bulkxcorr2d.restype = ctypes.c_ubyte
    L.lsqpeaklocate_lm.argtypes = [f32p, i32p, f32p, ci, ci, f32p, vp]
    L.lsqpeaklocate_lm.restype = None
    L.lsqpeaklocate_lm_batch.argtypes = [f32p, ci, i32p, ci, f32p, f32p, vp]
    L.lsqpeaklocate_lm_batch.restype = None
    L.peak_detectability.argtypes = [f32p, i32p]
    L.peak_detectability.restype = ctypes.c_float
    L.pivtools_cpu_supported.restype = ci
    L.peakfit_batch_available.restype = ci
    L.peakfit_batch_lanes.restype = ci
    L.codelet_lanes.restype = ci
    L.bulkxcorr2d_set_peakfit_impl.argtypes = [ci]
    L.bulkxcorr2d_set_peakfit_impl.restype = ci
    L.bulkxcorr2d_get_peakfit_impl.restype = ci
    L.bulkxcorr2d_peakfit_batch_available.restype = ci
    L.bulkxcorr2d_set_timing_enabled.argtypes = [ci]
    L.bulkxcorr2d_set_timing_enabled.restype = None
    L.bulkxcorr2d_reset_timing.restype = None
    L.bulkxcorr2d_get_timing.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    L.bulkxcorr2d_get_timing.restype = None
    L.convolve.argtypes = [f32p, f32p, f32p, i32p]
    L.convolve.restype = ctypes.c_uint
    L.xcorr.argtypes = [f32p, f32p, f32p, i32p]
    L.xcorr.restype = ctypes.c_uint
    L.fminvec.argtypes = [f32p, ci]
    L.fminvec.restype = ctypes.c_float
    L.fmaxvec.argtypes = [f32p, ci]
    L.fmaxvec.restype = ctypes.c_float
    L.pivb_xcorr_scratch_bytes.argtypes = [cll, ci, ci]
    L.pivb_xcorr_scratch_bytes.restype = csz
    L.pivb_correl_weight_dev.argtypes = [vp, ci, ci, vp, vp]
    L.pivb_correl_weight_dev.restype = ci
    L.pivb_xcorr_scratch_bytes_hw.argtypes = [cll, ci, ci, ci, ci]
    L.pivb_xcorr_scratch_bytes_hw.restype = csz
    L.pivb_xcorr_record_bytes.argtypes = [cll]
    L.pivb_xcorr_record_bytes.restype = csz
    L.pivb_xcorr_dev.argtypes = [vp, vp, cll, vp, ci, ci, ci, vp, vp, ci, ci, vp, vp, vp, ci, ci, ci, ci,
                                 ci, ci, vp, vp, vp, vp, vp, vp, vp, vp, vp, csz, vp]
    L.pivb_xcorr_dev.restype = ci
    if hasattr(L, "pivb_xcorr_dev_noalloc"):
        L.pivb_xcorr_dev_noalloc.argtypes = [vp, vp, cll, vp, ci, ci, ci, vp, vp, ci, ci, vp, vp, vp, ci, ci, ci,
                                             ci, ci, ci, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.pivb_xcorr_dev_noalloc.restype = ci
    L.pivb_device_info.argtypes = [ctypes.c_char_p, ci]
    L.pivb_device_info.restype = ci
    for opt in ("bulkxcorr2d_accumulate", "bulkxcorr2d_accumulate_triple"):
        if hasattr(L, opt):
            getattr(L, opt).restype = ctypes.c_ubyte
    if hasattr(L, "bulkxcorr2d_accumulate"):
        L.bulkxcorr2d_accumulate.argtypes = [f32p, f32p, f32p, i32p, ci, f32p, f32p, i32p, f32p, f32p,
                                             i32p, vp, f32p]
    if hasattr(L, "bulkxcorr2d_accumulate_triple"):
        L.bulkxcorr2d_accumulate_triple.argtypes = [f32p, f32p, f32p, i32p, ci, f32p, f32p, i32p, f32p,
                                                    f32p, f32p, f32p, i32p, vp, ci, ci, f32p, f32p,
                                                    f32p]
    L.pivb_accumulate_triple_dev.argtypes = [vp, vp, cll, vp, ci, ci, ci, vp, vp, ci, ci, vp, vp, vp, vp,
                                             ci, ci, ci, ci, ci, ci, vp, vp, vp, vp, vp, csz, vp]
    L.pivb_accumulate_triple_dev.restype = ci
    L.pivb_accumulate_dev.argtypes = [vp, vp, cll, vp, ci, ci, ci, vp, vp, ci, ci, vp, vp, ci, ci, ci, ci,
                                      vp, vp, vp, csz, vp]
    L.pivb_accumulate_dev.restype = ci
    L.pivb_accumulate_scratch_bytes.argtypes = [ci, cll]
    L.pivb_accumulate_scratch_bytes.restype = csz
    L.pivb_xcorr_jobs_max.restype = ci
    L.pivb_xcorr_jobs_record_bytes.argtypes = [ctypes.POINTER(XcorrJob), ci, ci]
    L.pivb_xcorr_jobs_record_bytes.restype = csz
    L.pivb_xcorr_jobs_dev.argtypes = [ctypes.POINTER(XcorrJob), ci, ci, ci, ci, vp, csz, vp]
    L.pivb_xcorr_jobs_dev.restype = ci
    L.pivb_xcorr_set_ctas_per_sm.argtypes = [ci, ci]
    L.pivb_xcorr_set_ctas_per_sm.restype = ci
    L.pivb_xcorr_get_ctas_per_sm.argtypes = [ci]
    L.pivb_xcorr_get_ctas_per_sm.restype = ci
    L.pivb_xcorr_max_ctas_per_sm.argtypes = [ci]
    L.pivb_xcorr_max_ctas_per_sm.restype = ci
    L.pivb_xcorr_set_record_block.argtypes = [ci]
    L.pivb_xcorr_set_record_block.restype = ci
    L._pivb_bound = True
    return L


def fusedwarp_lib() -> ctypes.CDLL:
    L = _load("libfusedwarp.so")
    if getattr(L, "_pivb_bound", False):
        return L
    L.fused_warp_set_impl.argtypes = [ci]
    L.fused_warp_set_impl.restype = None
    L.fused_warp_get_impl.restype = ci
    L.fused_symmetric_warp.argtypes = [f32p, f32p, f32p, f32p, f32p, f32p, ci, ci, ci, ci, f32p, f32p,
                                       ci, ci]
    L.fused_symmetric_warp.restype = ci
    L.fused_symmetric_warp_batch.argtypes = [f32p, f32p, f32p, f32p, f32p, f32p, ci, ci, ci, ci, ci,
                                             f32p, f32p, ci, ci, ci]
    L.fused_symmetric_warp_batch.restype = ci
    L.pivb_warp_dev.argtypes = [vp, vp, vp, vp, vp, vp, ci, ci, ci, ci, ci, cll, vp, ci, ci, ci, ci, vp]
    L.pivb_warp_dev.restype = ci
    L.pivb_warp_setup_dev.argtypes = [vp, ci, vp, ci, ci, ci, vp, vp]
    L.pivb_warp_setup_dev.restype = ci
    L.pivb_warp_table_bytes.argtypes = [ci, ci]
    L.pivb_warp_table_bytes.restype = csz
    L.pivb_warp_set_launch.argtypes = [ci, ci]
    L.pivb_warp_set_launch.restype = ci
    L.pivb_warp_get_launch.argtypes = [vp, vp]
    L.pivb_warp_get_launch.restype = None
    L._pivb_bound = True
    return L


def kspacefit_lib() -> ctypes.CDLL:
    L = _load("libkspacefit.so")
    if getattr(L, "_pivb_bound", False):
        return L
    L.kspace_lm_fit_batch.argtypes = [f64p, f64p, f64p, u8p, vp, ci, ci, ci, ci, ci, ci, f64p, i32p,
                                      f64p, f64p, f64p, f64p, f64p, f64p, i32p, i32p, u8p]
    L.kspace_lm_fit_batch.restype = ci
    L.kspace_lm_fit_max_threads.restype = ci
    L.kspace_fft2_centered.argtypes = [f64p, ci, ci, f64p, f64p]
    L.kspace_fft2_centered.restype = ci
    L.kspace_debug_prep.argtypes = [f64p, f64p, f64p, vp, ci, ci, f64p, ctypes.POINTER(ctypes.c_double)]
    L.kspace_debug_prep.restype = ci
    L.pivb_kspace_scratch_bytes.argtypes = [ci, ci, ci]
    L.pivb_kspace_scratch_bytes.restype = csz
    L.pivb_kspace_fit_dev.argtypes = [vp, vp, vp, vp, vp, ci, ci, ci, ci, ci, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                      vp, vp, vp, csz, vp]
    L.pivb_kspace_fit_dev.restype = ci
    L._pivb_bound = True
    return L


def pass_lib() -> ctypes.CDLL:
    L = _load("libpivb_pass.so")
    if getattr(L, "_pivb_bound", False):
        return L
    fl = ctypes.c_float
    L.pivb_validate_dev.argtypes = [vp, vp, vp, vp, vp, vp, ci, ci, ci, fl, fl, fl, fl, fl, ci, vp, vp, vp, vp,
                                    vp, vp]
    L.pivb_validate_dev.restype = ci
    L.pivb_floor_interp_dev.argtypes = [vp, ci, vp, ci, vp, vp, ci, vp, vp]
    L.pivb_floor_interp_dev.restype = ci
    L.pivb_infill_dev.argtypes = [vp, vp, vp, vp, ci, ci, ci, fl, fl, ci, ci, ctypes.c_double, vp, csz, vp]
    L.pivb_infill_dev.restype = ci
    L.pivb_infill_work_bytes.argtypes = [ci, ci, ci]
    L.pivb_infill_work_bytes.restype = csz
    L.pivb_pad_smooth_dev.argtypes = [vp, vp, ci, ci, ci, ci, ci, ci, ci, vp, ci, vp, vp, vp, vp]
    L.pivb_pad_smooth_dev.restype = ci
    L.pivb_remap_dev.argtypes = [vp, vp, ci, ci, ci, vp, vp, ci, ci, vp, vp, vp]
    L.pivb_remap_dev.restype = ci
    L.pivb_u16_to_f32_dev.argtypes = [vp, vp, cll, vp]
    L.pivb_u16_to_f32_dev.restype = ci
    L.pivb_frame_sum_dev.argtypes = [vp, cll, ci, cll, vp, vp, vp]
    L.pivb_frame_sum_dev.restype = ci
    L.pivb_frame_mean_dev.argtypes = [vp, cll, ci, vp, vp]
    L.pivb_frame_mean_dev.restype = ci
    L.pivb_center_frames_dev.argtypes = [vp, cll, ci, cll, vp, vp, cll, vp]
    L.pivb_center_frames_dev.restype = ci
    L.pivb_ensemble_finalize_dev.argtypes = [vp, vp, vp, vp, vp, vp, ci, ci, ci, ci, ci, vp, vp, vp, vp, vp, vp,
                                             ctypes.c_float, vp]
    L.pivb_pad_frames_dev.argtypes = [vp, cll, ci, ci, ci, vp, ci, ci, vp, ci, ci, cll, vp]
    L.pivb_pad_frames_dev.restype = ci
    L.pivb_ensemble_finalize_dev.restype = ci
    L.pivb_decode_frames_dev.argtypes = [vp, cll, ci, ci, ci, ci, ci, vp, cll, ci, ci, vp, cll, vp]
    L.pivb_decode_frames_dev.restype = ci
    L.pivb_validate_peaks_dev.argtypes = [vp, vp, vp, ci, ci, vp, vp, vp, ci, ci, ci, fl, fl, fl, fl, fl, ci,
                                          fl, ci, fl, fl, vp, vp, vp, vp, vp, vp, vp]
    L.pivb_validate_peaks_work_floats.argtypes = [ci, ci, ci]
    L.pivb_validate_peaks_work_floats.restype = cll
    L.pivb_validate_peaks_dev.restype = ci
    L.pivb_nearest_infill_dev.argtypes = [vp, vp, vp, vp, ci, ci, ci, ctypes.c_double, ctypes.c_double, vp]
    L.pivb_nearest_infill_dev.restype = ci
    L.pivb_gather_fill_dev.argtypes = [vp, vp, vp, ci, cll, vp, vp, vp]
    L.pivb_gather_fill_dev.restype = ci
    L.pivb_payload_bytes.argtypes = [cll, ci]
    L.pivb_payload_bytes.restype = cll
    L.pivb_unpack_pixels_dev.argtypes = [vp, cll, ci, cll, ci, ci, fl, ci, fl, vp, cll, vp]
    L.pivb_unpack_pixels_dev.restype = ci
    L._pivb_bound = True
    return L


def lavision_lib() -> ctypes.CDLL:
    """Host codecs of the LaVision containers (libpivb_lavision.so)."""
    L = _load("libpivb_lavision.so")
    if getattr(L, "_pivb_bound", False):
        return L
    llp = ctypes.POINTER(ctypes.c_longlong)
    L.pivb_davis_tokens_decode.argtypes = [vp, cll, llp, llp, vp, cll, llp]
    L.pivb_davis_tokens_decode.restype = ci
    L.pivb_lz4_block_decode.argtypes = [vp, cll, vp, cll]
    L.pivb_lz4_block_decode.restype = ci
    L.pivb_zlib_inflate_exact.argtypes = [vp, cll, vp, cll]
    L.pivb_zlib_inflate_exact.restype = ci
    L.pivb_zlib_inflate_prefix.argtypes = [vp, cll, vp, cll]
    L.pivb_zlib_inflate_prefix.restype = cll
    L.pivb_zlib_blocks_decode.argtypes = [vp, cll, cll, cll, cll, vp, cll, ci, llp, llp]
    L.pivb_zlib_blocks_decode.restype = ci
    L._pivb_bound = True
    return L


def dft_lib() -> ctypes.CDLL:
    L = _load("libpivb_dft.so")
    if getattr(L, "_pivb_bound", False):
        return L
    L.pivb_umma_selftest.argtypes = [vp, vp, vp, ci, ci, ci, vp, vp]
    L.pivb_umma_selftest.restype = ci
    L.pivb_wait_timeout_selftest.argtypes = [vp, ci, vp]
    L.pivb_wait_timeout_selftest.restype = ci
    L.pivb_dft_xcorr_dev.argtypes = [vp, vp, cll, vp, ci, ci, ci, vp, vp, ci, ci, vp, vp, vp, ci, ci, ci, ci,
                                     ci, ci, vp, vp, vp, vp, vp, vp, vp, vp, vp, csz, vp, vp]
    L.pivb_dft_xcorr_dev.restype = ci
    L._pivb_bound = True
    return L


def loaded_paths() -> list[str]:
    return [lib_path(n) for n in _cache]
