"""ctypes bindings for the CPU oracle (TEST INFRASTRUCTURE ONLY).

`lib/libpivoracle.so` is the project's C restatement of the reference path;
`_ref/libpeakfit_ref.so`, `_ref/libfusedwarp_ref.so`, `_ref/libbulkxcorr2d_ref.so`
and `_ref/libkspacefit_ref.so` are the reference's own fitter, warp, correlator and
k-space fitter compiled from its sources by `make -C oracle ref
PIVTOOLS_REF=<reference checkout>`.  Only the tests, the smoke check and bench.py's
CPU legs import this module.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libpivoracle.so")
REF_PEAKFIT = os.path.join(HERE, "_ref", "libpeakfit_ref.so")
REF_WARP = os.path.join(HERE, "_ref", "libfusedwarp_ref.so")
REF_BULK = os.path.join(HERE, "_ref", "libbulkxcorr2d_ref.so")
REF_KSPACE = os.path.join(HERE, "_ref", "libkspacefit_ref.so")

_f32 = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64 = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_vp = ctypes.c_void_p
_ci = ctypes.c_int


def ref_root() -> str | None:
    """The reference checkout named by $PIVTOOLS_REF, if it holds the C sources."""
    r = os.environ.get("PIVTOOLS_REF", "")
    return r if r and os.path.isfile(os.path.join(r, "pivtools_cli", "lib", "PIV_2d_cross_correlate.c")) else None


def build(with_ref: bool = True) -> None:
    """Compile the restatement (always) and, when $PIVTOOLS_REF names a reference
    checkout, the reference's own libraries from its sources."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if with_ref and ref_root():
        subprocess.run(["make", "-s", "-j4", "-C", HERE, "ref", f"PIVTOOLS_REF={ref_root()}"], check=True)


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.isfile(LIB_PATH):
        build(with_ref=False)
    L = ctypes.CDLL(LIB_PATH)
    L.orc_xcorr_plane.argtypes = [_f32, _f32, _ci, _ci, _f64]
    L.orc_correl_weight.argtypes = [_f32, _ci, _ci, _f32]
    L.orc_lsqpeaklocate_lm.argtypes = [_f32, _i32, _f32, _ci, _ci, _f32, _vp, _ci]
    L.orc_lsqpeaklocate_lm.restype = None
    L.orc_peak_detectability.argtypes = [_f32, _i32]
    L.orc_peak_detectability.restype = ctypes.c_float
    L.orc_bulkxcorr2d.argtypes = [_f32, _f32, _f32, _i32, _ci, _f32, _f32, _i32, _f32, _ci,
                                  _f32, _i32, _ci, _ci, _f32, _f32, _f32, _f32, _f32, _f32,
                                  _f32, _vp, _vp, _ci, _ci]
    L.orc_bulkxcorr2d.restype = ctypes.c_ubyte
    L.orc_accumulate_triple.argtypes = [_f32, _f32, _f32, _i32, _ci, _f32, _f32, _i32, _f32,
                                        _f32, _f32, _f32, _i32, _vp, _ci, _ci, _f32, _f32,
                                        _f32, _ci]
    L.orc_accumulate_triple.restype = ctypes.c_ubyte
    L.orc_accumulate.argtypes = [_f32, _f32, _f32, _i32, _ci, _f32, _f32, _i32, _f32, _f32,
                                 _i32, _vp, _f32, _ci]
    L.orc_accumulate.restype = ctypes.c_ubyte
    L.orc_fused_warp_batch.argtypes = [_f32, _f32, _f32, _f32, _f32, _f32, _ci, _ci, _ci, _ci,
                                       _ci, _f32, _f32, _ci, _ci, _ci, _ci]
    L.orc_kspace_lm_fit_batch.argtypes = [_f64, _f64, _f64, _u8, _vp, _ci, _ci, _ci, _ci, _ci,
                                          _f64, _i32, _f64, _f64, _f64, _f64, _f64, _f64, _i32,
                                          _i32, _u8, _ci]
    L.orc_kspace_fft2_centered.argtypes = [_f64, _ci, _ci, _f64, _f64]
    L.orc_fminvec.argtypes = [_f32, _ci]
    L.orc_fminvec.restype = ctypes.c_float
    L.orc_fmaxvec.argtypes = [_f32, _ci]
    L.orc_fmaxvec.restype = ctypes.c_float
    _lib = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data


def ref_peakfit() -> ctypes.CDLL | None:
    """The reference's own fitter compiled from source, or None if not built here."""
    if not os.path.isfile(REF_PEAKFIT):
        return None
    L = ctypes.CDLL(REF_PEAKFIT)
    L.lsqpeaklocate_lm.argtypes = [_f32, _i32, _f32, _ci, _ci, _f32, _vp]
    L.lsqpeaklocate_lm.restype = None
    L.lsqpeaklocate_lm_batch.argtypes = [_f32, _ci, _i32, _ci, _f32, _f32, _vp]
    L.lsqpeaklocate_lm_batch.restype = None
    L.peak_detectability.argtypes = [_f32, _i32]
    L.peak_detectability.restype = ctypes.c_float
    L.peakfit_batch_lanes.restype = ctypes.c_int
    return L


def ref_warp() -> ctypes.CDLL | None:
    if not os.path.isfile(REF_WARP):
        return None
    L = ctypes.CDLL(REF_WARP)
    L.fused_warp_set_impl.argtypes = [_ci]
    L.fused_symmetric_warp_batch.argtypes = [_f32, _f32, _f32, _f32, _f32, _f32, _ci, _ci,
                                             _ci, _ci, _ci, _f32, _f32, _ci, _ci, _ci]
    L.fused_symmetric_warp_batch.restype = ctypes.c_int
    return L


def ref_bulk() -> ctypes.CDLL | None:
    """The reference's own libbulkxcorr2d (correlator + fitters), or None if not built."""
    if not os.path.isfile(REF_BULK):
        return None
    L = ctypes.CDLL(REF_BULK)
    L.bulkxcorr2d.argtypes = [_f32, _f32, _f32, _i32, _ci, _f32, _f32, _i32, _f32, ctypes.c_bool,
                              _f32, _i32, _ci, _ci, _f32, _f32, _f32, _f32, _f32, _f32, _f32, _vp]
    L.bulkxcorr2d.restype = ctypes.c_ubyte
    L.bulkxcorr2d_accumulate_triple.argtypes = [_f32, _f32, _f32, _i32, _ci, _f32, _f32, _i32,
                                                _f32, _f32, _f32, _f32, _i32, _vp, _ci, _ci,
                                                _f32, _f32, _f32]
    L.bulkxcorr2d_accumulate_triple.restype = ctypes.c_ubyte
    L.bulkxcorr2d_set_peakfit_impl.argtypes = [_ci]
    L.bulkxcorr2d_set_peakfit_impl.restype = ctypes.c_int
    return L


def ref_kspace() -> ctypes.CDLL | None:
    """The reference's own libkspacefit, or None if not built."""
    if not os.path.isfile(REF_KSPACE):
        return None
    L = ctypes.CDLL(REF_KSPACE)
    L.kspace_lm_fit_batch.argtypes = [_f64, _f64, _f64, _u8, _vp, _ci, _ci, _ci, _ci, _ci, _ci,
                                      _f64, _i32, _f64, _f64, _f64, _f64, _f64, _f64, _i32,
                                      _i32, _u8]
    L.kspace_lm_fit_batch.restype = ctypes.c_int
    return L


def ref_bulkxcorr2d(A, B, mask, ctr_x, ctr_y, win_size, weight_a, weight_b, n_peaks=1,
                    peak_finder=3, ensemble=False, want_planes=False, peakfit_impl=0):
    """The reference's compiled bulkxcorr2d (PIV_2d_cross_correlate.c:203-397) with
    the output dict of bulkxcorr2d() below; outputs are zero-filled first, as the
    reference's caller does."""
    L = ref_bulk()
    if L is None:
        raise RuntimeError("reference correlator not built (make -C oracle ref)")
    A = np.ascontiguousarray(A, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    if A.ndim == 2:
        A, B = A[None], B[None]
    n, H, W = A.shape
    ny, nx = len(ctr_y), len(ctr_x)
    h, w = win_size
    shp = (n, n_peaks, ny, nx)
    out = {k: np.zeros(shp, np.float32) for k in ("pk_x", "pk_y", "pk_h", "sx", "sy", "sxy")}
    out["pk_ratio"] = np.zeros((n, ny, nx), np.float32)
    planes = np.zeros(n * ny * nx * h * w, np.float32) if want_planes else None
    if L.bulkxcorr2d_set_peakfit_impl(int(peakfit_impl)) != 0:
        raise RuntimeError("reference batch fitter unavailable")
    try:
        e = L.bulkxcorr2d(
            A, B, np.ascontiguousarray(mask, np.float32).ravel(), np.array([H, W], np.int32), n,
            np.ascontiguousarray(ctr_x, np.float32), np.ascontiguousarray(ctr_y, np.float32),
            np.array([ny, nx], np.int32), np.ascontiguousarray(weight_a, np.float32).ravel().copy(),
            bool(ensemble), np.ascontiguousarray(weight_b, np.float32).ravel(),
            np.array([h, w], np.int32), n_peaks, peak_finder, out["pk_x"], out["pk_y"],
            out["pk_h"], out["sx"], out["sy"], out["sxy"], out["pk_ratio"], _ptr(planes))
    finally:
        L.bulkxcorr2d_set_peakfit_impl(0)
    out["error"] = int(e)
    if planes is not None:
        out["planes"] = planes.reshape(n, ny, nx, h, w)
    return out


def ref_accumulate_triple(A, B, mask, ctr_x, ctr_y, win_size, w_ab_a, w_ab_b, w_auto_a,
                          w_auto_b, fit_size=None, mean_subtract=0, per_pair_norm=0):
    """The reference's compiled bulkxcorr2d_accumulate_triple
    (PIV_2d_cross_correlate.c:627-833) into zeroed sums; returns [AB, AA, BB]."""
    L = ref_bulk()
    if L is None:
        raise RuntimeError("reference correlator not built (make -C oracle ref)")
    A = np.ascontiguousarray(A, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    n, H, W = A.shape
    ny, nx = len(ctr_y), len(ctr_x)
    oh, ow = fit_size if fit_size is not None else win_size
    sums = [np.zeros(ny * nx * oh * ow, np.float32) for _ in range(3)]
    fs = None if fit_size is None else np.array(fit_size, np.int32)
    e = L.bulkxcorr2d_accumulate_triple(
        A, B, np.ascontiguousarray(mask, np.float32).ravel(), np.array([H, W], np.int32), n,
        np.ascontiguousarray(ctr_x, np.float32), np.ascontiguousarray(ctr_y, np.float32),
        np.array([ny, nx], np.int32), *[np.ascontiguousarray(x, np.float32).ravel() for x in
                                        (w_ab_a, w_ab_b, w_auto_a, w_auto_b)],
        np.array(win_size, np.int32), _ptr(fs), mean_subtract, per_pair_norm, *sums)
    if e:
        raise ValueError(f"reference accumulate_triple error {e}")
    return [s.reshape(ny, nx, oh, ow) for s in sums]


def ref_kspace_fit(R_AA, R_BB, R_AB, mask, corr_size, use_kx4=0, use_ky4=0, P_win=None,
                   n_threads=0):
    """The reference's compiled kspace_lm_fit_batch (kspace_lm_fit.c:669-884) with the
    output dict of kspace_fit() below."""
    L = ref_kspace()
    if L is None:
        raise RuntimeError("reference k-space fitter not built (make -C oracle ref)")
    h, w = corr_size
    R_AA = np.ascontiguousarray(R_AA, np.float64).ravel()
    R_BB = np.ascontiguousarray(R_BB, np.float64).ravel()
    R_AB = np.ascontiguousarray(R_AB, np.float64).ravel()
    n = R_AA.size // (h * w)
    m = np.ascontiguousarray(mask, np.uint8).ravel()
    P = None if P_win is None else np.ascontiguousarray(P_win, np.float64).ravel()
    o = dict(gauss_flat=np.zeros((n, 16)), status=np.zeros(n, np.int32),
             initial_guess=np.zeros((n, 16)), gain=np.zeros(n), N0=np.zeros(n),
             b4x=np.zeros(n), b4y=np.zeros(n), cost_per_pt=np.zeros(n),
             n_valid=np.zeros(n, np.int32), iters=np.zeros(n, np.int32),
             conv=np.zeros(n, np.uint8))
    r = L.kspace_lm_fit_batch(R_AA, R_BB, R_AB, m, _ptr(P), n, h, w, use_kx4, use_ky4, n_threads,
                              o["gauss_flat"], o["status"], o["initial_guess"], o["gain"],
                              o["N0"], o["b4x"], o["b4y"], o["cost_per_pt"], o["n_valid"],
                              o["iters"], o["conv"])
    o["ret"] = int(r)
    return o


# --------------------------------------------------------------------------- #
# numpy-facing helpers                                                         #
# --------------------------------------------------------------------------- #

def xcorr_plane(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    out = np.zeros(a.shape, np.float64)
    e = lib().orc_xcorr_plane(a, b, a.shape[0], a.shape[1], out)
    if e:
        raise ValueError(f"orc_xcorr_plane error {e}")
    return out


def correl_weight(w: np.ndarray) -> np.ndarray:
    w = np.ascontiguousarray(w, np.float32)
    out = np.zeros(w.shape, np.float32)
    if lib().orc_correl_weight(w, w.shape[0], w.shape[1], out):
        raise ValueError("orc_correl_weight failed")
    return out


def peakfit(plane, fit_type, n_peaks=1, weight=None, exp_mode=0):
    plane = np.ascontiguousarray(plane, np.float32)
    N = np.array(plane.shape, np.int32)
    loc = np.zeros(3 * n_peaks, np.float32)
    sd = np.zeros(3 * n_peaks, np.float32)
    w = None if weight is None else np.ascontiguousarray(weight, np.float32)
    lib().orc_lsqpeaklocate_lm(plane, N, loc, n_peaks, fit_type, sd, _ptr(w), exp_mode)
    return loc, sd


def detectability(plane) -> float:
    plane = np.ascontiguousarray(plane, np.float32)
    return float(lib().orc_peak_detectability(plane, np.array(plane.shape, np.int32)))


def bulkxcorr2d(A, B, mask, ctr_x, ctr_y, win_size, weight_a, weight_b, n_peaks=1,
                peak_finder=3, ensemble=False, want_planes=False, want_f64=False,
                peakfit_impl=0, n_threads=0):
    """Run the oracle bulkxcorr2d; returns a dict of outputs (numpy)."""
    A = np.ascontiguousarray(A, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    if A.ndim == 2:
        A, B = A[None], B[None]
    n, H, W = A.shape
    ny, nx = len(ctr_y), len(ctr_x)
    nwt = ny * nx
    h, w = win_size
    shp = (n, n_peaks, ny, nx)
    out = {k: np.zeros(shp, np.float32) for k in ("pk_x", "pk_y", "pk_h", "sx", "sy", "sxy")}
    out["pk_ratio"] = np.zeros((n, ny, nx), np.float32)
    planes = np.zeros(n * nwt * h * w, np.float32) if want_planes else None
    planes64 = np.zeros(n * nwt * h * w, np.float64) if want_f64 else None
    e = lib().orc_bulkxcorr2d(
        A, B, np.ascontiguousarray(mask, np.float32).ravel(), np.array([H, W], np.int32), n,
        np.ascontiguousarray(ctr_x, np.float32), np.ascontiguousarray(ctr_y, np.float32),
        np.array([ny, nx], np.int32), np.ascontiguousarray(weight_a, np.float32).ravel(),
        int(bool(ensemble)), np.ascontiguousarray(weight_b, np.float32).ravel(),
        np.array([h, w], np.int32), n_peaks, peak_finder, out["pk_x"], out["pk_y"],
        out["pk_h"], out["sx"], out["sy"], out["sxy"], out["pk_ratio"], _ptr(planes),
        _ptr(planes64), peakfit_impl, n_threads)
    out["error"] = int(e)
    if planes is not None:
        out["planes"] = planes.reshape(n, ny, nx, h, w)
    if planes64 is not None:
        out["planes_f64"] = planes64.reshape(n, ny, nx, h, w)
    return out


def accumulate_triple(A, B, mask, ctr_x, ctr_y, win_size, w_ab_a, w_ab_b, w_auto_a,
                      w_auto_b, fit_size=None, mean_subtract=0, per_pair_norm=0,
                      n_threads=0):
    A = np.ascontiguousarray(A, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    n, H, W = A.shape
    ny, nx = len(ctr_y), len(ctr_x)
    oh, ow = fit_size if fit_size is not None else win_size
    sums = [np.zeros(ny * nx * oh * ow, np.float32) for _ in range(3)]
    fs = None if fit_size is None else np.array(fit_size, np.int32)
    e = lib().orc_accumulate_triple(
        A, B, np.ascontiguousarray(mask, np.float32).ravel(), np.array([H, W], np.int32), n,
        np.ascontiguousarray(ctr_x, np.float32), np.ascontiguousarray(ctr_y, np.float32),
        np.array([ny, nx], np.int32), *[np.ascontiguousarray(x, np.float32).ravel() for x in
                                        (w_ab_a, w_ab_b, w_auto_a, w_auto_b)],
        np.array(win_size, np.int32), _ptr(fs), mean_subtract, per_pair_norm, *sums, n_threads)
    if e:
        raise ValueError(f"orc_accumulate_triple error {e}")
    return [s.reshape(ny, nx, oh, ow) for s in sums]


def fused_warp_batch(imgs_a, imgs_b, pred_dy, pred_dx, ctrs_y, ctrs_x, interp_mode=0,
                     shared_predictor=0, round_shifts=0, n_threads=0):
    imgs_a = np.ascontiguousarray(imgs_a, np.float32)
    imgs_b = np.ascontiguousarray(imgs_b, np.float32)
    N, H, W = imgs_a.shape
    pred_dy = np.ascontiguousarray(pred_dy, np.float32)
    pred_dx = np.ascontiguousarray(pred_dx, np.float32)
    nPY, nPX = pred_dy.shape[-2:]
    oa = np.zeros_like(imgs_a)
    ob = np.zeros_like(imgs_b)
    r = lib().orc_fused_warp_batch(imgs_a, imgs_b, oa, ob, pred_dy, pred_dx, N, H, W, nPY, nPX,
                                   np.ascontiguousarray(ctrs_y, np.float32),
                                   np.ascontiguousarray(ctrs_x, np.float32), interp_mode,
                                   shared_predictor, round_shifts, n_threads)
    if r:
        raise ValueError("orc_fused_warp_batch failed")
    return oa, ob


def kspace_fit(R_AA, R_BB, R_AB, mask, corr_size, use_kx4=0, use_ky4=0, P_win=None,
               n_threads=0):
    h, w = corr_size
    R_AA = np.ascontiguousarray(R_AA, np.float64).ravel()
    R_BB = np.ascontiguousarray(R_BB, np.float64).ravel()
    R_AB = np.ascontiguousarray(R_AB, np.float64).ravel()
    n = R_AA.size // (h * w)
    m = np.ascontiguousarray(mask, np.uint8).ravel()
    P = None if P_win is None else np.ascontiguousarray(P_win, np.float64).ravel()
    o = dict(gauss_flat=np.zeros((n, 16)), status=np.zeros(n, np.int32),
             initial_guess=np.zeros((n, 16)), gain=np.zeros(n), N0=np.zeros(n),
             b4x=np.zeros(n), b4y=np.zeros(n), cost_per_pt=np.zeros(n),
             n_valid=np.zeros(n, np.int32), iters=np.zeros(n, np.int32),
             conv=np.zeros(n, np.uint8))
    r = lib().orc_kspace_lm_fit_batch(R_AA, R_BB, R_AB, m, _ptr(P), n, h, w, use_kx4, use_ky4,
                                      o["gauss_flat"], o["status"], o["initial_guess"],
                                      o["gain"], o["N0"], o["b4x"], o["b4y"], o["cost_per_pt"],
                                      o["n_valid"], o["iters"], o["conv"], n_threads)
    o["ret"] = int(r)
    return o


# ---------------------------------------------------------------------------
# Ensemble finalise (pivtools_cli/piv/piv_backend/single_pass_accumulator.py)
# ---------------------------------------------------------------------------

def pair_envelope(wa, wb, corr_size):
    """Linear pair-count envelope E(s) = sum_x wa(x + s) wb(x), centre-cropped to
    corr_size with zero lag at corr_size // 2 and normalised to 1 there
    (single_pass_accumulator.py:52-102), by direct summation in FP64."""
    wa = np.asarray(wa, np.float64)
    wb = np.asarray(wb, np.float64)
    h, w = wa.shape
    ch, cw = corr_size
    env = np.zeros((ch, cw))
    for i in range(ch):
        for j in range(cw):
            sy, sx = i - ch // 2, j - cw // 2
            y0, y1 = max(0, -sy), min(h, h - sy)
            x0, x1 = max(0, -sx), min(w, w - sx)
            if y1 > y0 and x1 > x0:
                env[i, j] = np.sum(wa[y0 + sy:y1 + sy, x0 + sx:x1 + sx] * wb[y0:y1, x0:x1])
    return env / env[ch // 2, cw // 2]


def zero_plane_means(planes):
    """Subtract each window's plane mean (single_pass_accumulator.py:105-123);
    planes (n, h, w) float32."""
    p = np.asarray(planes, np.float32)
    return p - p.mean(axis=(1, 2), keepdims=True, dtype=np.float64).astype(np.float32)


def ensemble_finalize(sum_ab, sum_aa, sum_bb, n_pairs, bg=None, dc_zero=False, env_auto=None, env_ab=None,
                      ab_scale=None):
    """Averaged, background-subtracted, optionally DC-zeroed and envelope-divided,
    normalised ensemble planes, in float32 as the reference computes them
    (single_pass_accumulator.py:564-800): R = sum / N - bg; R -= mean; R /= E;
    single mode: R_AB *= sum area / particle area (ab_scale, :760-780);
    R /= sqrt(max(AA_c * BB_c, 1e-12)).  Inputs (n, h, w); returns
    (R_AA, R_BB, R_AB, norm)."""
    n = np.float32(n_pairs)
    R = [np.asarray(s, np.float32) / n for s in (sum_aa, sum_bb, sum_ab)]
    if bg is not None:
        bg_aa, bg_bb, bg_ab = bg
        R = [r - np.asarray(b, np.float32) for r, b in zip(R, (bg_aa, bg_bb, bg_ab))]
    if dc_zero:
        R = [zero_plane_means(r) for r in R]
    if env_auto is not None:
        ea = np.asarray(env_auto, np.float32)[None]
        eb = np.asarray(env_ab if env_ab is not None else env_auto, np.float32)[None]
        R = [R[0] / ea, R[1] / ea, R[2] / eb]
    h, w = R[0].shape[1:]
    c = (h // 2, w // 2)
    norm = np.sqrt(np.maximum(R[0][:, c[0], c[1]] * R[1][:, c[0], c[1]], np.float32(1e-12)))
    if ab_scale is not None:
        R[2] = R[2] * np.float32(ab_scale)
    R = [r / norm[:, None, None] for r in R]
    return R[0], R[1], R[2], norm


def image_method_means(batches_a, batches_b):
    """Phase A of the two-sweep 'image' background methods: the float32 frame sums
    of each batch (numpy sum over the pair axis, cpu_ensemble.py:1176-1177), summed
    across batches in float32 (dask_pipeline.py:1028-1033, 806-830), divided by the
    pair count and cast to float32 (pivtools_core/ensemble.py:199-200)."""
    tot, n = [None, None], 0
    for A, B in zip(batches_a, batches_b):
        for k, F in enumerate((A, B)):
            s = np.asarray(F, np.float32).sum(axis=0)
            tot[k] = s.copy() if tot[k] is None else tot[k] + s
        n += np.asarray(A).shape[0]
    return (tot[0] / n).astype(np.float32), (tot[1] / n).astype(np.float32)


def center_frames(frames, mean):
    """Phase B's `images -= A_mean` in float32 (cpu_ensemble.py:1290-1291)."""
    return np.asarray(frames, np.float32) - np.asarray(mean, np.float32)[None]


# ---------------------------------------------------------------------------
# Camera payload decode (pivtools_core/image_handling/readers/pivraw_reader.py:896-960,
# set_reader.py:1296-1345)
# ---------------------------------------------------------------------------

def decode_frames(raw, stride, n_frames, first_index, width, height, fmt, dark=None, dark_frames=2, rot=0):
    """Payloads (uint8, frame k at k * stride) -> float32 frames: Mono12p unpack
    (fmt 0) or the BayerRG8 mosaic (fmt 1), optional dark max(f, d) - d in the
    sensor type (odd 1-based indices take dark A, even dark B when dark_frames is
    2), the Bayer 2x2 superpixel sum, then np.rot90(., rot)."""
    raw = np.asarray(raw, np.uint8)
    npx = width * height

    def sensor(buf, k):
        if fmt == 0:
            b = buf[k * stride:k * stride + npx // 2 * 3].reshape(-1, 3).astype(np.uint16)
            p = np.empty((b.shape[0], 2), np.uint16)
            p[:, 0] = b[:, 0] | ((b[:, 1] & 0x0F) << 8)
            p[:, 1] = (b[:, 1] >> 4) | (b[:, 2] << 4)
            return p.reshape(height, width)
        return buf[k * stride:k * stride + npx].reshape(height, width).copy()

    out = []
    for k in range(n_frames):
        f = sensor(raw, k)
        if dark is not None:
            role = (first_index + k - 1) % 2 if dark_frames == 2 else 0
            d = sensor(np.asarray(dark, np.uint8), role)
            f = np.maximum(f, d) - d
        if fmt == 0:
            img = f.astype(np.float32)
        else:
            img = f.reshape(height // 2, 2, width // 2, 2).astype(np.float32).sum(axis=(1, 3))
        out.append(np.rot90(img, rot).astype(np.float32))
    return np.stack(out)


# ---------------------------------------------------------------------------
# Inter-pass outlier tests (pivtools_cli/piv/piv_backend/outlier_detection.py)
# ---------------------------------------------------------------------------

def median_outlier(ux, uy, eps=0.1, thr=2.0, size=5, masked=None):
    """Normalised median, vector-norm form (outlier_detection.py:87-243): the
    size x size neighbourhood without the node (grid edge and masked nodes
    excluded), residual norm over the median of the neighbour residual norms plus
    eps, non-finite residual flagged; 3x3 guard counting finite or masked cells
    (fewer than 6 flags); masked nodes never flagged."""
    ux = np.asarray(ux, np.float32)
    uy = np.asarray(uy, np.float32)
    ny, nx = ux.shape
    if masked is not None:
        masked = np.asarray(masked, bool)
        ux = np.where(masked, np.float32(np.nan), ux)
        uy = np.where(masked, np.float32(np.nan), uy)
    h = size // 2
    pu = np.pad(ux, h, constant_values=np.nan)
    pv = np.pad(uy, h, constant_values=np.nan)
    out = np.zeros((ny, nx), bool)
    with np.errstate(all="ignore"):
        for r in range(ny):
            for c in range(nx):
                wu = pu[r:r + size, c:c + size].ravel()
                wv = pv[r:r + size, c:c + size].ravel()
                k = size * size // 2
                nu = np.delete(wu, k)
                nv = np.delete(wv, k)
                if np.all(np.isnan(nu)):
                    mu = mv = np.nan
                else:
                    mu, mv = np.float32(np.nanmedian(nu)), np.float32(np.nanmedian(nv))
                r0 = np.sqrt((ux[r, c] - mu) ** 2 + (uy[r, c] - mv) ** 2)
                ri = np.sqrt((nu - mu) ** 2 + (nv - mv) ** 2)
                rm = np.float32(np.nanmedian(ri)) if np.any(np.isfinite(ri)) else np.nan
                nr = r0 / (rm + np.float32(eps))
                out[r, c] = (not np.isfinite(nr)) or nr > thr
        present = np.isfinite(ux) & np.isfinite(uy)
        if masked is not None:
            present |= masked
        pp = np.pad(present.astype(np.int32), 1)
        n_present = sum(pp[1 + dr:1 + dr + ny, 1 + dc:1 + dc + nx] for dr in (-1, 0, 1) for dc in (-1, 0, 1))
        out |= n_present < 6
        if masked is not None:
            out &= ~masked
    return out


NAN_MASKED, NAN_VALID, NAN_FIT_FAIL, NAN_LARGE_DISP = -1, 0, 1, 6
NAN_UNCLASSIFIED, NAN_OUTLIER, NAN_PEAK_MAG_NAN = 9, 10, 13


def pass_validation(pk_x, pk_y, pk_h, pred_dy, pred_dx, masked, thresh_x, thresh_y, peak_thr=0.25,
                    med_eps=0.1, med_thr=2.0, med_size=5):
    """One pass's validation of the primary peak for one pair, as the reference
    driver runs it (cpu_instantaneous.py:575-760; single peak, no secondary-peak
    substitution): masked windows and displacements beyond the gate are NaN-ed,
    the predictor is added, the failed vectors enter the peak-magnitude and
    normalised-median tests as zeros (outlier_detection.py:56-85, :87-243), NaN
    peak heights fail, and each invalid vector gets the reason code of the first
    stage that claimed it (nan_reason_codes.py:18-25).
    Returns (ux, uy, nan_mask, nan_reason): ux/uy NaN where invalid, 0 at masked."""
    x = np.asarray(pk_x, np.float32).copy()
    y = np.asarray(pk_y, np.float32).copy()
    h = np.asarray(pk_h, np.float32).copy()
    ny, nx = x.shape
    m = np.zeros((ny, nx), bool) if masked is None else np.asarray(masked, bool)
    with np.errstate(invalid="ignore"):
        large = (np.abs(x) > thresh_x) | (np.abs(y) > thresh_y)
    fit_fail = np.isnan(x) | np.isnan(y)
    gone = m | large
    x[gone] = np.nan
    y[gone] = np.nan
    h[gone] = np.nan
    if pred_dx is not None:
        x = x + np.asarray(pred_dx, np.float32)
        y = y + np.asarray(pred_dy, np.float32)
    nan_mask = np.isnan(x) | np.isnan(y) | m
    zx, zy = np.where(nan_mask, np.float32(0), x), np.where(nan_mask, np.float32(0), y)
    reason = np.zeros((ny, nx), np.int8)
    reason[fit_fail] = NAN_FIT_FAIL
    reason[large] = NAN_LARGE_DISP
    outlier = np.zeros((ny, nx), bool)
    with np.errstate(invalid="ignore"):
        if peak_thr >= 0:
            outlier |= (h < peak_thr) | np.isnan(h)
    if med_thr > 0:
        outlier |= median_outlier(zx, zy, med_eps, med_thr, med_size, masked=m if masked is not None else None)
    outlier &= ~m
    nan_mask |= outlier
    reason[outlier & (reason == NAN_VALID)] = NAN_OUTLIER
    nan_mask |= np.isnan(h)
    reason[np.isnan(h) & (reason == NAN_VALID)] = NAN_PEAK_MAG_NAN
    reason[nan_mask & (reason == NAN_VALID)] = NAN_UNCLASSIFIED
    reason[m] = NAN_MASKED
    ux = np.where(nan_mask, np.float32(np.nan), zx).astype(np.float32)
    uy = np.where(nan_mask, np.float32(np.nan), zy).astype(np.float32)
    ux[m] = 0.0
    uy[m] = 0.0
    return ux, uy, nan_mask, reason


# ---------------------------------------------------------------------------
# Coloured-floor lookup (pivtools_cli/piv/piv_backend/kspace_floor_psd.py:241-275)
# ---------------------------------------------------------------------------

def floor_fractions(pred):
    """|x - round(x)| of x = pred / 2 in float32 (interpolation_noise_psd.py:191-204,
    single_pass_accumulator.py:852-853)."""
    x = np.asarray(pred, np.float32) / np.float32(2.0)
    return np.abs(x - np.round(x))


def floor_interp(fs, P_grid, fx, fy):
    """Bilinear lookup of P_grid (nf, nf, h, w) [iy, ix] at per-window fractions,
    rounded through float32 as the driver stores it: (n, h*w)."""
    fx = np.asarray(fx, np.float64).ravel()
    fy = np.asarray(fy, np.float64).ravel()
    nf = len(fs)
    ix = np.clip(np.searchsorted(fs, fx) - 1, 0, nf - 2)
    iy = np.clip(np.searchsorted(fs, fy) - 1, 0, nf - 2)
    tx = np.clip((fx - fs[ix]) / (fs[ix + 1] - fs[ix]), 0.0, 1.0)
    ty = np.clip((fy - fs[iy]) / (fs[iy + 1] - fs[iy]), 0.0, 1.0)
    Pf = np.asarray(P_grid, np.float64).reshape(nf, nf, -1)
    out = (((1.0 - ty) * (1.0 - tx))[:, None] * Pf[iy, ix] + ((1.0 - ty) * tx)[:, None] * Pf[iy, ix + 1]
           + (ty * (1.0 - tx))[:, None] * Pf[iy + 1, ix] + (ty * tx)[:, None] * Pf[iy + 1, ix + 1])
    return out.astype(np.float32)
