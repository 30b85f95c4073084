"""Host-side interface of the correlation path.

`bulkxcorr2d` mirrors the reference driver's call of libbulkxcorr2d
(pivtools_cli/piv/piv_backend/cpu_instantaneous.py:505-555 and
_set_lib_arguments :1166-1280): the same arrays, the same output shapes
(N, nPeaks, nWinY, nWinX) and the same error-code handling.  `xcorr_device`
is the resident form: torch tensors on the GPU, no host copies.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

ERROR_NAMES = {
    1: "ERROR_NOMEM (out of memory)",
    2: "ERROR_NOPLAN_FWD (FFT forward plan failed)",
    4: "ERROR_NOPLAN_BWD (FFT backward plan failed)",
    8: "ERROR_NOPLAN (general plan error)",
    9: "ERROR_OUT_OF_BOUNDS (array access out of bounds)",
    16: "ERROR_CUDA (CUDA runtime failure)",
}


def _check(code: int, what: str = "bulkxcorr2d") -> None:
    if code != 0:
        raise RuntimeError(f"{what} failed with error {code}: {ERROR_NAMES.get(code, 'unknown')}")


def set_peakfit_impl(impl: str | int) -> None:
    """'scalar' (0) or 'batch' (1) peak-fit semantics (cpu_instantaneous.py:259-283)."""
    v = {"scalar": 0, "batch": 1}.get(impl, impl)
    if _lib.bulkxcorr2d_lib().bulkxcorr2d_set_peakfit_impl(int(v)) != 0:
        raise RuntimeError("peak_fit_impl selection refused")


def bulkxcorr2d(images_a, images_b, win_ctrs_x, win_ctrs_y, window_size, weight_a, weight_b=None,
                mask=None, n_peaks=1, peak_finder=3, ensemble=False, dump_planes=False):
    """Correlate N image pairs on the GPU; returns a dict of host arrays.

    images_*: (N, H, W) or (H, W) float32.  Output keys pk_loc_x, pk_loc_y,
    pk_height, sx, sy, sxy with shape (N, n_peaks, ny, nx), pk_ratio (N, ny, nx)
    and, with dump_planes, planes (N, ny, nx, h, w).
    """
    L = _lib.bulkxcorr2d_lib()
    A = np.ascontiguousarray(images_a, np.float32)
    B = np.ascontiguousarray(images_b, np.float32)
    if A.ndim == 2:
        A, B = A[None], B[None]
    N, H, W = A.shape
    cx = np.ascontiguousarray(win_ctrs_x, np.float32)
    cy = np.ascontiguousarray(win_ctrs_y, np.float32)
    ny, nx = len(cy), len(cx)
    h, w = window_size
    wa = np.ascontiguousarray(weight_a, np.float32)
    wb = wa if weight_b is None else np.ascontiguousarray(weight_b, np.float32)
    m = np.zeros((ny, nx), np.float32) if mask is None else np.ascontiguousarray(mask, np.float32)
    shape = (N, n_peaks, ny, nx)
    out = {k: np.zeros(shape, np.float32) for k in ("pk_loc_x", "pk_loc_y", "pk_height", "sx", "sy", "sxy")}
    out["pk_ratio"] = np.zeros((N, ny, nx), np.float32)
    planes = np.zeros(N * ny * nx * h * w, np.float32) if dump_planes else None
    code = L.bulkxcorr2d(A, B, m, np.array([H, W], np.int32), N, cx, cy, np.array([ny, nx], np.int32),
                         wa, bool(ensemble), wb, np.array([h, w], np.int32), int(n_peaks), int(peak_finder),
                         out["pk_loc_x"], out["pk_loc_y"], out["pk_height"], out["sx"], out["sy"],
                         out["sxy"], out["pk_ratio"],
                         None if planes is None else ctypes.c_void_p(planes.ctypes.data))
    _check(int(code))
    if planes is not None:
        out["planes"] = planes.reshape(N, ny, nx, h, w)
    return out


class DeviceCorrelator:
    """Resident correlation on torch CUDA tensors (one window size per call).

    Keeps the correlation weight of each (weight, size) on the device and a
    scratch buffer for deferred LM fits; launches on torch's current stream.
    """

    def __init__(self, device=None):
        import torch

        self.torch = torch
        self.device = torch.device("cuda" if device is None else device)
        self.L = _lib.bulkxcorr2d_lib()
        self._scratch = None
        self._cw = {}

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def correl_weight(self, weight_b):
        torch = self.torch
        key = (weight_b.data_ptr(), tuple(weight_b.shape))
        cw = self._cw.get(key)
        if cw is None:
            cw = torch.empty_like(weight_b)
            h, w = weight_b.shape
            _check(self.L.pivb_correl_weight_dev(weight_b.data_ptr(), h, w, cw.data_ptr(), self._stream()),
                   "pivb_correl_weight_dev")
            self._cw[key] = (cw, weight_b)   # keep weight alive: the key is its address
            return cw
        return cw[0]

    def scratch(self, nbytes: int):
        torch = self.torch
        if nbytes == 0:
            return None
        if self._scratch is None or self._scratch.numel() < nbytes:
            self._scratch = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        return self._scratch

    def run(self, A, B, ctr_x, ctr_y, weight_a, weight_b, out, mask=None, n_peaks=1, peak_finder=3,
            peakfit_impl=0, ensemble=False, planes=None, img_stride=None):
        """A, B: (N, H, W) float32 CUDA tensors (frames may be views with a common
        stride).  out: dict of preallocated CUDA tensors pk_loc_x ... pk_ratio."""
        N, H, W = A.shape
        ny, nx = ctr_y.numel(), ctr_x.numel()
        h, w = weight_a.shape
        cw = self.correl_weight(weight_b)
        total = N * ny * nx
        nbytes = int(self.L.pivb_xcorr_scratch_bytes_hw(total, h, w, n_peaks, peak_finder))
        scr = self.scratch(nbytes)
        stride = A.stride(0) if img_stride is None else img_stride
        code = self.L.pivb_xcorr_dev(
            A.data_ptr(), B.data_ptr(), stride, None if mask is None else mask.data_ptr(), H, W, N,
            ctr_x.data_ptr(), ctr_y.data_ptr(), ny, nx, weight_a.data_ptr(), weight_b.data_ptr(),
            cw.data_ptr(), h, w, int(ensemble), n_peaks, peak_finder, peakfit_impl,
            out["pk_loc_x"].data_ptr(), out["pk_loc_y"].data_ptr(), out["pk_height"].data_ptr(),
            out["sx"].data_ptr(), out["sy"].data_ptr(), out["sxy"].data_ptr(), out["pk_ratio"].data_ptr(),
            None if planes is None else planes.data_ptr(), None if scr is None else scr.data_ptr(),
            nbytes, self._stream())
        _check(int(code), "pivb_xcorr_dev")
