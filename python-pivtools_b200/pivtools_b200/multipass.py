"""GPU-resident multipass window-deformation PIV (instantaneous mode).

Follows the pass loop of the reference driver
(pivtools_cli/piv/piv_backend/cpu_instantaneous.py:381-927, :995-1133) for a
batch of N image pairs kept on the device:

  pass 0      correlate the raw frames;
  pass k > 0  remap the (smoothed, padded) predictor of pass k-1 to this pass's
              window centres, warp both frames symmetrically by it, correlate;
  every pass  gate large displacements (win/2 on pass 0, win/4 after), add the
              predictor, reject peak-magnitude and normalised-median outliers,
              infill, then (not on the last pass) pad onto the padded grid and
              smooth -- the predictor of the next pass.

Every step is a CUDA kernel launched on the caller's stream with no host
synchronisation, so a whole batch step can be captured as one CUDA graph.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib, geometry


@dataclass
class MultipassConfig:
    window_sizes: list = field(default_factory=lambda: [(128, 128), (64, 64), (32, 32), (32, 32)])
    overlaps: list = field(default_factory=lambda: [50, 50, 50, 75])
    window_type: str = "gaussian"
    peak_finder: int = 3
    peakfit_impl: int = 0
    interp_mode: int = 0            # 0 bicubic, 1 Lanczos-3
    warp_impl: int = 1
    predictor_smoothing: bool = True
    peak_mag_threshold: float = 0.25
    median_epsilon: float = 0.1
    median_threshold: float = 2.0
    median_size: int = 5
    infill: str = "biharmonic"      # infill between passes and after the last: least squares
                                    # "biharmonic" (the reference's default) or "harmonic", or "nearest"
    infill_max_iter: int = 2000     # conjugate-gradient iteration cap (exact solves need far fewer)
    infill_tol: float = 1e-12       # relative residual of the FP64 normal equations
    final_infill: bool = True
    predictor_fill: str = "harmonic"  # masked windows in the predictor: "harmonic", "nearest" or "none" (kept at 0)
    engine_32: str = "fft"          # 32 px passes: "fft" (FP32 FFT) or "dft" (tensor-core DFT-as-GEMM)
    sigma_threshold: float = 0.0    # > 0: the reference's `sigma` outlier method with this threshold
    div_vort: bool = False          # the reference's `div_vort` outlier method
    div_thresh: float | None = None  # its thresholds (None: 6 x 1.4826 x MAD of each pair's field)
    vort_thresh: float | None = None
    n_peaks: int = 1                # correlation peaks per window (the reference's num_peaks)
    secondary_peak: bool = False    # substitute the next peak for an invalid vector (needs n_peaks > 1)


def _gauss_taps(sigma: float, ksize: int):
    """Normalised taps of scipy.ndimage.gaussian_filter with truncate =
    (ksize-1)/(2 sigma) (cpu_instantaneous.py:1042-1048)."""
    if sigma <= 0:
        return np.ones(1, np.float32), 0
    truncate = (ksize - 1) / (2 * sigma)
    radius = int(truncate * sigma + 0.5)
    x = np.arange(-radius, radius + 1, dtype=np.float64)
    w = np.exp(-0.5 * (x / sigma) ** 2)
    return (w / w.sum()).astype(np.float32), radius


class MultipassPIV:
    """Multipass PIV for batches of N pairs of one image size on one GPU."""

    def __init__(self, image_shape, n_pairs: int, cfg: MultipassConfig | None = None, device=None,
                 vector_masks=None):
        """vector_masks: per-pass boolean (n_win_y, n_win_x) masked-window flags
        (geometry.compute_vector_masks), or None: masked windows are skipped by the
        correlator, stored as 0 with reason -1, never infill donors, and filled in
        the predictor (cpu_instantaneous.py:586-600, :836-850)."""
        import torch

        self.torch = torch
        self.cfg = cfg or MultipassConfig()
        self.device = torch.device("cuda" if device is None else device)
        self.H, self.W = image_shape
        self.N = n_pairs
        self.geo = geometry.multipass_geometry(image_shape, self.cfg.window_sizes, self.cfg.overlaps,
                                               self.cfg.window_type)
        self.Lx = _lib.bulkxcorr2d_lib()
        self.Lw = _lib.fusedwarp_lib()
        self.Lp = _lib.pass_lib()
        if self.cfg.engine_32 not in ("fft", "dft"):
            raise ValueError(f"engine_32 {self.cfg.engine_32!r}")
        if self.cfg.infill not in ("biharmonic", "harmonic", "nearest"):
            raise ValueError(f"infill {self.cfg.infill!r} (valid: 'biharmonic', 'harmonic', 'nearest')")
        self.infill_order = 2 if self.cfg.infill == "biharmonic" else 1
        if self.cfg.predictor_fill not in ("harmonic", "nearest", "none"):
            raise ValueError(f"predictor_fill {self.cfg.predictor_fill!r} (valid: 'harmonic', 'nearest', 'none')")
        if vector_masks is not None and len(vector_masks) != len(self.geo):
            raise ValueError(f"{len(vector_masks)} vector masks for {len(self.geo)} passes")
        P = int(self.cfg.n_peaks)
        if not 1 <= P <= 255:
            raise ValueError(f"n_peaks {P} outside 1..255")
        if P > 1 and self.cfg.engine_32 == "dft":
            raise ValueError("the tensor-core engine returns one peak per window: use engine_32='fft' with n_peaks > 1")
        self.P = P
        # the extended validation entry point: several peaks or further outlier tests
        self.full_validate = P > 1 or self.cfg.sigma_threshold > 0 or self.cfg.div_vort
        self.Ld = _lib.dft_lib() if self.cfg.engine_32 == "dft" else None
        dev, f32 = self.device, torch.float32
        # device status word of the tensor-core engine (1 = an MMA completion was not observed)
        self.dft_status = torch.zeros(1, dtype=torch.int32, device=dev)
        N, H, W = self.N, self.H, self.W
        self.warped = [torch.empty((N, H, W), dtype=f32, device=dev) for _ in range(2)]
        self.passes = []
        max_scratch = 0
        max_vec = 0
        max_pad = 0
        max_infill = 0
        for k, g in enumerate(self.geo):
            ny, nx = g.grid.n_win_y, g.grid.n_win_x
            nyp, nxp = len(g.ctrs_y_all), len(g.ctrs_x_all)
            w = torch.tensor(geometry.window_weight(g.window_size, self.cfg.window_type), device=dev)
            cw = torch.empty_like(w)
            p = dict(
                ny=ny, nx=nx, nyp=nyp, nxp=nxp, win=g.window_size[0], win_h=g.window_size[0],
                win_w=g.window_size[1], weight=w, cw=cw,
                cx=torch.tensor(g.grid.win_ctrs_x, device=dev), cy=torch.tensor(g.grid.win_ctrs_y, device=dev),
                cx_all=torch.tensor(g.ctrs_x_all, device=dev), cy_all=torch.tensor(g.ctrs_y_all, device=dev),
                # zero-filled once: skipped (masked) windows are never written
                out={k2: torch.zeros((N, P, ny, nx), dtype=f32, device=dev)
                     for k2 in ("pk_loc_x", "pk_loc_y", "pk_height", "sx", "sy", "sxy")},
                ratio=torch.zeros((N, ny, nx), dtype=f32, device=dev),
                ux=torch.empty((N, ny, nx), dtype=f32, device=dev),
                uy=torch.empty((N, ny, nx), dtype=f32, device=dev),
                invalid=torch.empty((N, ny, nx), dtype=torch.uint8, device=dev),
                reason=torch.empty((N, ny, nx), dtype=torch.int8, device=dev),
                pdy=torch.empty((N, nyp, nxp), dtype=f32, device=dev),
                pdx=torch.empty((N, nyp, nxp), dtype=f32, device=dev),
                spacing=(float(g.grid.win_spacing_y), float(g.grid.win_spacing_x)),
                pre=g.n_pre,
                # large-displacement gate: half the window on the first pass, a quarter
                # after (cpu_instantaneous.py:575-585), per axis
                thr=(g.window_size[1] / (2.0 if k == 0 else 4.0), g.window_size[0] / (2.0 if k == 0 else 4.0)),
                choice=(torch.empty((N, ny, nx), dtype=torch.uint8, device=dev) if self.full_validate
                        else None),
            )
            bm = None if vector_masks is None else np.asarray(vector_masks[k], bool)
            if bm is not None and bm.shape != (ny, nx):
                raise ValueError(f"pass {k}: vector mask shape {bm.shape} != window grid {(ny, nx)}")
            p["b_mask"] = np.zeros((ny, nx), bool) if bm is None else bm
            p["mask"] = None
            if bm is not None and bm.any():
                if bm.all():
                    raise ValueError(f"pass {k}: every window is masked")
                p["mask"] = torch.tensor(bm.astype(np.float32), device=dev)
                # (a broadcast view's astype keeps its odd strides: materialise C order)
                p["mask_u8"] = torch.tensor(np.ascontiguousarray(np.broadcast_to(bm, (N, ny, nx)), dtype=np.uint8),
                                            device=dev).contiguous()
                if self.cfg.predictor_fill == "nearest":
                    # donor of each masked window, fixed by the mask and the pitch
                    donor = geometry.nearest_donor_map(bm, (g.grid.win_spacing_y, g.grid.win_spacing_x))
                    p["donor"] = torch.tensor(donor.ravel(), dtype=torch.int32, device=dev)
            if k > 0:
                p["map_x"] = torch.tensor(g.pred_map_x, device=dev)
                p["map_y"] = torch.tensor(g.pred_map_y, device=dev)
                p["pred_dy"] = torch.empty((N, ny, nx), dtype=f32, device=dev)
                p["pred_dx"] = torch.empty((N, ny, nx), dtype=f32, device=dev)
            if k + 1 < len(self.geo):
                taps, rad = _gauss_taps(self.geo[k + 1].sd if self.cfg.predictor_smoothing else 0.0,
                                        self.geo[k + 1].ksize_filt[0])
                p["taps"] = torch.tensor(taps, device=dev)
                p["radius"] = rad
            # room for the per-window records, so every single-peak fit (3-point
            # included) runs in the thread-per-window record kernel
            wh, ww = g.window_size
            max_scratch = max(max_scratch,
                              int(self.Lx.pivb_xcorr_scratch_bytes_hw(N * ny * nx, wh, ww, P, self.cfg.peak_finder)),
                              int(self.Lx.pivb_xcorr_record_bytes(N * ny * nx)) if wh == ww else 0)
            max_vec = max(max_vec, N * ny * nx)
            max_pad = max(max_pad, N * nyp * nxp)
            max_infill = max(max_infill, int(self.Lp.pivb_infill_work_bytes(N, ny, nx)))
            self.passes.append(p)
        self.scratch = torch.empty(max(max_scratch, 256), dtype=torch.uint8, device=dev)
        nval = 8 * max_vec + 2 * N if self.full_validate else 2 * max_vec
        self.work = torch.empty(max(nval, max_pad), dtype=f32, device=dev)
        self.infill_work = torch.empty(max(max_infill, 256), dtype=torch.uint8, device=dev)
        # predictor copies with the masked windows filled (the stored field keeps 0 there)
        self.fill = (torch.empty((2, max_vec), dtype=f32, device=dev)
                     if any(self._fills(k) for k in range(len(self.passes))) else None)
        # warp tables per pass (centres of the previous pass's padded grid)
        tb = int(self.Lw.pivb_warp_table_bytes(H, W))
        self.tables = [None] + [torch.empty(tb, dtype=torch.uint8, device=dev) for _ in self.geo[1:]]
        s = self._stream()
        for k in range(1, len(self.geo)):
            prev = self.passes[k - 1]
            self._ok(self.Lw.pivb_warp_setup_dev(prev["cy_all"].data_ptr(), prev["nyp"], prev["cx_all"].data_ptr(),
                                                 prev["nxp"], H, W, self.tables[k].data_ptr(), s), "warp setup")
        for p in self.passes:
            self._ok(self.Lx.pivb_correl_weight_dev(p["weight"].data_ptr(), p["win_h"], p["win_w"], p["cw"].data_ptr(), s),
                     "correlation weight")
        self.launches_per_step = self._count_launches()
        self.planes = None
        self._last_n = self.N
        # the set-up above (zero fills, correlation weights, warp tables) ran on the
        # stream current at construction; finish it before run() is called from
        # any other stream (a serving engine runs on its own)
        torch.cuda.current_stream(self.device).synchronize()

    def keep_planes(self, on: bool = True):
        """Keep every window's correlation plane of every pass on the device (the
        reference's dump_correlation_planes, cpu_instantaneous.py:425-432):
        N x n_windows x win^2 floats per pass, for save_corr_plane_dump."""
        torch = self.torch
        self.planes = None
        if on:
            self.planes = [torch.zeros((self.N, p["ny"], p["nx"], p["win_h"], p["win_w"]), dtype=torch.float32,
                                       device=self.device) for p in self.passes]
            torch.cuda.current_stream(self.device).synchronize()

    # ------------------------------------------------------------------ #
    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    @staticmethod
    def _ok(code, what):
        if code != 0:
            raise RuntimeError(f"{what} failed with code {code}")

    def _fills(self, k):
        return (k + 1 < len(self.passes) and self.passes[k]["mask"] is not None
                and self.cfg.predictor_fill in ("harmonic", "nearest"))

    def _count_launches(self):
        n = 0
        for k in range(len(self.geo)):
            n += 1 if self._fills(k) else 0                  # predictor fill of masked windows
            n += 1                                        # correlation
            n += 1 if (3 <= self.cfg.peak_finder <= 6) else 0  # deferred fit (record kernel)
            n += 2 if self.cfg.median_threshold > 0 else 1  # validate (+ median)
            if self.full_validate:                        # choices, substitution rounds, final
                extra = (1 if self.cfg.sigma_threshold > 0 else 0) + (3 if self.cfg.div_vort else 0)
                n += 2 + (2 * (self.P - 1) if self.cfg.secondary_peak and self.P > 1 else 1) + extra
                if self.cfg.secondary_peak and self.P > 1:
                    n += extra * (self.P - 1)
                if self.cfg.median_threshold <= 0 and extra:
                    n += 1                                # the finalising pass of the median kernel
            if k + 1 < len(self.geo) or self.cfg.final_infill:
                n += 1                                    # infill
            if k + 1 < len(self.geo):
                n += 1 + (4 if self.passes[k]["radius"] > 0 else 0)   # pad (+ smoothing)
            if k > 0:
                n += 2                                    # remap, warp
        return n

    def run(self, A, B, n=None):
        """A, B: (N, H, W) float32 CUDA tensors.  Returns (ux, uy) of the final pass
        (device tensors, views into internal buffers).  n (<= N) processes only the
        first n pairs (a partly filled batch); every pair's result is independent of
        the others in the batch."""
        N = self._batch(n)
        for k in range(len(self.passes)):
            fa, fb = self.stage_pre(k, A, B, N)
            self._correlate(k, fa, fb, N)
            self.stage_post(k, N)
        self._last_n = N
        last = self.passes[-1]
        return last["ux"], last["uy"]

    def _batch(self, n):
        N = self.N if n is None else int(n)
        if not 1 <= N <= self.N:
            raise ValueError(f"n = {N} outside 1..{self.N}")
        return N

    # The pass split into stages, so that a scheduler can interleave several
    # engines' passes and pack their correlations into shared launches
    # (serving.PivServer(packed=True)).  run() is stage_pre, the correlation and
    # stage_post for each pass in turn.
    def stage_pre(self, k, A, B, N):
        """Pass k's frames: the raw frames on pass 0, else the predictor of pass
        k-1 remapped to this pass's windows and both frames warped by it."""
        if k == 0:
            return A, B
        cfg, p, prev = self.cfg, self.passes[k], self.passes[k - 1]
        s = self._stream()
        H, W = self.H, self.W
        self._ok(self.Lp.pivb_remap_dev(prev["pdy"].data_ptr(), prev["pdx"].data_ptr(), N, prev["nyp"],
                                        prev["nxp"], p["map_y"].data_ptr(), p["map_x"].data_ptr(), p["ny"],
                                        p["nx"], p["pred_dy"].data_ptr(), p["pred_dx"].data_ptr(), s), "remap")
        fa, fb = self.warped
        self._ok(self.Lw.pivb_warp_dev(A.data_ptr(), B.data_ptr(), fa.data_ptr(), fb.data_ptr(),
                                       prev["pdy"].data_ptr(), prev["pdx"].data_ptr(), N, H, W, prev["nyp"],
                                       prev["nxp"], H * W, self.tables[k].data_ptr(), cfg.interp_mode, 0, 0,
                                       cfg.warp_impl, s), "warp")
        return fa, fb

    def _correlate(self, k, fa, fb, N):
        cfg, p = self.cfg, self.passes[k]
        s = self._stream()
        H, W = self.H, self.W
        o = p["out"]
        scr = self.scratch
        mptr = None if p["mask"] is None else p["mask"].data_ptr()
        args = (fa.data_ptr(), fb.data_ptr(), H * W, mptr, H, W, N, p["cx"].data_ptr(), p["cy"].data_ptr(),
                p["ny"], p["nx"], p["weight"].data_ptr(), p["weight"].data_ptr(), p["cw"].data_ptr(), p["win_h"],
                p["win_w"], 0, self.P, cfg.peak_finder, cfg.peakfit_impl, o["pk_loc_x"].data_ptr(),
                o["pk_loc_y"].data_ptr(), o["pk_height"].data_ptr(), o["sx"].data_ptr(), o["sy"].data_ptr(),
                o["sxy"].data_ptr(), p["ratio"].data_ptr(),
                None if self.planes is None else self.planes[k].data_ptr(), scr.data_ptr(), scr.numel())
        if self.Ld is not None and p["win_h"] == 32 and p["win_w"] == 32:
            self._ok(self.Ld.pivb_dft_xcorr_dev(*args, self.dft_status.data_ptr(), s), "correlation (tensor core)")
        else:
            self._ok(self.Lx.pivb_xcorr_dev(*args, s), "correlation")

    def packable(self, k):
        """Whether pass k's correlation can join a packed launch (square windows,
        one peak, the FFT engine, no plane dump)."""
        p = self.passes[k]
        return (p["win_h"] == p["win_w"] and self.planes is None and 3 <= self.cfg.peak_finder <= 6 and self.P == 1
                and not (self.Ld is not None and p["win_h"] == 32))

    def job(self, k, fa, fb, N):
        """Pass k's correlation as one job of a packed launch (_lib.XcorrJob)."""
        p = self.passes[k]
        o = p["out"]
        return _lib.XcorrJob(fa.data_ptr(), fb.data_ptr(), self.H * self.W,
                             None if p["mask"] is None else p["mask"].data_ptr(), self.H, self.W, N,
                             p["cx"].data_ptr(), p["cy"].data_ptr(), p["ny"], p["nx"], p["weight"].data_ptr(),
                             p["weight"].data_ptr(), p["cw"].data_ptr(), o["pk_loc_x"].data_ptr(),
                             o["pk_loc_y"].data_ptr(), o["pk_height"].data_ptr(), o["sx"].data_ptr(),
                             o["sy"].data_ptr(), o["sxy"].data_ptr(), p["ratio"].data_ptr())

    def stage_post(self, k, N):
        """Validation, infilling and (before the last pass) the next predictor."""
        cfg, p = self.cfg, self.passes[k]
        s = self._stream()
        o = p["out"]
        mptr = None if p["mask"] is None else p["mask"].data_ptr()
        pred_dy = p["pred_dy"] if k > 0 else None
        pred_dx = p["pred_dx"] if k > 0 else None
        thr_x, thr_y = p["thr"]
        if self.full_validate:
            self._ok(self.Lp.pivb_validate_peaks_dev(
                o["pk_loc_x"].data_ptr(), o["pk_loc_y"].data_ptr(), o["pk_height"].data_ptr(), self.P,
                int(bool(cfg.secondary_peak)), None if pred_dy is None else pred_dy.data_ptr(),
                None if pred_dx is None else pred_dx.data_ptr(), mptr, N, p["ny"], p["nx"], thr_x, thr_y,
                cfg.peak_mag_threshold, cfg.median_epsilon, cfg.median_threshold, cfg.median_size,
                float(cfg.sigma_threshold), int(bool(cfg.div_vort)),
                -1.0 if cfg.div_thresh is None else float(cfg.div_thresh),
                -1.0 if cfg.vort_thresh is None else float(cfg.vort_thresh),
                p["ux"].data_ptr(), p["uy"].data_ptr(), p["invalid"].data_ptr(), p["reason"].data_ptr(),
                p["choice"].data_ptr(), self.work.data_ptr(), s), "validate (peaks)")
        else:
            self._validate_one_peak(p, o, pred_dy, pred_dx, mptr, N, thr_x, thr_y, s)
        self._post_infill(k, N, mptr, s)

    def _validate_one_peak(self, p, o, pred_dy, pred_dx, mptr, N, thr_x, thr_y, s):
        cfg = self.cfg
        self._ok(self.Lp.pivb_validate_dev(
            o["pk_loc_x"].data_ptr(), o["pk_loc_y"].data_ptr(), o["pk_height"].data_ptr(),
            None if pred_dy is None else pred_dy.data_ptr(), None if pred_dx is None else pred_dx.data_ptr(),
            mptr, N, p["ny"], p["nx"], thr_x, thr_y, cfg.peak_mag_threshold, cfg.median_epsilon,
            cfg.median_threshold, cfg.median_size, p["ux"].data_ptr(), p["uy"].data_ptr(),
            p["invalid"].data_ptr(), p["reason"].data_ptr(), self.work.data_ptr(), s), "validate")

    def _post_infill(self, k, N, mptr, s):
        cfg, p = self.cfg, self.passes[k]
        last = k + 1 == len(self.passes)
        if (not last or cfg.final_infill) and cfg.infill == "nearest":
            self._ok(self.Lp.pivb_nearest_infill_dev(p["ux"].data_ptr(), p["uy"].data_ptr(), p["invalid"].data_ptr(),
                                                     mptr, N, p["ny"], p["nx"], p["spacing"][0], p["spacing"][1], s),
                     "infill (nearest)")
        elif not last or cfg.final_infill:
            self._ok(self.Lp.pivb_infill_dev(p["ux"].data_ptr(), p["uy"].data_ptr(), p["invalid"].data_ptr(), mptr,
                                             N, p["ny"], p["nx"], p["spacing"][0], p["spacing"][1],
                                             self.infill_order, cfg.infill_max_iter, cfg.infill_tol,
                                             self.infill_work.data_ptr(), self.infill_work.numel(), s), "infill")
        if not last:
            src_x, src_y = p["ux"], p["uy"]
            if self._fills(k):
                # harmonic fill of the masked windows, every other window fixed
                # (infilling.py:808-874 with the harmonic least-squares fill)
                nv = N * p["ny"] * p["nx"]
                src_x, src_y = self.fill[0, :nv], self.fill[1, :nv]
                if cfg.predictor_fill == "nearest":
                    self._ok(self.Lp.pivb_gather_fill_dev(p["ux"].data_ptr(), p["uy"].data_ptr(),
                                                          p["donor"].data_ptr(), N, p["ny"] * p["nx"],
                                                          src_x.data_ptr(), src_y.data_ptr(), s), "predictor fill")
                else:
                    src_x.copy_(p["ux"].reshape(-1)[:nv])
                    src_y.copy_(p["uy"].reshape(-1)[:nv])
                    self._ok(self.Lp.pivb_infill_dev(src_x.data_ptr(), src_y.data_ptr(), p["mask_u8"].data_ptr(),
                                                     None, N, p["ny"], p["nx"], p["spacing"][0], p["spacing"][1],
                                                     1, cfg.infill_max_iter, cfg.infill_tol,
                                                     self.infill_work.data_ptr(), self.infill_work.numel(), s),
                             "predictor fill")
            self._ok(self.Lp.pivb_pad_smooth_dev(src_x.data_ptr(), src_y.data_ptr(), N, p["ny"], p["nx"],
                                                 p["nyp"], p["nxp"], p["pre"][0], p["pre"][1],
                                                 p["taps"].data_ptr(), p["radius"], p["pdy"].data_ptr(),
                                                 p["pdx"].data_ptr(), self.work.data_ptr(), s), "pad/smooth")
        if last:
            self._last_n = N

    def collect(self, n=None):
        """Per-pair results of the last run, every pass, as host PIVResult objects
        (the reference's PIVPassResult fields, cpu_instantaneous.py:875-910):
        infilled ux/uy, nan_mask, nan_reason, peak_mag (NaN where gated),
        peak_ratio, peak_choice, the predictor added on this pass, window grid.
        With keep_planes on, each pass carries the correlation-plane payload."""
        from .results import PIVPassResult, PIVResult

        torch = self.torch
        n = self._last_n if n is None else int(n)
        torch.cuda.current_stream(self.device).synchronize()
        out = [PIVResult() for _ in range(n)]
        for k, (p, g) in enumerate(zip(self.passes, self.geo)):
            ny, nx = p["ny"], p["nx"]
            o = {key: v[:n].cpu().numpy() for key, v in p["out"].items()}
            ux, uy = p["ux"][:n].cpu().numpy(), p["uy"][:n].cpu().numpy()
            reason = p["reason"][:n].cpu().numpy()
            nan_mask = p["invalid"][:n].cpu().numpy().astype(bool) | (reason == -1)
            ratio = p["ratio"][:n].cpu().numpy()
            if k > 0:
                pred = torch.stack((p["pred_dy"][:n], p["pred_dx"][:n]), dim=-1).cpu().numpy()
            else:
                pred = np.zeros((n, ny, nx, 2), np.float32)
            # masked windows and peaks beyond the displacement gate: the reference NaNs
            # their heights (cpu_instantaneous.py:602-607), peak by peak
            thr_x, thr_y = p["thr"]
            with np.errstate(invalid="ignore"):
                gone = (np.abs(o["pk_loc_x"]) > thr_x) | (np.abs(o["pk_loc_y"]) > thr_y)
            gone |= p["b_mask"][None, None]
            peak_mag = np.where(gone, np.float32(np.nan), o["pk_height"])
            if self.full_validate:
                choice = p["choice"][:n].cpu().numpy().astype(np.intp)
            else:
                choice = np.where(nan_mask, 0, 1).astype(np.intp)
            planes = None if self.planes is None else self.planes[k][:n].cpu().numpy()
            for i in range(n):
                pr = PIVPassResult(
                    n_windows=np.array([ny, nx], dtype=np.int32), ux_mat=ux[i].copy(), uy_mat=uy[i].copy(),
                    nan_mask=nan_mask[i].copy(), nan_reason=reason[i].copy(), peak_mag=peak_mag[i].copy(),
                    peak_ratio=ratio[i].copy(), peak_choice=choice[i].copy(),
                    predictor_field=pred[i].copy(), b_mask=p["b_mask"].copy(),
                    window_size=tuple(self.cfg.window_sizes[k]), win_ctrs_x=g.grid.win_ctrs_x,
                    win_ctrs_y=g.grid.win_ctrs_y)
                if planes is not None:
                    pr.debug_dump = {
                        "planes": planes[i], "peak_finder": int(self.cfg.peak_finder),
                        "pk_loc_x_raw": o["pk_loc_x"][i], "pk_loc_y_raw": o["pk_loc_y"][i],
                        "pk_height_raw": o["pk_height"][i], "pk_ratio_raw": ratio[i], "sx": o["sx"][i],
                        "sy": o["sy"][i], "sxy": o["sxy"][i]}
                out[i].add_pass(pr)
        return out

    def pass_inputs(self, k, A, B):
        """The frames pass k of the last run correlated, rebuilt on the device: the
        raw frames for pass 0, else both frames warped again by pass k-1's padded
        predictor (still held in its buffers).  Returns device tensors (views of
        internal buffers for k > 0, overwritten by the next run or call)."""
        if k == 0:
            return A, B
        n = self._last_n
        prev = self.passes[k - 1]
        fa, fb = self.warped
        self._ok(self.Lw.pivb_warp_dev(A.data_ptr(), B.data_ptr(), fa.data_ptr(), fb.data_ptr(),
                                       prev["pdy"].data_ptr(), prev["pdx"].data_ptr(), n, self.H, self.W,
                                       prev["nyp"], prev["nxp"], self.H * self.W, self.tables[k].data_ptr(),
                                       self.cfg.interp_mode, 0, 0, self.cfg.warp_impl, self._stream()), "warp")
        return fa[:n], fb[:n]

    def vectors_per_step(self) -> int:
        p = self.passes[-1]
        return self.N * p["ny"] * p["nx"]

    def windows_per_step(self) -> int:
        return self.N * sum(p["ny"] * p["nx"] for p in self.passes)


class HostPipeline:
    """End-to-end multipass from pinned host memory: uint16 frames in, float32
    vector fields out.

    The batch is processed in chunks of `chunk` pairs (one MultipassPIV of that
    batch size).  While chunk c is computed, chunk c+1's frames cross PCIe on a
    copy stream into the other of two uint16 staging slots; frames are converted
    to float32 on the GPU (the reference's readers convert on the host), and each
    chunk's final field is read back right after its last pass.
    """

    def __init__(self, image_shape, chunk: int, cfg: MultipassConfig | None = None, device=None,
                 vector_masks=None, graph: bool = True):
        """graph: after the first chunk, replay the chunk's passes as one captured
        CUDA graph (the conversions and copies stay stream operations)."""
        import torch

        self.torch = torch
        self.mp = MultipassPIV(image_shape, chunk, cfg, device, vector_masks)
        self.use_graph = graph
        self._graph = None
        dev = self.mp.device
        H, W = image_shape
        self.C = chunk
        self.u16 = [[torch.empty((chunk, H, W), dtype=torch.uint16, device=dev) for _ in range(2)] for _ in range(2)]
        self.f32 = [torch.empty((chunk, H, W), dtype=torch.float32, device=dev) for _ in range(2)]
        self.copy_stream = torch.cuda.Stream(device=dev)
        self.ev_h2d = [torch.cuda.Event() for _ in range(2)]
        self.ev_conv = [torch.cuda.Event() for _ in range(2)]
        # results leave through a staging copy on a second copy stream, so a
        # chunk's read-back overlaps the next chunk's passes
        last = self.mp.passes[-1]
        self.out_stage = [torch.empty((2, chunk, last["ny"], last["nx"]), dtype=torch.float32, device=dev)
                          for _ in range(2)]
        self.d2h_stream = torch.cuda.Stream(device=dev)
        self.ev_done = [torch.cuda.Event() for _ in range(2)]
        self.ev_d2h = [torch.cuda.Event() for _ in range(2)]
        self._d2h_used = [False, False]
        self._slot = 0
        self.Lp = _lib.pass_lib()

    def run(self, Ah, Bh, ux_out, uy_out):
        """Ah, Bh: pinned uint16 (N, H, W) host tensors, N a multiple of the chunk;
        ux_out, uy_out: pinned float32 (N, ny, nx) host tensors, complete once the
        current stream passes finish() (or after a device synchronisation)."""
        torch = self.torch
        if not all(t.is_pinned() for t in (Ah, Bh, ux_out, uy_out)):
            raise ValueError("HostPipeline.run needs page-locked host tensors (use .pin_memory())")
        comp = torch.cuda.current_stream(self.mp.device)
        C = self.C
        n_chunks = Ah.shape[0] // C
        for c in range(n_chunks):
            # staging slots alternate across calls too, so the next call's first
            # chunk crosses PCIe while this call's last chunk computes; a slot is
            # refilled only after its previous frames were converted
            s = self._slot
            self._slot ^= 1
            sl = slice(c * C, (c + 1) * C)
            self.copy_stream.wait_event(self.ev_conv[s])
            with torch.cuda.stream(self.copy_stream):
                self.u16[s][0].copy_(Ah[sl], non_blocking=True)
                self.u16[s][1].copy_(Bh[sl], non_blocking=True)
                self.ev_h2d[s].record(self.copy_stream)
            comp.wait_event(self.ev_h2d[s])
            st = ctypes.c_void_p(comp.cuda_stream)
            for k in range(2):
                src, dst = self.u16[s][k], self.f32[k]
                if self.Lp.pivb_u16_to_f32_dev(src.data_ptr(), dst.data_ptr(), src.numel(), st) != 0:
                    raise RuntimeError("u16 -> f32 conversion failed")
            self.ev_conv[s].record(comp)
            if self._graph is not None:
                self._graph.replay()
                last = self.mp.passes[-1]
                ux, uy = last["ux"], last["uy"]
            else:
                ux, uy = self.mp.run(self.f32[0], self.f32[1])
            # the staging slot is refilled only after its previous read-back
            if self._d2h_used[s]:
                comp.wait_event(self.ev_d2h[s])
            stage = self.out_stage[s]
            stage[0].copy_(ux)
            stage[1].copy_(uy)
            self.ev_done[s].record(comp)
            self.d2h_stream.wait_event(self.ev_done[s])
            with torch.cuda.stream(self.d2h_stream):
                ux_out[sl].copy_(stage[0], non_blocking=True)
                uy_out[sl].copy_(stage[1], non_blocking=True)
                self.ev_d2h[s].record(self.d2h_stream)
            self._d2h_used[s] = True
        if self.use_graph and self._graph is None:
            # every lazy set-up has run once: capture the chunk's passes (capture
            # records, it does not execute)
            comp.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self.mp.run(self.f32[0], self.f32[1])
            torch.cuda.current_stream(self.mp.device).synchronize()
            self._graph = g
        return ux_out, uy_out

    def finish(self):
        """Make the current stream wait for every read-back issued so far (the
        host result tensors are complete once the stream reaches this point)."""
        comp = self.torch.cuda.current_stream(self.mp.device)
        for s in range(2):
            if self._d2h_used[s]:
                comp.wait_event(self.ev_d2h[s])
