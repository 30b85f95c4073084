"""GPU-resident ensemble PIV pass: accumulate, finalise, k-space fit.

Follows the reference's single-pass ensemble for one pass, std or single mode
(pivtools_cli/piv/piv_backend/cpu_ensemble.py:188-225, 590-676, 700-760,
single_pass_accumulator.py:292-320, 352-506, 508-800,
kspace_lm_fitting.py:804-961):

  accumulate  per batch of pairs: the AB, AA and BB correlation sums of every
              window (bulkxcorr2d_accumulate_triple, Kahan-compensated FP32 across
              batches) and the frame sums for the mean images;
  two sweeps  the 'image' background methods (pivtools_core/ensemble.py:142-204,
              cpu_ensemble.py:1104-1330): a first sweep sums the frames only
              (accumulate_means), end_means forms the mean images, and the second
              sweep (accumulate) correlates each frame minus its mean image;
  finalise    mean images, their correlation as the background term ('correlation'
              methods), the per-window plane-mean removal ('+dc_zero'), the
              optional pair-count envelope divide, the normalisation by the auto
              peaks, FP64 planes;
  fit         the k-space LM fit of every window (libkspacefit).

All sums, planes and fit outputs stay on the device; every step is a kernel of
the repo's libraries launched on the caller's stream.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib, geometry

_METHODS = {
    # method: (per-pair window-mean removal in the correlator, subtract the
    #          mean-image correlation at finalise, zero the plane means, two
    #          sweeps with the mean images subtracted from each frame)
    # (pivtools_core/config.py:2495-2631, single_pass_accumulator.py:575-680)
    "correlation": (0, True, False, False),
    "correlation+dc_zero": (0, True, True, False),
    "window_mean": (1, False, False, False),
    "correlation+window_mean": (1, True, False, False),
    "image": (0, False, False, True),
    "image+window_mean": (1, False, False, True),
    "image+dc_zero": (0, False, True, True),
}


def pair_envelope(wa, wb, corr_size):
    """Linear pair-count envelope E(s) = (wa * wb)(s) of two window weights,
    centre-cropped to corr_size (zero lag at corr_size // 2) and normalised to 1
    there (single_pass_accumulator.py:52-102): FP64, zero-padded FFT."""
    wa = np.asarray(wa, np.float64)
    wb = np.asarray(wb, np.float64)
    h, w = wa.shape
    ch, cw = corr_size
    if wa.shape != wb.shape:
        raise ValueError(f"window weights must share a shape, got {wa.shape} vs {wb.shape}")
    if ch > h or cw > w:
        raise ValueError(f"corr_size {tuple(corr_size)} exceeds envelope support {(h, w)}")
    full = np.fft.fftshift(np.fft.ifft2(np.fft.fft2(wa, s=(2 * h, 2 * w)) *
                                        np.conj(np.fft.fft2(wb, s=(2 * h, 2 * w)))).real)
    env = full[h - ch // 2:h - ch // 2 + ch, w - cw // 2:w - cw // 2 + cw]
    centre = env[ch // 2, cw // 2]
    if abs(centre - env.max()) > 1e-9 * env.max():
        raise ValueError(f"envelope centre {centre:.12f} != max {env.max():.12f}: centering is off")
    env = env / centre
    if np.any(env <= 0.0):
        raise ValueError("pair-count envelope has non-positive entries inside the plane")
    return env


class EnsemblePIV:
    """One ensemble pass over frames of one size on one GPU: std mode (both frames
    weighted by one window) or single mode (cpu_ensemble.py:188-225, 700-760:
    frame A weighted by the small window centred in the sum window ('singlepix'),
    frame B and both auto planes by the whole sum window ('bsingle'), frames
    zero-padded so the sum window fits around every small window, planes stored
    at the fitting window)."""

    def __init__(self, image_shape, window=(16, 16), overlap=75, window_type="square",
                 background="correlation+dc_zero", envelope_divide=False, device=None, runtype="std",
                 sum_window=None, fit_window=None, per_pair_normalization=False):
        import torch

        if background not in _METHODS:
            raise ValueError(f"Invalid ensemble_background_subtraction_method {background!r}. "
                             f"Must be one of {sorted(_METHODS)}")
        if runtype not in ("std", "single"):
            raise ValueError(f"ensemble_type must be 'std' or 'single', got {runtype!r}")
        if per_pair_normalization and background != "window_mean":
            # pivtools_core/validation.py:544-552
            raise ValueError("ensemble_piv.per_pair_normalization requires background_subtraction_method exactly "
                             f"'window_mean', got {background!r}")
        self.torch = torch
        self.device = torch.device("cuda" if device is None else device)
        self.H, self.W = image_shape
        self.win = tuple(window)
        self.runtype = runtype
        self.mean_subtract, self.use_bg, self.dc_zero, self.two_sweep = _METHODS[background]
        self.per_pair_norm = 1 if per_pair_normalization else 0
        self.background = background
        if runtype == "single":
            if sum_window is None:
                raise ValueError("ensemble_sum_window must be defined when using 'single' mode in ensemble_type")
            self.sum_window = tuple(int(v) for v in sum_window)
            self.corr = tuple(int(v) for v in (fit_window if fit_window is not None else self.sum_window))
            if self.corr[0] > self.sum_window[0] or self.corr[1] > self.sum_window[1]:
                raise ValueError(f"sum_fitting_window {self.corr} must be <= sum_window {self.sum_window}")
            # grid and padding of the padded frame (window_utils.py:276-463)
            self.grid, self.padding = geometry.compute_window_centers_single_mode(image_shape, self.win,
                                                                                  self.sum_window, overlap)
            wa = geometry.window_weight(self.win, "singlepix", self.sum_window)
            wb = geometry.window_weight(self.sum_window, "bsingle", self.sum_window)
            self.comp_size = self.sum_window
            # the AB plane's normalisation correction (single_pass_accumulator.py:760-780)
            self.ab_scale = float(np.float32((self.sum_window[0] * self.sum_window[1]) / (self.win[0] * self.win[1])))
        else:
            if fit_window is not None or sum_window is not None:
                raise ValueError("sum_window and fit_window belong to single mode")
            self.sum_window = None
            self.corr = self.win
            self.grid = geometry.compute_window_centers(image_shape, self.win, overlap)
            self.padding = (0, 0, 0, 0)
            wa = wb = geometry.window_weight(self.win, window_type)
            self.comp_size = self.win
            self.ab_scale = 1.0
        if self.comp_size[0] != self.comp_size[1]:
            raise ValueError(f"the GPU accumulation takes square computation windows, got {self.comp_size}")
        pt, pb, pl, pr = self.padding
        self.Hp, self.Wp = self.H + pt + pb, self.W + pl + pr       # frame size the correlator reads
        g = self.grid
        self.n_win = g.n_win_y * g.n_win_x
        h, w = self.corr
        dev, f32 = self.device, torch.float32
        self.weight_a = torch.tensor(wa, dtype=f32, device=dev)       # AB weight of frame A
        self.weight = torch.tensor(wb, dtype=f32, device=dev)         # AB weight of frame B, both auto planes
        self._wb_host = np.asarray(wb, np.float64)
        self.cx = torch.tensor(g.win_ctrs_x, dtype=f32, device=dev)
        self.cy = torch.tensor(g.win_ctrs_y, dtype=f32, device=dev)
        self.env = self.env_ab = None
        if envelope_divide:
            # std: every plane shares E = W * W; single: the autos E = B * B, AB the
            # A * B trapezoid (single_pass_accumulator.py:690-730)
            self.env = torch.tensor(pair_envelope(wb, wb, self.corr), dtype=f32, device=dev)
            self.env_ab = (torch.tensor(pair_envelope(wa, wb, self.corr), dtype=f32, device=dev)
                           if runtype == "single" else self.env)
        plane = self.n_win * h * w
        self.sums = torch.zeros((3, plane), dtype=f32, device=dev)       # AB, AA, BB
        self.comp = torch.zeros((3, plane), dtype=f32, device=dev)
        self.bg = torch.zeros((3, plane), dtype=f32, device=dev)
        self.fsum = torch.zeros((2, self.H * self.W), dtype=f32, device=dev)   # frame sums A, B
        self.fcomp = torch.zeros_like(self.fsum)
        self.fmean = torch.zeros_like(self.fsum)
        self.planes = torch.zeros((3, self.n_win, h, w), dtype=torch.float64, device=dev)  # AA, BB, AB
        self.norm = torch.zeros(self.n_win, dtype=f32, device=dev)
        self.Lx = _lib.bulkxcorr2d_lib()
        self.Lp = _lib.pass_lib()
        self.Lk = _lib.kspacefit_lib()
        sb = int(self.Lx.pivb_accumulate_scratch_bytes(self.comp_size[0], self.n_win))
        self.scratch = torch.empty(max(sb, 256), dtype=torch.uint8, device=dev)
        self.n_pairs = 0
        self.n_means = 0              # pairs of the first sweep (two-sweep methods)
        self.means_ready = False
        self._centered = None         # (2, n, Hp, Wp) centred / padded frames the correlator reads
        # zero fills above ran on the construction stream: finish them before use
        # from another stream
        torch.cuda.current_stream(self.device).synchronize()

    @property
    def window_centres(self):
        """Window centres (x, y) in the coordinates of the unpadded frame."""
        pt, _, pl, _ = self.padding
        return self.grid.win_ctrs_x - pl, self.grid.win_ctrs_y - pt

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    @staticmethod
    def _ok(code, what):
        if code != 0:
            raise RuntimeError(f"{what} failed with code {code}")

    def reset(self):
        for t in (self.sums, self.comp, self.fsum, self.fcomp):
            t.zero_()
        self.n_pairs = 0
        self.n_means = 0
        self.means_ready = False

    def _triple(self, A, B, n, mean_subtract, out, comp, s):
        """bulkxcorr2d_accumulate_triple over n frames of the correlator's size
        (Hp x Wp): AB weights (A, B), auto weights (B, B) (cpu_ensemble.py:1000-1013)."""
        g = self.grid
        ch, cw = self.comp_size
        h, w = self.corr
        wa, wb = self.weight_a.data_ptr(), self.weight.data_ptr()
        self._ok(self.Lx.pivb_accumulate_triple_dev(
            A.data_ptr(), B.data_ptr(), self.Hp * self.Wp, None, self.Hp, self.Wp, n, self.cx.data_ptr(),
            self.cy.data_ptr(), g.n_win_y, g.n_win_x, wa, wb, wb, wb, ch, cw, h, w, mean_subtract,
            self.per_pair_norm, out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(),
            None if comp is None else comp.data_ptr(), self.scratch.data_ptr(), self.scratch.numel(), s),
            "accumulate_triple")

    def _frame_sums(self, A, B, n, s):
        npix = self.H * self.W
        for k, F in enumerate((A, B)):
            self._ok(self.Lp.pivb_frame_sum_dev(F.data_ptr(), npix, n, npix, self.fsum[k].data_ptr(),
                                                self.fcomp[k].data_ptr(), s), "frame sum")

    def _check_batch(self, A, B):
        torch = self.torch
        if A.shape != B.shape or A.dim() != 3 or tuple(A.shape[1:]) != (self.H, self.W):
            raise ValueError(f"frames must be (n, {self.H}, {self.W}) pairs of one shape")
        if A.dtype != torch.float32 or B.dtype != torch.float32 or not (A.is_contiguous() and B.is_contiguous()):
            raise ValueError("frames must be contiguous float32 tensors")

    def accumulate_means(self, A, B):
        """First sweep of the 'image' methods: add a batch of pairs (n, H, W)
        float32 to the frame sums only (compute_warp_sums_only,
        cpu_ensemble.py:1104-1190)."""
        if not self.two_sweep:
            raise ValueError(f"accumulate_means belongs to the two-sweep 'image' methods, not {self.background!r}")
        if self.means_ready:
            raise RuntimeError("the first sweep is closed (end_means was called); reset() starts over")
        self._check_batch(A, B)
        n = int(A.shape[0])
        self._frame_sums(A, B, n, self._stream())
        self.n_means += n

    def end_means(self):
        """Close the first sweep: the mean images sum / n (pivtools_core/ensemble.py:
        199-200) of this process's pairs."""
        return self._end_means(self.fsum, self.n_means)

    def end_means_distributed(self, group=None):
        """Close the first sweep across the ranks of `group` (pairs sharded): one
        all-reduce combines the frame sums and pair counts, so every rank
        subtracts the ensemble's mean images (the reference reduces the workers'
        warp sums the same way, pivtools_core/ensemble.py:179-200)."""
        from . import ensemble_dist as ed

        if not self.two_sweep:
            raise ValueError(f"end_means belongs to the two-sweep 'image' methods, not {self.background!r}")
        fsum, n = ed.all_reduce_frame_sums(self.fsum, self.fcomp, self.n_means, group)
        return self._end_means(fsum, n)

    def _end_means(self, fsum, n):
        if not self.two_sweep:
            raise ValueError(f"end_means belongs to the two-sweep 'image' methods, not {self.background!r}")
        if self.means_ready:
            raise RuntimeError("end_means was already called")
        if n == 0:
            raise RuntimeError("end_means before any accumulate_means")
        s = self._stream()
        npix = self.H * self.W
        for k in range(2):
            self._ok(self.Lp.pivb_frame_mean_dev(fsum[k].data_ptr(), npix, n, self.fmean[k].data_ptr(), s),
                     "frame mean")
        self.n_means = n
        self.means_ready = True
        return {"A_mean": self.fmean[0].view(self.H, self.W), "B_mean": self.fmean[1].view(self.H, self.W),
                "n_pairs": n}

    def _scratch_pair(self, n):
        if self._centered is None or self._centered.shape[1] < n:
            self._centered = self.torch.empty((2, n, self.Hp, self.Wp), dtype=self.torch.float32, device=self.device)
        return self._centered[0, :n], self._centered[1, :n]

    def _prepare(self, A, B, n, s, in_place):
        """The frames the correlator reads: as given (std mode); minus the mean
        images for the 'image' methods (cpu_ensemble.py:1290-1291), in place for
        the pipeline's own staging buffers, else into scratch; in single mode
        zero-padded (and centred first) into scratch (cpu_ensemble.py:962-972,
        1314-1324).  The caller's tensors are never modified."""
        npix = self.H * self.W
        if self.runtype == "single":
            outs = self._scratch_pair(n)
            for k, (F, O) in enumerate(zip((A, B), outs)):
                self._ok(self.Lp.pivb_pad_frames_dev(F.data_ptr(), npix, n, self.H, self.W,
                                                     self.fmean[k].data_ptr() if self.two_sweep else None,
                                                     self.padding[0], self.padding[2], O.data_ptr(), self.Hp,
                                                     self.Wp, self.Hp * self.Wp, s), "pad frames")
            return outs
        if not self.two_sweep:
            return A, B
        outs = (A, B) if in_place else self._scratch_pair(n)
        for k, (F, O) in enumerate(zip((A, B), outs)):
            self._ok(self.Lp.pivb_center_frames_dev(F.data_ptr(), npix, n, npix, self.fmean[k].data_ptr(),
                                                    O.data_ptr(), npix, s), "centre frames")
        return outs

    def accumulate(self, A, B):
        """Add a batch of pairs: A, B (n, H, W) float32 CUDA tensors.  For the
        'image' methods this is the second sweep: each frame minus the mean
        images of the first is correlated (correlate_mean_subtracted_batch,
        cpu_ensemble.py:1192-1330); the caller's tensors are not modified."""
        self._accumulate(A, B, in_place=False)

    def _accumulate(self, A, B, in_place):
        self._check_batch(A, B)
        n = int(A.shape[0])
        s = self._stream()
        if self.two_sweep:
            if not self.means_ready:
                raise RuntimeError(f"{self.background!r} sweeps twice: accumulate_means over every pair, then "
                                   "end_means, before accumulate")
        else:
            self._frame_sums(A, B, n, s)        # of the unpadded frames (cpu_ensemble.py:955-960)
        A, B = self._prepare(A, B, n, s, in_place)
        self._triple(A, B, n, self.mean_subtract, self.sums, self.comp, s)
        self.n_pairs += n

    def accumulate_host(self, Ah, Bh, chunk: int = 16):
        """Add pairs from page-locked uint16 host frames Ah, Bh (n, H, W): chunks
        cross PCIe on a copy stream into two alternating staging slots while the
        previous chunk is converted to float32 on the GPU and accumulated on the
        caller's stream.  Equal, bit for bit, to accumulate() called on the same
        frames in float32, chunk by chunk (for the 'image' methods the mean images
        are subtracted in the staging buffers)."""
        self._stream_host(Ah, Bh, chunk, lambda a, b: self._accumulate(a, b, in_place=True))

    def accumulate_means_host(self, Ah, Bh, chunk: int = 16):
        """The first sweep of the 'image' methods from page-locked uint16 host
        frames, staged as in accumulate_host."""
        if not self.two_sweep:
            raise ValueError(f"accumulate_means belongs to the two-sweep 'image' methods, not {self.background!r}")
        self._stream_host(Ah, Bh, chunk, self.accumulate_means)

    def _stream_host(self, Ah, Bh, chunk, sink):
        import ctypes as C

        torch = self.torch
        if not (Ah.is_pinned() and Bh.is_pinned()):
            raise ValueError("accumulate_host needs page-locked host frames (use .pin_memory())")
        if Ah.dtype != torch.uint16 or Bh.dtype != torch.uint16 or Ah.shape != Bh.shape:
            raise ValueError("accumulate_host takes two uint16 frame stacks of one shape")
        n, H, W = Ah.shape
        if (H, W) != (self.H, self.W):
            raise ValueError(f"frames {H}x{W} do not match the pass's {self.H}x{self.W}")
        st = self.__dict__.get("_stage")
        if st is None or st["chunk"] != chunk:
            dev = self.device
            st = dict(chunk=chunk, slot=0, copy=torch.cuda.Stream(device=dev),
                      u16=[[torch.empty((chunk, H, W), dtype=torch.uint16, device=dev) for _ in range(2)]
                           for _ in range(2)],
                      f32=[torch.empty((chunk, H, W), dtype=torch.float32, device=dev) for _ in range(2)],
                      ev_h2d=[torch.cuda.Event() for _ in range(2)], ev_conv=[torch.cuda.Event() for _ in range(2)])
            self._stage = st
        comp = torch.cuda.current_stream(self.device)
        cs = C.c_void_p(comp.cuda_stream)
        for c0 in range(0, n, chunk):
            k = min(chunk, n - c0)
            sl = st["slot"]
            st["slot"] ^= 1
            st["copy"].wait_event(st["ev_conv"][sl])
            with torch.cuda.stream(st["copy"]):
                st["u16"][sl][0][:k].copy_(Ah[c0:c0 + k], non_blocking=True)
                st["u16"][sl][1][:k].copy_(Bh[c0:c0 + k], non_blocking=True)
                st["ev_h2d"][sl].record(st["copy"])
            comp.wait_event(st["ev_h2d"][sl])
            for j in range(2):
                self._ok(self.Lp.pivb_u16_to_f32_dev(st["u16"][sl][j].data_ptr(), st["f32"][j].data_ptr(), k * H * W,
                                                     cs), "u16 -> f32")
            st["ev_conv"][sl].record(comp)
            sink(st["f32"][0][:k], st["f32"][1][:k])

    def finalize(self):
        """Background, DC zero, envelope, normalisation -> FP64 planes (AA, BB, AB)
        of shape (n_win, h, w) on the device, and the normalisation factors."""
        if self.n_pairs == 0:
            raise RuntimeError("finalize before any accumulate")
        self._finalize(self.sums, self.n_pairs, self.fsum, 0, self.n_win, self.planes, self.norm)
        return {"R_AA": self.planes[0], "R_BB": self.planes[1], "R_AB": self.planes[2], "norm": self.norm}

    def finalize_distributed(self, group=None):
        """Finalise across the ranks of `group` (one GPU each, pairs sharded):
        one exchange combines the sums (ensemble_dist.exchange_sums), then this
        rank finalises its block of windows.  Returns the block's planes and
        (start, stop); `fit` then fits the block and `gather_fit` joins them."""
        from . import ensemble_dist as ed

        h, w = self.corr
        block, fsum, n_tot, (a, b) = ed.exchange_sums(self.sums, self.comp, self.fsum, self.fcomp, self.n_pairs,
                                                      self.n_win, h * w, group)
        torch = self.torch
        nb = b - a
        self.block = (a, b)
        self.planes = torch.zeros((3, nb, h, w), dtype=torch.float64, device=self.device)
        self.norm = torch.zeros(max(nb, 1), dtype=torch.float32, device=self.device)
        if nb > 0:
            self._finalize(block.reshape(3, -1), n_tot, fsum, a, b, self.planes, self.norm)
        return {"R_AA": self.planes[0], "R_BB": self.planes[1], "R_AB": self.planes[2], "norm": self.norm,
                "windows": (a, b), "n_pairs": n_tot}

    def _finalize(self, sums, n_pairs, fsum, w0, w1, planes, norm):
        """Finalise windows [w0, w1): sums (3, (w1 - w0) * h * w) for those windows,
        fsum (2, H * W) frame sums over n_pairs pairs."""
        s = self._stream()
        h, w = self.corr
        hw = h * w
        bg = None
        if self.use_bg:
            npix = self.H * self.W
            for k in range(2):
                self._ok(self.Lp.pivb_frame_mean_dev(fsum[k].data_ptr(), npix, n_pairs, self.fmean[k].data_ptr(), s),
                         "frame mean")
            self.bg.zero_()
            MA, MB = self.fmean[0].view(1, self.H, self.W), self.fmean[1].view(1, self.H, self.W)
            if self.runtype == "single":        # padded like the pairs (single_pass_accumulator.py:402-410)
                PA, PB = self._scratch_pair(1)
                for F, O in ((MA, PA), (MB, PB)):
                    self._ok(self.Lp.pivb_pad_frames_dev(F.data_ptr(), npix, 1, self.H, self.W, None,
                                                         self.padding[0], self.padding[2], O.data_ptr(), self.Hp,
                                                         self.Wp, self.Hp * self.Wp, s), "pad frames")
                MA, MB = PA, PB
            self._triple(MA, MB, 1, self.mean_subtract, self.bg, None, s)
            bg = self.bg[:, w0 * hw:w1 * hw]
        env = None if self.env is None else self.env.data_ptr()
        env_ab = None if self.env_ab is None else self.env_ab.data_ptr()
        self._ok(self.Lp.pivb_ensemble_finalize_dev(
            sums[0].data_ptr(), sums[1].data_ptr(), sums[2].data_ptr(),
            None if bg is None else bg[0].data_ptr(), None if bg is None else bg[1].data_ptr(),
            None if bg is None else bg[2].data_ptr(), n_pairs, w1 - w0, h, w, int(self.dc_zero), env, env_ab,
            planes[2].data_ptr(), planes[0].data_ptr(), planes[1].data_ptr(), norm.data_ptr(), self.ab_scale, s),
            "ensemble finalize")

    def gather_fit(self, fit, group=None):
        """All-gather the per-window fit outputs of every rank's block."""
        from . import ensemble_dist as ed

        return {k: ed.gather_rows(v, self.n_win, group) for k, v in fit.items()}

    def floor_regressor(self, predictor=None, warp_kernel="lanczos"):
        """Coloured-floor regressor P_win (n, h*w) FP64 on the device for the windows
        of the finalised planes (kspace_floor_psd.py, single_pass_accumulator.py:814-887):
        the P grid of this pass's chain (window weight, envelope when divided,
        window-mean hole when the method removes window means) looked up per window
        at the fractions of predictor / 2.  predictor: (n_win_y, n_win_x, 2) [dy, dx]
        on the full window grid (None on a first pass: zero shift everywhere)."""
        from . import floor_psd

        torch = self.torch
        dev = self.device
        h, w = self.corr
        a, b = getattr(self, "block", (0, self.n_win))
        n = b - a
        pdy = pdx = None
        nf = 2
        if predictor is not None:
            pr = torch.as_tensor(predictor, dtype=torch.float32, device=dev).reshape(self.n_win, 2)
            if not bool(torch.isfinite(pr).all()):
                raise ValueError("non-finite predictor: the coloured-floor fractions are undefined")
            pdy, pdx = pr[a:b, 0].contiguous(), pr[a:b, 1].contiguous()
            half = pr[a:b] * 0.5
            if float((half - torch.round(half)).abs().max()) > 0.0:
                nf = floor_psd.N_FRACS
        hole = self.mean_subtract == 1
        key = (nf, warp_kernel, hole)
        cache = self.__dict__.setdefault("_p_grids", {})
        if key not in cache:
            # the auto envelope and the frame-B weight: the sum window in single mode
            # (single_pass_accumulator.py:863-874)
            env = self.env.cpu().numpy().astype(np.float64) if self.env is not None else np.ones((h, w))
            fs, P = floor_psd.build_p_grid(env, warp_kernel, hole, self._wb_host.astype(np.float32), n_fracs=nf)
            cache[key] = (torch.tensor(fs, dtype=torch.float64, device=dev),
                          torch.tensor(P, dtype=torch.float64, device=dev).contiguous())
        fs_d, P_d = cache[key]
        out = torch.empty((max(n, 1), h * w), dtype=torch.float64, device=dev)
        if n > 0:
            self._ok(self.Lp.pivb_floor_interp_dev(fs_d.data_ptr(), nf, P_d.data_ptr(), h * w,
                                                   None if pdy is None else pdy.data_ptr(),
                                                   None if pdx is None else pdx.data_ptr(), n, out.data_ptr(),
                                                   self._stream()), "floor regressor")
        return out[:n]

    def fit(self, mask=None, use_kx4=0, use_ky4=0, floor="flat", predictor=None, warp_kernel="lanczos"):
        """k-space LM fit of the finalised planes, flat or coloured noise floor
        (`floor_regressor`).  Returns device tensors: gauss (n_win, 16) and status
        (n_win,), plus diagnostics."""
        torch = self.torch
        dev = self.device
        h, w = self.corr
        n = int(self.planes.shape[1])
        if floor not in ("flat", "coloured"):
            raise ValueError(f"kspace floor {floor!r} (valid: 'flat', 'coloured')")
        if floor == "flat" and predictor is not None:
            raise ValueError("a predictor only enters the coloured floor")
        p_win = self.floor_regressor(predictor, warp_kernel) if floor == "coloured" else None
        m = (torch.zeros(n, dtype=torch.uint8, device=dev) if mask is None
             else torch.as_tensor(mask, dtype=torch.uint8, device=dev).reshape(n))
        o = {
            "gauss": torch.zeros((n, 16), dtype=torch.float64, device=dev),
            "status": torch.zeros(n, dtype=torch.int32, device=dev),
            "init": torch.zeros((n, 16), dtype=torch.float64, device=dev),
        }
        for k in ("gain", "N0", "b4x", "b4y", "cost_per_pt"):
            o[k] = torch.zeros(n, dtype=torch.float64, device=dev)
        o["n_valid"] = torch.zeros(n, dtype=torch.int32, device=dev)
        o["iters"] = torch.zeros(n, dtype=torch.int32, device=dev)
        o["conv"] = torch.zeros(n, dtype=torch.uint8, device=dev)
        sb = int(self.Lk.pivb_kspace_scratch_bytes(n, h, w))
        scratch = torch.empty(max(sb, 256), dtype=torch.uint8, device=dev)
        self._ok(self.Lk.pivb_kspace_fit_dev(
            self.planes[0].data_ptr(), self.planes[1].data_ptr(), self.planes[2].data_ptr(), m.data_ptr(),
            None if p_win is None else p_win.data_ptr(),
            n, h, w, use_kx4, use_ky4, o["gauss"].data_ptr(), o["status"].data_ptr(), o["init"].data_ptr(),
            o["gain"].data_ptr(), o["N0"].data_ptr(), o["b4x"].data_ptr(), o["b4y"].data_ptr(),
            o["cost_per_pt"].data_ptr(), o["n_valid"].data_ptr(), o["iters"].data_ptr(), o["conv"].data_ptr(),
            scratch.data_ptr(), scratch.numel(), self._stream()), "kspace fit")
        return o
