"""Window geometry and weights of the PIVtools correlation path (host logic).

Restates the reference's interrogation-grid rules so that the GPU path receives
exactly the arrays the reference drivers pass to its C libraries:

* window centres: pivtools_core/window_utils.py:142-274 (compute_window_centers),
  and for ensemble single mode window_utils.py:79-128, 276-525
  (compute_padding_for_single_mode, compute_window_centers_single_mode)
* window weights: pivtools_cli/piv/piv_backend/base.py:52-134 (_window_weight_fun)
* padded predictor grids and smoothing kernels: base.py:136-318
  (_cache_window_padding_unified)
* predictor remap coordinates: base.py:404-482 (_cache_interpolation_grids_unified)
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

BUILT_FFT_SIZES = (8, 12, 16, 24, 32, 48, 64, 96, 128)  # pivtools_core/fft_sizes.py:16


@dataclass
class WindowGrid:
    win_ctrs_x: np.ndarray
    win_ctrs_y: np.ndarray
    n_win_x: int
    n_win_y: int
    win_spacing_x: int
    win_spacing_y: int


def compute_window_centers(image_shape, window_size, overlap) -> WindowGrid:
    """Centres of the full windows that fit the image (window_utils.py:142-255).

    x centres start at (w-1)/2; y centres are anchored to the bottom edge and
    returned ascending.
    """
    H, W = image_shape
    wh, ww = window_size
    if wh > H or ww > W:
        raise ValueError(f"Window size {window_size} exceeds image dimensions {image_shape}")
    if overlap < 0 or overlap >= 100:
        raise ValueError(f"Overlap must be in range [0, 100), got {overlap}")
    sx = max(1, round((1 - overlap / 100) * ww))
    sy = max(1, round((1 - overlap / 100) * wh))
    fx, lx = (ww - 1) / 2.0, W - (ww + 1) / 2.0
    fy, ly = (wh - 1) / 2.0, H - (wh + 1) / 2.0
    nx = max(1, int(np.floor((lx - fx) / sx)) + 1)
    ny = max(1, int(np.floor((ly - fy) / sy)) + 1)
    cx = np.linspace(fx, fx + sx * (nx - 1), nx, dtype=np.float32)
    cy = np.linspace(ly - sy * (ny - 1), ly, ny, dtype=np.float32)
    return WindowGrid(cx, cy, nx, ny, sx, sy)


def compute_padding_for_single_mode(window_size, sum_window):
    """(top, bottom, left, right) zero padding that lets the sum window sit around
    every small window (window_utils.py:79-128): ceil on top/left, floor on
    bottom/right of half the size difference."""
    dh, dw = sum_window[0] - window_size[0], sum_window[1] - window_size[1]
    return (int(np.ceil(dh / 2)), int(np.floor(dh / 2)), int(np.ceil(dw / 2)), int(np.floor(dw / 2)))


def compute_window_centers_single_mode(image_shape, window_size, sum_window, overlap):
    """Ensemble single-mode grid (window_utils.py:276-463): spacing from the small
    window, centres in the coordinates of the zero-padded frame (the small
    window's standard-mode centres shifted by the padding; y anchored to the
    bottom and ascending).  Returns (WindowGrid in padded coordinates, padding)."""
    H, W = image_shape
    wh, ww = window_size
    sh, sw = sum_window
    if sh < wh or sw < ww:
        raise ValueError(f"SumWindow {tuple(sum_window)} must be >= window_size {tuple(window_size)} for single mode")
    if wh > H or ww > W:
        raise ValueError(f"Window size {window_size} exceeds image dimensions {image_shape}")
    if overlap < 0 or overlap >= 100:
        raise ValueError(f"Overlap must be in range [0, 100), got {overlap}")
    pt, pb, pl, pr = compute_padding_for_single_mode(window_size, sum_window)
    Nx, Ny = W + pl + pr, H + pt + pb
    sx = max(1, round((1 - overlap / 100) * ww))
    sy = max(1, round((1 - overlap / 100) * wh))
    fx, fy = pl + (ww - 1) / 2.0, pt + (wh - 1) / 2.0
    lx, ly = pl + W - (ww + 1) / 2.0, pt + H - (wh + 1) / 2.0
    nx = max(1, int(np.floor((lx - fx) / sx)) + 1)
    ny = max(1, int(np.floor((ly - fy) / sy)) + 1)
    cx = np.linspace(fx, fx + sx * (nx - 1), nx, dtype=np.float32)
    cy = np.linspace(ly - sy * (ny - 1), ly, ny, dtype=np.float32)
    if cx[-1] + (sw - 1) / 2.0 >= Nx or cy[-1] + (sh - 1) / 2.0 >= Ny:
        raise ValueError("Single mode window centers exceed padded image bounds")
    return WindowGrid(cx, cy, nx, ny, sx, sy), (pt, pb, pl, pr)


def compute_vector_masks(pixel_mask, image_shape, window_sizes, overlaps, threshold=0.5):
    """Per-pass masked-window flags (n_win_y, n_win_x) from a boolean pixel mask
    (H, W) (load_images.py:827-990, standard passes): a window is masked when the
    masked pixels inside its footprint [floor(c - (w-1)/2 + 0.5),
    floor(c + (w-1)/2 + 0.5)], clipped to the image, exceed threshold * h * w.
    Counts come from an integral image (exact integers)."""
    H, W = image_shape
    m = np.asarray(pixel_mask, bool)
    if m.shape != (H, W):
        raise ValueError(f"pixel mask shape {m.shape} is not the image shape {(H, W)}")
    S = np.zeros((H + 1, W + 1), np.int64)
    S[1:, 1:] = np.cumsum(np.cumsum(m, axis=0, dtype=np.int64), axis=1)
    out = []
    for (wy, wx), ov in zip(window_sizes, overlaps):
        g = compute_window_centers(image_shape, (wy, wx), ov)
        hy, hx = (wy - 1) / 2.0, (wx - 1) / 2.0
        cy = g.win_ctrs_y.astype(np.float64)
        cx = g.win_ctrs_x.astype(np.float64)
        y0 = np.clip(np.floor(cy - hy + 0.5).astype(np.int64), 0, H)
        y1 = np.clip(np.floor(cy + hy + 0.5).astype(np.int64) + 1, 0, H)
        x0 = np.clip(np.floor(cx - hx + 0.5).astype(np.int64), 0, W)
        x1 = np.clip(np.floor(cx + hx + 0.5).astype(np.int64) + 1, 0, W)
        cnt = (S[y1[:, None], x1[None, :]] - S[y0[:, None], x1[None, :]] - S[y1[:, None], x0[None, :]]
               + S[y0[:, None], x0[None, :]])
        ok = (y1 > y0)[:, None] & (x1 > x0)[None, :]
        out.append(ok & (cnt / (wy * wx) > threshold))
    return out


def window_weight(wsize, window_type: str, sum_window=None) -> np.ndarray:
    """2-D correlation weighting window (base.py:52-134), float32."""
    m, n = wsize
    t = window_type.lower()
    if t == "blackman":
        a0, a1, a2 = 0.42659, 0.49656, 0.076849
        dmax = np.sqrt(((m + 1) / 2) ** 2 + ((n + 1) / 2) ** 2)
        ii, jj = np.meshgrid(np.arange(m), np.arange(n), indexing="ij")
        d = np.sqrt((ii - (m - 1) / 2) ** 2 + (jj - (n - 1) / 2) ** 2)
        th = d / dmax * np.pi + np.pi
        w = (a0 - a1 * np.cos(th) + a2 * np.cos(2 * th)).astype(np.float32)
        w[w <= 0] = 0.01
        return w
    if t == "square":
        return np.ones((m, n), np.float32)
    if t == "bsingle":
        if sum_window is None:
            raise ValueError("SumWindow must be provided for 'bsingle'")
        return np.ones(sum_window, np.float32)
    if t in ("gaussian", "gaussiantop"):
        wx = np.arange(-m / 2 + 0.5, m / 2, dtype=np.float32)
        wy = np.arange(-n / 2 + 0.5, n / 2, dtype=np.float32)
        xm, ym = np.meshgrid(wx, wy, indexing="ij")
        w = np.exp(-0.5 * ((xm / np.float32(m / 2)) ** 2 + (ym / np.float32(n / 2)) ** 2))
        w = w.astype(np.float32)
        if t == "gaussiantop":
            if m > 6 and n > 6:
                c = np.tile(np.array([[1, 0], [0, 0]], np.float32), (m // 2, n // 2))
                c = np.roll(np.roll(c, int(np.ceil(m / 4)), axis=0), int(np.ceil(n / 4)), axis=1)
            else:
                c = np.zeros((m, n), np.float32)
                c[m // 2 - 1: m // 2 + 3, n // 2 - 1: n // 2 + 3] = 1
            w = w * c
        return np.ascontiguousarray(w, np.float32)
    if t == "singlepix":
        if sum_window is None:
            raise ValueError("SumWindow must be provided for 'singlepix'")
        w = np.zeros(sum_window, np.float32)
        r0 = int(np.ceil((sum_window[0] - m) / 2))
        c0 = int(np.ceil((sum_window[1] - n) / 2))
        w[r0:r0 + m, c0:c0 + n] = 1.0
        return w
    raise ValueError(f"Unrecognized window type '{window_type}'")


def _pad_axis(ctrs: np.ndarray, spacing: int, size: int):
    """Padded centres before/after the grid, at least two on each side (base.py:198-240)."""
    pre = np.arange(1, ctrs[0] - spacing / 2, spacing)
    if pre.size == 0:
        pre = np.array([1])
    pre = pre - 1
    while len(pre) < 2:
        pre = np.concatenate([[max(0, pre[0] - spacing)], pre])
    post = np.arange(size, ctrs[-1] + spacing / 2, -spacing)
    if post.size == 0:
        post = np.array([size])
    post = post - 1
    while len(post) < 2:
        post = np.concatenate([post, [min(size - 1, post[-1] + spacing)]])
    allc = np.concatenate([pre, ctrs, post[::-1]])
    return allc.astype(np.float32), len(pre), len(post)


@dataclass
class PassGeometry:
    window_size: tuple
    overlap: float
    grid: WindowGrid
    ctrs_x_all: np.ndarray     # padded centres (predictor grid of this pass)
    ctrs_y_all: np.ndarray
    n_pre: tuple               # (y, x)
    n_post: tuple
    ksize_filt: tuple
    sd: float
    pred_map_x: np.ndarray | None = None   # fractional index of this pass's centres
    pred_map_y: np.ndarray | None = None   # on the previous pass's padded grid


def multipass_geometry(image_shape, window_sizes, overlaps, window_type="gaussian",
                       first_pass_ksize=(0, 0)):
    """Per-pass grids of the instantaneous multipass driver (instantaneous mode:
    first-pass smoothing kernel (0, 0); base.py:136-318, 404-482)."""
    H, W = image_shape
    out: list[PassGeometry] = []
    for k, (ws, ov) in enumerate(zip(window_sizes, overlaps)):
        g = compute_window_centers((H, W), tuple(ws), ov)
        ax, pre_x, post_x = _pad_axis(g.win_ctrs_x.astype(np.float64), g.win_spacing_x, W)
        ay, pre_y, post_y = _pad_axis(g.win_ctrs_y.astype(np.float64), g.win_spacing_y, H)
        if k == 0:
            ks = tuple(first_pass_ksize)
            sd = 0.0 if ks == (0, 0) else float(np.sqrt(np.prod(ks)) / 3 * 0.65)
        else:
            prev = out[-1]
            kf = np.round(np.array(window_sizes[k - 1]) /
                          np.array((prev.grid.win_spacing_y, prev.grid.win_spacing_x))).astype(int) + 1
            kf = [int(v) for v in kf.tolist()]
            ks = (kf[0] + (kf[0] % 2 == 0), kf[1] + (kf[1] % 2 == 0))
            sd = float(np.sqrt(np.prod(ks)) / 3 * 0.65)
        pg = PassGeometry(tuple(ws), ov, g, ax, ay, (pre_y, pre_x), (post_y, post_x), ks, sd)
        if k > 0:
            prev = out[-1]
            px, py = prev.ctrs_x_all, prev.ctrs_y_all
            wy, wx = np.meshgrid(g.win_ctrs_y, g.win_ctrs_x, indexing="ij")
            pg.pred_map_x = np.interp(wx.ravel(), px, np.arange(len(px))).reshape(wx.shape).astype(np.float32)
            pg.pred_map_y = np.interp(wy.ravel(), py, np.arange(len(py))).reshape(wy.shape).astype(np.float32)
        out.append(pg)
    return out


def nearest_donor_map(mask, spacing):
    """Flat index of each window's donor for the 'nearest' predictor fill of the
    masked windows (infilling.py:114-141, 808-874): the nearest unmasked window in
    physical distance (pitch (py, px) in pixels), chosen among equidistant donors
    as scipy's Euclidean distance transform chooses; every unmasked window maps to
    itself.  Computed once per pass geometry on the host (the mask is shared by all
    pairs); the fill itself is a gather on the GPU (pivb_gather_fill_dev)."""
    from scipy import ndimage as ndi

    m = np.asarray(mask, bool)
    ny, nx = m.shape
    donor = ~m
    if not donor.any():
        raise ValueError("every window is masked: no donor for the nearest fill")
    iy, ix = ndi.distance_transform_edt(~donor, sampling=(float(spacing[0]), float(spacing[1])),
                                       return_distances=False, return_indices=True)
    idx = (iy * nx + ix).astype(np.int32)
    idx[donor] = np.flatnonzero(donor).astype(np.int32)
    return idx.reshape(ny, nx)
