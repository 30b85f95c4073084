"""The reference's instantaneous multipass on the CPU (TEST / BASELINE INFRASTRUCTURE).

Runs the pass loop of the reference driver (pivtools_cli/piv/piv_backend/
cpu_instantaneous.py:381-927 and :995-1133) over the reference's own C libraries
compiled from its sources (`_ref/libbulkxcorr2d_ref.so`, `_ref/libfusedwarp_ref.so`,
built by `make -C oracle ref`), for a batch of image pairs in one call per
library, as the driver does:

  pass 0      bulkxcorr2d on the raw frames;
  pass k > 0  Gaussian smoothing of the padded predictor (scipy gaussian_filter,
              mode 'nearest', :1040-1048), cv2.remap of it to this pass's window
              centres (INTER_CUBIC, BORDER_REPLICATE, :1050-1071),
              fused_symmetric_warp_batch of both frames (:1112), bulkxcorr2d;
  every pass  the large-displacement gate, predictor addition, peak-magnitude and
              normalised-median outliers (:575-760; outlier_detection.py:56-243),
              least-squares infilling (infilling.py:200-283, harmonic or
              biharmonic), edge padding onto the padded grid (:836-860).

The glue between the library calls is this module's restatement of the
driver's NumPy/SciPy code (the same library calls where the driver makes them:
scipy.ndimage.gaussian_filter, cv2.remap, scipy.sparse splu).  Used by bench.py's
reference arm and CPU baseline; never by the product.
"""

from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)
import oracle as O  # noqa: E402


def set_threads(n: int) -> None:
    """Set the OpenMP thread count of the reference libraries (libgomp is shared
    by every library loaded in this process)."""
    try:
        ctypes.CDLL("libgomp.so.1").omp_set_num_threads(int(n))
    except OSError:
        os.environ["OMP_NUM_THREADS"] = str(int(n))


# ---------------------------------------------------------------------------
# Least-squares infilling (infilling.py:150-283): minimise the sum of squared
# finite differences of order 1 (harmonic) or 2 (biharmonic) along y and x, in
# physical units, over the fill nodes with every known node fixed; equations
# touching an excluded node are dropped; normal equations solved by sparse LU.
# ---------------------------------------------------------------------------

def _difference_operator(ny, nx, pitch, order):
    import scipy.sparse as sp

    coef = {1: (-1.0, 1.0), 2: (1.0, -2.0, 1.0)}[order]
    idx = np.arange(ny * nx).reshape(ny, nx)
    rows, cols, vals = [], [], []
    r0 = 0
    for axis, h in ((0, pitch[0]), (1, pitch[1])):
        n = (ny, nx)[axis]
        if n <= order:
            continue
        scale = 1.0 / h ** order
        taps = []
        for j in range(order + 1):
            taps.append(idx[j:n - order + j, :].ravel() if axis == 0 else idx[:, j:n - order + j].ravel())
        m = taps[0].size
        rr = r0 + np.arange(m)
        for t, c in zip(taps, coef):
            rows.append(rr)
            cols.append(t)
            vals.append(np.full(m, scale * c))
        r0 += m
    if r0 == 0:
        return sp.csr_matrix((0, ny * nx))
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(r0, ny * nx))


def fill_least_squares(fields, fill, pitch, order, exclude=None):
    """fields (K, ny, nx); fill, exclude (ny, nx) bool.  Returns float64 fields
    with the fill nodes solved; raises ValueError when a group of fill nodes has
    no equation reaching a known node, or no known node exists."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components
    from scipy.sparse.linalg import splu

    fields = np.asarray(fields, np.float64)
    fill = np.asarray(fill, bool)
    excl = np.zeros_like(fill) if exclude is None else np.asarray(exclude, bool)
    out = fields.copy()
    if not fill.any():
        return out
    known = ~fill & ~excl
    if not known.any():
        raise ValueError("least-squares fill: no known node")
    K, ny, nx = fields.shape
    L = _difference_operator(ny, nx, pitch, order)
    f, k, e = fill.ravel(), known.ravel(), excl.ravel()
    Lf = L[:, f].tocsr()
    keep = (np.diff(Lf.indptr) > 0) & ~(np.diff(L[:, e].tocsr().indptr) > 0)
    Lf = Lf[keep]
    Lk = L[:, k].tocsr()[keep]
    A = (Lf.T @ Lf).tocsc()
    n_groups, group = connected_components(A, directed=False)
    anchored = np.zeros(n_groups, bool)
    anchored[np.unique(group[Lf[np.diff(Lk.indptr) > 0].indices])] = True
    if not anchored.all():
        raise ValueError("least-squares fill: a group of fill nodes is not linked to a known node")
    rhs = Lf.T @ (-(Lk @ fields[:, known].T))
    X = np.asarray(splu(A).solve(np.asarray(rhs))).reshape(-1, K)
    out[:, fill] = X.T
    return out


# ---------------------------------------------------------------------------
# Validation between passes (cpu_instantaneous.py:575-760, one peak)
# ---------------------------------------------------------------------------

def fill_nearest(fields, fill, pitch, exclude=None):
    """Nearest-donor fill of a (K, ny, nx) stack sharing one fill pattern
    (infilling.py:114-141): every fill cell takes the values of the nearest cell,
    in physical distance, that is neither filled nor excluded and finite in every
    field, through scipy's Euclidean feature transform as the reference calls it."""
    from scipy import ndimage as ndi

    fields = np.asarray(fields, np.float64)
    fill = np.asarray(fill, bool)
    exclude = np.zeros_like(fill) if exclude is None else np.asarray(exclude, bool)
    out = fields.copy()
    if not fill.any():
        return out
    donor = ~fill & ~exclude & np.all(np.isfinite(fields), axis=0)
    if not donor.any():
        raise ValueError("no donor for the nearest fill")
    iy, ix = ndi.distance_transform_edt(~donor, sampling=pitch, return_distances=False, return_indices=True)
    out[:, fill] = fields[:, iy, ix][:, fill]
    return out


def _nanmedian_last(a):
    """Median over the last axis ignoring NaN; rows without NaN go through the
    partition-based np.median (the reference uses bottleneck's nanmedian, which
    numpy's masked-sort nanmedian is many times slower than), the few grid-edge
    rows with NaN through np.nanmedian."""
    with np.errstate(all="ignore"):
        out = np.median(a, axis=-1)
        holes = np.isnan(a).any(axis=-1)
        if holes.any():
            out[holes] = np.nanmedian(a[holes], axis=-1)
    return out.astype(np.float32)


def median_flags(zx, zy, eps=0.1, thr=2.0, size=5):
    """Normalised-median outliers of (N, ny, nx) fields (outlier_detection.py:87-243)
    on the zero-filled fields, vectorised over windows: the size x size
    neighbourhood without the node (cells beyond the grid excluded), residual
    norm over the median neighbour residual norm + eps, non-finite flagged, and
    the 3x3 presence guard (fewer than 6 present cells flagged)."""
    from numpy.lib.stride_tricks import sliding_window_view

    h = size // 2
    N, ny, nx = zx.shape
    pad = ((0, 0), (h, h), (h, h))
    pu = np.pad(zx.astype(np.float32), pad, constant_values=np.nan)
    pv = np.pad(zy.astype(np.float32), pad, constant_values=np.nan)
    centre = size * size // 2
    sel = np.r_[0:centre, centre + 1:size * size]
    nu = sliding_window_view(pu, (size, size), axis=(1, 2)).reshape(N, ny, nx, -1)[..., sel]
    nv = sliding_window_view(pv, (size, size), axis=(1, 2)).reshape(N, ny, nx, -1)[..., sel]
    with np.errstate(all="ignore"):
        mu = _nanmedian_last(nu)
        mv = _nanmedian_last(nv)
        r0 = np.sqrt((zx - mu) ** 2 + (zy - mv) ** 2)
        ri = np.sqrt((nu - mu[..., None]) ** 2 + (nv - mv[..., None]) ** 2)
        rm = _nanmedian_last(ri)
        nr = r0 / (rm + np.float32(eps))
        flag = ~np.isfinite(nr) | (nr > thr)
    present = np.pad((np.isfinite(zx) & np.isfinite(zy)).astype(np.int32), ((0, 0), (1, 1), (1, 1)))
    n_present = sum(present[:, 1 + dr:1 + dr + ny, 1 + dc:1 + dc + nx] for dr in (-1, 0, 1) for dc in (-1, 0, 1))
    return flag | (n_present < 6)


def validate(pk_x, pk_y, pk_h, pred_dy, pred_dx, thresh_x, thresh_y, peak_thr=0.25, eps=0.1, med_thr=2.0, size=5):
    """(N, ny, nx) primary-peak outputs -> (ux, uy, invalid) with NaN at invalid."""
    x = pk_x.astype(np.float32).copy()
    y = pk_y.astype(np.float32).copy()
    h = pk_h.astype(np.float32).copy()
    with np.errstate(invalid="ignore"):
        gone = (np.abs(x) > thresh_x) | (np.abs(y) > thresh_y)
    x[gone] = np.nan
    y[gone] = np.nan
    h[gone] = np.nan
    if pred_dx is not None:
        x = x + pred_dx
        y = y + pred_dy
    bad = np.isnan(x) | np.isnan(y)
    zx = np.where(bad, np.float32(0), x)
    zy = np.where(bad, np.float32(0), y)
    with np.errstate(invalid="ignore"):
        out = (h < peak_thr) | np.isnan(h)
    if med_thr > 0:
        out |= median_flags(zx, zy, eps, med_thr, size)
    bad |= out
    return np.where(bad, np.float32(np.nan), zx), np.where(bad, np.float32(np.nan), zy), bad


def sigma_flags(ux, uy, thr):
    """Local 8-neighbour sigma test on the vector norm, per (ny, nx) field
    (outlier_detection.py:246-319, combine 'norm')."""
    from scipy import ndimage as ndi

    v = np.sqrt(ux ** 2 + uy ** 2).astype(np.float32)
    finite = np.isfinite(v).astype(np.float32)
    v0 = np.where(np.isfinite(v), v, np.float32(0.0))
    sum9 = ndi.uniform_filter(v0, size=3, mode="constant", cval=0.0) * 9.0
    sumsq9 = ndi.uniform_filter(v0 * v0, size=3, mode="constant", cval=0.0) * 9.0
    cnt9 = ndi.uniform_filter(finite, size=3, mode="constant", cval=0.0) * 9.0
    sum8 = sum9 - v0
    sumsq8 = sumsq9 - v0 * v0
    cnt8 = cnt9 - finite
    with np.errstate(invalid="ignore", divide="ignore"):
        mean8 = sum8 / cnt8
        var8 = (sumsq8 / cnt8) - mean8 * mean8
    std8 = np.sqrt(np.maximum(var8, 0.0))
    with np.errstate(invalid="ignore"):
        return ((np.abs(v - mean8) > thr * std8) | ~np.isfinite(v) | ~np.isfinite(mean8) | (std8 == 0)
                | (cnt8 < 1))


def divvort_flags(ux, uy, div_thresh=None, vort_thresh=None):
    """Divergence/vorticity test of one (ny, nx) field (outlier_detection.py:322-380):
    periodic central differences, thresholds 6 x 1.4826 x MAD unless given."""
    dudx = 0.5 * (np.roll(ux, -1, 1) - np.roll(ux, 1, 1))
    dudy = 0.5 * (np.roll(ux, -1, 0) - np.roll(ux, 1, 0))
    dvdx = 0.5 * (np.roll(uy, -1, 1) - np.roll(uy, 1, 1))
    dvdy = 0.5 * (np.roll(uy, -1, 0) - np.roll(uy, 1, 0))
    div = dudx + dvdy
    vort = dvdx - dudy

    def thresh(f, given):
        if given is not None:
            return given
        fin = f[np.isfinite(f)]
        if fin.size == 0:
            return np.inf
        med = np.median(fin)
        return 6 * (1.4826 * np.median(np.abs(fin - med)))

    with np.errstate(invalid="ignore"):
        return (np.abs(div) > thresh(div, div_thresh)) | (np.abs(vort) > thresh(vort, vort_thresh))


def validate_peaks(pk_x, pk_y, pk_h, pred_dy, pred_dx, thresh_x, thresh_y, secondary=True, peak_thr=0.25,
                   eps=0.1, med_thr=2.0, size=5, sigma_thr=0.0, divvort=False, div_thr=None, vort_thr=None):
    """(N, P, ny, nx) peak outputs -> (ux, uy, invalid, reason, choice): the driver's
    validation with several peaks and the secondary-peak substitution
    (cpu_instantaneous.py:589-760; no masked windows), in its order of steps: gate
    and predictor on every peak, primary outlier tests on the zero-filled field,
    then per round the next peak for every invalid vector with peaks left, judged
    afresh and tested on the field of the current choices (NaN cells drop out of
    the medians), then the NaN-height and unclassified codes."""
    x = pk_x.astype(np.float32).copy()
    y = pk_y.astype(np.float32).copy()
    h = pk_h.astype(np.float32).copy()
    N, P, ny, nx = x.shape
    with np.errstate(invalid="ignore"):
        large = (np.abs(x) > thresh_x) | (np.abs(y) > thresh_y)
    fit_fail0 = np.isnan(x[:, 0]) | np.isnan(y[:, 0])
    large0 = large[:, 0]
    x[large] = np.nan
    y[large] = np.nan
    h[large] = np.nan
    if pred_dx is not None:
        x += pred_dx[:, None]
        y += pred_dy[:, None]
    ux = x[:, 0].copy()
    uy = y[:, 0].copy()
    nan_mask = np.isnan(ux) | np.isnan(uy)
    ux[nan_mask] = 0.0
    uy[nan_mask] = 0.0
    choice = np.ones((N, ny, nx), np.intp)
    reason = np.zeros((N, ny, nx), np.int8)
    reason[fit_fail0] = 1
    reason[large0] = 6

    def outliers(fx, fy, pm):
        with np.errstate(invalid="ignore"):
            o = (pm < peak_thr) | np.isnan(pm) if peak_thr >= 0 else np.zeros(fx.shape, bool)
        if med_thr > 0:
            o = o | median_flags(fx, fy, eps, med_thr, size)
        for n in range(fx.shape[0]):
            if sigma_thr > 0:
                o[n] |= sigma_flags(fx[n], fy[n], sigma_thr)
            if divvort:
                o[n] |= divvort_flags(fx[n], fy[n], div_thr, vort_thr)
        return o

    out = outliers(ux, uy, h[:, 0])
    nan_mask |= out
    reason[out & (reason == 0)] = 10
    if secondary:
        for _ in range(1, P):
            active = nan_mask & (choice < P)
            if not active.any():
                break
            choice[active] += 1
            idx = choice[:, None] - 1
            ux = np.take_along_axis(x, idx, axis=1)[:, 0]
            uy = np.take_along_axis(y, idx, axis=1)[:, 0]
            sub_nan = np.isnan(ux) | np.isnan(uy)
            nan_mask[active] = sub_nan[active]
            reason[active] = np.where(sub_nan[active], 13, 0)
            pm = np.take_along_axis(h, idx, axis=1)[:, 0]
            re = active & outliers(ux, uy, pm) & ~sub_nan
            nan_mask |= re
            reason[re] = 12
    pm = np.take_along_axis(h, choice[:, None] - 1, axis=1)[:, 0]
    nan_mask |= np.isnan(pm)
    reason[np.isnan(pm) & (reason == 0)] = 13
    reason[nan_mask & (reason == 0)] = 9
    ux = np.where(nan_mask, np.float32(np.nan), ux).astype(np.float32)
    uy = np.where(nan_mask, np.float32(np.nan), uy).astype(np.float32)
    choice[nan_mask] = 0
    return ux, uy, nan_mask, reason, choice


# ---------------------------------------------------------------------------
# The pass loop
# ---------------------------------------------------------------------------

class RefMultipass:
    """The reference's multipass for batches of pairs of one image shape.

    geo: the pass geometries (pivtools_b200.geometry.multipass_geometry: window
    grids, padded predictor grids, remap maps, smoothing widths) -- the
    reference's base.py:136-482 restated.  infill: 'biharmonic' (the reference's
    default, config.yaml:60-66) or 'harmonic'."""

    def __init__(self, geo, window_type="gaussian", peak_finder=3, infill="biharmonic", final_infill=True,
                 smoothing=True, n_peaks=1, secondary_peak=False, interp_mode=0):
        self.bulk = O.ref_bulk()
        self.warp = O.ref_warp()
        if self.bulk is None or self.warp is None:
            raise RuntimeError("the reference libraries are not built (make -C oracle ref PIVTOOLS_REF=...)")
        import cv2  # noqa: F401  (the driver's predictor remap)

        from pivtools_b200 import geometry

        self.geo = geo
        self.weights = [geometry.window_weight(g.window_size, window_type) for g in geo]
        self.finder = peak_finder
        self.order = {"nearest": 0, "harmonic": 1, "biharmonic": 2}[infill]
        self.final_infill = final_infill
        self.smoothing = smoothing
        self.n_peaks = n_peaks
        self.secondary = secondary_peak
        self.interp_mode = interp_mode            # 0 bicubic, 1 Lanczos-3 (image_warp_interpolation)
        self.warp.fused_warp_set_impl(1)        # the SIMD route, the reference's default

    def run(self, A, B):
        """A, B: (N, H, W) float32.  Returns the final pass's (ux, uy) (N, ny, nx)."""
        import cv2
        from scipy.ndimage import gaussian_filter

        A = np.ascontiguousarray(A, np.float32)
        B = np.ascontiguousarray(B, np.float32)
        N, H, W = A.shape
        old = None
        self.history = []          # per pass: (ux, uy, invalid) after validation and infilling
        for k, (g, w) in enumerate(zip(self.geo, self.weights)):
            ny, nx = g.grid.n_win_y, g.grid.n_win_x
            pdy = pdx = None
            fa, fb = A, B
            if k > 0:
                prev = self.geo[k - 1]
                if self.smoothing and g.sd > 0:
                    tr = (g.ksize_filt[0] - 1) / (2 * g.sd)
                    for i in range(N):
                        for d in range(2):
                            old[i, ..., d] = gaussian_filter(old[i, ..., d], sigma=g.sd, truncate=tr, mode="nearest")
                pdy = np.empty((N, ny, nx), np.float32)
                pdx = np.empty((N, ny, nx), np.float32)
                for i in range(N):
                    pdy[i] = cv2.remap(old[i, ..., 0], g.pred_map_x, g.pred_map_y, cv2.INTER_CUBIC,
                                       borderMode=cv2.BORDER_REPLICATE)
                    pdx[i] = cv2.remap(old[i, ..., 1], g.pred_map_x, g.pred_map_y, cv2.INTER_CUBIC,
                                       borderMode=cv2.BORDER_REPLICATE)
                fa = np.zeros_like(A)
                fb = np.zeros_like(B)
                ody = np.ascontiguousarray(old[..., 0])
                odx = np.ascontiguousarray(old[..., 1])
                if self.warp.fused_symmetric_warp_batch(A, B, fa, fb, ody, odx, N, H, W, ody.shape[1], ody.shape[2],
                                                        prev.ctrs_y_all, prev.ctrs_x_all, self.interp_mode, 0, 0) != 0:
                    raise RuntimeError("reference fused_symmetric_warp_batch failed")
            mask = np.zeros((ny, nx), np.float32)
            r = O.ref_bulkxcorr2d(fa, fb, mask, g.grid.win_ctrs_x, g.grid.win_ctrs_y, g.window_size, w, w,
                                  n_peaks=self.n_peaks, peak_finder=self.finder)
            if r["error"]:
                raise RuntimeError(f"reference bulkxcorr2d error {r['error']}")
            div = 2.0 if k == 0 else 4.0
            if self.n_peaks > 1:
                ux, uy, bad, _, _ = validate_peaks(r["pk_x"], r["pk_y"], r["pk_h"], pdy, pdx, g.window_size[1] / div,
                                                   g.window_size[0] / div, secondary=self.secondary)
            else:
                ux, uy, bad = validate(r["pk_x"][:, 0], r["pk_y"][:, 0], r["pk_h"][:, 0], pdy, pdx,
                                       g.window_size[1] / div, g.window_size[0] / div)
            last = k + 1 == len(self.geo)
            if not last or self.final_infill:
                pitch = (float(g.grid.win_spacing_y), float(g.grid.win_spacing_x))
                for i in range(N):
                    if bad[i].any():
                        if self.order == 0:
                            f = fill_nearest(np.stack([ux[i], uy[i]]), bad[i], pitch).astype(np.float32)
                        else:
                            f = fill_least_squares(np.stack([ux[i], uy[i]]), bad[i], pitch, self.order)
                        ux[i], uy[i] = f[0], f[1]
            self.history.append((ux.copy(), uy.copy(), bad.copy()))
            if not last:
                (py0, px0), (py1, px1) = g.n_pre, g.n_post
                old = np.pad(np.stack([uy, ux], axis=-1), ((0, 0), (py0, py1), (px0, px1), (0, 0)), mode="edge")
        return ux, uy
