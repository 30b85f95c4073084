"""Seeded inputs of the correlator fixtures (xcorr_ref.npz).

`make_golden.py xcorr` runs each case through the reference's own libbulkxcorr2d
(compiled from its sources under oracle/_ref) and stores the outputs; the tests
rebuild the same inputs here and run them through the oracle and the GPU C-ABI.
Inputs are rebuilt, not stored: each case's frames are checked against a stored
float64 checksum first, so a change of the generator fails loudly instead of
comparing different images.
"""

from __future__ import annotations

import numpy as np

from pivtools_b200 import geometry, synthetic

SIZES = (8, 12, 16, 24, 32, 48, 64, 96, 128)
OUT_KEYS = ("pk_x", "pk_y", "pk_h", "sx", "sy", "sxy", "pk_ratio")


def _grid(shape, win, overlap):
    g = geometry.compute_window_centers(shape, win, overlap)
    return np.asarray(g.win_ctrs_x, np.float32), np.asarray(g.win_ctrs_y, np.float32)


def _case(name, A, B, cx, cy, win, wa, wb, mask=None, finder=3, n_peaks=1, ensemble=False, impl=0,
          plane_idx=None):
    ny, nx = len(cy), len(cx)
    if A.ndim == 2:
        A, B = A[None], B[None]
    return dict(name=name, A=np.ascontiguousarray(A, np.float32), B=np.ascontiguousarray(B, np.float32),
                cx=cx, cy=cy, win=tuple(win), wa=np.ascontiguousarray(wa, np.float32),
                wb=np.ascontiguousarray(wb, np.float32),
                mask=np.zeros((ny, nx), np.float32) if mask is None else np.asarray(mask, np.float32),
                finder=finder, n_peaks=n_peaks, ensemble=ensemble, impl=impl,
                plane_idx=np.arange(0) if plane_idx is None else np.asarray(plane_idx, np.int64))


def config1_cases():
    """The single-pair workload at full size: one 1024^2 pair (seed 1), 32 px
    gaussian-weighted windows at 50% (63 x 63), 3-point and LM fits."""
    A, B, _ = synthetic.particle_pair((1024, 1024), seed=1)
    cx, cy = _grid(A.shape, (32, 32), 50)
    w = geometry.window_weight((32, 32), "gaussian")
    idx = np.arange(0, len(cx) * len(cy), 62)
    out = [_case("c1_g3", A, B, cx, cy, (32, 32), w, w, finder=3, plane_idx=idx)]
    for f in (4, 5, 6):
        out.append(_case(f"c1_g{f}", A, B, cx, cy, (32, 32), w, w, finder=f))
    out.append(_case("c1_g6_batch", A, B, cx, cy, (32, 32), w, w, finder=6, impl=1))
    return out


def size_cases():
    """Every built window size on a small pair: 3-point and gauss5 fits, the
    corner window masked, planes of the first eight windows."""
    out = []
    for n in SIZES:
        side = max(160, 3 * n)
        A, B, _ = synthetic.particle_pair((side, side + 16), seed=300 + n)
        cx, cy = _grid(A.shape, (n, n), 50)
        wt = "blackman" if n in (24, 96) else "gaussian"
        w = geometry.window_weight((n, n), wt)
        mask = np.zeros((len(cy), len(cx)), np.float32)
        mask[0, 0] = 1.0
        out.append(_case(f"n{n}_g3", A, B, cx, cy, (n, n), w, w, mask=mask, finder=3, plane_idx=np.arange(8)))
        out.append(_case(f"n{n}_g5", A, B, cx, cy, (n, n), w, w, mask=mask, finder=5))
    return out


def feature_cases():
    """Multiple peaks, ensemble mode (no mean subtraction), two pairs in one call,
    square and asymmetric weights."""
    out = []
    A, B, _ = synthetic.particle_pair((192, 208), seed=41)
    cx, cy = _grid(A.shape, (32, 32), 50)
    wg = geometry.window_weight((32, 32), "gaussian")
    ws = geometry.window_weight((32, 32), "square")
    out.append(_case("peaks3_g3", A, B, cx, cy, (32, 32), wg, wg, finder=3, n_peaks=3))
    out.append(_case("peaks2_g6", A, B, cx, cy, (32, 32), wg, wg, finder=6, n_peaks=2))
    out.append(_case("ensemble_g3", A, B, cx, cy, (32, 32), ws, ws, finder=3, ensemble=True,
                     plane_idx=np.arange(4)))
    out.append(_case("asym_w_g3", A, B, cx, cy, (32, 32), ws, wg, finder=3, plane_idx=np.arange(4)))
    A2, B2, _ = synthetic.particle_pair((192, 208), seed=42, flow="uniform", flow_kwargs=dict(u=-2.4, v=5.3))
    out.append(_case("two_pairs_g4", np.stack([A, A2]), np.stack([B, B2]), cx, cy, (32, 32), wg, wg, finder=4))
    return out


def edge_cases():
    """The reference's edge handling: windows reaching outside the frame are
    skipped (outputs stay at the caller's zeros), a NaN inside a window, a window
    of zeros (zero energy), a random 10% of windows masked."""
    out = []
    A, B, _ = synthetic.particle_pair((160, 176), seed=51)
    cx, cy = _grid(A.shape, (32, 32), 50)
    cx_o = np.concatenate([[-20.0, 3.0], cx, [A.shape[1] - 4.0, A.shape[1] + 30.0]]).astype(np.float32)
    cy_o = np.concatenate([[-9.0], cy, [A.shape[0] + 2.0]]).astype(np.float32)
    w = geometry.window_weight((32, 32), "gaussian")
    out.append(_case("oob_g3", A, B, cx_o, cy_o, (32, 32), w, w, finder=3))
    An, Bn = A.copy(), B.copy()
    An[40:44, 60:64] = np.nan
    out.append(_case("nan_g3", An, Bn, cx, cy, (32, 32), w, w, finder=3))
    out.append(_case("nan_g6", An, Bn, cx, cy, (32, 32), w, w, finder=6))
    Az, Bz = A.copy(), B.copy()
    Az[:64, :64] = 0.0
    Bz[:64, :64] = 0.0
    out.append(_case("zero_g3", Az, Bz, cx, cy, (32, 32), w, w, finder=3))
    rng = np.random.default_rng(53)
    mask = (rng.random((len(cy), len(cx))) < 0.1).astype(np.float32)
    out.append(_case("masked_g3", A, B, cx, cy, (32, 32), w, w, mask=mask, finder=3))
    return out


def rect_cases():
    """Rectangular windows (nWindowSize = {h, w} with h != w)."""
    out = []
    for h, wd in ((16, 32), (32, 16), (24, 48), (64, 32), (32, 128)):
        A, B, _ = synthetic.particle_pair((192, 256), seed=60 + h + wd)
        cx, cy = _grid(A.shape, (h, wd), 50)
        w = geometry.window_weight((h, wd), "gaussian")
        out.append(_case(f"rect{h}x{wd}_g3", A, B, cx, cy, (h, wd), w, w, finder=3, plane_idx=np.arange(4)))
        out.append(_case(f"rect{h}x{wd}_g6", A, B, cx, cy, (h, wd), w, w, finder=6))
    return out


def all_cases():
    return config1_cases() + size_cases() + feature_cases() + edge_cases() + rect_cases()


def checksum(case) -> float:
    a = np.nan_to_num(case["A"].astype(np.float64), nan=-1.0)
    b = np.nan_to_num(case["B"].astype(np.float64), nan=-1.0)
    return float(a.sum() + 2.0 * b.sum() + (a * np.arange(a.size).reshape(a.shape) % 7).sum())


# ----------------------------------------------------------------------------
# ensemble triple accumulation (PIV_2d_cross_correlate.c:627-833)
# ----------------------------------------------------------------------------

def triple_cases():
    """Four pairs at the ensemble workload's density, 16 px square windows at 75%
    (and 32 px gaussian at 50% with a 24 x 24 crop), every combination of
    bMeanSubtract and bPerPairNorm.  The fixture keeps every fifth window's sums
    (`keep`)."""
    frames = [synthetic.particle_pair((96, 112), seed=70 + k, density=0.02, flow="ensemble_rows")[:2]
              for k in range(4)]
    A = np.stack([f[0] for f in frames])
    B = np.stack([f[1] for f in frames])
    out = []
    cx, cy = _grid(A.shape[1:], (16, 16), 75)
    sq = geometry.window_weight((16, 16), "square")
    for ms in (0, 1):
        for pn in (0, 1):
            out.append(dict(name=f"t16_ms{ms}_pn{pn}", A=A, B=B, cx=cx, cy=cy, win=(16, 16), fit=None,
                            w=(sq, sq, sq, sq), ms=ms, pn=pn, keep=np.arange(0, len(cx) * len(cy), 5)))
    cx, cy = _grid(A.shape[1:], (32, 32), 50)
    g = geometry.window_weight((32, 32), "gaussian")
    sq = geometry.window_weight((32, 32), "square")
    out.append(dict(name="t32_crop_ms1_pn1", A=A, B=B, cx=cx, cy=cy, win=(32, 32), fit=(24, 24),
                    w=(g, sq, sq, sq), ms=1, pn=1, keep=np.arange(len(cx) * len(cy))))
    # ensemble single mode: 4 px particle windows at 50% inside a 16 px sum window,
    # zero-padded frames, singlepix frame-A weight, bsingle elsewhere, 12 x 12 crop
    grid, (pt, pb, pl, pr) = geometry.compute_window_centers_single_mode(A.shape[1:], (4, 4), (16, 16), 50)
    PA = np.pad(A, ((0, 0), (pt, pb), (pl, pr)))
    PB = np.pad(B, ((0, 0), (pt, pb), (pl, pr)))
    sp = geometry.window_weight((4, 4), "singlepix", (16, 16))
    bs = geometry.window_weight((16, 16), "bsingle", (16, 16))
    for ms in (0, 1):
        out.append(dict(name=f"t16_single_ms{ms}", A=PA, B=PB, cx=grid.win_ctrs_x, cy=grid.win_ctrs_y, win=(16, 16),
                        fit=(12, 12), w=(sp, bs, bs, bs), ms=ms, pn=0,
                        keep=np.arange(0, grid.n_win_x * grid.n_win_y, 7)))
    return out


# ----------------------------------------------------------------------------
# comparison against a fixture
# ----------------------------------------------------------------------------

def near_tie(plane, rel=1e-5):
    """True if the two largest positive 3x3 local maxima of the search region are
    within `rel` of each other (argmax order is then not stable to rounding)."""
    n0, n1 = plane.shape
    vals = []
    for i in range(n0 // 4, n0 * 3 // 4):
        for j in range(n1 // 4, n1 * 3 // 4):
            v = plane[i, j]
            if v > 0 and v >= plane[max(i - 1, 0):i + 2, max(j - 1, 0):j + 2].max():
                vals.append(v)
    vals = sorted(vals, reverse=True)
    return len(vals) >= 2 and (vals[0] - vals[1]) <= rel * abs(vals[0])


def compare(case, out, ref, planes=None):
    """Statistics of one output dict (keys pk_x ... pk_ratio, arrays shaped as
    the reference's) against the fixture arrays `ref` (dict name -> array).
    `planes` (n_windows, h, w), when given, are the compared side's full planes
    (for the plane error and the near-tie classification)."""
    rx, ry = ref["pk_x"], ref["pk_y"]
    ox, oy = np.asarray(out["pk_x"]), np.asarray(out["pk_y"])
    nan_r, nan_o = np.isnan(rx), np.isnan(ox)
    d = np.maximum(np.abs(rx - ox), np.abs(ry - oy))
    both = ~nan_r & ~nan_o
    st = dict(n=int(rx.size), nan_flip=int((nan_r != nan_o).sum()),
              zeros_equal=bool(np.array_equal(rx == 0, ox == 0) and np.array_equal(ry == 0, oy == 0)),
              n_far=int((d[both] > 0.005).sum()), max_d=float(d[both].max()) if both.any() else 0.0,
              median_d=float(np.median(d[both])) if both.any() else 0.0)
    far = (nan_r != nan_o) | (both & (d > 0.005))
    st["far_idx"] = np.nonzero(far.ravel())[0]
    if planes is not None and len(case["plane_idx"]):
        R = ref["planes"]
        P = np.asarray(planes)[case["plane_idx"]]
        sc = np.abs(R).reshape(len(R), -1).max(axis=1)
        sc[sc == 0] = 1.0
        st["plane_rel"] = float((np.abs(P - R).reshape(len(R), -1).max(axis=1) / sc).max())
    hk = both & (ref["pk_h"] != 0) & np.isfinite(ref["pk_h"]) & np.isfinite(np.asarray(out["pk_h"]))
    st["height_rel"] = float((np.abs(np.asarray(out["pk_h"])[hk] - ref["pk_h"][hk]) / np.abs(ref["pk_h"][hk])).max()) \
        if hk.any() else 0.0
    return st
