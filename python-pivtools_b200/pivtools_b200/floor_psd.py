"""Coloured noise-floor shape P(k; fx, fy) for the k-space ensemble fit.

The k-space fit models the white sensor-noise floor of F_ref = sqrt(|F_AA||F_BB|)
as N0 * P(k; fx, fy): white noise coloured by the warp kernel at the window's
fractional shift (fx, fy), the weighted window-mean removal and the envelope
divide (pivtools_cli/piv/piv_backend/kspace_floor_psd.py:1-275).  This module
builds the table of P over a grid of fractions, once per pass, on the host in
FP64 (a few hundred 16 x 16 planes); the per-window bilinear lookup that turns
the table into the fit's (n_windows, h*w) regressor runs on the GPU
(`pivb_floor_interp_dev`), next to the planes it goes with.

Closed form for one (fx, fy), with w the correlation pixel weight (sh, sw),
r_x, r_y the autocorrelations of the warp-kernel taps at fx, fy, A(tau) the
zero-padded lag autocorrelation of w, v = (r_y (x) r_x) * w (separable, zero
padded), q = sum(w v), W = DFT(w), V = DFT(w v):

    E(k) = sum_tau r_y r_x A(tau) cos(k . tau)                      (T1)
           - (2 / sum w) Re[conj(W) V] + q |W|^2 / (sum w)^2        (mean hole)

then lag space (inverse DFT, fftshift), central (h, w) crop, divide by the
envelope, centred DFT, magnitude.  The grid is normalised to unit mean at
(fx, fy) = (0, 0).  All grid cells are evaluated together (broadcast over the
fraction axes).
"""

from __future__ import annotations

import numpy as np

KEYS_A = -0.75
N_FRACS = 21


def _keys_taps(f):
    """Keys cubic weights (a = -0.75) at offsets -1, 0, 1, 2 for fractions f (n,)."""
    a = KEYS_A
    f = np.asarray(f, np.float64)
    f2, f3 = f * f, f * f * f
    return np.stack([a * f3 - 2 * a * f2 + a * f,
                     (a + 2) * f3 - (a + 3) * f2 + 1.0,
                     -(a + 2) * f3 + (2 * a + 3) * f2 - a * f,
                     -a * f3 + a * f2], axis=-1)


def _lanczos_taps(f):
    """Normalised Lanczos-3 weights at offsets -2..3 for fractions f (n,)."""
    f = np.asarray(f, np.float64)
    t = f[:, None] - np.arange(-2, 4, dtype=np.float64)[None, :]
    pt = np.pi * t
    with np.errstate(invalid="ignore", divide="ignore"):
        w = (np.sin(pt) / pt) * (np.sin(pt / 3.0) / (pt / 3.0))
    w = np.where(np.abs(t) < 1e-12, 1.0, w)
    w = np.where(np.abs(t) >= 3.0, 0.0, w)
    s = w.sum(axis=1, keepdims=True)
    unit = np.zeros_like(w)
    unit[:, 2] = 1.0
    return np.where(s < 1e-12, unit, w / np.where(s < 1e-12, 1.0, s))


TAPS = {"cubic": _keys_taps, "lanczos": _lanczos_taps}


def tap_autocorr(f, kernel="lanczos"):
    """(taus, r): r[i, t] = sum_j c[i, j] c[i, j + taus[t]] of the kernel taps
    c at fractions f (n,); the taps sit at consecutive integer offsets."""
    if kernel not in TAPS:
        raise ValueError(f"unknown warp kernel {kernel!r} (valid: {sorted(TAPS)})")
    c = TAPS[kernel](np.atleast_1d(f))
    n = c.shape[1]
    taus = np.arange(-(n - 1), n)
    r = np.zeros((c.shape[0], len(taus)))
    for t, tau in enumerate(taus):
        lo, hi = max(0, -tau), min(n, n - tau)
        r[:, t] = (c[:, lo:hi] * c[:, lo + tau:hi + tau]).sum(axis=1)
    return taus, r


def _shifted(a, tau, axis):
    """out(x) = a(x + tau) along axis, zero outside."""
    out = np.zeros_like(a)
    n = a.shape[axis]
    if abs(tau) >= n:
        return out
    src = [slice(None)] * a.ndim
    dst = [slice(None)] * a.ndim
    if tau >= 0:
        src[axis], dst[axis] = slice(tau, n), slice(0, n - tau)
    else:
        src[axis], dst[axis] = slice(0, n + tau), slice(-tau, n)
    out[tuple(dst)] = a[tuple(src)]
    return out


def _centred_dft2(x):
    return np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(x, axes=(-2, -1))), axes=(-2, -1))


def floor_grid(env_auto, weight_B, kernel="lanczos", hole=True, fs_y=None, fs_x=None):
    """Unnormalised |F| floor shape for every (fy, fx) pair: (len(fs_y), len(fs_x), h, w).

    env_auto (h, w): the envelope the planes were divided by (ones if none);
    weight_B (sh, sw): the correlation pixel weight, sh >= h, sw >= w."""
    env = np.asarray(env_auto, np.float64)
    w = np.asarray(weight_B, np.float64)
    h, wd = env.shape
    sh, sw = w.shape
    if w.ndim != 2 or sh < h or sw < wd:
        raise ValueError(f"weight_B shape {w.shape} does not cover the envelope {env.shape}")
    taus, ry = tap_autocorr(fs_y, kernel)          # (ny, T)
    _, rx = tap_autocorr(fs_x, kernel)             # (nx, T)
    T = len(taus)
    # lag autocorrelation of the weight and the shifted weights
    A = np.array([[float((w * _shifted(_shifted(w, int(ty), 0), int(tx), 1)).sum()) for tx in taus]
                  for ty in taus])                                      # (T, T)
    wx = np.stack([_shifted(w, int(t), 1) for t in taus])               # (T, sh, sw)
    vx = np.einsum("xt,tab->xab", rx, wx)                               # (nx, sh, sw)
    vxy = np.stack([_shifted(vx, int(t), 1) for t in taus], axis=1)     # (nx, T, sh, sw): rows shifted
    v = np.einsum("yt,xtab->yxab", ry, vxy)                             # (ny, nx, sh, sw)
    sumB = w.sum()
    q = (w[None, None] * v).sum(axis=(2, 3))                            # (ny, nx)
    my, mx = np.arange(sh), np.arange(sw)
    PY = np.exp(-2j * np.pi * np.outer(my, taus) / sh)                  # (sh, T)
    PX = np.exp(-2j * np.pi * np.outer(mx, taus) / sw)                  # (sw, T)
    Bc = ry[:, None, :, None] * rx[None, :, None, :] * A[None, None]    # (ny, nx, T, T)
    T1 = np.einsum("yxts,at,bs->yxab", Bc, PY, PX).real
    if hole:
        W = np.fft.fft2(w)
        V = np.fft.fft2(w[None, None] * v)
        E = (T1 - (2.0 / sumB) * np.real(np.conj(W)[None, None] * V)
             + (q / sumB ** 2)[..., None, None] * (np.abs(W) ** 2)[None, None])
        if np.abs(E[..., 0, 0]).max() > 1e-9 * np.abs(q).max():
            raise AssertionError("weighted-mean hole is not zero at DC")
        E[..., 0, 0] = 0.0
    else:
        E = T1
    R = np.fft.fftshift(np.fft.ifft2(E).real, axes=(-2, -1))
    y0, x0 = (sh - h) // 2, (sw - wd) // 2
    return np.abs(_centred_dft2(R[..., y0:y0 + h, x0:x0 + wd] / env))


def build_p_grid(env_auto, kernel, hole, weight_B, n_fracs=N_FRACS):
    """(fs, P_grid): fs = linspace(0, 0.5, n_fracs); P_grid (n_fracs, n_fracs, h, w)
    indexed [iy (fy), ix (fx)], unit mean at (0, 0) (kspace_floor_psd.py:206-238)."""
    fs = np.linspace(0.0, 0.5, n_fracs)
    P = floor_grid(env_auto, weight_B, kernel, hole, fs, fs)
    return fs, P / P[0, 0].mean()
