"""Seeded synthetic particle-image pairs (test and benchmark inputs).

Particle model (the reference test generator's local-patch Gaussian rendering,
unit-tests/synthetic_piv.py:22-75): each particle adds I*exp(-r^2/(2 sigma^2))
within +-3 sigma of its centre.  Defaults follow the benchmark workloads:
sigma = 0.6 px, peak intensity U[1000, 4000], 0.05 particles/pixel, Poisson
shot noise on a 100-count background, uint16 clipping, float32 output.  Frame B
renders every particle at x + u(x).  Rendering runs in numpy, or on a CUDA
device through torch for benchmark-sized batches; positions and intensities
always come from numpy.random.default_rng(seed).
"""

from __future__ import annotations

import numpy as np


def _render_np(shape, xs, ys, amp, sigma):
    h, w = shape
    img = np.zeros(h * w, np.float64)
    r = int(np.ceil(3.0 * sigma))
    x0 = np.floor(xs).astype(np.int64)
    y0 = np.floor(ys).astype(np.int64)
    inv = 1.0 / (2.0 * sigma * sigma)
    for dy in range(-r, r + 1):
        yy = y0 + dy
        for dx in range(-r, r + 1):
            xx = x0 + dx
            ok = (yy >= 0) & (yy < h) & (xx >= 0) & (xx < w)
            d2 = (xx - xs) ** 2 + (yy - ys) ** 2
            np.add.at(img, (yy * w + xx)[ok], (amp * np.exp(-d2 * inv))[ok])
    return img.reshape(h, w)


def _render_torch(shape, xs, ys, amp, sigma, device):
    import torch

    h, w = shape
    xs = torch.as_tensor(xs, device=device, dtype=torch.float64)
    ys = torch.as_tensor(ys, device=device, dtype=torch.float64)
    amp = torch.as_tensor(amp, device=device, dtype=torch.float64)
    img = torch.zeros(h * w, device=device, dtype=torch.float64)
    r = int(np.ceil(3.0 * sigma))
    x0 = torch.floor(xs).long()
    y0 = torch.floor(ys).long()
    inv = 1.0 / (2.0 * sigma * sigma)
    for dy in range(-r, r + 1):
        yy = y0 + dy
        for dx in range(-r, r + 1):
            xx = x0 + dx
            ok = (yy >= 0) & (yy < h) & (xx >= 0) & (xx < w)
            d2 = (xx - xs) ** 2 + (yy - ys) ** 2
            img.index_add_(0, (yy * w + xx)[ok], (amp * torch.exp(-d2 * inv))[ok])
    return img.reshape(h, w)


def smooth_field(rng, shape, std, corr_len):
    """Gaussian random field: white noise filtered by a Gaussian of width corr_len,
    rescaled to the requested standard deviation."""
    from scipy.ndimage import gaussian_filter

    f = gaussian_filter(rng.standard_normal(shape), sigma=corr_len / 2.0, mode="wrap")
    s = f.std()
    return f * (std / s) if s > 0 else f


def uniform_grf_flow(rng, shape, mean=(3.3, -1.7), std=0.5, corr_len=40.0):
    """Uniform shift plus isotropic GRF (u, v) in px; returns (u, v) on the pixel grid."""
    u = mean[0] + smooth_field(rng, shape, std, corr_len)
    v = mean[1] + smooth_field(rng, shape, std, corr_len)
    return u, v


def channel_flow(rng, shape, peak=12.0, re_tau=1000.0, rms_frac=0.08, corr_len=24.0):
    """Turbulent-channel-like field: log-law mean u+(y+) across the height (wall at
    both edges) scaled to `peak` px, plus isotropic Gaussian fluctuations of rms
    rms_frac*peak."""
    h, w = shape
    y = (np.arange(h) + 0.5) / h                       # 0..1 across the channel
    yw = np.minimum(y, 1.0 - y) * 2.0 * re_tau         # wall units from the nearer wall
    kappa, B = 0.41, 5.2
    uplus = np.where(yw < 11.0, yw, np.log(np.maximum(yw, 1e-9)) / kappa + B)
    prof = uplus / uplus.max() * peak
    u = prof[:, None] + smooth_field(rng, shape, rms_frac * peak, corr_len)
    v = smooth_field(rng, shape, rms_frac * peak, corr_len)
    return u, v


def ensemble_row_statistics(yn, peak=4.0, uu_max=0.6, vv_max=0.3, rho=-0.4):
    """Prescribed per-row statistics of the ensemble flow at normalised height yn:
    mean streamwise displacement (parabolic profile, `peak` px at the centre),
    variances <u'u'>, <v'v'> (largest near the walls) and covariance <u'v'> with
    correlation coefficient rho.  Returns (mean_u, (uu, vv, uv))."""
    yn = np.asarray(yn, np.float64)
    mean_u = peak * 4.0 * yn * (1.0 - yn)
    shape_ = 0.35 + 0.65 * (1.0 - 4.0 * yn * (1.0 - yn))
    uu = uu_max * shape_
    vv = vv_max * shape_
    uv = rho * np.sqrt(uu * vv)
    return mean_u, (uu, vv, uv)


def ensemble_row_displacements(rng, yn, **kw):
    """Per-particle (u, v) drawn from the row's joint Gaussian."""
    mean_u, (uu, vv, uv) = ensemble_row_statistics(yn, **kw)
    z1, z2 = rng.standard_normal((2, len(yn)))
    su = np.sqrt(uu)
    rho_ = uv / np.maximum(su * np.sqrt(vv), 1e-30)
    du = mean_u + su * z1
    dv = np.sqrt(vv) * (rho_ * z1 + np.sqrt(1.0 - rho_ ** 2) * z2)
    return du, dv


def particle_pair(shape, seed, density=0.05, sigma=0.6, i_range=(1000.0, 4000.0), background=100.0,
                  flow="uniform_grf", device=None, flow_kwargs=None):
    """One image pair (A, B) as float32 arrays (numpy, or torch tensors on `device`)
    plus the displacement field (u, v) used for frame B."""
    rng = np.random.default_rng(seed)
    h, w = shape
    n = int(round(density * h * w))
    margin = 8.0
    xs = rng.uniform(-margin, w + margin, n)
    ys = rng.uniform(-margin, h + margin, n)
    amp = rng.uniform(i_range[0], i_range[1], n)
    kw = flow_kwargs or {}
    if flow == "uniform_grf":
        u, v = uniform_grf_flow(rng, shape, **kw)
    elif flow == "channel":
        u, v = channel_flow(rng, shape, **kw)
    elif flow == "uniform":
        u = np.full(shape, kw.get("u", 0.0))
        v = np.full(shape, kw.get("v", 0.0))
    elif flow == "ensemble_rows":
        u = v = None
    else:
        raise ValueError(flow)
    xi = np.clip(np.round(xs).astype(np.int64), 0, w - 1)
    yi = np.clip(np.round(ys).astype(np.int64), 0, h - 1)
    if flow == "ensemble_rows":
        # every particle draws its own displacement from the row's joint Gaussian
        du, dv = ensemble_row_displacements(rng, ys / h, **kw)
        xb, yb = xs + du, ys + dv
        u, v = ensemble_row_statistics(np.linspace(0.0, 1.0, h), **kw)
    else:
        xb = xs + u[yi, xi]
        yb = ys + v[yi, xi]
    seed_a, seed_b = rng.integers(0, 2**62, 2)
    if device is None:
        ia = _render_np(shape, xs, ys, amp, sigma)
        ib = _render_np(shape, xb, yb, amp, sigma)
        na = np.random.default_rng(seed_a).poisson(ia + background)
        nb = np.random.default_rng(seed_b).poisson(ib + background)
        A = np.clip(na, 0, 65535).astype(np.uint16).astype(np.float32)
        B = np.clip(nb, 0, 65535).astype(np.uint16).astype(np.float32)
        return A, B, (u, v)
    import torch

    ia = _render_torch(shape, xs, ys, amp, sigma, device)
    ib = _render_torch(shape, xb, yb, amp, sigma, device)
    ga = torch.Generator(device=device).manual_seed(int(seed_a) & 0x7FFFFFFF)
    gb = torch.Generator(device=device).manual_seed(int(seed_b) & 0x7FFFFFFF)
    A = torch.clamp(torch.poisson(ia + background, generator=ga), 0, 65535).float()
    B = torch.clamp(torch.poisson(ib + background, generator=gb), 0, 65535).float()
    return A, B, (u, v)


def channel_batch_torch(n_pairs, shape, seed, device, peak=12.0, re_tau=1000.0, rms_frac=0.08, corr_len=24.0,
                        density=0.05, sigma=0.6, i_range=(1000.0, 4000.0), background=100.0):
    """Benchmark batch of channel-flow pairs rendered on the GPU: (A, B) as
    (n_pairs, H, W) float32 CUDA tensors.  Fluctuation fields are Gaussian random
    fields made by spectral filtering on the device; particles come from
    numpy.random.default_rng(seed + pair)."""
    import torch

    h, w = shape
    y = (np.arange(h) + 0.5) / h
    yw = np.minimum(y, 1.0 - y) * 2.0 * re_tau
    uplus = np.where(yw < 11.0, yw, np.log(np.maximum(yw, 1e-9)) / 0.41 + 5.2)
    prof = torch.tensor(uplus / uplus.max() * peak, device=device, dtype=torch.float64)
    ky = torch.fft.fftfreq(h, device=device, dtype=torch.float64)[:, None]
    kx = torch.fft.fftfreq(w, device=device, dtype=torch.float64)[None, :]
    filt = torch.exp(-2.0 * (np.pi * corr_len / 2.0) ** 2 * (kx * kx + ky * ky))
    A = torch.empty((n_pairs, h, w), dtype=torch.float32, device=device)
    B = torch.empty_like(A)
    for k in range(n_pairs):
        g = torch.Generator(device=device).manual_seed(int(seed) * 1000003 + k)
        fields = []
        for _ in range(2):
            f = torch.fft.ifft2(torch.fft.fft2(torch.randn((h, w), generator=g, device=device,
                                                           dtype=torch.float64)) * filt).real
            fields.append(f * (rms_frac * peak / f.std()))
        u = prof[:, None] + fields[0]
        v = fields[1]
        rng = np.random.default_rng(seed * 7919 + k)
        n = int(round(density * h * w))
        xs = rng.uniform(-8.0, w + 8.0, n)
        ys = rng.uniform(-8.0, h + 8.0, n)
        amp = rng.uniform(i_range[0], i_range[1], n)
        xi = torch.as_tensor(np.clip(np.round(xs), 0, w - 1).astype(np.int64), device=device)
        yi = torch.as_tensor(np.clip(np.round(ys), 0, h - 1).astype(np.int64), device=device)
        xs_t = torch.as_tensor(xs, device=device)
        ys_t = torch.as_tensor(ys, device=device)
        xb = (xs_t + u[yi, xi]).cpu().numpy()
        yb = (ys_t + v[yi, xi]).cpu().numpy()
        ia = _render_torch(shape, xs, ys, amp, sigma, device)
        ib = _render_torch(shape, xb, yb, amp, sigma, device)
        A[k] = torch.clamp(torch.poisson(ia + background, generator=g), 0, 65535).float()
        B[k] = torch.clamp(torch.poisson(ib + background, generator=g), 0, 65535).float()
    return A, B
