"""Several correlation peaks per window, the secondary-peak substitution and the
further outlier tests (local sigma, divergence/vorticity) of the resident
multipass (pivb_validate_peaks_dev, MultipassConfig(n_peaks, secondary_peak,
sigma_threshold, div_vort)) against the oracle's restatement of the reference driver
(oracle/ref_multipass.validate_peaks: cpu_instantaneous.py:589-760) and against
the reference's pass loop over its compiled libraries."""

import ctypes

import numpy as np
import pytest

from pivtools_b200 import _lib

pytestmark = pytest.mark.gpu


def _peaks(rng, N, P, ny, nx):
    """Peak arrays with a smooth truth, outliers on the first peak that a later
    peak can rescue, fit failures (NaN), peaks beyond the gate and weak or NaN
    heights."""
    yy, xx = np.mgrid[0:ny, 0:nx]
    tx = (1.5 * np.sin(xx / 6.0) + 0.5 * np.cos(yy / 5.0)).astype(np.float32)
    ty = (0.8 * np.cos(xx / 7.0) - 0.3 * np.sin(yy / 4.0)).astype(np.float32)
    x = np.empty((N, P, ny, nx), np.float32)
    y = np.empty_like(x)
    h = rng.uniform(0.3, 1.0, x.shape).astype(np.float32)
    for n in range(N):
        x[n] = tx + rng.normal(0, 0.05, (P, ny, nx))
        y[n] = ty + rng.normal(0, 0.05, (P, ny, nx))
        for k in range(P):
            bad = rng.random((ny, nx)) < (0.12 if k == 0 else 0.35)
            x[n, k][bad] = rng.uniform(-6, 6, bad.sum())
            y[n, k][bad] = rng.uniform(-6, 6, bad.sum())
        nanf = rng.random((P, ny, nx)) < 0.03
        x[n][nanf] = np.nan
        y[n][nanf] = np.nan
        weak = rng.random((P, ny, nx)) < 0.04
        h[n][weak] = rng.uniform(0.0, 0.2, weak.sum())
        hn = rng.random((P, ny, nx)) < 0.01
        h[n][hn] = np.nan
    return x, y, h


@pytest.mark.parametrize("P,secondary,with_pred,sigma,divvort", [
    (3, True, True, 0.0, False), (2, True, False, 0.0, False), (3, False, True, 0.0, False),
    (4, True, True, 0.0, False), (3, True, True, 2.0, False), (3, True, True, 0.0, True),
    (1, False, True, 2.0, True), (3, True, False, 1.5, True)])
def test_validate_peaks_matches_oracle(cuda, P, secondary, with_pred, sigma, divvort):
    import torch

    import ref_multipass as RM

    rng = np.random.default_rng(40 + P + 10 * secondary)
    N, ny, nx = 2, 37, 45
    x, y, h = _peaks(rng, N, P, ny, nx)
    pdy = pdx = None
    if with_pred:
        pdy = rng.normal(0, 1.0, (N, ny, nx)).astype(np.float32)
        pdx = rng.normal(0, 1.0, (N, ny, nx)).astype(np.float32)
    thr_x, thr_y = 4.0, 4.0
    ox, oy, obad, oreason, ochoice = RM.validate_peaks(x, y, h, pdy, pdx, thr_x, thr_y, secondary=secondary,
                                                       sigma_thr=sigma, divvort=divvort)
    L = _lib.pass_lib()
    dev = cuda
    t = {k: torch.tensor(v, device=dev) for k, v in (("x", x), ("y", y), ("h", h))}
    tp = {k: (None if v is None else torch.tensor(v, device=dev)) for k, v in (("dy", pdy), ("dx", pdx))}
    ux = torch.empty((N, ny, nx), device=dev)
    uy = torch.empty_like(ux)
    inv = torch.empty((N, ny, nx), dtype=torch.uint8, device=dev)
    rc = torch.empty((N, ny, nx), dtype=torch.int8, device=dev)
    ch = torch.empty((N, ny, nx), dtype=torch.uint8, device=dev)
    work = torch.empty(int(L.pivb_validate_peaks_work_floats(N, ny, nx)), device=dev)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ptr = lambda v: None if v is None else v.data_ptr()   # noqa: E731
    assert L.pivb_validate_peaks_dev(t["x"].data_ptr(), t["y"].data_ptr(), t["h"].data_ptr(), P, int(secondary),
                                     ptr(tp["dy"]), ptr(tp["dx"]), None, N, ny, nx, thr_x, thr_y, 0.25, 0.1, 2.0, 5,
                                     sigma, int(divvort), -1.0, -1.0, ux.data_ptr(), uy.data_ptr(), inv.data_ptr(),
                                     rc.data_ptr(), ch.data_ptr(), work.data_ptr(), s) == 0
    torch.cuda.synchronize()
    gbad = inv.cpu().numpy().astype(bool)
    assert np.array_equal(gbad, obad)
    assert np.array_equal(rc.cpu().numpy(), oreason)
    assert np.array_equal(ch.cpu().numpy().astype(np.intp), ochoice)
    assert np.array_equal(ux.cpu().numpy(), ox, equal_nan=True)
    assert np.array_equal(uy.cpu().numpy(), oy, equal_nan=True)
    if secondary and P > 1:
        assert (ochoice > 1).sum() > 20          # the case exercises the substitution
        assert (oreason == 12).sum() > 0 and (oreason == 13).sum() > 0


def test_one_peak_path_equals_validate_dev(cuda):
    """n_peaks 1 through the multi-peak entry point equals pivb_validate_dev."""
    import torch

    rng = np.random.default_rng(9)
    N, ny, nx = 2, 30, 33
    x, y, h = _peaks(rng, N, 1, ny, nx)
    dev = cuda
    L = _lib.pass_lib()
    t = [torch.tensor(v, device=dev) for v in (x, y, h)]
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    outs = []
    for multi in (False, True):
        ux = torch.empty((N, ny, nx), device=dev)
        uy = torch.empty_like(ux)
        inv = torch.empty((N, ny, nx), dtype=torch.uint8, device=dev)
        rc = torch.empty((N, ny, nx), dtype=torch.int8, device=dev)
        work = torch.empty(int(L.pivb_validate_peaks_work_floats(N, ny, nx)), device=dev)
        if multi:
            ch = torch.empty((N, ny, nx), dtype=torch.uint8, device=dev)
            assert L.pivb_validate_peaks_dev(t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), 1, 1, None, None,
                                             None, N, ny, nx, 4.0, 4.0, 0.25, 0.1, 2.0, 5, 0.0, 0, -1.0, -1.0,
                                             ux.data_ptr(), uy.data_ptr(), inv.data_ptr(), rc.data_ptr(),
                                             ch.data_ptr(), work.data_ptr(), s) == 0
        else:
            assert L.pivb_validate_dev(t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), None, None, None, N, ny,
                                       nx, 4.0, 4.0, 0.25, 0.1, 2.0, 5, ux.data_ptr(), uy.data_ptr(), inv.data_ptr(),
                                       rc.data_ptr(), work.data_ptr(), s) == 0
        torch.cuda.synchronize()
        outs.append([v.cpu().numpy() for v in (ux, uy, inv, rc)])
    for a, b in zip(*outs):
        assert np.array_equal(a, b, equal_nan=True)


def test_multipass_secondary_matches_reference_pipeline(cuda, oracle):
    """Three peaks with substitution through the whole resident multipass against
    the reference's pass loop over its compiled libraries (same statistical bar
    as the one-peak pipeline test: small plane differences travel through the
    predictors)."""
    import torch

    if oracle.ref_bulk() is None or oracle.ref_warp() is None:
        pytest.skip("reference libraries not built here (make -C oracle ref PIVTOOLS_REF=...)")
    import ref_multipass as RM

    from pivtools_b200 import multipass, synthetic

    HW = (512, 512)
    cfg = multipass.MultipassConfig(window_sizes=[(64, 64), (32, 32), (32, 32)], overlaps=[50, 50, 75], n_peaks=3,
                                    secondary_peak=True)
    # sparse particles and strong fluctuations: weak correlations, outliers that a
    # second or third peak can replace
    A, B = synthetic.channel_batch_torch(1, HW, seed=78, device=cuda, peak=8.0, rms_frac=0.25, density=0.01)
    mp = multipass.MultipassPIV(HW, 1, cfg, device=cuda)
    mp.run(A, B)
    torch.cuda.synchronize()
    rm = RM.RefMultipass(mp.geo, window_type=cfg.window_type, peak_finder=cfg.peak_finder, infill=cfg.infill,
                         n_peaks=3, secondary_peak=True)
    rm.run(A.cpu().numpy(), B.cpu().numpy())
    subst = 0
    for k, (p, (rx, ry, rbad)) in enumerate(zip(mp.passes, rm.history)):
        gx, gy = p["ux"][0].cpu().numpy(), p["uy"][0].cpu().numpy()
        gbad = p["invalid"][0].cpu().numpy().astype(bool)
        subst += int((p["choice"][0].cpu().numpy() > 1).sum())
        d = np.maximum(np.abs(gx - rx[0]), np.abs(gy - ry[0]))
        print(f"\npass {k}: invalid {int(gbad.sum())} (reference {int(rbad[0].sum())}), flags equal "
              f"{(gbad == rbad[0]).mean():.4f}, within 1e-3 px {(d <= 1e-3).mean():.4f}")
        assert (gbad == rbad[0]).mean() >= 0.995, k
        assert (d <= 1e-3).mean() >= 0.99, k
    assert subst > 0
    res = mp.collect()[0]
    assert res.passes[-1].peak_mag.shape[0] == 3


def test_multipass_three_peaks_without_substitution_equals_one_peak(cuda):
    """n_peaks 3 without substitution: the primary peak's fields equal the
    one-peak run bit for bit."""
    import torch

    from pivtools_b200 import multipass, synthetic

    HW = (384, 384)
    A, B = synthetic.channel_batch_torch(2, HW, seed=79, device=cuda, peak=6.0)
    res = []
    for P in (1, 3):
        cfg = multipass.MultipassConfig(window_sizes=[(64, 64), (32, 32)], overlaps=[50, 50], n_peaks=P)
        mp = multipass.MultipassPIV(HW, 2, cfg, device=cuda)
        ux, uy = mp.run(A, B)
        torch.cuda.synchronize()
        res.append((ux.cpu().numpy().copy(), uy.cpu().numpy().copy(), mp.passes[-1]["invalid"].cpu().numpy().copy()))
    for a, b in zip(*res):
        assert np.array_equal(a, b, equal_nan=True)
