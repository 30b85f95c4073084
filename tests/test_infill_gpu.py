"""GPU least-squares infilling (pivb_infill_dev) against the reference's own
infill_harmonic and infill_biharmonic (pivtools_cli/piv/piv_backend/
infilling.py:336-421; fixture golden/infill_ref.npz from make_golden.py infill):
filled values within 1e-5 px (the solve is FP64 conjugate gradients to a 1e-12
relative residual; outputs are float32), known and excluded cells untouched,
several pairs in one launch, bit-identical on a repeated call."""

import ctypes
import os
import sys

import numpy as np
import pytest

from pivtools_b200 import _lib

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLD)
from infill_cases import infill_cases  # noqa: E402


def _run(torch, dev, U, V, fill, excl, pitch, order):
    L = _lib.pass_lib()
    N, ny, nx = U.shape
    tu = torch.tensor(U, device=dev)
    tv = torch.tensor(V, device=dev)
    tb = torch.tensor(fill.astype(np.uint8), device=dev)
    tm = None if excl is None else torch.tensor(excl.astype(np.float32), device=dev)
    nb = int(L.pivb_infill_work_bytes(N, ny, nx))
    work = torch.empty(nb, dtype=torch.uint8, device=dev)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.pivb_infill_dev(tu.data_ptr(), tv.data_ptr(), tb.data_ptr(), None if tm is None else tm.data_ptr(), N,
                             ny, nx, pitch[0], pitch[1], order, 2000, 1e-12, work.data_ptr(), nb, s) == 0
    torch.cuda.synchronize()
    return tu.cpu().numpy(), tv.cpu().numpy()


@pytest.mark.parametrize("method,order", [("harmonic", 1), ("biharmonic", 2)])
def test_infill_matches_reference(cuda, method, order):
    import torch

    g = np.load(os.path.join(GOLD, "infill_ref.npz"))
    for k, c in enumerate(infill_cases()):
        U, V = c["ux"].copy(), c["uy"].copy()
        U[c["fill"]] = np.nan
        V[c["fill"]] = np.nan
        # the same field three times in one launch (one CTA per pair)
        gu, gv = _run(torch, cuda, np.stack([U] * 3), np.stack([V] * 3), np.stack([c["fill"]] * 3), c["exclude"],
                      c["pitch"], order)
        for n in range(3):
            for got, key, src in ((gu[n], "ux", U), (gv[n], "uy", V)):
                ref = g[f"c{k}_{method}_{key}"]
                assert np.abs(got[c["fill"]] - ref[c["fill"]]).max() <= 1e-5, (k, method, key)
                keep = ~c["fill"]
                assert np.array_equal(got[keep], src[keep]), (k, key)   # known and excluded cells untouched
        assert np.array_equal(gu[0], gu[1]) and np.array_equal(gu[0], gu[2])


def test_infill_is_deterministic_and_handles_no_donor(cuda):
    import torch

    rng = np.random.default_rng(4)
    ny, nx = 61, 67
    U = rng.normal(2.0, 0.5, (2, ny, nx)).astype(np.float32)
    V = rng.normal(-1.0, 0.5, (2, ny, nx)).astype(np.float32)
    fill = rng.random((2, ny, nx)) < 0.1
    fill[1] = True                       # pair 1: no valid vector at all -> zeros
    U[fill] = np.nan
    V[fill] = np.nan
    a = _run(torch, cuda, U, V, fill, None, (16.0, 16.0), 2)
    b = _run(torch, cuda, U, V, fill, None, (16.0, 16.0), 2)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert np.isfinite(a[0]).all() and np.isfinite(a[1]).all()
    assert np.all(a[0][1] == 0.0) and np.all(a[1][1] == 0.0)


def test_nearest_infill_matches_reference(cuda):
    """pivb_nearest_infill_dev equals the reference's infill_nearest bit for bit
    (same donors, ties included) on every fixture case, with several pairs in one
    launch; a pair without donors keeps 0."""
    import torch

    g = np.load(os.path.join(GOLD, "infill_ref.npz"))
    L = _lib.pass_lib()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for k, c in enumerate(infill_cases()):
        U, V = c["ux"].copy(), c["uy"].copy()
        U[c["fill"]] = np.nan
        V[c["fill"]] = np.nan
        ny, nx = U.shape
        tu = torch.tensor(np.stack([U, U]), device=cuda)
        tv = torch.tensor(np.stack([V, V]), device=cuda)
        fill2 = np.stack([c["fill"], np.ones_like(c["fill"])])       # pair 1: everything to fill
        tb = torch.tensor(fill2.astype(np.uint8), device=cuda)
        tm = None if c["exclude"] is None else torch.tensor(c["exclude"].astype(np.float32), device=cuda)
        assert L.pivb_nearest_infill_dev(tu.data_ptr(), tv.data_ptr(), tb.data_ptr(),
                                         None if tm is None else tm.data_ptr(), 2, ny, nx, c["pitch"][0],
                                         c["pitch"][1], s) == 0
        torch.cuda.synchronize()
        gu, gv = tu.cpu().numpy(), tv.cpu().numpy()
        assert np.array_equal(gu[0], g[f"c{k}_nearest_ux"].astype(np.float32)), k
        assert np.array_equal(gv[0], g[f"c{k}_nearest_uy"].astype(np.float32)), k
        assert np.all(gu[1] == 0.0) and np.all(gv[1] == 0.0)


def test_multipass_nearest_infill_matches_oracle_pipeline(cuda, oracle):
    """The resident multipass with infill 'nearest' against the reference's pass
    loop over its compiled libraries with the nearest fill (statistical bar of the
    pipeline tests)."""
    import torch

    if oracle.ref_bulk() is None or oracle.ref_warp() is None:
        pytest.skip("reference libraries not built here")
    import ref_multipass as RM

    from pivtools_b200 import multipass, synthetic

    HW = (512, 512)
    cfg = multipass.MultipassConfig(window_sizes=[(64, 64), (32, 32), (32, 32)], overlaps=[50, 50, 75],
                                    infill="nearest")
    A, B = synthetic.channel_batch_torch(1, HW, seed=83, device=cuda, peak=8.0, rms_frac=0.2, density=0.02)
    mp = multipass.MultipassPIV(HW, 1, cfg, device=cuda)
    mp.run(A, B)
    torch.cuda.synchronize()
    rm = RM.RefMultipass(mp.geo, window_type=cfg.window_type, peak_finder=cfg.peak_finder, infill="nearest")
    rm.run(A.cpu().numpy(), B.cpu().numpy())
    for k, (p, (rx, ry, rbad)) in enumerate(zip(mp.passes, rm.history)):
        gx, gy = p["ux"][0].cpu().numpy(), p["uy"][0].cpu().numpy()
        gbad = p["invalid"][0].cpu().numpy().astype(bool)
        d = np.maximum(np.abs(gx - rx[0]), np.abs(gy - ry[0]))
        assert (gbad == rbad[0]).mean() >= 0.995, k
        assert (d <= 1e-3).mean() >= 0.99, k
