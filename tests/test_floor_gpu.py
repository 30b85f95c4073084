"""Coloured-floor regressor on the GPU (pivb_floor_interp_dev): bit-exact to the
reference's interp_P on its own P grid, and the coloured k-space fit of a
resident ensemble pass against the oracle fit given the same regressor."""

import ctypes
import os

import numpy as np
import pytest

from pivtools_b200 import _lib, ensemble, floor_psd, synthetic

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _interp(cuda, fs, P, pdy, pdx, n_win):
    import torch

    L = _lib.pass_lib()
    fs_d = torch.tensor(fs, dtype=torch.float64, device=cuda)
    P_d = torch.tensor(np.ascontiguousarray(P), dtype=torch.float64, device=cuda)
    hw = P.shape[-1] * P.shape[-2]
    out = torch.full((n_win, hw), -1.0, dtype=torch.float64, device=cuda)
    dy = None if pdy is None else torch.tensor(pdy, device=cuda)
    dx = None if pdx is None else torch.tensor(pdx, device=cuda)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.pivb_floor_interp_dev(fs_d.data_ptr(), len(fs), P_d.data_ptr(), hw,
                                   None if dy is None else dy.data_ptr(), None if dx is None else dx.data_ptr(),
                                   n_win, out.data_ptr(), s) == 0
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_floor_lookup_bit_exact_to_reference(cuda):
    g = np.load(os.path.join(GOLD, "floor_ref.npz"))
    n = g["pred_dx"].size
    for ci in range(4):
        got = _interp(cuda, g[f"c{ci}_fs"], g[f"c{ci}_P"], g["pred_dy"], g["pred_dx"], n)
        assert np.array_equal(got, g[f"c{ci}_Pwin"].astype(np.float64)), ci


def test_floor_lookup_without_predictor_and_full_grid(oracle, cuda):
    g = np.load(os.path.join(GOLD, "floor_ref.npz"))
    got = _interp(cuda, g["c0_fs"], g["c0_P"], None, None, 37)
    want = g["c0_P"][0, 0].reshape(-1).astype(np.float32).astype(np.float64)
    assert np.array_equal(got, np.broadcast_to(want, got.shape))
    fs, P = floor_psd.build_p_grid(g["c2_env"], "cubic", True, g["c2_w"])           # 21 x 21 grid
    rng = np.random.default_rng(4)
    pdy = rng.normal(0, 4, 5000).astype(np.float32)
    pdx = rng.normal(0, 4, 5000).astype(np.float32)
    got = _interp(cuda, fs, P, pdy, pdx, 5000)
    want = oracle.floor_interp(fs, P, oracle.floor_fractions(pdx), oracle.floor_fractions(pdy))
    assert np.array_equal(got, want.astype(np.float64))


@pytest.mark.parametrize("method,kernel", [("window_mean", "lanczos"), ("correlation+dc_zero", "cubic")])
def test_coloured_fit_matches_oracle(oracle, cuda, method, kernel):
    import torch

    shape, win = (128, 160), (16, 16)
    out = [synthetic.particle_pair(shape, seed=900 + k, flow="uniform_grf")[:2] for k in range(8)]
    A = np.stack([p[0] for p in out]).astype(np.float32)
    B = np.stack([p[1] for p in out]).astype(np.float32)
    ep = ensemble.EnsemblePIV(shape, win, 75, "gaussian", background=method, envelope_divide=True, device=cuda)
    ep.accumulate(torch.tensor(A, device=cuda), torch.tensor(B, device=cuda))
    fin = ep.finalize()
    g = ep.grid
    rng = np.random.default_rng(8)
    pred = rng.normal(0, 2, (g.n_win_y, g.n_win_x, 2)).astype(np.float32)
    fit = ep.fit(floor="coloured", predictor=pred, warp_kernel=kernel)
    P_win = ep.floor_regressor(pred, kernel).cpu().numpy()
    torch.cuda.synchronize()
    env = ep.env.cpu().numpy().astype(np.float64)
    fs, P = floor_psd.build_p_grid(env, kernel, method == "window_mean", ep.weight.cpu().numpy())
    want = oracle.floor_interp(fs, P, oracle.floor_fractions(pred[..., 1].ravel()),
                               oracle.floor_fractions(pred[..., 0].ravel()))
    assert np.array_equal(P_win, want.astype(np.float64))
    n_win = g.n_win_y * g.n_win_x
    R = [fin[k].cpu().numpy() for k in ("R_AA", "R_BB", "R_AB")]
    ref = oracle.kspace_fit(*R, np.zeros(n_win, np.uint8), win, P_win=P_win)
    st = fit["status"].cpu().numpy()
    assert np.array_equal(st, ref["status"])
    ok = st == 0
    assert ok.sum() >= 0.5 * n_win
    gg = fit["gauss"].cpu().numpy()
    assert np.abs(gg[ok, 9:12] - ref["gauss_flat"][ok, 9:12]).max() < 1e-8
    assert np.abs(gg[ok, 14:16] - ref["gauss_flat"][ok, 14:16]).max() < 1e-8
    np.testing.assert_allclose(fit["N0"].cpu().numpy()[ok], ref["N0"][ok], rtol=1e-6, atol=1e-12)
    # a first pass (no predictor) uses the 2 x 2 grid: every window gets the (0, 0) shape
    P0 = ep.floor_regressor(None, kernel).cpu().numpy()
    assert np.array_equal(P0, np.broadcast_to(P0[0], P0.shape))
