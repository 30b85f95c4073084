"""GPU parity of the ensemble accumulators (bulkxcorr2d_accumulate[_triple]) through
the C-ABI against the FP64 oracle: accumulated planes within 1e-5 of each
window's plane magnitude, += semantics into caller-zeroed sums, masked windows
untouched."""

import numpy as np
import pytest

from pivtools_b200 import _lib, geometry, synthetic

pytestmark = pytest.mark.gpu


def _stack(n_pairs, shape, seed):
    A, B = [], []
    for k in range(n_pairs):
        a, b, _ = synthetic.particle_pair(shape, seed=seed + k, density=0.02)
        A.append(a)
        B.append(b)
    return np.stack(A), np.stack(B)


def _triple_gpu(A, B, mask, g, win, wab_a, wab_b, waa, wbb, fit, ms, ppn, init=None):
    L = _lib.bulkxcorr2d_lib()
    n, H, W = A.shape
    oh, ow = fit if fit is not None else win
    nwt = g.n_win_y * g.n_win_x
    outs = [np.zeros(nwt * oh * ow, np.float32) if init is None else init[k].copy() for k in range(3)]
    fs = None if fit is None else np.array(fit, np.int32)
    code = L.bulkxcorr2d_accumulate_triple(
        np.ascontiguousarray(A), np.ascontiguousarray(B), mask.ravel(), np.array([H, W], np.int32), n,
        g.win_ctrs_x, g.win_ctrs_y, np.array([g.n_win_y, g.n_win_x], np.int32), wab_a.ravel(), wab_b.ravel(),
        waa.ravel(), wbb.ravel(), np.array(win, np.int32), None if fs is None else fs.ctypes.data, ms, ppn, *outs)
    assert code == 0
    return [o.reshape(g.n_win_y, g.n_win_x, oh, ow) for o in outs]


def _close(got, ref, rel=1e-5):
    scale = np.abs(ref).reshape(ref.shape[0], ref.shape[1], -1).max(axis=2)[..., None, None]
    scale = np.maximum(scale, 1e-30)
    err = np.abs(got - ref) / scale
    assert err.max() <= rel, float(err.max())


@pytest.mark.parametrize("win,ov,fit", [(16, 75, None), (16, 75, (12, 12)), (32, 50, None), (64, 50, (32, 32))])
@pytest.mark.parametrize("ms,ppn", [(0, 0), (1, 0), (1, 1)])
def test_triple_matches_oracle(oracle, cuda, win, ov, fit, ms, ppn):
    A, B = _stack(5, (160, 192), seed=40 + win)
    g = geometry.compute_window_centers(A.shape[1:], (win, win), ov)
    mask = np.zeros((g.n_win_y, g.n_win_x), np.float32)
    mask[1, 2] = 1.0
    wsq = geometry.window_weight((win, win), "square")
    wab_a = geometry.window_weight((win // 2, win // 2), "singlepix", sum_window=(win, win))
    got = _triple_gpu(A, B, mask, g, (win, win), wab_a, wsq, wsq, wsq, fit, ms, ppn)
    ref = oracle.accumulate_triple(A, B, mask, g.win_ctrs_x, g.win_ctrs_y, (win, win), wab_a, wsq, wsq, wsq,
                                   fit_size=fit, mean_subtract=ms, per_pair_norm=ppn)
    for k in range(3):
        live = np.ones((g.n_win_y, g.n_win_x), bool)
        live[1, 2] = False
        _close(got[k][live][None], ref[k][live][None])
        assert np.all(got[k][1, 2] == 0)


@pytest.mark.parametrize("n_pairs", [64, 150])
def test_long_call_matches_oracle(oracle, cuda, n_pairs):
    """Many pairs in one call: the spectra of up to 64 pairs are summed in FP32
    before one inverse transform per block; the planes still match the oracle's
    per-pair Kahan sums within 1e-5 of each plane's magnitude."""
    A, B = _stack(n_pairs, (96, 112), seed=900)
    g = geometry.compute_window_centers(A.shape[1:], (16, 16), 75)
    mask = np.zeros((g.n_win_y, g.n_win_x), np.float32)
    w = geometry.window_weight((16, 16), "square")
    got = _triple_gpu(A, B, mask, g, (16, 16), w, w, w, w, None, 0, 0)
    ref = oracle.accumulate_triple(A, B, mask, g.win_ctrs_x, g.win_ctrs_y, (16, 16), w, w, w, w)
    for k in range(3):
        _close(got[k], ref[k])


def test_plus_equals_semantics(oracle, cuda):
    A, B = _stack(3, (128, 128), seed=7)
    g = geometry.compute_window_centers(A.shape[1:], (16, 16), 50)
    mask = np.zeros((g.n_win_y, g.n_win_x), np.float32)
    w = geometry.window_weight((16, 16), "square")
    first = _triple_gpu(A, B, mask, g, (16, 16), w, w, w, w, None, 1, 0)
    nwt = g.n_win_y * g.n_win_x
    second = _triple_gpu(A, B, mask, g, (16, 16), w, w, w, w, None, 1, 0,
                         init=[f.reshape(-1) for f in first])
    for a, b in zip(first, second):
        np.testing.assert_allclose(b, 2 * a, rtol=2e-6, atol=1e-6 * np.abs(a).max())
    assert nwt > 0


def test_accumulate_ab_matches_oracle(oracle, cuda):
    L = _lib.bulkxcorr2d_lib()
    A, B = _stack(4, (128, 160), seed=11)
    n, H, W = A.shape
    g = geometry.compute_window_centers((H, W), (32, 32), 50)
    mask = np.zeros((g.n_win_y, g.n_win_x), np.float32)
    w = geometry.window_weight((32, 32), "gaussian")
    out = np.zeros(g.n_win_y * g.n_win_x * 32 * 32, np.float32)
    code = L.bulkxcorr2d_accumulate(A, B, mask.ravel(), np.array([H, W], np.int32), n, g.win_ctrs_x, g.win_ctrs_y,
                                    np.array([g.n_win_y, g.n_win_x], np.int32), w.ravel(), w.ravel(),
                                    np.array([32, 32], np.int32), None, out)
    assert code == 0
    ref = np.zeros_like(out)
    e = oracle.lib().orc_accumulate(A, B, mask.ravel(), np.array([H, W], np.int32), n, g.win_ctrs_x, g.win_ctrs_y,
                                    np.array([g.n_win_y, g.n_win_x], np.int32), w.ravel(), w.ravel(),
                                    np.array([32, 32], np.int32), None, ref, 0)
    assert e == 0
    _close(out.reshape(g.n_win_y, g.n_win_x, 32, 32), ref.reshape(g.n_win_y, g.n_win_x, 32, 32))
