"""CPU checks: the C-ABI libraries load and export every declared symbol, and the
host-side grid rules reproduce the reference's numbers."""

import ctypes
import os
import re

import numpy as np
import pytest

from pivtools_b200 import _lib, geometry

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
HEADER_LIB = {
    "libbulkxcorr2d.h": "libbulkxcorr2d.so",
    "libfusedwarp.h": "libfusedwarp.so",
    "libkspacefit.h": "libkspacefit.so",
    "libpivb_pass.h": "libpivb_pass.so",
    "libpivb_dft.h": "libpivb_dft.so",
    "libpivb_lavision.h": "libpivb_lavision.so",
}


def _declared(header):
    txt = open(os.path.join(INCLUDE, header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", txt)
    skip = {"if", "for", "while", "return", "sizeof", "defined"}
    return sorted({n for n in names if n not in skip})


@pytest.mark.parametrize("header", sorted(HEADER_LIB))
def test_library_exports_every_declared_symbol(header):
    path = _lib.lib_path(HEADER_LIB[header])
    if not os.path.isfile(os.path.join(INCLUDE, header)):
        pytest.skip(f"{header} not written yet")
    assert os.path.isfile(path), f"{path} not built"
    L = ctypes.CDLL(path)
    missing = [n for n in _declared(header) if not hasattr(L, n)]
    assert not missing, missing


def test_selectors_without_gpu():
    L = _lib.bulkxcorr2d_lib()
    assert L.pivtools_cpu_supported() == 1
    assert L.bulkxcorr2d_set_peakfit_impl(1) == 0 and L.bulkxcorr2d_get_peakfit_impl() == 1
    assert L.bulkxcorr2d_set_peakfit_impl(0) == 0 and L.bulkxcorr2d_get_peakfit_impl() == 0
    assert L.peakfit_batch_lanes() == L.codelet_lanes() <= 16
    W = _lib.fusedwarp_lib()
    assert W.fused_warp_get_impl() == 1
    W.fused_warp_set_impl(0)
    assert W.fused_warp_get_impl() == 0
    W.fused_warp_set_impl(1)


def test_config1_grid():
    g = geometry.compute_window_centers((1024, 1024), (32, 32), 50)
    assert (g.n_win_y, g.n_win_x) == (63, 63)
    assert g.win_ctrs_x[0] == 15.5 and g.win_spacing_x == 16
    assert g.win_ctrs_y[-1] == 1024 - 33 / 2.0


def test_config2_grids():
    geo = geometry.multipass_geometry((2048, 2048), [(128, 128), (64, 64), (32, 32), (32, 32)],
                                      [50, 50, 50, 75])
    counts = [g.grid.n_win_y * g.grid.n_win_x for g in geo]
    assert counts == [31 ** 2, 63 ** 2, 127 ** 2, 253 ** 2]
    assert sum(counts) == 85068
    for g in geo[1:]:
        assert g.pred_map_x.shape == (g.grid.n_win_y, g.grid.n_win_x)
        assert g.ksize_filt[0] % 2 == 1
    assert geo[0].sd == 0.0 and geo[1].ksize_filt == (3, 3)


def test_config3_grid():
    g = geometry.compute_window_centers((1024, 1024), (16, 16), 75)
    assert g.n_win_y * g.n_win_x == 64009


@pytest.mark.parametrize("wt", ["gaussian", "square", "blackman", "gaussianTOP"])
def test_window_weights(wt):
    w = geometry.window_weight((32, 32), wt)
    assert w.shape == (32, 32) and w.dtype == np.float32 and np.all(w >= 0)
    if wt == "gaussian":
        assert abs(float(w[15, 15]) - np.exp(-0.5 * 2 * (0.5 / 16) ** 2)) < 1e-6


def test_single_mode_grid_weights_and_envelopes():
    """Ensemble single mode against the reference's own functions
    (tests/golden/make_golden.py ensemble): the padded grid and its padding
    (window_utils.py), the singlepix / bsingle weights (base.py) and the two
    envelopes of the finalise (single_pass_accumulator.py:52-102, 706-716)."""
    from pivtools_b200 import ensemble

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "ensemble_ref.npz"))
    k = 0
    while f"single{k}_case" in g.files:
        H, W, wh, ww, sh, sw, ov = (int(v) for v in g[f"single{k}_case"])
        grid, pad = geometry.compute_window_centers_single_mode((H, W), (wh, ww), (sh, sw), ov)
        meta = g[f"single{k}_meta"]
        assert [grid.n_win_x, grid.n_win_y, grid.win_spacing_x, grid.win_spacing_y, *pad] == meta.tolist(), k
        assert np.array_equal(grid.win_ctrs_x, g[f"single{k}_cx"]) and np.array_equal(grid.win_ctrs_y, g[f"single{k}_cy"])
        k += 1
    assert k == 4
    for key in [f for f in g.files if f.startswith("sp_") and f.endswith("_wa")]:
        _, win, sumw, fit = key[:-3].split("_")
        win, sumw, fit = (int(win),) * 2, (int(sumw),) * 2, (int(fit),) * 2
        wa = geometry.window_weight(win, "singlepix", sumw)
        wb = geometry.window_weight(sumw, "bsingle", sumw)
        assert np.array_equal(wa, g[key]) and np.array_equal(wb, g[key[:-3] + "_wb"])
        np.testing.assert_allclose(ensemble.pair_envelope(wb, wb, fit), g[key[:-3] + "_env_auto"], rtol=1e-12,
                                   atol=1e-14)
        np.testing.assert_allclose(ensemble.pair_envelope(wa, wb, fit), g[key[:-3] + "_env_ab"], rtol=1e-12,
                                   atol=1e-14)
    with pytest.raises(ValueError, match="must be >="):
        geometry.compute_window_centers_single_mode((64, 64), (16, 16), (8, 8), 50)
    with pytest.raises(ValueError, match="exceeds envelope support"):
        ensemble.pair_envelope(np.ones((8, 8)), np.ones((8, 8)), (16, 16))
    wa, wb = np.zeros((16, 16)), np.zeros((16, 16))
    wa[0:4, 0:4] = 1.0                                   # windows 8 px apart: the envelope peak leaves the centre
    wb[8:12, 8:12] = 1.0
    with pytest.raises(ValueError, match="centering is off"):
        ensemble.pair_envelope(wa, wb, (16, 16))
