"""Pin the oracle's correlator restatement to the reference's own correlator.

The fixtures (`golden/xcorr_ref.npz`, `golden/triple_ref.npz`) hold the outputs of
the reference's libbulkxcorr2d, built from its sources (PIV_2d_cross_correlate.c,
xcorr.c, codelet_fft.c, peak_locate_lm*.c and the codelet headers its generator
writes) by `make -C oracle ref`, on the seeded cases of `golden/xcorr_cases.py`:
the single-pair workload at full size (1024^2, 32 px at 50%), every window size
8-128, multiple peaks, ensemble mode, asymmetric weights, windows outside the
frame, NaN and zero-energy windows, masked windows, rectangular windows, and
bulkxcorr2d_accumulate_triple with every mean/normalisation option.

Bars for the restatement (FP64 planes rounded once to float, against the
reference's FP32 codelet planes): planes within 1e-6 of each plane's peak; the
3-point fit's NaN pattern identical and displacements within 1e-3 px; LM fits
(gauss4-6) flip at most 5% of NaN sentinels (the trust rule's hard threshold
meets 1e-7 plane differences) and disagree by more than 0.005 px on at most 2% of
the windows both fit; skipped windows identical; accumulated sums within 1e-6
of each plane's peak.  When the reference library itself is present, the
restatement is also run against it live on a second config-1 seed.
"""

import os
import sys

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLD)
import xcorr_cases as XC  # noqa: E402


def _ref(g, name):
    r = {k: g[f"{name}__{k}"] for k in XC.OUT_KEYS}
    if f"{name}__planes" in g:
        r["planes"] = g[f"{name}__planes"]
    return r


@pytest.fixture(scope="module")
def fixture():
    return np.load(os.path.join(GOLD, "xcorr_ref.npz"))


@pytest.mark.parametrize("case", XC.all_cases(), ids=lambda c: c["name"])
def test_restated_correlator_matches_reference(oracle, fixture, case):
    nm = case["name"]
    assert XC.checksum(case) == float(fixture[f"{nm}__checksum"]), "case inputs changed"
    want = bool(len(case["plane_idx"]))
    o = oracle.bulkxcorr2d(case["A"], case["B"], case["mask"], case["cx"], case["cy"], case["win"], case["wa"],
                           case["wb"], n_peaks=case["n_peaks"], peak_finder=case["finder"],
                           ensemble=case["ensemble"], want_planes=want, peakfit_impl=case["impl"])
    assert o["error"] == int(fixture[f"{nm}__error"])
    h, w = case["win"]
    st = XC.compare(case, o, _ref(fixture, nm), o["planes"].reshape(-1, h, w) if want else None)
    assert st["zeros_equal"], nm
    if want:
        assert st["plane_rel"] <= 1e-6, st["plane_rel"]
    assert st["height_rel"] <= 1e-4, st["height_rel"]
    if case["finder"] == 3:
        assert st["nan_flip"] == 0 and st["max_d"] <= 1e-3, st
    else:
        assert st["nan_flip"] <= 0.05 * st["n"], st
        assert st["n_far"] <= max(1, 0.02 * st["n"]), st
    r = fixture[f"{nm}__pk_ratio"]
    assert np.array_equal(r == 0, o["pk_ratio"] == 0) or case["finder"] != 3, nm
    ok = (r > 0) & (o["pk_ratio"] > 0)
    close = np.abs(o["pk_ratio"][ok] - r[ok]) <= 1e-3 * np.abs(r[ok])
    assert close.sum() >= 0.99 * ok.sum(), (nm, close.mean())


@pytest.mark.parametrize("case", XC.triple_cases(), ids=lambda c: c["name"])
def test_restated_triple_matches_reference(oracle, case):
    g = np.load(os.path.join(GOLD, "triple_ref.npz"))
    s = oracle.accumulate_triple(case["A"], case["B"], np.zeros((len(case["cy"]), len(case["cx"])), np.float32),
                                 case["cx"], case["cy"], case["win"], *case["w"], fit_size=case["fit"],
                                 mean_subtract=case["ms"], per_pair_norm=case["pn"])
    for k, v in zip(("ab", "aa", "bb"), s):
        R = g[f"{case['name']}__{k}"]
        V = v.reshape(-1, *v.shape[2:])[case["keep"]]
        sc = np.abs(R).reshape(len(R), -1).max(axis=1)
        sc[sc == 0] = 1.0
        assert (np.abs(V - R).reshape(len(R), -1).max(axis=1) / sc).max() <= 1e-6, k


def test_restated_correlator_live_against_reference_library(oracle):
    """A second full-size pair straight through the compiled reference library."""
    if oracle.ref_bulk() is None:
        pytest.skip("reference correlator not built here (make -C oracle ref PIVTOOLS_REF=...)")
    from pivtools_b200 import geometry, synthetic

    A, B, _ = synthetic.particle_pair((1024, 1024), seed=2)
    g = geometry.compute_window_centers(A.shape, (32, 32), 50)
    w = geometry.window_weight((32, 32), "gaussian")
    m = np.zeros((g.n_win_y, g.n_win_x), np.float32)
    r = oracle.ref_bulkxcorr2d(A, B, m, g.win_ctrs_x, g.win_ctrs_y, (32, 32), w, w, want_planes=True)
    o = oracle.bulkxcorr2d(A, B, m, g.win_ctrs_x, g.win_ctrs_y, (32, 32), w, w, want_planes=True)
    sc = np.abs(r["planes"]).max(axis=(-1, -2))
    assert (np.abs(r["planes"] - o["planes"]).max(axis=(-1, -2)) / sc).max() <= 1e-6
    assert np.array_equal(np.isnan(r["pk_x"]), np.isnan(o["pk_x"]))
    d = np.maximum(np.abs(r["pk_x"] - o["pk_x"]), np.abs(r["pk_y"] - o["pk_y"]))
    assert np.nanmax(d) <= 1e-3


def test_correlation_weight_matches_reference(oracle, fixture):
    """numel / (wB (*) wB), the fit patch's loss-of-correlation weight
    (PIV_2d_cross_correlate.c:216-222, xcorr.c:204-271): the oracle's FP64 direct
    sum against the reference's FP32 zero-padded-FFT convolve, square and
    rectangular windows, three weight types, within 2e-6 relative."""
    from pivtools_b200 import geometry

    for h, w in fixture["cw_sizes"]:
        for wt in ("gaussian", "blackman", "square"):
            ref = fixture[f"cw_{wt}_{h}x{w}"]
            got = oracle.correl_weight(geometry.window_weight((int(h), int(w)), wt))
            assert (np.abs(got - ref) / np.abs(ref)).max() <= 2e-6, (h, w, wt)
