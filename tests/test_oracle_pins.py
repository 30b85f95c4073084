"""Pin the CPU oracle (the checker) to the reference.

The oracle's restatements must reproduce the reference's own outputs:
  * peak fitter, scalar and batch routes: bit-exact against fixtures produced by
    the reference's peak_locate_lm*.c compiled from source (tests/golden);
  * fused warp: bit-exact against the reference's fused_warp.c scalar route;
  * k-space fit: the reference's own parity contract against its NumPy oracle
    (status equality, |dSigma|, |dmu| < 1e-8; test_kspace_c_fit.py:53-54);
  * correlation planes: against a brute-force FP64 circular correlation, the
    reference's codelet gate (test_codelet_gate.c:33-49).
"""

import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _eq(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


def test_peakfit_scalar_matches_reference_fixture(oracle):
    g = np.load(os.path.join(GOLD, "peakfit_ref.npz"))
    n_checked = 0
    for si, shape in enumerate(g["shapes"]):
        planes = g[f"s{si}_planes"]
        for k in range(planes.shape[0]):
            t = int(g[f"s{si}_types"][k])
            m = int(g[f"s{si}_npeaks"][k])
            w = g[f"s{si}_weights"][k] if g[f"s{si}_hasw"][k] else None
            loc, sd = oracle.peakfit(planes[k], t, n_peaks=m, weight=w)
            assert _eq(loc, g[f"s{si}_loc"][k, :3 * m]), (tuple(shape), k, t, loc, g[f"s{si}_loc"][k])
            assert _eq(sd, g[f"s{si}_sd"][k, :3 * m]), (tuple(shape), k, t)
            assert _eq(np.float32(oracle.detectability(planes[k])), g[f"s{si}_ratio"][k])
            n_checked += 1
    assert n_checked >= 140


def test_peakfit_batch_matches_reference_fixture(oracle):
    g = np.load(os.path.join(GOLD, "peakfit_ref.npz"))
    for k in range(g["batch_planes"].shape[0]):
        loc, sd = oracle.peakfit(g["batch_planes"][k], int(g["batch_types"][k]), exp_mode=1)
        assert _eq(loc, g["batch_loc"][k]), k
        assert _eq(sd, g["batch_sd"][k]), k


def test_warp_matches_reference_fixture(oracle):
    g = np.load(os.path.join(GOLD, "warp_ref.npz"))
    for mode in (0, 1):
        for rs in (0, 1):
            oa, ob = oracle.fused_warp_batch(g["imgs_a"], g["imgs_b"], g["pred_dy"], g["pred_dx"],
                                             g["ctrs_y"], g["ctrs_x"], interp_mode=mode, round_shifts=rs)
            assert _eq(oa, g[f"out_a_m{mode}_r{rs}"]), (mode, rs)
            assert _eq(ob, g[f"out_b_m{mode}_r{rs}"]), (mode, rs)


@pytest.mark.parametrize("shape", ["gaussian", "kx4", "ky4", "kx4+ky4"])
@pytest.mark.parametrize("floor", ["flat", "coloured"])
def test_kspace_matches_reference_numpy_oracle(oracle, shape, floor):
    g = np.load(os.path.join(GOLD, "kspace_ref.npz"))
    corr = tuple(int(v) for v in g["corr"])
    o = oracle.kspace_fit(g["R_AA"], g["R_BB"], g["R_AB"], g["mask"], corr,
                          use_kx4=int("kx4" in shape), use_ky4=int("ky4" in shape),
                          P_win=g["P_win"] if floor == "coloured" else None)
    key = f"{shape}_{floor}"
    st_ref = g[f"{key}_status"]
    assert np.array_equal(o["status"], st_ref)
    ok = (o["status"] == 0) & (st_ref == 0)
    assert ok.any()
    gp = g[f"{key}_gauss"]
    assert np.abs(o["gauss_flat"][ok, 9:12] - gp[ok, 9:12]).max() < 1e-8
    assert np.abs(o["gauss_flat"][ok, 14:16] - gp[ok, 14:16]).max() < 1e-8
    np.testing.assert_allclose(o["initial_guess"], g[f"{key}_init"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("n", [8, 12, 16, 24, 32, 48])
def test_xcorr_plane_is_circular_correlation(oracle, n):
    rng = np.random.default_rng(n)
    a = rng.normal(size=(n, n)).astype(np.float32)
    b = rng.normal(size=(n, n)).astype(np.float32)
    got = oracle.xcorr_plane(a, b)
    ref = np.zeros((n, n))
    ad, bd = a.astype(np.float64), b.astype(np.float64)
    for r in range(n):
        for c in range(n):
            s = (r - n // 2, c - n // 2)
            ref[r, c] = np.sum(np.roll(ad, (-s[0], -s[1]), axis=(0, 1)) * bd)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-9 * np.abs(ref).max())


def test_oracle_recovers_known_shift(oracle):
    from pivtools_b200 import geometry, synthetic

    A, B, _ = synthetic.particle_pair((128, 128), seed=3, flow="uniform", flow_kwargs={"u": 3.3, "v": -1.7})
    g = geometry.compute_window_centers((128, 128), (32, 32), 50)
    w = geometry.window_weight((32, 32), "gaussian")
    o = oracle.bulkxcorr2d(A, B, np.zeros((g.n_win_y, g.n_win_x)), g.win_ctrs_x, g.win_ctrs_y, (32, 32), w, w)
    dx = np.nanmedian(o["pk_x"])
    dy = np.nanmedian(o["pk_y"])
    assert abs(dx - 3.3) < 0.05 and abs(dy + 1.7) < 0.05


def test_oracle_matches_live_reference_fitter(oracle):
    R = oracle.ref_peakfit()
    if R is None:
        pytest.skip("reference fitter not compiled in this checkout (fixture test covers it)")
    rng = np.random.default_rng(99)
    for k in range(200):
        t = (3, 4, 5, 6)[k % 4]
        p = rng.gamma(2.0, 50.0, (33, 33)).astype(np.float32)
        p[16, 16] += 800.0
        loc, sd = oracle.peakfit(p, t)
        l2 = np.zeros(3, np.float32)
        s2 = np.zeros(3, np.float32)
        R.lsqpeaklocate_lm(p, np.array([33, 33], np.int32), l2, 1, t, s2, None)
        assert _eq(loc, l2) and _eq(sd, s2)


def test_ensemble_finalise_restatement_matches_reference_fixture(oracle):
    """Pair-count envelope and plane-mean removal against the reference's own
    functions (fixture from tests/golden/make_golden.py ensemble)."""
    g = np.load(os.path.join(GOLD, "ensemble_ref.npz"))
    for wtype in ("square", "gaussian", "blackman"):
        for n in (16, 32):
            env = oracle.pair_envelope(g[f"w_{wtype}_{n}"], g[f"w_{wtype}_{n}"], (n, n))
            np.testing.assert_allclose(env, g[f"env_{wtype}_{n}"], rtol=1e-12, atol=1e-14)
    got = oracle.zero_plane_means(g["dc_in"].reshape(7, 16, 16)).ravel()
    np.testing.assert_allclose(got, g["dc_out"], rtol=0, atol=2e-6)


ROTS = {"none": 0, "cw90": 3, "ccw90": 1, "180": 2}


def test_ingest_decode_restatement_matches_reference_fixture(oracle):
    """Mono12p / BayerRG8 payload decode with and without the in-run dark, every
    view rotation, against the reference's own decode (fixture from
    tests/golden/make_golden.py ingest)."""
    g = np.load(os.path.join(GOLD, "ingest_ref.npz"))
    W, H, n = int(g["W"]), int(g["H"]), int(g["n"])
    for fi, fmt in enumerate(("Mono12p", "BayerRG8")):
        for view, rot in ROTS.items():
            for with_dark in (0, 1):
                got = oracle.decode_frames(g[f"{fmt}_raw"], int(g[f"{fmt}_stride"]), n, 1, W, H, fi,
                                           g[f"{fmt}_dark"] if with_dark else None, 2, rot)
                assert np.array_equal(got, g[f"{fmt}_{view}_{with_dark}"]), (fmt, view, with_dark)


def test_median_outlier_restatement_matches_reference_fixture(oracle):
    """Normalised-median outlier test against the reference's own function
    (fixture from tests/golden/make_golden.py validate): zeroed failed vectors,
    masked windows, sizes 3 and 5."""
    g = np.load(os.path.join(GOLD, "validate_ref.npz"))
    for case in range(4):
        m = g[f"c{case}_masked"] if case >= 2 else None
        for size in (3, 5):
            got = oracle.median_outlier(g[f"c{case}_ux"], g[f"c{case}_uy"], 0.1, 2.0, size, masked=m)
            assert np.array_equal(got, g[f"c{case}_s{size}_median"]), (case, size)
        assert np.array_equal(g[f"c{case}_pk"] < 0.25, g[f"c{case}_peakmag"]) or \
            np.array_equal((g[f"c{case}_pk"] < 0.25) | np.isnan(g[f"c{case}_pk"]), g[f"c{case}_peakmag"])


def test_pass_validation_outlier_stage_matches_reference_fixture(oracle):
    """The outlier stage of the pass-validation restatement is the OR of the
    reference's peak-magnitude and median tests with masked windows exempt, and
    the reason codes follow the first claiming stage (fixture fields, no gate)."""
    g = np.load(os.path.join(GOLD, "validate_ref.npz"))
    for case in range(4):
        m = g[f"c{case}_masked"] if case >= 2 else None
        ux, uy, pk = g[f"c{case}_ux"], g[f"c{case}_uy"], g[f"c{case}_pk"]
        _, _, nan_mask, reason = oracle.pass_validation(ux, uy, pk, None, None, m, 1e6, 1e6, 0.25, 0.1, 2.0, 5)
        mk = np.zeros(ux.shape, bool) if m is None else m
        flagged = (g[f"c{case}_s5_median"] | g[f"c{case}_peakmag"]) & ~mk
        assert np.array_equal(nan_mask, flagged | mk)
        assert np.array_equal(reason == 10, flagged) and np.array_equal(reason == -1, mk)
        assert np.all(reason[~(flagged | mk)] == 0)


def test_floor_grid_and_lookup_match_reference_fixture(oracle):
    """Coloured-floor P grid (package builder) and per-window lookup (oracle
    restatement) against the reference's build_P_grid / interp_P
    (fixture from tests/golden/make_golden.py floor)."""
    from pivtools_b200 import floor_psd

    g = np.load(os.path.join(GOLD, "floor_ref.npz"))
    cases = [("lanczos", True), ("lanczos", False), ("cubic", True), ("cubic", False)]
    fx, fy = oracle.floor_fractions(g["pred_dx"]), oracle.floor_fractions(g["pred_dy"])
    for ci, (kernel, hole) in enumerate(cases):
        fs, P = floor_psd.build_p_grid(g[f"c{ci}_env"], kernel, hole, g[f"c{ci}_w"], n_fracs=5)
        assert np.array_equal(fs, g[f"c{ci}_fs"])
        np.testing.assert_allclose(P, g[f"c{ci}_P"], rtol=1e-13, atol=1e-13 * np.abs(P).max())
        got = oracle.floor_interp(g[f"c{ci}_fs"], g[f"c{ci}_P"], fx, fy)
        assert np.array_equal(got, g[f"c{ci}_Pwin"]), ci


def test_vector_masks_match_reference_fixture():
    """Per-pass masked-window flags from a pixel mask against the reference's
    compute_vector_mask (fixture from tests/golden/make_golden.py vmask)."""
    from pivtools_b200 import geometry

    g = np.load(os.path.join(GOLD, "vmask_ref.npz"))
    for ci in range(2):
        pm = g[f"c{ci}_pixel_mask"]
        for ti, thr in enumerate((0.0, 0.5, 0.9)):
            got = geometry.compute_vector_masks(pm, pm.shape, [(64, 64), (32, 32), (16, 16)], [50, 50, 75], thr)
            for k in range(3):
                ref = g[f"c{ci}_t{ti}_p{k}"]
                assert ref.any() and np.array_equal(got[k], ref), (ci, thr, k)


@pytest.mark.parametrize("shape", ["gaussian", "kx4", "ky4", "kx4+ky4"])
@pytest.mark.parametrize("floor", ["flat", "coloured"])
def test_kspace_matches_reference_c_library(oracle, shape, floor):
    """The restated fitter against the reference's compiled kspace_lm_fit.c
    (fixture golden/kspace_c_ref.npz): equal statuses, Sigma and mu within 1e-8."""
    g = np.load(os.path.join(GOLD, "kspace_ref.npz"))
    c = np.load(os.path.join(GOLD, "kspace_c_ref.npz"))
    corr = tuple(int(v) for v in g["corr"])
    o = oracle.kspace_fit(g["R_AA"], g["R_BB"], g["R_AB"], g["mask"], corr,
                          use_kx4=int("kx4" in shape), use_ky4=int("ky4" in shape),
                          P_win=g["P_win"] if floor == "coloured" else None)
    key = f"{shape}_{floor}"
    assert np.array_equal(o["status"], c[f"{key}_status"])
    ok = o["status"] == 0
    assert ok.any()
    gp = c[f"{key}_gauss_flat"]
    assert np.abs(o["gauss_flat"][ok, 9:12] - gp[ok, 9:12]).max() < 1e-8
    assert np.abs(o["gauss_flat"][ok, 14:16] - gp[ok, 14:16]).max() < 1e-8
    np.testing.assert_allclose(o["initial_guess"], c[f"{key}_initial_guess"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("method,order", [("harmonic", 1), ("biharmonic", 2)])
def test_least_squares_fill_matches_reference(method, order):
    """The restated least-squares infill (oracle/ref_multipass.py) against the
    reference's own infill_harmonic / infill_biharmonic (golden/infill_ref.npz)."""
    import sys

    sys.path.insert(0, GOLD)
    import ref_multipass as RM
    from infill_cases import infill_cases

    g = np.load(os.path.join(GOLD, "infill_ref.npz"))
    for k, c in enumerate(infill_cases()):
        U, V = c["ux"].copy(), c["uy"].copy()
        U[c["fill"]] = np.nan
        V[c["fill"]] = np.nan
        out = RM.fill_least_squares(np.stack([U, V]), c["fill"], c["pitch"], order, c["exclude"])
        np.testing.assert_allclose(out[0], g[f"c{k}_{method}_ux"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(out[1], g[f"c{k}_{method}_uy"], rtol=0, atol=1e-9)
