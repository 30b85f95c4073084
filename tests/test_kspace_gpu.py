"""GPU parity of libkspacefit (through its C-ABI).

Contract of the reference's own C-vs-NumPy gate (test_kspace_c_fit.py:48-146):
identical status per window; |dSigma| and |dmu| < 1e-8 on jointly converged
windows; initial guesses equal.  Checked against fixtures produced by the
reference's NumPy oracle and against the project's CPU restatement.
"""

import os

import numpy as np
import pytest

from pivtools_b200 import _lib

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _gpu_fit(R_AA, R_BB, R_AB, mask, corr, ukx, uky, P=None):
    L = _lib.kspacefit_lib()
    h, w = corr
    n = R_AA.size // (h * w)
    o = dict(gauss=np.zeros((n, 16)), status=np.zeros(n, np.int32), init=np.zeros((n, 16)), gain=np.zeros(n),
             N0=np.zeros(n), b4x=np.zeros(n), b4y=np.zeros(n), cpp=np.zeros(n), nv=np.zeros(n, np.int32),
             it=np.zeros(n, np.int32), conv=np.zeros(n, np.uint8))
    Pp = None if P is None else np.ascontiguousarray(P, np.float64)
    r = L.kspace_lm_fit_batch(np.ascontiguousarray(R_AA, np.float64), np.ascontiguousarray(R_BB, np.float64),
                              np.ascontiguousarray(R_AB, np.float64), np.ascontiguousarray(mask, np.uint8),
                              None if Pp is None else Pp.ctypes.data, n, h, w, ukx, uky, 0, o["gauss"], o["status"],
                              o["init"], o["gain"], o["N0"], o["b4x"], o["b4y"], o["cpp"], o["nv"], o["it"], o["conv"])
    assert r == 0
    return o


@pytest.mark.parametrize("shape", ["gaussian", "kx4", "ky4", "kx4+ky4"])
@pytest.mark.parametrize("floor", ["flat", "coloured"])
def test_matches_reference_numpy_oracle(cuda, oracle, shape, floor):
    g = np.load(os.path.join(GOLD, "kspace_ref.npz"))
    corr = tuple(int(v) for v in g["corr"])
    ukx, uky = int("kx4" in shape), int("ky4" in shape)
    P = g["P_win"] if floor == "coloured" else None
    o = _gpu_fit(g["R_AA"], g["R_BB"], g["R_AB"], g["mask"], corr, ukx, uky, P)
    key = f"{shape}_{floor}"
    assert np.array_equal(o["status"], g[f"{key}_status"])
    ok = (o["status"] == 0) & (g[f"{key}_status"] == 0)
    assert ok.any()
    gp = g[f"{key}_gauss"]
    assert np.abs(o["gauss"][ok, 9:12] - gp[ok, 9:12]).max() < 1e-8
    assert np.abs(o["gauss"][ok, 14:16] - gp[ok, 14:16]).max() < 1e-8
    np.testing.assert_allclose(o["init"], g[f"{key}_init"], rtol=0, atol=1e-12)
    # and against the CPU restatement, diagnostics included
    c = oracle.kspace_fit(g["R_AA"], g["R_BB"], g["R_AB"], g["mask"], corr, ukx, uky, P_win=P)
    assert np.array_equal(o["status"], c["status"])
    assert np.array_equal(o["nv"], c["n_valid"])
    np.testing.assert_allclose(o["gain"][ok], c["gain"][ok], rtol=1e-7)


@pytest.mark.parametrize("n", [8, 12, 16, 24, 32])
def test_fft2_centered_matches_numpy(cuda, n):
    L = _lib.kspacefit_lib()
    rng = np.random.default_rng(n)
    x = rng.normal(size=(n, n))
    re = np.zeros((n, n))
    im = np.zeros((n, n))
    assert L.kspace_fft2_centered(np.ascontiguousarray(x), n, n, re, im) == 0
    ref = np.fft.fft2(np.fft.ifftshift(x))
    np.testing.assert_allclose(re, ref.real, atol=1e-12 * np.abs(ref).max())
    np.testing.assert_allclose(im, ref.imag, atol=1e-12 * np.abs(ref).max())


def test_debug_prep_regressor(cuda):
    import ctypes

    L = _lib.kspacefit_lib()
    g = np.load(os.path.join(GOLD, "kspace_ref.npz"))
    h, w = (int(v) for v in g["corr"])
    P = h * w
    aa, bb, ab = (np.ascontiguousarray(g[k][:P]) for k in ("R_AA", "R_BB", "R_AB"))
    Pc = np.ascontiguousarray(g["P_win"][:P])
    Dv = np.zeros(P)
    seed = ctypes.c_double(0.0)
    assert L.kspace_debug_prep(aa, bb, ab, Pc.ctypes.data, h, w, Dv, ctypes.byref(seed)) == 0
    Faa = np.fft.fft2(np.fft.ifftshift(aa.reshape(h, w)))
    Fbb = np.fft.fft2(np.fft.ifftshift(bb.reshape(h, w)))
    Fr = np.sqrt(np.abs(Faa) * np.abs(Fbb))
    Pn = np.fft.ifftshift(Pc.reshape(h, w))
    np.testing.assert_allclose(Dv.reshape(h, w), Pn / np.maximum(Fr, 1e-30), rtol=1e-10)
    ky, kx = np.meshgrid(np.fft.fftfreq(h), np.fft.fftfreq(w), indexing="ij")
    tail = (kx ** 2 + ky ** 2) >= 0.35 ** 2
    med = float(np.clip(np.median((Fr / np.maximum(Pn, 1e-30))[tail]), 1e-3, 10.0))
    assert abs(seed.value - med) < 1e-10 * max(1.0, med)


def test_all_masked_and_bad_size(cuda):
    L = _lib.kspacefit_lib()
    n, h = 3, 16
    z = np.ones(n * h * h)
    o = _gpu_fit(z, z, z, np.ones(n, np.uint8), (h, h), 0, 0)
    assert np.all(o["status"] == -1)
    assert np.all(np.isnan(o["init"][:, 6:9]))      # all-masked batch mirrors the defaults
    assert L.kspace_lm_fit_max_threads() > 0
    re = np.zeros(100)
    assert L.kspace_fft2_centered(np.zeros(100), 10, 10, re, re.copy()) == -1
