"""GPU parity of libfusedwarp (through its C-ABI).

impl 0 must equal the reference's scalar route bit for bit and impl 1 its
default SIMD route (fixtures produced by the reference's fused_warp.c compiled
from source); larger seeded cases are checked against the oracle restatement.
The reference's own accuracy bar against cv2.remap (mean error < 0.1% of the
range, test_fused_warp.py:1-14) is checked on a smooth field.
"""

import os

import numpy as np
import pytest

from pivtools_b200 import _lib, geometry, synthetic

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _warp(ia, ib, pdy, pdx, cy, cx, mode, rs=0, impl=0, shared=0):
    L = _lib.fusedwarp_lib()
    L.fused_warp_set_impl(impl)
    N, H, W = ia.shape
    oa = np.zeros_like(ia)
    ob = np.zeros_like(ib)
    nPY, nPX = pdy.shape[-2:]
    r = L.fused_symmetric_warp_batch(np.ascontiguousarray(ia), np.ascontiguousarray(ib), oa, ob,
                                     np.ascontiguousarray(pdy), np.ascontiguousarray(pdx), N, H, W, nPY, nPX,
                                     np.ascontiguousarray(cy), np.ascontiguousarray(cx), mode, shared, rs)
    L.fused_warp_set_impl(1)
    assert r == 0
    return oa, ob


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("rs", [0, 1])
def test_scalar_route_bit_exact(cuda, mode, rs):
    g = np.load(os.path.join(GOLD, "warp_ref.npz"))
    oa, ob = _warp(g["imgs_a"], g["imgs_b"], g["pred_dy"], g["pred_dx"], g["ctrs_y"], g["ctrs_x"], mode, rs, impl=0)
    assert np.array_equal(oa, g[f"out_a_m{mode}_r{rs}"])
    assert np.array_equal(ob, g[f"out_b_m{mode}_r{rs}"])


@pytest.mark.parametrize("mode", [0, 1])
def test_simd_route_bit_exact(cuda, mode):
    g = np.load(os.path.join(GOLD, "warp_ref.npz"))
    oa, ob = _warp(g["imgs_a"], g["imgs_b"], g["pred_dy"], g["pred_dx"], g["ctrs_y"], g["ctrs_x"], mode, 0, impl=1)
    assert np.array_equal(oa, g[f"simd_a_m{mode}"])
    assert np.array_equal(ob, g[f"simd_b_m{mode}"])


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("shared", [0, 1])
def test_against_oracle_multipass_grid(cuda, oracle, mode, shared):
    H, W = 200, 264
    A, B, _ = synthetic.particle_pair((H, W), seed=21, flow="channel", flow_kwargs={"peak": 6.0})
    geo = geometry.multipass_geometry((H, W), [(32, 32), (16, 16)], [50, 50])
    g0 = geo[0]
    ny, nx = len(g0.ctrs_y_all), len(g0.ctrs_x_all)
    rng = np.random.default_rng(3)
    n = 3
    pdy = rng.normal(0, 1.5, (1 if shared else n, ny, nx)).astype(np.float32)
    pdx = (3.0 + rng.normal(0, 1.5, (1 if shared else n, ny, nx))).astype(np.float32)
    ia = np.stack([A] * n)
    ib = np.stack([B] * n)
    oa, ob = _warp(ia, ib, pdy, pdx, g0.ctrs_y_all, g0.ctrs_x_all, mode, impl=0, shared=shared)
    ra, rb = oracle.fused_warp_batch(ia, ib, pdy, pdx, g0.ctrs_y_all, g0.ctrs_x_all, interp_mode=mode,
                                     shared_predictor=shared)
    assert np.array_equal(oa, ra) and np.array_equal(ob, rb)
    oa1, _ = _warp(ia, ib, pdy, pdx, g0.ctrs_y_all, g0.ctrs_x_all, mode, impl=1, shared=shared)
    assert np.abs(oa1 - ra).max() <= 1e-3 * max(1.0, np.abs(ra).max()) / 255.0 * 255.0


def test_against_cv2_remap(cuda):
    cv2 = pytest.importorskip("cv2")
    H, W = 128, 160
    A, B, _ = synthetic.particle_pair((H, W), seed=5, flow="uniform", flow_kwargs={"u": 0.0, "v": 0.0})
    cy = np.linspace(0, H - 1, 9).astype(np.float32)
    cx = np.linspace(0, W - 1, 11).astype(np.float32)
    yy, xx = np.meshgrid(cy, cx, indexing="ij")
    pdx = (2.0 * np.sin(yy / 40.0)).astype(np.float32)[None]
    pdy = (1.0 * np.cos(xx / 50.0)).astype(np.float32)[None]
    oa, _ = _warp(A[None], B[None], pdy, pdx, cy, cx, 0, impl=1)
    # dense predictor with the same bicubic upsampling, then cv2 bicubic remap of A
    iy = np.interp(np.arange(H), cy, np.arange(len(cy))).astype(np.float32)
    ix = np.interp(np.arange(W), cx, np.arange(len(cx))).astype(np.float32)
    my, mx = np.meshgrid(iy, ix, indexing="ij")
    ddx = cv2.remap(pdx[0], mx, my, cv2.INTER_CUBIC, borderMode=cv2.BORDER_REPLICATE)
    ddy = cv2.remap(pdy[0], mx, my, cv2.INTER_CUBIC, borderMode=cv2.BORDER_REPLICATE)
    gy, gx = np.meshgrid(np.arange(H, dtype=np.float32), np.arange(W, dtype=np.float32), indexing="ij")
    ref = cv2.remap(A, gx - 0.5 * ddx, gy - 0.5 * ddy, cv2.INTER_CUBIC, borderMode=cv2.BORDER_CONSTANT, borderValue=0)
    inner = (slice(4, H - 4), slice(4, W - 4))
    rng_ = float(A.max() - A.min())
    err = np.abs(oa[0][inner] - ref[inner])
    assert err.mean() < 1e-3 * rng_
    assert np.percentile(err, 99.9) < 5e-2 * rng_


def test_bad_arguments_return_one(cuda):
    L = _lib.fusedwarp_lib()
    z = np.zeros((1, 8, 8), np.float32)
    c = np.zeros(2, np.float32)
    p = np.zeros((1, 2, 2), np.float32)
    assert L.fused_symmetric_warp_batch(z, z, z.copy(), z.copy(), p, p, 0, 8, 8, 2, 2, c, c, 0, 0, 0) == 1
