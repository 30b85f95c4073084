"""The 'nearest' fill of a predictor's masked windows (masking.predictor_fill:
nearest): the donor map of pivtools_b200.geometry.nearest_donor_map, applied as a
gather, equals the reference's fill_masked_predictor(..., 'nearest')
(infilling.py:808-874) on its own outputs (tests/golden/pfill_ref.npz, written by
tests/golden/make_golden.py pfill): blob, edge and stripe masks, isotropic and
anisotropic pitches.  The GPU gather is checked in the gpu-marked test."""

import ctypes
import os

import numpy as np
import pytest

from pivtools_b200 import _lib, geometry

GOLD = os.path.join(os.path.dirname(__file__), "golden", "pfill_ref.npz")


def _cases():
    z = np.load(GOLD)
    for k in range(int(z["n_cases"])):
        yield k, z[f"c{k}_field"], z[f"c{k}_mask"], tuple(z[f"c{k}_pitch"]), z[f"c{k}_filled"]


def test_donor_map_reproduces_reference_fill():
    for k, field, mask, pitch, ref in _cases():
        idx = geometry.nearest_donor_map(mask, pitch).ravel()
        ny, nx = mask.shape
        flat = field.reshape(field.shape[0], ny * nx, 2)
        got = flat[:, idx].reshape(field.shape)
        assert np.array_equal(got, ref), k
        assert np.array_equal(idx.reshape(ny, nx)[~mask], np.flatnonzero(~mask)), k


def test_donor_map_refuses_fully_masked_grid():
    with pytest.raises(ValueError):
        geometry.nearest_donor_map(np.ones((4, 5), bool), (16.0, 16.0))


@pytest.mark.gpu
def test_gather_fill_on_gpu_equals_reference(cuda):
    import torch

    L = _lib.pass_lib()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for k, field, mask, pitch, ref in _cases():
        N = field.shape[0]
        ny, nx = mask.shape
        idx = torch.tensor(geometry.nearest_donor_map(mask, pitch).ravel(), dtype=torch.int32, device=cuda)
        uy = torch.tensor(np.ascontiguousarray(field[..., 0]), device=cuda)
        ux = torch.tensor(np.ascontiguousarray(field[..., 1]), device=cuda)
        ox, oy = torch.empty_like(ux), torch.empty_like(uy)
        assert L.pivb_gather_fill_dev(ux.data_ptr(), uy.data_ptr(), idx.data_ptr(), N, ny * nx, ox.data_ptr(),
                                      oy.data_ptr(), s) == 0
        torch.cuda.synchronize()
        assert np.array_equal(oy.cpu().numpy(), ref[..., 0]), k
        assert np.array_equal(ox.cpu().numpy(), ref[..., 1]), k


@pytest.mark.gpu
def test_multipass_nearest_predictor_fill(cuda):
    """With a vector mask, the nearest fill changes the predictor only through the
    masked windows: the fields outside the mask's reach match the harmonic run on
    the first pass and every pass runs."""
    import torch

    from pivtools_b200 import multipass, synthetic

    HW = (384, 384)
    sizes, ovl = [(64, 64), (32, 32)], [50, 50]
    geo = geometry.multipass_geometry(HW, sizes, ovl, "gaussian")
    masks = []
    for g in geo:
        ny, nx = g.grid.n_win_y, g.grid.n_win_x
        yy, xx = np.mgrid[0:ny, 0:nx]
        masks.append((yy - ny / 2) ** 2 + (xx - nx / 3) ** 2 < (ny / 6) ** 2)
    A, B = synthetic.channel_batch_torch(1, HW, seed=81, device=cuda, peak=6.0)
    out = {}
    for fill in ("nearest", "harmonic"):
        cfg = multipass.MultipassConfig(window_sizes=sizes, overlaps=ovl, predictor_fill=fill)
        mp = multipass.MultipassPIV(HW, 1, cfg, device=cuda, vector_masks=masks)
        mp.run(A, B)
        torch.cuda.synchronize()
        out[fill] = [(p["ux"].cpu().numpy().copy(), p["pdx"].cpu().numpy().copy()) for p in mp.passes]
    # the first pass sees no predictor: identical
    assert np.array_equal(out["nearest"][0][0], out["harmonic"][0][0], equal_nan=True)
    # its padded predictor differs (the masked windows are filled differently)
    assert not np.array_equal(out["nearest"][0][1], out["harmonic"][0][1])
    assert np.isfinite(out["nearest"][1][0]).all()


def test_multipass_config_refusals_without_gpu():
    """Configuration errors are refused before any device work."""
    from pivtools_b200 import multipass

    HW = (256, 256)
    with pytest.raises(ValueError, match="predictor_fill"):
        multipass.MultipassPIV(HW, 1, multipass.MultipassConfig(predictor_fill="linear"), device="cuda:0")
    with pytest.raises(ValueError, match="one peak"):
        multipass.MultipassPIV(HW, 1, multipass.MultipassConfig(n_peaks=2, engine_32="dft"), device="cuda:0")
    with pytest.raises(ValueError, match="n_peaks"):
        multipass.MultipassPIV(HW, 1, multipass.MultipassConfig(n_peaks=0), device="cuda:0")
