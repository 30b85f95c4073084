"""DFT-as-GEMM correlation on the tensor core (libpivb_dft, 32 x 32 and 64 x 64
windows) against the FP64 oracle and the FP32 FFT path, through the C-ABI.

Split-precision BF16 hi + lo operands with three products keep ~16 significant
bits per GEMM operand, so the bars are those of the tensor-core variant:
correlation planes within 1e-4 of each plane's peak magnitude (FP64 oracle),
RMS displacement difference at most 0.01 px, the same NaN sentinels except
documented near-ties, and LM fits (which amplify plane noise) within 0.02 px.
"""

import ctypes

import numpy as np
import pytest

from pivtools_b200 import _lib, geometry, synthetic

pytestmark = pytest.mark.gpu
SIZES = (32, 64)
KEYS = ("pk_x", "pk_y", "pk_h", "sx", "sy", "sxy", "ratio")


def _case(torch, dev, seed, N, shape=(256, 288), overlap=50, flow="uniform_grf"):
    A, B, _ = synthetic.particle_pair(shape, seed=seed, flow=flow)
    g = geometry.compute_window_centers(A.shape, (N, N), overlap)
    w = geometry.window_weight((N, N), "gaussian")
    return A, B, g, w


def _run(L, torch, dev, A, B, g, w, finder, dft, planes=True, impl=0):
    N = w.shape[0]
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    tA, tB = torch.tensor(A[None], device=dev), torch.tensor(B[None], device=dev)
    tw = torch.tensor(w, device=dev)
    cw = torch.empty_like(tw)
    Lx = _lib.bulkxcorr2d_lib()
    assert Lx.pivb_correl_weight_dev(tw.data_ptr(), N, N, cw.data_ptr(), s) == 0
    cx, cy = torch.tensor(g.win_ctrs_x, device=dev), torch.tensor(g.win_ctrs_y, device=dev)
    shp = (1, 1, g.n_win_y, g.n_win_x)
    out = {k: torch.full(shp, -7.0, device=dev) for k in KEYS}
    total = g.n_win_y * g.n_win_x
    pl = torch.zeros((total, N, N), device=dev) if planes else None
    nbytes = int(Lx.pivb_xcorr_scratch_bytes(total, 1, finder))
    scratch = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=dev)
    args = [tA.data_ptr(), tB.data_ptr(), tA.stride(0), None, A.shape[0], A.shape[1], 1, cx.data_ptr(),
            cy.data_ptr(), g.n_win_y, g.n_win_x, tw.data_ptr(), tw.data_ptr(), cw.data_ptr(), N, N, 0, 1, finder,
            impl] + [out[k].data_ptr() for k in KEYS] + [None if pl is None else pl.data_ptr(), scratch.data_ptr(),
                                                         nbytes]
    if dft:
        st = torch.zeros(1, dtype=torch.int32, device=dev)
        assert L.pivb_dft_xcorr_dev(*args, st.data_ptr(), s) == 0
        torch.cuda.synchronize()
        assert st.item() == 0
    else:
        assert Lx.pivb_xcorr_dev(*args, s) == 0
        torch.cuda.synchronize()
    res = {k: v.cpu().numpy().ravel() for k, v in out.items()}
    if pl is not None:
        res["planes"] = pl.cpu().numpy()
    return res


@pytest.mark.parametrize("N", SIZES)
def test_dft_planes_and_gauss3_against_oracle(oracle, cuda, N):
    import torch

    L = _lib.dft_lib()
    A, B, g, w = _case(torch, cuda, 301, N, shape=(256, 288) if N == 32 else (384, 416))
    got = _run(L, torch, cuda, A, B, g, w, 3, dft=True)
    orc = oracle.bulkxcorr2d(A, B, np.zeros((g.n_win_y, g.n_win_x), np.float32), g.win_ctrs_x, g.win_ctrs_y, (N, N),
                             w, w, peak_finder=3, want_planes=True, want_f64=True)
    R = orc["planes_f64"].reshape(-1, N, N)
    P = got["planes"]
    scale = np.abs(R).reshape(len(R), -1).max(axis=1)
    err = np.abs(P - R).reshape(len(R), -1).max(axis=1)
    rel = err / scale
    assert np.all(rel <= 1e-4), float(rel.max())
    gx, ox = got["pk_x"], orc["pk_x"].ravel()
    gy, oy = got["pk_y"], orc["pk_y"].ravel()
    both = np.isfinite(gx) & np.isfinite(ox)
    assert (np.isnan(gx) != np.isnan(ox)).mean() < 0.01
    d = np.hypot(gx - ox, gy - oy)[both]
    assert np.sqrt(np.mean(d ** 2)) <= 0.01, float(np.sqrt(np.mean(d ** 2)))
    np.testing.assert_allclose(got["pk_h"][both], orc["pk_h"].ravel()[both], rtol=2e-3)


@pytest.mark.parametrize("N", SIZES)
@pytest.mark.parametrize("finder", [4, 6])
def test_dft_lm_fits_track_fft_path(cuda, finder, N):
    import torch

    L = _lib.dft_lib()
    A, B, g, w = _case(torch, cuda, 310 + finder, N, shape=(320, 320) if N == 32 else (448, 448), overlap=75)
    got = _run(L, torch, cuda, A, B, g, w, finder, dft=True, planes=False)
    ref = _run(L, torch, cuda, A, B, g, w, finder, dft=False, planes=False)
    both = np.isfinite(got["pk_x"]) & np.isfinite(ref["pk_x"])
    assert both.mean() > 0.8
    d = np.hypot(got["pk_x"] - ref["pk_x"], got["pk_y"] - ref["pk_y"])[both]
    assert np.sqrt(np.mean(d ** 2)) <= 0.02 and np.percentile(d, 99) <= 0.05


@pytest.mark.parametrize("N", SIZES)
def test_dft_batch_of_frames_and_ragged_groups(cuda, N):
    """Several frames per call, a window count that is not a multiple of the
    window group (eight windows at 32 px, four at 64 px), a masked window and an
    out-of-bounds centre."""
    import torch

    L = _lib.dft_lib()
    Lx = _lib.bulkxcorr2d_lib()
    shape = (160, 176) if N == 32 else (320, 352)
    frames = [synthetic.particle_pair(shape, seed=330 + k)[:2] for k in range(3)]
    A = np.stack([f[0] for f in frames]); B = np.stack([f[1] for f in frames])
    g = geometry.compute_window_centers(A.shape[1:], (N, N), 50)
    cxs = np.array(g.win_ctrs_x, np.float32)
    cxs[-1] = shape[1] - 1.0   # pushes the last column of windows out of the frame
    w = geometry.window_weight((N, N), "gaussian")
    mask = np.zeros((g.n_win_y, g.n_win_x), np.float32)
    mask[1, 2] = 1.0
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    dev = cuda
    tA, tB = torch.tensor(A, device=dev), torch.tensor(B, device=dev)
    tw = torch.tensor(w, device=dev)
    cw = torch.empty_like(tw)
    assert Lx.pivb_correl_weight_dev(tw.data_ptr(), N, N, cw.data_ptr(), s) == 0
    cx, cy, tm = torch.tensor(cxs, device=dev), torch.tensor(g.win_ctrs_y, device=dev), torch.tensor(mask, device=dev)
    total = 3 * g.n_win_y * g.n_win_x
    assert total % (8 if N == 32 else 4) != 0
    res = []
    for fn in ("dft", "fft"):
        out = {k: torch.full((3, 1, g.n_win_y, g.n_win_x), -7.0, device=dev) for k in KEYS}
        args = [tA.data_ptr(), tB.data_ptr(), tA.stride(0), tm.data_ptr(), A.shape[1], A.shape[2], 3, cx.data_ptr(),
                cy.data_ptr(), g.n_win_y, g.n_win_x, tw.data_ptr(), tw.data_ptr(), cw.data_ptr(), N, N, 0, 1, 3, 0] + \
            [out[k].data_ptr() for k in KEYS] + [None, None, 0]
        if fn == "dft":
            st = torch.zeros(1, dtype=torch.int32, device=dev)
            assert L.pivb_dft_xcorr_dev(*args, st.data_ptr(), s) == 0
        else:
            assert Lx.pivb_xcorr_dev(*args, s) == 0
        torch.cuda.synchronize()
        res.append({k: v.cpu().numpy() for k, v in out.items()})
    d, f = res
    # skipped windows (masked, out of bounds) are left untouched by both paths
    untouched_d = d["pk_x"] == -7.0
    untouched_f = f["pk_x"] == -7.0
    assert np.array_equal(untouched_d, untouched_f) and untouched_d.sum() >= 3 * (1 + g.n_win_y)
    live = ~untouched_d & np.isfinite(d["pk_x"]) & np.isfinite(f["pk_x"])
    assert np.max(np.abs(d["pk_x"][live] - f["pk_x"][live])) < 0.02


def test_dft_rejects_unsupported(cuda):
    L = _lib.dft_lib()
    args = [1, 1, 0, None, 64, 64, 1, 1, 1, 1, 1, 1, 1, 1, 48, 48, 0, 1, 3, 0] + [1] * 7 + [None, None, 0, 1, None]
    assert L.pivb_dft_xcorr_dev(*args) == 8          # 48 x 48 not on this path
    args[14], args[15] = 32, 64
    assert L.pivb_dft_xcorr_dev(*args) == 8          # nor rectangular windows
    args[14] = args[15] = 32
    args[17] = 2
    assert L.pivb_dft_xcorr_dev(*args) == 9          # n_peaks > 1
