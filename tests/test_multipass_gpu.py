"""GPU multipass: the inter-pass glue kernels against NumPy/SciPy restatements of
the reference's Python steps, and the resident multipass driver against known
displacement fields."""

import ctypes

import numpy as np
import pytest

from pivtools_b200 import _lib, geometry, multipass, synthetic

pytestmark = pytest.mark.gpu


def _t(x, dev, dtype=None):
    import torch

    return torch.as_tensor(np.ascontiguousarray(x), device=dev, dtype=dtype)


def _stream():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _validate(L, cuda, pk_x, pk_y, pk_h, pdy, pdx, mask, thr, size, peak_thr=0.25, med_thr=2.0, reasons=False):
    import torch

    N, ny, nx = pk_x.shape
    ux = torch.empty((N, ny, nx), device=cuda)
    uy = torch.empty_like(ux)
    inv = torch.empty((N, ny, nx), dtype=torch.uint8, device=cuda)
    rc = torch.full((N, ny, nx), 99, dtype=torch.int8, device=cuda)
    work = torch.empty(2 * N * ny * nx, device=cuda)
    T = [_t(a, cuda) for a in (pk_x, pk_y, pk_h)]
    P = [None if a is None else _t(a, cuda) for a in (pdy, pdx, mask)]
    assert L.pivb_validate_dev(T[0].data_ptr(), T[1].data_ptr(), T[2].data_ptr(),
                               *[None if t is None else t.data_ptr() for t in P], N, ny, nx, thr, thr, peak_thr, 0.1,
                               med_thr, size, ux.data_ptr(), uy.data_ptr(), inv.data_ptr(),
                               rc.data_ptr() if reasons else None, work.data_ptr(), _stream()) == 0
    torch.cuda.synchronize()
    out = (inv.cpu().numpy().astype(bool), ux.cpu().numpy(), uy.cpu().numpy())
    return out + (rc.cpu().numpy(),) if reasons else out


def test_median_matches_reference_fixture(cuda):
    """The GPU normalised-median test on the reference's own fixture fields
    (outlier_detection.median_outlier_detection, tests/golden/validate_ref.npz)."""
    import os

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "validate_ref.npz"))
    L = _lib.pass_lib()
    for case in range(4):
        ux, uy = g[f"c{case}_ux"][None], g[f"c{case}_uy"][None]
        mask = g[f"c{case}_masked"].astype(np.float32) if case >= 2 else None
        for size in (3, 5):
            inv, _, _ = _validate(L, cuda, ux, uy, np.ones_like(ux), None, None, mask, 1e6, size)
            assert np.array_equal(inv[0], g[f"c{case}_s{size}_median"]), (case, size)


def test_validate_matches_restatement(oracle, cuda):
    """Gate, predictor, peak magnitude and the median test on a field with failed
    fits: failed and gated vectors enter the median test as zeros, as the
    reference driver passes them (cpu_instantaneous.py:592-674)."""
    L = _lib.pass_lib()
    rng = np.random.default_rng(3)
    N, ny, nx = 2, 23, 31
    pk_x = rng.normal(0.5, 0.3, (N, ny, nx)).astype(np.float32)
    pk_y = rng.normal(-0.2, 0.3, (N, ny, nx)).astype(np.float32)
    pk_h = rng.uniform(0.1, 0.9, (N, ny, nx)).astype(np.float32)
    pk_x[0, 5, 5] = 9.0            # gate
    pk_x[1, 7, 8] = np.nan          # failed fit
    pk_x[1, 7, 9] = np.nan
    pk_x[0, 10, 10] += 3.0          # outlier
    pdx = rng.normal(4.0, 0.1, (N, ny, nx)).astype(np.float32)
    pdy = rng.normal(1.0, 0.1, (N, ny, nx)).astype(np.float32)
    inv, ux, uy = _validate(L, cuda, pk_x, pk_y, pk_h, pdy, pdx, None, 8.0, 5)
    gate = (np.abs(pk_x) > 8) | (np.abs(pk_y) > 8)
    gx = np.where(gate, np.nan, pk_x) + pdx
    gy = np.where(gate, np.nan, pk_y) + pdy
    for n in range(N):
        failed = np.isnan(gx[n]) | np.isnan(gy[n])
        zx, zy = np.where(failed, 0.0, gx[n]), np.where(failed, 0.0, gy[n])
        bad = failed | (pk_h[n] < 0.25) | oracle.median_outlier(zx, zy, 0.1, 2.0, 5)
        assert np.array_equal(inv[n], bad)
        ok = ~bad
        assert np.array_equal(ux[n][ok], gx[n][ok]) and np.all(np.isnan(ux[n][bad]))
    assert inv[0, 5, 5] and inv[1, 7, 8] and inv[0, 10, 10]


@pytest.mark.parametrize("peak_thr", [0.25, -1.0])
@pytest.mark.parametrize("med_thr", [2.0, 0.0])
@pytest.mark.parametrize("masked", [False, True])
def test_validation_reason_codes(oracle, cuda, med_thr, masked, peak_thr):
    """ux/uy, the invalid flags and the int8 reason codes of every stage against
    the restatement of the reference driver's validation (fit failure, large
    displacement, masked window, peak magnitude, median outlier, NaN peak height)."""
    L = _lib.pass_lib()
    rng = np.random.default_rng(11)
    N, ny, nx = 3, 21, 26
    pk_x = rng.normal(0.5, 0.3, (N, ny, nx)).astype(np.float32)
    pk_y = rng.normal(-0.2, 0.3, (N, ny, nx)).astype(np.float32)
    pk_h = rng.uniform(0.1, 0.9, (N, ny, nx)).astype(np.float32)
    sel = lambda f: rng.random((N, ny, nx)) < f
    pk_x[sel(0.03)] = np.nan                         # fit failures
    pk_y[sel(0.02)] = 11.0                           # large displacement
    pk_x[sel(0.03)] += 4.0                           # outliers
    nanh = sel(0.02)
    pk_h[nanh] = np.nan                              # NaN height with a finite location
    pdx = rng.normal(2.0, 0.1, (N, ny, nx)).astype(np.float32)
    pdy = rng.normal(-1.0, 0.1, (N, ny, nx)).astype(np.float32)
    mask = None
    if masked:
        mask = np.zeros((ny, nx), np.float32)
        mask[:, :2] = 1.0
        mask[9:12, 12:15] = 1.0
    inv, ux, uy, rc = _validate(L, cuda, pk_x, pk_y, pk_h, pdy, pdx, mask, 8.0, 5, peak_thr=peak_thr,
                                med_thr=med_thr, reasons=True)
    for n in range(N):
        ox, oy, onan, orc = oracle.pass_validation(pk_x[n], pk_y[n], pk_h[n], pdy[n], pdx[n],
                                                   None if mask is None else mask.astype(bool), 8.0, 8.0,
                                                   peak_thr, 0.1, med_thr, 5)
        m = np.zeros((ny, nx), bool) if mask is None else mask.astype(bool)
        assert np.array_equal(rc[n], orc), (n, np.argwhere(rc[n] != orc)[:5])
        assert np.array_equal(inv[n] | m, onan)
        assert np.array_equal(ux[n], ox, equal_nan=True) and np.array_equal(uy[n], oy, equal_nan=True)
    codes = set(np.unique(rc).tolist())
    assert {0, 1, 6}.issubset(codes) and ((-1 in codes) == masked)
    assert (10 in codes) == (peak_thr >= 0 or med_thr > 0) and (13 in codes) == (peak_thr < 0)


def test_pad_smooth_and_remap(cuda):
    import torch
    from scipy.ndimage import gaussian_filter

    L = _lib.pass_lib()
    rng = np.random.default_rng(9)
    N, ny, nx, pre, post = 2, 9, 12, (2, 3), (2, 2)
    ux = rng.normal(size=(N, ny, nx)).astype(np.float32)
    uy = rng.normal(size=(N, ny, nx)).astype(np.float32)
    nyp, nxp = ny + pre[0] + post[0], nx + pre[1] + post[1]
    taps, rad = multipass._gauss_taps(0.65, 3)
    tux, tuy = _t(ux, cuda), _t(uy, cuda)
    pdy = torch.empty((N, nyp, nxp), device=cuda)
    pdx = torch.empty_like(pdy)
    work = torch.empty(N * nyp * nxp, device=cuda)
    tt = _t(taps, cuda)
    assert L.pivb_pad_smooth_dev(tux.data_ptr(), tuy.data_ptr(), N, ny, nx, nyp, nxp, pre[0], pre[1], tt.data_ptr(),
                                 rad, pdy.data_ptr(), pdx.data_ptr(), work.data_ptr(), _stream()) == 0
    torch.cuda.synchronize()
    for n in range(N):
        ref = np.pad(uy[n], ((pre[0], post[0]), (pre[1], post[1])), mode="edge")
        ref = gaussian_filter(ref.astype(np.float64), sigma=0.65, truncate=2 / (2 * 0.65), mode="nearest")
        np.testing.assert_allclose(pdy[n].cpu().numpy(), ref, atol=1e-5)
    # remap at fractional coordinates, inside and across the border, exactly as
    # the reference driver's cv2.remap(INTER_CUBIC, BORDER_REPLICATE)
    import cv2

    my = rng.uniform(-2.0, nyp + 1.0, (23, 29)).astype(np.float32)
    mx = rng.uniform(-2.0, nxp + 1.0, (23, 29)).astype(np.float32)
    my[0, :8] = (np.arange(8, dtype=np.float32) + np.float32(0.5)) / np.float32(64.0) + np.float32(3.0)  # half steps
    oy = torch.empty((N, 23, 29), device=cuda)
    ox = torch.empty_like(oy)
    tmy, tmx = _t(my, cuda), _t(mx, cuda)
    assert L.pivb_remap_dev(pdy.data_ptr(), pdx.data_ptr(), N, nyp, nxp, tmy.data_ptr(), tmx.data_ptr(), 23, 29,
                            oy.data_ptr(), ox.data_ptr(), _stream()) == 0
    torch.cuda.synchronize()
    for n in range(N):
        for plane, got in ((pdy, oy), (pdx, ox)):
            ref = cv2.remap(plane[n].cpu().numpy(), mx, my, cv2.INTER_CUBIC, borderMode=cv2.BORDER_REPLICATE)
            assert np.array_equal(got[n].cpu().numpy(), ref)


@pytest.mark.parametrize("flow", ["uniform", "channel"])
def test_multipass_recovers_displacement(cuda, flow):
    import torch

    H = W = 384
    N = 2
    kw = {"u": 3.3, "v": -1.7} if flow == "uniform" else {"peak": 6.0}
    pairs = [synthetic.particle_pair((H, W), seed=60 + k, flow=flow, flow_kwargs=kw) for k in range(N)]
    A = torch.tensor(np.stack([p[0] for p in pairs]), device=cuda)
    B = torch.tensor(np.stack([p[1] for p in pairs]), device=cuda)
    cfg = multipass.MultipassConfig(window_sizes=[(64, 64), (32, 32), (32, 32)], overlaps=[50, 50, 75])
    mp = multipass.MultipassPIV((H, W), N, cfg, device=cuda)
    ux, uy = mp.run(A, B)
    torch.cuda.synchronize()
    g = mp.geo[-1].grid
    err = []
    for n in range(N):
        u, v = pairs[n][2]
        # truth: flow at the window centre, symmetric-warp convention (midpoint)
        iy = np.clip(np.round(g.win_ctrs_y).astype(int), 0, H - 1)
        ix = np.clip(np.round(g.win_ctrs_x).astype(int), 0, W - 1)
        tu = u[np.ix_(iy, ix)]
        tv = v[np.ix_(iy, ix)]
        inner = (slice(2, -2), slice(2, -2))
        err.append(np.hypot(ux[n].cpu().numpy() - tu, uy[n].cpu().numpy() - tv)[inner])
    err = np.concatenate([e.ravel() for e in err])
    assert np.isfinite(err).all()
    assert np.sqrt(np.mean(err ** 2)) < (0.1 if flow == "uniform" else 0.35)
    # graph capture of a whole step reproduces the eager result
    ref = (ux.clone(), uy.clone())
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        mp.run(A, B)
    s.synchronize()
    gph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(gph, stream=s):
        mp.run(A, B)
    gph.replay()
    torch.cuda.synchronize()
    assert torch.equal(ux, ref[0]) and torch.equal(uy, ref[1])


@pytest.mark.parametrize("engine", ["fft", "dft"])
def test_collect_and_result_files(cuda, oracle, tmp_path, engine):
    """Per-pass results of a step: every pass's validation (reason codes, invalid
    flags) against the restatement applied to that pass's raw peaks and predictor,
    the kept planes against the raw peak positions, and the .mat / plane-dump
    files read back."""
    import scipy.io
    import torch

    from pivtools_b200 import results

    H = W = 256
    N = 2
    pairs = [synthetic.particle_pair((H, W), seed=80 + k, flow="channel", flow_kwargs={"peak": 6.0})
             for k in range(N)]
    A = np.stack([p[0] for p in pairs])
    B = np.stack([p[1] for p in pairs])
    B[1, 96:160, 96:160] = np.random.default_rng(0).uniform(0, 1, (64, 64)).astype(np.float32)   # decorrelated patch
    cfg = multipass.MultipassConfig(window_sizes=[(64, 64), (32, 32), (32, 32)], overlaps=[50, 50, 75],
                                    engine_32=engine)
    mp = multipass.MultipassPIV((H, W), N, cfg, device=cuda)
    mp.keep_planes()
    mp.run(torch.tensor(A, device=cuda), torch.tensor(B, device=cuda))
    res = mp.collect()
    assert len(res) == N and all(len(r.passes) == 3 for r in res)
    n_invalid = 0
    for n, r in enumerate(res):
        for k, pr in enumerate(r.passes):
            dd = pr.debug_dump
            win = pr.window_size[0]
            thr = win / 2.0 if k == 0 else win / 4.0
            pred = pr.predictor_field
            assert k > 0 or not pred.any()
            _, _, onan, orc = oracle.pass_validation(dd["pk_loc_x_raw"][0], dd["pk_loc_y_raw"][0],
                                                     dd["pk_height_raw"][0], pred[..., 0], pred[..., 1], None,
                                                     thr, thr, cfg.peak_mag_threshold, cfg.median_epsilon,
                                                     cfg.median_threshold, cfg.median_size)
            assert np.array_equal(pr.nan_reason, orc), (n, k)
            assert np.array_equal(pr.nan_mask, onan) and np.array_equal(pr.nan_mask, pr.nan_reason != 0)
            assert np.array_equal(pr.peak_choice, (~pr.nan_mask).astype(np.intp))
            assert np.isfinite(pr.ux_mat).all() and np.isfinite(pr.uy_mat).all()
            assert np.array_equal(np.isnan(pr.peak_mag[0]), (pr.nan_reason == 6) | np.isnan(dd["pk_height_raw"][0]))
            n_invalid += int(pr.nan_mask.sum())
            # on valid windows the raw peak sits at the kept plane's largest 3x3
            # local maximum inside the central half (the correlator's peak search);
            # on failed ones a 3-point estimate over a flat peak can land far away
            ok = pr.nan_reason == 0
            P = dd["planes"]
            q, h2 = win // 4, win // 2
            core = P[..., q:q + h2, q:q + h2]
            locmax = np.ones(core.shape, bool)
            for a in (-1, 0, 1):
                for b in (-1, 0, 1):
                    locmax &= ~(P[..., q + a:q + a + h2, q + b:q + b + h2] > core)
            cand = np.where(locmax & (core > 0), core, -1.0).reshape(core.shape[:2] + (h2 * h2,))
            am = cand.argmax(axis=-1)
            py, px = am // h2 + q - h2, am % h2 + q - h2
            assert np.abs(px - dd["pk_loc_x_raw"][0])[ok].max() <= 1.0
            assert np.abs(py - dd["pk_loc_y_raw"][0])[ok].max() <= 1.0
    assert n_invalid > 0
    path = results.save_piv_result_distributed(res[1], tmp_path, 2)
    st = scipy.io.loadmat(path)["piv_result"]
    assert st.shape == (1, 3)
    for k, pr in enumerate(res[1].passes):
        assert np.array_equal(st["ux"][0, k], results.to_half(pr.ux_mat))
        assert np.array_equal(st["nan_reason"][0, k], pr.nan_reason)
        assert np.array_equal(st["n_windows"][0, k].ravel(), pr.n_windows)
    dump = np.load(results.save_corr_plane_dump(res[1], tmp_path, 2))
    assert dump["pass2_planes"].shape == (res[1].passes[2].n_windows[0], res[1].passes[2].n_windows[1], 32, 32)


@pytest.mark.parametrize("engine", ["fft", "dft"])
def test_multipass_with_vector_masks(cuda, oracle, engine):
    """Masked windows (from a pixel mask, geometry.compute_vector_masks) are
    skipped, stored as 0 with reason -1 and kept out of the infill; the
    predictor is filled across them, so the next pass's predictor there follows
    the flow instead of the stored zeros; every pass's reason codes equal the
    restatement given the mask."""
    import torch

    H = W = 384
    N = 2
    pairs = [synthetic.particle_pair((H, W), seed=120 + k, flow="uniform", flow_kwargs={"u": 3.3, "v": -1.7})
             for k in range(N)]
    A = torch.tensor(np.stack([p[0] for p in pairs]), device=cuda)
    B = torch.tensor(np.stack([p[1] for p in pairs]), device=cuda)
    pm = np.zeros((H, W), bool)
    pm[140:250, 100:210] = True
    cfg = multipass.MultipassConfig(window_sizes=[(64, 64), (32, 32), (32, 32)], overlaps=[50, 50, 75],
                                    engine_32=engine)
    vm = geometry.compute_vector_masks(pm, (H, W), cfg.window_sizes, cfg.overlaps, 0.5)
    assert all(m.any() for m in vm)
    mp = multipass.MultipassPIV((H, W), N, cfg, device=cuda, vector_masks=vm)
    ux, uy = mp.run(A, B)
    res = mp.collect()
    for n, r in enumerate(res):
        for k, pr in enumerate(r.passes):
            m = vm[k]
            assert np.array_equal(pr.b_mask, m)
            assert np.all(pr.nan_reason[m] == -1) and np.all(pr.nan_reason[~m] != -1)
            assert np.all(pr.ux_mat[m] == 0) and np.all(pr.uy_mat[m] == 0)
            assert np.isfinite(pr.ux_mat).all()
            thr = pr.window_size[0] / 2.0 if k == 0 else pr.window_size[0] / 4.0
            pred = pr.predictor_field
            raw = mp.passes[k]["out"]
            _, _, onan, orc = oracle.pass_validation(
                raw["pk_loc_x"][n, 0].cpu().numpy(), raw["pk_loc_y"][n, 0].cpu().numpy(),
                raw["pk_height"][n, 0].cpu().numpy(), pred[..., 0], pred[..., 1], m, thr, thr,
                cfg.peak_mag_threshold, cfg.median_epsilon, cfg.median_threshold, cfg.median_size)
            assert np.array_equal(pr.nan_reason, orc), (n, k)
            if k > 0:
                # the predictor under the mask follows the flow (filled), not 0
                assert np.abs(pred[m][:, 1] - 3.3).max() < 0.3 and np.abs(pred[m][:, 0] + 1.7).max() < 0.3
        fin = r.passes[-1]
        ok = ~vm[-1]
        err = np.hypot(fin.ux_mat[ok] - 3.3, fin.uy_mat[ok] + 1.7)
        assert np.sqrt(np.mean(err ** 2)) < 0.1


def test_u16_to_f32_conversion(cuda):
    import torch

    L = _lib.pass_lib()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(5)
    for n in (1, 3, 4, 1021, 1 << 20):                   # ragged tails and a large case
        src = torch.tensor(rng.integers(0, 65536, n).astype(np.int32)).to(torch.uint16).to(cuda)
        dst = torch.full((n,), -1.0, device=cuda)
        assert L.pivb_u16_to_f32_dev(src.data_ptr(), dst.data_ptr(), n, s) == 0
        torch.cuda.synchronize()
        assert torch.equal(dst.cpu(), src.cpu().to(torch.int32).to(torch.float32))
    # misaligned pointers are refused before any launch
    buf = torch.zeros(64, dtype=torch.uint16, device=cuda)
    out = torch.zeros(64, device=cuda)
    assert L.pivb_u16_to_f32_dev(buf.data_ptr() + 2, out.data_ptr(), 16, s) == 1
    assert L.pivb_u16_to_f32_dev(buf.data_ptr(), out.data_ptr() + 4, 16, s) == 1
    assert L.pivb_u16_to_f32_dev(buf.data_ptr(), out.data_ptr(), 0, s) == 1


def test_host_pipeline_matches_resident_batch(cuda):
    """uint16 pinned frames, chunked and overlapped with compute, give the same
    fields as one resident batch of float32 frames."""
    import torch

    H = W = 256
    N, C = 4, 2
    pairs = [synthetic.particle_pair((H, W), seed=80 + k, flow="channel", flow_kwargs={"peak": 5.0})
             for k in range(N)]
    A16 = np.stack([np.clip(np.round(p[0]), 0, 65535) for p in pairs]).astype(np.int32)
    B16 = np.stack([np.clip(np.round(p[1]), 0, 65535) for p in pairs]).astype(np.int32)
    cfg = multipass.MultipassConfig(window_sizes=[(64, 64), (32, 32)], overlaps=[50, 50])
    mp = multipass.MultipassPIV((H, W), N, cfg, device=cuda)
    ux, uy = mp.run(torch.tensor(A16, dtype=torch.float32, device=cuda),
                    torch.tensor(B16, dtype=torch.float32, device=cuda))
    torch.cuda.synchronize()
    pipe = multipass.HostPipeline((H, W), C, cfg, device=cuda)
    Ah = torch.tensor(A16).to(torch.uint16).pin_memory()
    Bh = torch.tensor(B16).to(torch.uint16).pin_memory()
    g = mp.geo[-1].grid
    oux = torch.empty((N, g.n_win_y, g.n_win_x)).pin_memory()
    ouy = torch.empty_like(oux).pin_memory()
    for _ in range(2):                                   # twice: slots and events are reused
        oux.fill_(7.0)
        ouy.fill_(7.0)
        pipe.run(Ah, Bh, oux, ouy)
        torch.cuda.synchronize()
        assert torch.equal(oux, ux.cpu()) and torch.equal(ouy, uy.cpu())


def test_multipass_tensor_core_engine_tracks_fft(cuda):
    """The 32 px passes on the tensor-core DFT-as-GEMM engine give the FFT
    engine's field within the split-BF16 precision (planes 1e-4 of the peak)."""
    import torch

    H = W = 384
    N = 2
    pairs = [synthetic.particle_pair((H, W), seed=70 + k, flow="channel", flow_kwargs={"peak": 6.0})
             for k in range(N)]
    A = torch.tensor(np.stack([p[0] for p in pairs]), device=cuda)
    B = torch.tensor(np.stack([p[1] for p in pairs]), device=cuda)
    res = []
    for eng in ("fft", "dft"):
        cfg = multipass.MultipassConfig(window_sizes=[(64, 64), (32, 32), (32, 32)], overlaps=[50, 50, 75],
                                        engine_32=eng)
        mp = multipass.MultipassPIV((H, W), N, cfg, device=cuda)
        ux, uy = mp.run(A, B)
        torch.cuda.synchronize()
        assert mp.dft_status.item() == 0
        res.append((ux.cpu().numpy().copy(), uy.cpu().numpy().copy()))
    d = np.hypot(res[0][0] - res[1][0], res[0][1] - res[1][1])
    assert np.isfinite(d).all()
    assert np.median(d) < 1e-3 and np.percentile(d, 99) < 0.05
