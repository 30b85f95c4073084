"""The GPU-resident ensemble pass (pivtools_b200.ensemble.EnsemblePIV):
accumulate in batches, finalise (background of the mean images, plane-mean
removal, envelope divide, normalisation) and k-space fit, against the oracle's
restatement of the same steps (oracle accumulate_triple, ensemble_finalize,
kspace_fit) on the same seeded pairs."""

import numpy as np
import pytest

from pivtools_b200 import ensemble, geometry, synthetic

pytestmark = pytest.mark.gpu


def _pairs(n, shape, seed):
    out = [synthetic.particle_pair(shape, seed=seed + k, flow="uniform_grf")[:2] for k in range(n)]
    return np.stack([p[0] for p in out]).astype(np.float32), np.stack([p[1] for p in out]).astype(np.float32)


@pytest.mark.parametrize("method,env", [("correlation+dc_zero", False), ("correlation", True), ("window_mean", False),
                                        ("image", False), ("image+window_mean", True), ("image+dc_zero", False)])
def test_ensemble_pass_matches_oracle(oracle, cuda, method, env):
    import torch

    shape, win = (128, 160), (16, 16)
    A, B = _pairs(10, shape, 700)
    ep = ensemble.EnsemblePIV(shape, win, 75, "square", background=method, envelope_divide=env, device=cuda)
    ms, use_bg, dc, two = ensemble._METHODS[method]
    if two:                                  # stationary structure for the mean images to remove
        A += np.linspace(0, 40, shape[1], dtype=np.float32)[None, None]
        B += np.linspace(0, 40, shape[1], dtype=np.float32)[None, None]
    batches = (slice(0, 4), slice(4, 10))
    dA = [torch.tensor(A[sl], device=cuda) for sl in batches]
    dB = [torch.tensor(B[sl], device=cuda) for sl in batches]
    if two:                                                     # first sweep: the mean images
        for a, b in zip(dA, dB):
            ep.accumulate_means(a, b)
        means = ep.end_means()
    for a, b in zip(dA, dB):                                    # two batches
        ep.accumulate(a, b)
    fin = ep.finalize()
    fit = ep.fit()
    torch.cuda.synchronize()

    g = ep.grid
    w = geometry.window_weight(win, "square")
    mask = np.zeros((g.n_win_y, g.n_win_x), np.float32)
    CA, CB = A, B
    if two:
        mA, mB = oracle.image_method_means([A[sl] for sl in batches], [B[sl] for sl in batches])
        assert means["n_pairs"] == 10
        np.testing.assert_allclose(means["A_mean"].cpu().numpy(), mA, rtol=1e-6)
        np.testing.assert_allclose(means["B_mean"].cpu().numpy(), mB, rtol=1e-6)
        CA, CB = oracle.center_frames(A, mA), oracle.center_frames(B, mB)
        assert np.array_equal(dA[1].cpu().numpy(), A[4:10])     # the caller's frames are untouched
    s_ab, s_aa, s_bb = oracle.accumulate_triple(CA, CB, mask, g.win_ctrs_x, g.win_ctrs_y, win, w, w, w, w,
                                                mean_subtract=ms)
    n_win = g.n_win_y * g.n_win_x
    bg = None
    if use_bg:
        mA = (A.astype(np.float64).sum(0) / 10).astype(np.float32)
        mB = (B.astype(np.float64).sum(0) / 10).astype(np.float32)
        b_ab, b_aa, b_bb = oracle.accumulate_triple(mA[None], mB[None], mask, g.win_ctrs_x, g.win_ctrs_y, win,
                                                    w, w, w, w, mean_subtract=ms)
        bg = [x.reshape(n_win, *win) for x in (b_aa, b_bb, b_ab)]
    e = oracle.pair_envelope(w, w, win) if env else None
    R_AA, R_BB, R_AB, norm = oracle.ensemble_finalize(s_ab.reshape(n_win, *win), s_aa.reshape(n_win, *win),
                                                      s_bb.reshape(n_win, *win), 10, bg=bg, dc_zero=dc,
                                                      env_auto=e)
    for got, ref in ((fin["R_AA"], R_AA), (fin["R_BB"], R_BB), (fin["R_AB"], R_AB)):
        got = got.cpu().numpy()
        scale = np.abs(ref).reshape(n_win, -1).max(axis=1)[:, None, None]
        assert np.all(np.abs(got - ref) <= 2e-4 * scale + 1e-7), float(np.max(np.abs(got - ref) / scale))
    np.testing.assert_allclose(fin["norm"].cpu().numpy(), norm, rtol=2e-4)

    ref_fit = oracle.kspace_fit(R_AA, R_BB, R_AB, np.zeros(n_win, np.uint8), win)
    st_g, st_o = fit["status"].cpu().numpy(), ref_fit["status"]
    assert (st_g == st_o).mean() >= 0.95
    both = (st_g == 0) & (st_o == 0)
    assert both.sum() >= 0.5 * n_win
    gg, go = fit["gauss"].cpu().numpy()[both], ref_fit["gauss_flat"][both]
    # fitted displacement (cols 14-15) and Reynolds stresses (cols 9-11)
    assert np.max(np.abs(gg[:, 14:16] - go[:, 14:16])) < 2e-3
    np.testing.assert_allclose(gg[:, 9:12], go[:, 9:12], rtol=5e-3, atol=1e-4)


@pytest.mark.parametrize("method,env,win,sumw,fit", [
    ("correlation+dc_zero", False, (4, 4), (16, 16), None), ("window_mean", True, (4, 4), (16, 16), (12, 12)),
    ("image", True, (8, 8), (32, 32), (24, 24)), ("correlation", True, (5, 5), (16, 16), None),
    ("image+dc_zero", False, (6, 6), (16, 16), (16, 16))])
def test_single_mode_matches_oracle(oracle, cuda, method, env, win, sumw, fit):
    """Ensemble single mode (singlepix frame-A weight inside the sum window,
    bsingle frame B and auto planes, zero-padded frames, planes at the fitting
    window, the AB area correction) against the oracle's restatement of the
    reference's steps on the same pairs."""
    import torch

    shape = (96, 112)
    A, B = _pairs(6, shape, 770)
    ep = ensemble.EnsemblePIV(shape, win, 50, "square", background=method, envelope_divide=env, device=cuda,
                              runtype="single", sum_window=sumw, fit_window=fit)
    ms, use_bg, dc, two = ensemble._METHODS[method]
    batches = (slice(0, 2), slice(2, 6))
    dA = [torch.tensor(A[sl], device=cuda) for sl in batches]
    dB = [torch.tensor(B[sl], device=cuda) for sl in batches]
    if two:
        for a, b in zip(dA, dB):
            ep.accumulate_means(a, b)
        ep.end_means()
    for a, b in zip(dA, dB):
        ep.accumulate(a, b)
    fin = ep.finalize()
    torch.cuda.synchronize()

    g = ep.grid
    corr = fit or sumw
    assert tuple(fin["R_AB"].shape[1:]) == corr
    pt, pb, pl, pr = ep.padding
    wa = geometry.window_weight(win, "singlepix", sumw)
    wb = geometry.window_weight(sumw, "bsingle", sumw)
    mask = np.zeros((g.n_win_y, g.n_win_x), np.float32)
    pad = lambda F: np.pad(F, ((0, 0), (pt, pb), (pl, pr)))      # noqa: E731
    CA, CB = A, B
    if two:
        mA, mB = oracle.image_method_means([A[sl] for sl in batches], [B[sl] for sl in batches])
        CA, CB = oracle.center_frames(A, mA), oracle.center_frames(B, mB)
    s_ab, s_aa, s_bb = oracle.accumulate_triple(pad(CA), pad(CB), mask, g.win_ctrs_x, g.win_ctrs_y, sumw, wa, wb,
                                                wb, wb, fit_size=corr, mean_subtract=ms)
    n_win = g.n_win_y * g.n_win_x
    bg = None
    if use_bg:
        mA = (A.astype(np.float64).sum(0) / 6).astype(np.float32)
        mB = (B.astype(np.float64).sum(0) / 6).astype(np.float32)
        b_ab, b_aa, b_bb = oracle.accumulate_triple(pad(mA[None]), pad(mB[None]), mask, g.win_ctrs_x, g.win_ctrs_y,
                                                    sumw, wa, wb, wb, wb, fit_size=corr, mean_subtract=ms)
        bg = [x.reshape(n_win, *corr) for x in (b_aa, b_bb, b_ab)]
    e_auto = oracle.pair_envelope(wb, wb, corr) if env else None
    e_ab = oracle.pair_envelope(wa, wb, corr) if env else None
    R_AA, R_BB, R_AB, norm = oracle.ensemble_finalize(
        s_ab.reshape(n_win, *corr), s_aa.reshape(n_win, *corr), s_bb.reshape(n_win, *corr), 6, bg=bg, dc_zero=dc,
        env_auto=e_auto, env_ab=e_ab, ab_scale=(sumw[0] * sumw[1]) / (win[0] * win[1]))
    for got, ref in ((fin["R_AA"], R_AA), (fin["R_BB"], R_BB), (fin["R_AB"], R_AB)):
        got = got.cpu().numpy()
        scale = np.abs(ref).reshape(n_win, -1).max(axis=1)[:, None, None]
        assert np.all(np.abs(got - ref) <= 2e-4 * scale + 1e-7), float(np.max(np.abs(got - ref) / scale))
    np.testing.assert_allclose(fin["norm"].cpu().numpy(), norm, rtol=2e-4)
    cx, cy = ep.window_centres                                  # unpadded-frame coordinates
    assert float(cx[0]) == (win[1] - 1) / 2.0


def test_single_mode_refusals(cuda):
    with pytest.raises(ValueError, match="sum_window must be defined"):
        ensemble.EnsemblePIV((64, 64), (4, 4), 50, runtype="single", device=cuda)
    with pytest.raises(ValueError, match="must be <="):
        ensemble.EnsemblePIV((64, 64), (4, 4), 50, runtype="single", sum_window=(16, 16), fit_window=(20, 20),
                             device=cuda)
    with pytest.raises(ValueError, match="square"):
        ensemble.EnsemblePIV((64, 64), (4, 4), 50, runtype="single", sum_window=(16, 32), device=cuda)
    with pytest.raises(ValueError, match="per_pair_normalization"):
        ensemble.EnsemblePIV((64, 64), (16, 16), 75, background="correlation", per_pair_normalization=True,
                             device=cuda)


def test_two_sweep_order_and_refusals(cuda):
    import torch

    with pytest.raises(ValueError, match="Invalid ensemble_background_subtraction_method"):
        ensemble.EnsemblePIV((64, 64), (16, 16), 75, "square", background="image+correlation", device=cuda)
    a = torch.rand((2, 64, 64), device=cuda)
    ep = ensemble.EnsemblePIV((64, 64), (16, 16), 75, "square", background="image", device=cuda)
    with pytest.raises(RuntimeError, match="sweeps twice"):
        ep.accumulate(a, a)                                    # second sweep before the means
    with pytest.raises(RuntimeError, match="before any accumulate_means"):
        ep.end_means()
    ep.accumulate_means(a, a)
    ep.end_means()
    with pytest.raises(RuntimeError, match="closed"):
        ep.accumulate_means(a, a)
    with pytest.raises(RuntimeError, match="already"):
        ep.end_means()
    with pytest.raises(ValueError, match="float32"):
        ep.accumulate(a.double(), a.double())
    ep.accumulate(a, a)
    ep.reset()
    assert not ep.means_ready and ep.n_pairs == 0
    plain = ensemble.EnsemblePIV((64, 64), (16, 16), 75, "square", background="correlation", device=cuda)
    with pytest.raises(ValueError, match="two-sweep"):
        plain.accumulate_means(a, a)


def test_image_method_from_uint16_host_frames(cuda):
    """Both sweeps of the 'image' method streamed from page-locked uint16 host
    frames equal the float32 device path bit for bit."""
    import torch

    shape, win = (128, 160), (16, 16)
    A, B = _pairs(7, shape, 740)
    A16 = np.clip(np.round(A), 0, 65535).astype(np.int32)
    B16 = np.clip(np.round(B), 0, 65535).astype(np.int32)
    Ah = torch.tensor(A16).to(torch.uint16).pin_memory()
    Bh = torch.tensor(B16).to(torch.uint16).pin_memory()
    host = ensemble.EnsemblePIV(shape, win, 75, "square", background="image+dc_zero", device=cuda)
    dev = ensemble.EnsemblePIV(shape, win, 75, "square", background="image+dc_zero", device=cuda)
    host.accumulate_means_host(Ah, Bh, chunk=3)
    host.end_means()
    host.accumulate_host(Ah, Bh, chunk=3)
    fa = [torch.tensor(A16[c0:c0 + 3], dtype=torch.float32, device=cuda) for c0 in range(0, 7, 3)]
    fb = [torch.tensor(B16[c0:c0 + 3], dtype=torch.float32, device=cuda) for c0 in range(0, 7, 3)]
    for a, b in zip(fa, fb):
        dev.accumulate_means(a, b)
    dev.end_means()
    for a, b in zip(fa, fb):
        dev.accumulate(a, b)
    torch.cuda.synchronize()
    assert host.n_pairs == dev.n_pairs == 7 and host.n_means == 7
    for x, y in ((host.sums, dev.sums), (host.comp, dev.comp), (host.fmean, dev.fmean)):
        assert torch.equal(x, y)


def test_distributed_finalise_single_rank_equals_local(cuda):
    """The multi-GPU finalise path on a one-rank group (GPU tensors through gloo)
    gives the local finalise's planes and fits."""
    import datetime
    import os
    import socket

    import torch

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.distributed.init_process_group("gloo", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        shape, win = (128, 128), (16, 16)
        A, B = _pairs(6, shape, 760)
        ep = ensemble.EnsemblePIV(shape, win, 75, "square", device=cuda)
        ep.accumulate(torch.tensor(A, device=cuda), torch.tensor(B, device=cuda))
        loc = {k: v.clone() for k, v in ep.finalize().items()}
        fit_loc = ep.fit()
        dist = ep.finalize_distributed()
        assert dist["windows"] == (0, ep.n_win) and dist["n_pairs"] == 6
        for k in ("R_AA", "R_BB", "R_AB"):
            ref = loc[k].cpu().numpy()
            scale = np.abs(ref).reshape(ref.shape[0], -1).max(axis=1)[:, None, None]
            assert np.all(np.abs(dist[k].cpu().numpy() - ref) <= 1e-5 * scale)
        fit = ep.gather_fit(ep.fit())
        torch.cuda.synchronize()
        st_l, st_d = fit_loc["status"].cpu().numpy(), fit["status"].cpu().numpy()
        assert (st_l == st_d).mean() > 0.95
        ok = (st_l == 0) & (st_d == 0)
        np.testing.assert_allclose(fit["gauss"].cpu().numpy()[ok][:, 14:16],
                                   fit_loc["gauss"].cpu().numpy()[ok][:, 14:16], atol=1e-3)
    finally:
        torch.distributed.destroy_process_group()


def test_accumulate_from_uint16_host_frames(cuda):
    """Pairs streamed from page-locked uint16 host frames (chunked, staged on a
    copy stream) accumulate exactly as the same frames in float32, chunk by chunk."""
    import torch

    shape, win = (128, 160), (16, 16)
    A, B = _pairs(7, shape, 730)
    A16 = np.clip(np.round(A), 0, 65535).astype(np.int32)
    B16 = np.clip(np.round(B), 0, 65535).astype(np.int32)
    host = ensemble.EnsemblePIV(shape, win, 75, "square", device=cuda)
    dev = ensemble.EnsemblePIV(shape, win, 75, "square", device=cuda)
    Ah = torch.tensor(A16).to(torch.uint16).pin_memory()
    Bh = torch.tensor(B16).to(torch.uint16).pin_memory()
    for _ in range(2):                                   # staging slots and events reused
        host.accumulate_host(Ah, Bh, chunk=3)
    for _ in range(2):
        for c0 in range(0, 7, 3):
            dev.accumulate(torch.tensor(A16[c0:c0 + 3], dtype=torch.float32, device=cuda),
                           torch.tensor(B16[c0:c0 + 3], dtype=torch.float32, device=cuda))
    torch.cuda.synchronize()
    assert host.n_pairs == dev.n_pairs == 14
    for a, b in ((host.sums, dev.sums), (host.comp, dev.comp), (host.fsum, dev.fsum)):
        assert torch.equal(a, b)
    fa, fb = host.finalize(), dev.finalize()
    torch.cuda.synchronize()
    assert torch.equal(fa["R_AB"], fb["R_AB"]) and torch.equal(fa["R_AA"], fb["R_AA"])
    with pytest.raises(ValueError):
        host.accumulate_host(torch.tensor(A16).to(torch.uint16), Bh)          # pageable
