"""The request loop with continuous batching (pivtools_b200.serving.PivServer):
a request's field is the same alone and in a mix of shapes and schedules (and at
any slot of a shared batch), and a short Poisson run completes every request."""

import time

import numpy as np
import pytest

from pivtools_b200 import serving, synthetic

pytestmark = pytest.mark.gpu


def _pair(shape, seed):
    import torch

    A, B, _ = synthetic.particle_pair(shape, seed=seed, flow="channel", flow_kwargs={"peak": 4.0})
    return (torch.tensor(A.astype(np.int32)).to(torch.uint16).pin_memory(),
            torch.tensor(B.astype(np.int32)).to(torch.uint16).pin_memory())


def _same(a, b):
    a, b = a.numpy(), b.numpy()
    return np.array_equal(a, b, equal_nan=True)


def test_result_same_alone_and_in_mix(cuda):
    srv = serving.PivServer(device=cuda, max_batch=4)
    A, B = _pair((256, 256), 901)
    alone = srv.submit(A, B, (64, 32))
    srv.drain()
    assert alone.finished and np.isfinite(alone.ux.numpy()).all()
    others = [(_pair((256, 256), 910 + k), (64, 32)) for k in range(2)]
    others += [(_pair((192, 320), 920), (32,)), (_pair((256, 256), 921), (32,)),
               (_pair((320, 256), 922), (64, 32, 16))]
    mix = []
    for (a, b), sch in others[:2]:
        mix.append(srv.submit(a, b, sch))            # same class first: the request lands in slot 2
    again = srv.submit(A, B, (64, 32))
    for (a, b), sch in others[2:]:
        mix.append(srv.submit(a, b, sch))
    srv.drain()
    assert all(r.finished for r in mix + [again])
    assert _same(again.ux, alone.ux) and _same(again.uy, alone.uy)


@pytest.mark.parametrize("packed", [False, True], ids=["per-class", "packed"])
def test_short_poisson_run_completes(cuda, packed):
    srv = serving.PivServer(device=cuda, max_batch=4, packed=packed)
    pool = {(256, 256): _pair((256, 256), 930), (384, 256): _pair((384, 256), 931)}
    scheds = [(32,), (64, 32)]
    # warm the engines
    for shp, (a, b) in pool.items():
        for sch in scheds:
            srv.submit(a, b, sch)
    srv.drain()
    arr = serving.poisson_arrivals(60.0, 1.0, seed=3)
    rng = np.random.default_rng(4)
    reqs = []
    t0 = time.perf_counter()
    i = 0
    while i < len(arr) or not srv.idle():
        now = time.perf_counter() - t0
        while i < len(arr) and arr[i] <= now:
            shp = list(pool)[rng.integers(len(pool))]
            a, b = pool[shp]
            reqs.append(srv.submit(a, b, scheds[rng.integers(len(scheds))], arrival=t0 + arr[i]))
            i += 1
        srv.poll()
        assert time.perf_counter() - t0 < 30.0
        time.sleep(2e-4)
    lat = np.array([r.done - r.arrival for r in reqs])
    assert len(reqs) == len(arr) and all(r.finished for r in reqs)
    assert np.all(lat > 0) and np.percentile(lat, 99) < 5.0


def test_packed_rounds_equal_per_class_engines(cuda):
    """Packed mode: the waiting requests of every class run as one round whose
    correlations of one window size share a launch; every request's field is
    bit-identical to the per-class engines' result."""
    work = [((256, 256), 940, (64, 32)), ((192, 320), 941, (32,)), ((256, 256), 942, (64, 32)),
            ((320, 256), 943, (64, 32, 16)), ((256, 384), 944, (32,)), ((256, 256), 945, (128, 64, 32))]
    pairs = [(_pair(shp, seed), sch) for shp, seed, sch in work]
    ref_srv = serving.PivServer(device=cuda, max_batch=4)
    ref = [ref_srv.submit(a, b, sch) for (a, b), sch in pairs]
    ref_srv.drain()
    srv = serving.PivServer(device=cuda, max_batch=4, packed=True)
    got = [srv.submit(a, b, sch) for (a, b), sch in pairs]
    srv.drain()
    assert srv.pack_stats["rounds"] >= 1
    assert srv.pack_stats["packed_launches"] < srv.pack_stats["jobs"]       # launches were shared
    for r, g in zip(ref, got):
        assert g.finished and _same(g.ux, r.ux) and _same(g.uy, r.uy)


def test_packed_jobs_equal_single_calls(cuda):
    """pivb_xcorr_jobs_dev on jobs of different frame sizes, grids, masks and
    batch sizes equals each job's own pivb_xcorr_dev call bit for bit."""
    import ctypes

    import torch

    from pivtools_b200 import _lib, geometry

    L = _lib.bulkxcorr2d_lib()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    n = 32
    w = torch.tensor(geometry.window_weight((n, n), "gaussian"), device=cuda)
    cw = torch.empty_like(w)
    assert L.pivb_correl_weight_dev(w.data_ptr(), n, n, cw.data_ptr(), s) == 0
    keep, jobs, refs = [], [], []
    for k, (shape, npairs, masked) in enumerate((((160, 224), 1, False), ((256, 256), 2, True), ((192, 160), 3, False))):
        fr = [synthetic.particle_pair(shape, seed=950 + 10 * k + i)[:2] for i in range(npairs)]
        A = torch.tensor(np.stack([f[0] for f in fr]), device=cuda)
        B = torch.tensor(np.stack([f[1] for f in fr]), device=cuda)
        g = geometry.compute_window_centers(shape, (n, n), 50)
        cx, cy = torch.tensor(g.win_ctrs_x, device=cuda), torch.tensor(g.win_ctrs_y, device=cuda)
        m = None
        if masked:
            mm = np.zeros((g.n_win_y, g.n_win_x), np.float32)
            mm[1:3, 2:4] = 1.0
            m = torch.tensor(mm, device=cuda)
        outs = [{key: torch.full((npairs, 1, g.n_win_y, g.n_win_x), -3.0, device=cuda)
                 for key in ("x", "y", "h", "sx", "sy", "sxy")} for _ in range(2)]
        rat = [torch.full((npairs, g.n_win_y, g.n_win_x), -3.0, device=cuda) for _ in range(2)]
        keep += [A, B, cx, cy, m, outs, rat]
        o, r = outs[0], rat[0]
        jobs.append(_lib.XcorrJob(A.data_ptr(), B.data_ptr(), shape[0] * shape[1], None if m is None else m.data_ptr(),
                                  shape[0], shape[1], npairs, cx.data_ptr(), cy.data_ptr(), g.n_win_y, g.n_win_x,
                                  w.data_ptr(), w.data_ptr(), cw.data_ptr(), o["x"].data_ptr(), o["y"].data_ptr(),
                                  o["h"].data_ptr(), o["sx"].data_ptr(), o["sy"].data_ptr(), o["sxy"].data_ptr(),
                                  r.data_ptr()))
        o, r = outs[1], rat[1]
        total = npairs * g.n_win_y * g.n_win_x
        nb = int(L.pivb_xcorr_record_bytes(total))
        scr = torch.empty(nb, dtype=torch.uint8, device=cuda)
        keep.append(scr)
        assert L.pivb_xcorr_dev(A.data_ptr(), B.data_ptr(), shape[0] * shape[1], None if m is None else m.data_ptr(),
                                shape[0], shape[1], npairs, cx.data_ptr(), cy.data_ptr(), g.n_win_y, g.n_win_x,
                                w.data_ptr(), w.data_ptr(), cw.data_ptr(), n, n, 0, 1, 6, 0, o["x"].data_ptr(),
                                o["y"].data_ptr(), o["h"].data_ptr(), o["sx"].data_ptr(), o["sy"].data_ptr(),
                                o["sxy"].data_ptr(), r.data_ptr(), None, scr.data_ptr(), nb, s) == 0
        refs.append((outs, rat))
    arr = (_lib.XcorrJob * len(jobs))(*jobs)
    nb = int(L.pivb_xcorr_jobs_record_bytes(arr, len(jobs), n))
    rec = torch.empty(nb, dtype=torch.uint8, device=cuda)
    assert L.pivb_xcorr_jobs_dev(arr, len(jobs), n, 6, 0, rec.data_ptr(), nb, s) == 0
    torch.cuda.synchronize()
    for outs, rat in refs:
        for key in outs[0]:
            assert np.array_equal(outs[0][key].cpu().numpy(), outs[1][key].cpu().numpy(), equal_nan=True), key
        assert np.array_equal(rat[0].cpu().numpy(), rat[1].cpu().numpy(), equal_nan=True)
