"""The distributed ensemble chain end to end: two gloo ranks (two processes on
the one GPU; their kernels never wait on each other, every exchange goes through
the host) each accumulate half of the pairs with EnsemblePIV, combine the
compensated sums with finalize_distributed (one reduce-scatter by window block),
k-space-fit their own block and all-gather the fit rows.  The gathered result
must equal a single process's accumulate -> finalize -> fit over all the pairs:
planes within 1e-5 of each plane's peak, statuses equal on at least 98% of the
windows, fitted displacements within 1e-3 px and stresses within 0.5%."""

import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pivtools_b200 import ensemble, synthetic

pytestmark = pytest.mark.gpu

SHAPE, WIN, N_PAIRS = (128, 160), (16, 16), 8


def _pairs():
    out = [synthetic.particle_pair(SHAPE, seed=880 + k, density=0.02, flow="ensemble_rows")[:2]
           for k in range(N_PAIRS)]
    return np.stack([p[0] for p in out]).astype(np.float32), np.stack([p[1] for p in out]).astype(np.float32)


def _worker(rank, world, port, q):
    import torch

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        A, B = _pairs()
        ep = ensemble.EnsemblePIV(SHAPE, WIN, 75, "square", device=dev)
        ep.accumulate(torch.tensor(A[rank::world], device=dev), torch.tensor(B[rank::world], device=dev))
        fin = ep.finalize_distributed()
        planes = {k: fin[k].cpu().numpy() for k in ("R_AA", "R_BB", "R_AB")}
        fit = ep.gather_fit(ep.fit())
        torch.cuda.synchronize()
        q.put((rank, fin["windows"], fin["n_pairs"], planes,
               fit["status"].cpu().numpy(), fit["gauss"].cpu().numpy()))
    except Exception as e:       # report instead of leaving the parent waiting
        q.put((rank, "error", repr(e), None, None, None))
        raise
    finally:
        torch.distributed.destroy_process_group()


def test_two_rank_ensemble_chain_equals_one_rank(cuda):
    import torch

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in range(2)), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=120)
    for r in res:
        assert r[1] != "error", r[2]
    assert all(p.exitcode == 0 for p in procs)

    A, B = _pairs()
    ep = ensemble.EnsemblePIV(SHAPE, WIN, 75, "square", device=cuda)
    ep.accumulate(torch.tensor(A, device=cuda), torch.tensor(B, device=cuda))
    loc = {k: v.cpu().numpy() for k, v in ep.finalize().items() if k != "norm"}
    fit = ep.fit()
    torch.cuda.synchronize()
    st_l, g_l = fit["status"].cpu().numpy(), fit["gauss"].cpu().numpy()

    covered = 0
    for rank, (a, b), n_tot, planes, st_d, g_d in res:
        assert n_tot == N_PAIRS
        covered += b - a
        for k in ("R_AA", "R_BB", "R_AB"):
            ref = loc[k][a:b]
            scale = np.abs(ref).reshape(len(ref), -1).max(axis=1)[:, None, None]
            assert np.all(np.abs(planes[k] - ref) <= 1e-5 * scale), (rank, k)
        assert (st_d == st_l).mean() >= 0.98
        ok = (st_d == 0) & (st_l == 0)
        assert ok.mean() > 0.5
        assert np.abs(g_d[ok, 14:16] - g_l[ok, 14:16]).max() < 1e-3
        np.testing.assert_allclose(g_d[ok, 9:12], g_l[ok, 9:12], rtol=5e-3, atol=1e-4)
    assert covered == ep.n_win
