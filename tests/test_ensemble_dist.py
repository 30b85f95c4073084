"""Cross-rank exchange of the multi-GPU ensemble pass (pivtools_b200.ensemble_dist),
run as two gloo ranks on CPU tensors: window blocks, the reduce-scatter of the
compensated plane sums, the all-reduce of the frame sums and pair counts, and the
all-gather of per-window fit rows."""

import os
import socket

import numpy as np
import torch
import torch.multiprocessing as mp

from pivtools_b200 import ensemble_dist as ed

N_WIN, HW, NPIX = 37, 16, 50


def _rank_data(r):
    g = torch.Generator().manual_seed(100 + r)
    sums = torch.randn((3, N_WIN * HW), generator=g) * 1000
    comps = torch.randn((3, N_WIN * HW), generator=g) * 1e-4
    fsum = torch.randn((2, NPIX), generator=g) * 100
    fcomp = torch.randn((2, NPIX), generator=g) * 1e-5
    return sums, comps, fsum, fcomp, 3 + r


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        sums, comps, fsum, fcomp, n = _rank_data(rank)
        block, fr, n_tot, (a, b) = ed.exchange_sums(sums, comps, fsum, fcomp, n, N_WIN, HW)
        rows = torch.arange(a, b, dtype=torch.float64)[:, None] * torch.ones((1, 16), dtype=torch.float64)
        full = ed.gather_rows(rows, N_WIN)
        fm, n_m = ed.all_reduce_frame_sums(fsum, fcomp, n, None)     # first sweep of the 'image' methods
        q.put((rank, block.numpy(), fr.numpy(), n_tot, (a, b), full.numpy(), fm.numpy(), n_m))
    finally:
        torch.distributed.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_window_blocks_cover_all_windows():
    for n, w in ((37, 2), (64009, 8), (5, 8), (8, 8)):
        blocks = ed.window_blocks(n, w)
        assert blocks[0][0] == 0 and blocks[-1][1] == n
        assert all(blocks[i][1] == blocks[i + 1][0] for i in range(w - 1))
        sizes = [b - a for a, b in blocks]
        assert max(sizes) - min(sizes) <= 1


def test_two_rank_exchange_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    data = [_rank_data(r) for r in range(world)]
    tot = sum((d[0].double() - d[1].double()) for d in data).reshape(3, N_WIN, HW)
    ftot = sum((d[2].double() - d[3].double()) for d in data)
    for rank, block, fr, n_tot, (a, b), full, fm, n_m in res:
        assert n_tot == n_m == sum(d[4] for d in data)
        np.testing.assert_allclose(block, tot[:, a:b].float().numpy(), rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(fr, ftot.float().numpy(), rtol=1e-6, atol=1e-6)
        assert np.array_equal(fm, fr)
        assert np.array_equal(full[:, 0], np.arange(N_WIN, dtype=np.float64))
