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


def test_short_poisson_run_completes(cuda):
    srv = serving.PivServer(device=cuda, max_batch=4)
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
