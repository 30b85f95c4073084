"""Host-side logic of the serving loop and the launch autotuner, on the CPU.

The libraries and the GPU are replaced by fakes: the autotuner's coordinate
search runs against a timing model whose fastest settings are known, and the
serving helpers that need no device (arrivals, engine sizing, schedules) are
checked directly.
"""

import json
import types

import numpy as np
import pytest


def _fake_mp(sizes=((128, 128), (64, 64), (32, 32)), finder=3):
    cfg = types.SimpleNamespace(window_sizes=list(sizes), overlaps=[50] * len(sizes),
                                peak_finder=finder, interp_mode=0)
    return types.SimpleNamespace(cfg=cfg, device="cuda:0", H=2048, W=2048, N=64)


class _FakeLibs:
    """Records what the tuner applies and times the step from the settings."""

    def __init__(self, best_rows=8, best_by=2, best_caps=None, best_tb=64, top=4):
        self.best = dict(rows=best_rows, by=best_by, caps=best_caps or {64: 3}, tb=best_tb)
        self.top = top
        self.state = dict(rows=16, by=4, caps={}, tb=128)
        self.applied = []
        self.timed = 0

    def apply(self, s):
        self.applied.append(json.loads(json.dumps(s)))
        if "warp_rows" in s:
            self.state["rows"], self.state["by"] = int(s["warp_rows"]), int(s["warp_block_y"])
        for n, c in s.get("ctas_per_sm", {}).items():
            self.state["caps"][int(n)] = int(c)
        if "record_block" in s:
            self.state["tb"] = int(s["record_block"])

    def time_step(self, *_a):
        # 100 ms, less 5 ms for each setting at its fastest value
        self.timed += 1
        st, b = self.state, self.best
        t = 100.0
        t -= 5.0 * ((st["rows"], st["by"]) == (b["rows"], b["by"]))
        t -= sum(5.0 for n, c in b["caps"].items() if st["caps"].get(n, 0) == c)
        t -= 5.0 * (st["tb"] == b["tb"])
        return t


@pytest.fixture
def tuner(monkeypatch):
    import torch
    from pivtools_b200 import autotune

    libs = _FakeLibs()
    monkeypatch.setattr(autotune, "apply", libs.apply)
    monkeypatch.setattr(autotune, "_time_step", libs.time_step)
    monkeypatch.setattr(autotune, "_key", lambda mp: f"fake|{mp.H}x{mp.W}|finder{mp.cfg.peak_finder}")
    monkeypatch.setattr(autotune._lib, "bulkxcorr2d_lib",
                        lambda: types.SimpleNamespace(pivb_xcorr_max_ctas_per_sm=lambda n: libs.top))
    monkeypatch.setattr(torch.cuda, "Stream", lambda device=None: object())
    return autotune, libs


def test_autotune_finds_the_fastest_settings_and_caches_them(tuner, tmp_path):
    autotune, libs = tuner
    cache = str(tmp_path / "tune" / "autotune.json")
    out = autotune.tune(_fake_mp(), None, None, cache=cache)
    assert out["cached"] is False
    s = out["settings"]
    assert (s["warp_rows"], s["warp_block_y"]) == (8, 2)
    assert s["record_block"] == 64
    # caps tried from the occupancy maximum down: top-1 and top-2 for each size
    assert s["ctas_per_sm"] == {128: 0, 64: 3, 32: 0}
    assert out["step_ms_default"] == 100.0 and out["step_ms_tuned"] == 85.0
    # the best settings are left applied
    assert libs.applied[-1]["warp_rows"] == 8 and libs.state["tb"] == 64
    # trials, each value once: the default step, the 11 other warp shapes, caps
    # top-1 and top-2 for each of 3 sizes, the 2 other record blocks
    assert out["trials"] == 1 + 11 + 6 + 2 == libs.timed

    with open(cache) as f:
        assert "fake|2048x2048|finder3" in json.load(f)
    libs.applied.clear()
    libs.timed = 0
    again = autotune.tune(_fake_mp(), None, None, cache=cache)
    assert again["cached"] is True and libs.timed == 0
    assert libs.applied == [json.loads(json.dumps(s))]


def test_autotune_keeps_defaults_below_min_gain(tuner, tmp_path):
    autotune, libs = tuner
    libs.time_step = lambda *_a: 100.0            # nothing is faster
    autotune._time_step = libs.time_step
    out = autotune.tune(_fake_mp(finder=0), None, None, cache=None)
    s = out["settings"]
    assert (s["warp_rows"], s["warp_block_y"], s["record_block"]) == (16, 4, 128)
    assert s["ctas_per_sm"] == {128: 0, 64: 0, 32: 0}
    # no fit kernel for the argmax-only finder: record blocks are not tried
    assert not any(a.get("record_block") in (32, 64) for a in libs.applied)


def test_autotune_unreadable_cache_is_a_miss(tuner, tmp_path):
    autotune, libs = tuner
    cache = tmp_path / "autotune.json"
    cache.write_text("{not json")
    out = autotune.tune(_fake_mp(), None, None, cache=str(cache))
    assert out["cached"] is False and libs.timed > 0


def test_poisson_arrivals_seeded_sorted_and_at_rate():
    from pivtools_b200 import serving

    a = serving.poisson_arrivals(200.0, 60.0, seed=5)
    b = serving.poisson_arrivals(200.0, 60.0, seed=5)
    assert np.array_equal(a, b)
    assert np.all(np.diff(a) > 0) and a[0] > 0 and a[-1] < 60.0
    # 12,000 expected; Poisson std ~110
    assert abs(len(a) - 12000) < 600
    assert len(serving.poisson_arrivals(200.0, 60.0, seed=6)) != len(a) or not np.array_equal(
        serving.poisson_arrivals(200.0, 60.0, seed=6), a)


def test_serving_engine_size_and_schedule():
    from pivtools_b200 import serving

    cfg = serving.schedule_config([128, 64, 32, 16], overlap=50)
    assert cfg.window_sizes == [(128, 128), (64, 64), (32, 32), (16, 16)]
    assert cfg.overlaps == [50, 50, 50, 50]
    # four float32 frames and two uint16 frames per pair, 10% margin, 64 MiB of grids
    nb = serving.PivServer._engine_bytes((2048, 4096), (32,), 4)
    assert nb == int(4 * 2048 * 4096 * 20 * 1.1) + (64 << 20)
    # the largest class of the serving mix fits the 120 GB budget many times over
    assert 120e9 // nb >= 50


def test_no_cpu_path():
    """Without a GPU the resident pipelines refuse to start: there is no CPU
    fallback behind them."""
    import torch
    from pivtools_b200 import ensemble, multipass

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    cfg = multipass.MultipassConfig(window_sizes=[(32, 32)], overlaps=[50])
    with pytest.raises(RuntimeError):
        multipass.MultipassPIV((256, 256), 1, cfg)
    with pytest.raises(RuntimeError):
        ensemble.EnsemblePIV((256, 256), window=(16, 16), overlap=75)
