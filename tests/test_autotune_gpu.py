"""The launch-shape autotuner (pivtools_b200.autotune): results are bit-identical
under every launch setting it may choose, it leaves the best setting applied and
never slower than the default by more than timing noise, and its cache replays."""

import numpy as np
import pytest

from pivtools_b200 import autotune, multipass, synthetic

pytestmark = pytest.mark.gpu


def _fields(mp):
    return [(p["ux"].cpu().numpy().copy(), p["uy"].cpu().numpy().copy()) for p in mp.passes]


def test_results_identical_under_every_setting(cuda):
    import torch

    HW = (512, 640)
    A, B = synthetic.channel_batch_torch(2, HW, seed=31, device=cuda, peak=6.0)
    mp = multipass.MultipassPIV(HW, 2, device=cuda)
    autotune.reset()
    mp.run(A, B)
    torch.cuda.synchronize()
    ref = _fields(mp)
    for s in ({"warp_rows": 4, "warp_block_y": 1, "record_block": 32, "ctas_per_sm": {32: 1, 64: 1, 128: 1}},
              {"warp_rows": 32, "warp_block_y": 2, "record_block": 64, "ctas_per_sm": {32: 2}}):
        autotune.apply(s)
        mp.run(A, B)
        torch.cuda.synchronize()
        for (rx, ry), (gx, gy) in zip(ref, _fields(mp)):
            assert np.array_equal(rx, gx, equal_nan=True) and np.array_equal(ry, gy, equal_nan=True)
    autotune.reset()
    with pytest.raises(ValueError):
        autotune.apply({"warp_rows": 0, "warp_block_y": 4})


def test_tune_and_cache(cuda, tmp_path):
    HW = (512, 512)
    A, B = synthetic.channel_batch_torch(2, HW, seed=32, device=cuda, peak=6.0)
    mp = multipass.MultipassPIV(HW, 2, device=cuda)
    cache = str(tmp_path / "tune.json")
    out = autotune.tune(mp, A, B, reps=2, cache=cache)
    assert not out["cached"] and out["trials"] > 10
    assert out["step_ms_tuned"] <= out["step_ms_default"] * 1.05
    assert autotune.current()["warp_rows"] == out["settings"]["warp_rows"]
    again = autotune.tune(mp, A, B, cache=cache)
    assert again["cached"] and again["settings"]["warp_rows"] == out["settings"]["warp_rows"]
    autotune.reset()
