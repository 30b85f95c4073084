"""Launch-shape autotuner for the multipass step.

The kernels' data layouts (lanes per FFT column, plane strides, register caps)
are fixed at compile time by measurement; what stays open at run time, and
depends on the GPU and the workload's shape, is tuned here on the caller's own
step:

  * correlation: resident CTAs per SM for each window size of the schedule
    (``pivb_xcorr_set_ctas_per_sm``: from the occupancy maximum down), which
    sets how many windows share an SM;
  * warp: output rows per thread and block height
    (``pivb_warp_set_launch``);
  * per-window fit kernel: block size (``pivb_xcorr_set_record_block``).

A coordinate search times the whole resident step (CUDA events on the step's
stream, median of `reps` replays after one warm-up) for each candidate of one
setting with the others held, keeps a candidate only if it beats the current
best by more than `min_gain`, and moves to the next setting.  Results are cached
per (GPU name, frame shape, batch, schedule) in a JSON file so later processes
apply them without measuring.  Settings are process-wide launch parameters of
the libraries; results are bit-identical under every setting (they change only
how work is spread over the GPU).
"""

from __future__ import annotations

import ctypes
import json
import os
import statistics

from . import _lib

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "pivtools_b200", "autotune.json")
WARP_ROWS = (4, 8, 16, 32)
WARP_BLOCK_Y = (1, 2, 4)
RECORD_BLOCKS = (32, 64, 128)


def _key(mp) -> str:
    import torch

    name = torch.cuda.get_device_name(mp.device)
    sizes = "-".join(f"{h}x{w}@{o}" for (h, w), o in zip(mp.cfg.window_sizes, mp.cfg.overlaps))
    return f"{name}|{mp.H}x{mp.W}|n{mp.N}|{sizes}|finder{mp.cfg.peak_finder}|interp{mp.cfg.interp_mode}"


def current() -> dict:
    """The libraries' current launch settings."""
    Lx, Lw = _lib.bulkxcorr2d_lib(), _lib.fusedwarp_lib()
    r, b = ctypes.c_int(), ctypes.c_int()
    Lw.pivb_warp_get_launch(ctypes.byref(r), ctypes.byref(b))
    return {"warp_rows": r.value, "warp_block_y": b.value,
            "ctas_per_sm": {n: Lx.pivb_xcorr_get_ctas_per_sm(n) for n in (8, 12, 16, 24, 32, 48, 64, 96, 128)}}


def apply(settings: dict) -> None:
    """Set the libraries' launch settings (a dict as `tune` returns)."""
    Lx, Lw = _lib.bulkxcorr2d_lib(), _lib.fusedwarp_lib()
    if "warp_rows" in settings:
        if Lw.pivb_warp_set_launch(int(settings["warp_rows"]), int(settings["warp_block_y"])) != 0:
            raise ValueError(f"warp launch settings out of range: {settings}")
    for n, c in settings.get("ctas_per_sm", {}).items():
        if Lx.pivb_xcorr_set_ctas_per_sm(int(n), int(c)) != 0:
            raise ValueError(f"ctas per SM out of range: {n}: {c}")
    if "record_block" in settings:
        if Lx.pivb_xcorr_set_record_block(int(settings["record_block"])) != 0:
            raise ValueError(f"record block out of range: {settings['record_block']}")


def reset() -> None:
    """Back to the compiled defaults."""
    apply({"warp_rows": 16, "warp_block_y": 4, "record_block": 128,
           "ctas_per_sm": {n: 0 for n in (8, 12, 16, 24, 32, 48, 64, 96, 128)}})


def _time_step(mp, A, B, stream, reps):
    import torch

    with torch.cuda.stream(stream):
        mp.run(A, B)                                   # warm-up under the candidate settings
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for a, b in ev:
            a.record(stream)
            mp.run(A, B)
            b.record(stream)
    stream.synchronize()
    return statistics.median(a.elapsed_time(b) for a, b in ev)


def tune(mp, A, B, reps: int = 3, min_gain: float = 0.01, cache: str | None = DEFAULT_CACHE,
         use_cache: bool = True) -> dict:
    """Tune the launch settings for MultipassPIV `mp` on frames A, B (its batch)
    and leave the best applied.  Returns the settings with the step times
    measured before and after (ms), and whether they came from the cache."""
    import torch

    key = _key(mp)
    if use_cache and cache and os.path.isfile(cache):
        try:
            with open(cache) as f:
                hit = json.load(f).get(key)
        except (OSError, ValueError):
            hit = None
        if hit:
            apply(hit["settings"])
            return dict(hit, cached=True)
    Lx = _lib.bulkxcorr2d_lib()
    stream = torch.cuda.Stream(device=mp.device)
    reset()
    best = {"warp_rows": 16, "warp_block_y": 4, "record_block": 128,
            "ctas_per_sm": {int(h): 0 for (h, w) in mp.cfg.window_sizes if h == w}}
    t_best = t0 = _time_step(mp, A, B, stream, reps)
    trials = [dict(best, ctas_per_sm=dict(best["ctas_per_sm"]))]

    def attempt(cand):
        nonlocal best, t_best
        apply(cand)
        t = _time_step(mp, A, B, stream, reps)
        trials.append(dict(cand, ms=t))
        if t < t_best * (1.0 - min_gain):
            best, t_best = cand, t
        apply(best)

    # each candidate value is measured once: the default is not retried after
    # another value has replaced it
    for rows in WARP_ROWS:
        for by in WARP_BLOCK_Y:
            if (rows, by) != (16, 4):
                attempt(dict(best, warp_rows=rows, warp_block_y=by))
    for n in sorted(best["ctas_per_sm"]):
        top = int(Lx.pivb_xcorr_max_ctas_per_sm(n))
        for c in range(top - 1, max(top - 3, 0), -1):
            cap = dict(best["ctas_per_sm"])
            cap[n] = c
            attempt(dict(best, ctas_per_sm=cap))
    if mp.cfg.peak_finder in (3, 4, 5, 6):
        for tb in RECORD_BLOCKS:
            if tb != 128:
                attempt(dict(best, record_block=tb))
    apply(best)
    out = {"settings": best, "step_ms_default": t0, "step_ms_tuned": t_best, "trials": len(trials), "key": key}
    if cache:
        try:
            os.makedirs(os.path.dirname(cache), exist_ok=True)
            data = {}
            if os.path.isfile(cache):
                with open(cache) as f:
                    data = json.load(f)
            data[key] = out
            with open(cache, "w") as f:
                json.dump(data, f, indent=1, default=str)
        except (OSError, ValueError):
            pass
    return dict(out, cached=False)
