"""Benchmark: multipass window-deformation PIV, 64 pairs of 2048x2048 per GPU.

Workload (one step): 64 image pairs of 2048^2 (0.05 ppp Gaussian particles,
sigma 0.6 px, intensities U[1000, 4000], Poisson noise on a 100-count
background; turbulent-channel-like flow with a 12 px log-law peak and 8% rms
fluctuations), four passes of 128/64/32/32 px windows at 50/50/50/75% overlap,
bicubic symmetric warp by the smoothed predictor before passes 2-4, 3-point
Gaussian subpixel fit, normalised-median validation and infilling between
passes.  Metric: output vectors (the final pass's 253x253 grid per pair) per
second.  Inputs (4.3 GB of float32 frames) exceed the 126 MB L2, so no flush is
needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun every rank processes its own 64 pairs (instantaneous PIV shards
by pair, no collective): weak scaling, value = all ranks' vectors / max time.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "python-pivtools_b200"))

METRIC = "vectors/s and p50/p99 pair latency on 1 B200 at ≤0.01 px RMS vs FP64 oracle"
WORKLOAD = "multipass window-deformation PIV, 64 pairs 2048x2048, passes 128/64/32/32 px at 50/50/50/75%"
HW = (2048, 2048)
PEAK_FINDER = 3        # the multipass workload's subpixel fit (--peak-finder; 3-point by default)
INTERP = 0             # image warp interpolation (--interp): 0 bicubic (default), 1 Lanczos-3
# FP32 CUDA-core peak, nominal: 148 SMs x 128 lanes x 2 flops x 1.965 GHz (no measured figure)
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--pairs", type=int, default=64)
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--cpu-pairs", type=int, default=2, help="CPU baseline leg: pairs in its batch")
    ap.add_argument("--ref-pairs", type=int, default=4, help="reference arm: pairs per (sampled) step")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the per-pass RMS against FP64")
    ap.add_argument("--no-autotune", action="store_true", help="keep the compiled launch defaults")
    ap.add_argument("--workload", default="multipass", choices=["multipass", "ensemble", "serve", "dft", "ingest"],
                    help="multipass: the headline line (default); ensemble: the 1024^2 16 px ensemble pass; "
                         "serve: Poisson request stream with continuous batching")
    ap.add_argument("--chunk", type=int, default=32, help="e2e: pairs per host-to-device chunk")
    ap.add_argument("--interp", default="cubic", choices=["cubic", "lanczos"],
                    help="multipass: image warp interpolation (the reference's image_warp_interpolation)")
    ap.add_argument("--peak-finder", type=int, default=3, choices=[3, 4, 5, 6],
                    help="multipass: subpixel fit, gauss3 (3-point) or the gauss4/5/6 Levenberg-Marquardt fits")
    ap.add_argument("--ensemble-bg", default="correlation+dc_zero",
                    choices=["correlation", "correlation+dc_zero", "window_mean", "correlation+window_mean", "image",
                             "image+window_mean", "image+dc_zero"],
                    help="ensemble: background subtraction method (the 'image' ones sweep each batch twice)")
    ap.add_argument("--no-dft-leg", action="store_true",
                    help="skip the tensor-core workload leg of the default run")
    ap.add_argument("--dft-frames", type=int, nargs=2, default=[49, 13], metavar=("F64", "F32"),
                    help="dft: 4096^2 mosaic frames of 64 px and of 32 px windows (smaller for profiling)")
    ap.add_argument("--engine32", default="fft", choices=["fft", "dft"],
                    help="32 px passes on the FP32 FFT path or the tensor-core DFT-as-GEMM path")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: offered pairs/s")
    ap.add_argument("--duration", type=float, default=60.0, help="serve: seconds of arrivals")
    ap.add_argument("--packed", action="store_true",
                    help="serve: packed rounds (one correlation launch per window size and pass)")
    ap.add_argument("--no-serve", action="store_true",
                    help="multipass: skip the served-latency leg (Poisson arrivals, --rate for --duration s)")
    return ap.parse_args()


def _pci_bus_id(index):
    """PCI bus id ("domain:bus:device.function") of CUDA device `index`, or None."""
    try:
        import torch

        p = torch.cuda.get_device_properties(index)
        return f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
    except Exception:
        return None


class ClockSampler:
    """SM clocks and throttle reasons sampled while the timed region runs.

    Read-only NVML queries every `period_s` (20 ms), else `nvidia-smi` every 0.2 s
    when NVML cannot be used.  The GPU is found by its PCI bus id, so the samples
    are of the device the step runs on even where CUDA_VISIBLE_DEVICES renumbers
    the devices."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index, period_s=0.02):
        self.index = index
        self.period = period_s
        self.rows = []
        self._stop = threading.Event()
        self._t = None
        self.bus_id = _pci_bus_id(index)
        self._nvml = None
        self._shutdown = None
        self.source = "nvidia-smi"
        try:
            import pynvml as nv

            nv.nvmlInit()
            self._shutdown = nv.nvmlShutdown
            h = nv.nvmlDeviceGetHandleByPciBusId(self.bus_id) if self.bus_id else nv.nvmlDeviceGetHandleByIndex(index)
            self._nvml = (nv, h)
            self.source = "nvml"
        except Exception:
            self._nvml = None

    def _nvml_row(self):
        nv, h = self._nvml
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        try:
            pw = f"{nv.nvmlDeviceGetPowerUsage(h) / 1000.0:.2f}"
        except Exception:
            pw = "[N/A]"
        r = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
        bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
        return [str(self.index), str(sm), str(mx), pw, hex(r)] + ["Active" if r & b else "Not Active" for b in bits]

    def _smi_row(self):
        ids = [self.bus_id, str(self.index)] if self.bus_id else [str(self.index)]
        for i in ids:
            out = subprocess.run(["nvidia-smi", f"--id={i}", f"--query-gpu={self.QUERY}",
                                  "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                 timeout=5).stdout.strip()
            row = [c.strip() for c in out.split(",")] if out else []
            if len(row) == 9:
                return row
            self.bus_id = None                 # not accepted as an id: use the index from now on
        return None

    def _run(self):
        while not self._stop.is_set():
            if self._nvml is not None:
                try:
                    self.rows.append(self._nvml_row())
                except Exception:
                    self._nvml, self.source = None, "nvidia-smi"
                    continue
                self._stop.wait(self.period)
            else:
                try:
                    row = self._smi_row()
                    if row:
                        self.rows.append(row)
                except Exception:
                    pass
                self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)
        if self._shutdown is not None:
            try:
                self._shutdown()
            except Exception:
                pass
            self._shutdown = None

    def summary(self):
        rows = [r for r in self.rows if len(r) == 9]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = self.REASONS
        reasons = sorted({names[k] for r in rows for k in range(4) if "Active" in r[5 + k] and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "source": self.source}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


def _dist():
    import torch

    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local))
    return ws, rank, local


def _workload_config(n_pairs, ws, vec_step, win_step):
    """The workload as both arms state it (identical keys and values)."""
    return {"workload": WORKLOAD, "pairs_per_step_per_gpu": n_pairs, "image": "2048x2048 uint16 counts",
            "passes": "128/64/32/32 px, 50/50/50/75%", "window_weight": "gaussian", "peak_finder": f"gauss{PEAK_FINDER}",
            "warp": f"{'Lanczos-3' if INTERP else 'bicubic'} symmetric, smoothed predictor",
            "validation": "gate win/2 then win/4; peak_mag 0.25; normalised median 5x5 (eps 0.1, thr 2)",
            "infill": "least squares between passes and after the last",
            "vectors_per_step_per_gpu": vec_step, "windows_per_step_per_gpu": win_step,
            "l2": "inputs 4.3 GB > L2, no flush", "parallelism": f"dp{ws} (pairs)"}


def _ref_frames(n_pairs, seed):
    """Host frames of the workload for the CPU arms (the same generator as the GPU
    arm's, run on the host)."""
    from pivtools_b200 import synthetic

    A, B = synthetic.channel_batch_torch(n_pairs, HW, seed=seed, device="cpu")
    return A.numpy(), B.numpy()


def _ref_pipeline():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_multipass as RM
    from pivtools_b200 import geometry, multipass

    cfg = multipass.MultipassConfig(peak_finder=PEAK_FINDER, interp_mode=INTERP)
    geo = geometry.multipass_geometry(HW, cfg.window_sizes, cfg.overlaps, cfg.window_type)
    return RM, RM.RefMultipass(geo, window_type=cfg.window_type, peak_finder=cfg.peak_finder,
                               infill=cfg.infill, final_infill=cfg.final_infill, interp_mode=cfg.interp_mode)


def _cpu_baseline(n_pairs: int):
    """CPU leg: the reference's multipass (its compiled libbulkxcorr2d and
    libfusedwarp, built from its sources, under OpenMP on every host core; the
    driver's glue restated in NumPy/SciPy/cv2) on n_pairs pairs in one batch, then
    one pair on one thread.  Returns the cpu_baseline object."""
    RM, rm = _ref_pipeline()
    A, B = _ref_frames(n_pairs, seed=900)
    cores = os.cpu_count() or 1
    RM.set_threads(cores)
    rm.run(A[:1], B[:1])                        # load libraries, warm caches
    t0 = time.perf_counter()
    rm.run(A, B)
    dt = time.perf_counter() - t0
    RM.set_threads(1)
    t1 = time.perf_counter()
    rm.run(A[:1], B[:1])
    dt1 = time.perf_counter() - t1
    RM.set_threads(cores)
    vec = 64009
    return {"value": n_pairs * vec / dt, "unit": "vectors/s", "cores": cores, "kind": "reference",
            "value_1_thread": vec / dt1,
            "sample": f"{n_pairs} pairs of the workload in one batch through the reference's compiled "
                      f"libbulkxcorr2d + libfusedwarp (OpenMP, {cores} threads; glue in NumPy/SciPy/cv2, "
                      f"biharmonic infill): {dt:.2f} s; 1 pair on 1 thread: {dt1:.2f} s"}


def run_reference(args):
    """The reference's own CPU path on this workload: every step is one batch of
    --ref-pairs pairs (a bounded sample of the 64-pair step) through the
    reference's pass loop over its compiled libraries, all host threads."""
    ws, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    RM, rm = _ref_pipeline()
    P = args.ref_pairs
    A, B = _ref_frames(P, seed=2026)
    cores = os.cpu_count() or 1
    RM.set_threads(cores)
    for _ in range(args.warmup):
        rm.run(A, B)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        rm.run(A, B)
        times.append(time.perf_counter() - t0)
    ms = statistics.median(times) * 1e3
    vec = 64009
    value = P * vec / (ms * 1e-3)
    geo_win = 31 * 31 + 63 * 63 + 127 * 127 + 253 * 253
    sample = (f"{P} pairs per step (of the 64-pair workload step) through the reference's compiled "
              f"libbulkxcorr2d + libfusedwarp, OpenMP {cores} threads, glue in NumPy/SciPy/cv2, biharmonic "
              f"infill; median of {args.steps} steps")
    line = {"metric": METRIC, "value": value, "unit": "vectors/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": _workload_config(64, ws, 64 * vec, 64 * geo_win),
            "impl": "reference", "sample_pairs_per_step": P,
            "cpu_baseline": {"value": value, "unit": "vectors/s", "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "vectors/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _pipeline_vs_reference(mp, A, B):
    """Pair 0's whole multipass (warps, validation, biharmonic infill,
    smoothing, remap) against the reference's pass loop over its compiled
    libraries on the same frames: per pass the largest and RMS displacement
    difference and the share of equal invalid flags; None when the reference
    libraries are not built."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    if O.ref_bulk() is None or O.ref_warp() is None:
        return None
    import ref_multipass as RM

    rm = RM.RefMultipass(mp.geo, window_type=mp.cfg.window_type, peak_finder=mp.cfg.peak_finder,
                         infill=mp.cfg.infill, final_infill=mp.cfg.final_infill)
    rm.run(A[:1].cpu().numpy(), B[:1].cpu().numpy())
    out = []
    for k, (p, (rx, ry, rbad)) in enumerate(zip(mp.passes, rm.history)):
        gx, gy = p["ux"][0].cpu().numpy(), p["uy"][0].cpu().numpy()
        gbad = p["invalid"][0].cpu().numpy().astype(bool)
        d = np.hypot(gx - rx[0], gy - ry[0])
        out.append({"pass": k, "max_px": float(d.max()), "rms_px": float(np.sqrt(np.mean(d * d))),
                    "invalid_flags_equal": float((gbad == rbad[0]).mean()), "invalid": int(gbad.sum())})
    return out


def _rms_vs_fp64(mp, A, B):
    """Per pass, pair 0: the resident pipeline's 3-point displacements against
    the FP64 oracle (and, when built, the reference's compiled correlator) on the
    same frames the pass correlated.  RMS over windows both fit."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from pivtools_b200 import geometry

    out = []
    for k, (p, g) in enumerate(zip(mp.passes, mp.geo)):
        fa, fb = mp.pass_inputs(k, A[:1], B[:1])
        fa, fb = fa[0].cpu().numpy(), fb[0].cpu().numpy()
        gx = p["out"]["pk_loc_x"][0, 0].cpu().numpy()
        gy = p["out"]["pk_loc_y"][0, 0].cpu().numpy()
        w = geometry.window_weight(g.window_size, mp.cfg.window_type)
        m = np.zeros((p["ny"], p["nx"]), np.float32)
        row = {"pass": k, "window": g.window_size[0], "windows": int(gx.size)}
        for name, fn in (("fp64", O.bulkxcorr2d), ("reference", O.ref_bulkxcorr2d if O.ref_bulk() else None)):
            if fn is None:
                continue
            r = fn(fa, fb, m, g.grid.win_ctrs_x, g.grid.win_ctrs_y, g.window_size, w, w)
            rx, ry = r["pk_x"][0, 0], r["pk_y"][0, 0]
            both = np.isfinite(gx) & np.isfinite(rx)
            row[f"rms_px_vs_{name}"] = float(np.sqrt(np.mean((gx - rx)[both] ** 2 + (gy - ry)[both] ** 2)))
            row[f"nan_flips_vs_{name}"] = int((np.isnan(gx) != np.isnan(rx)).sum())
        out.append(row)
    return out


def run_b200(args):
    import torch

    from pivtools_b200 import multipass, synthetic

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    N = args.pairs
    A, B = synthetic.channel_batch_torch(N, HW, seed=2026 + rank, device=dev)
    mp = multipass.MultipassPIV(HW, N, multipass.MultipassConfig(engine_32=args.engine32, peak_finder=PEAK_FINDER,
                                                                  interp_mode=INTERP), device=dev)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 1)):
            mp.run(A, B)
    stream.synchronize()
    tuned = None
    if not args.no_autotune:
        # launch shapes measured on this workload before the graph is captured
        # (a fresh measurement every run: no cache)
        from pivtools_b200 import autotune

        tuned = autotune.tune(mp, A, B, reps=3, cache=None)
    graph = None
    if not args.no_graph:
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            mp.run(A, B)
        for _ in range(args.warmup):
            graph.replay()
        torch.cuda.synchronize()

    def step():
        if graph is not None:
            graph.replay()
        else:
            mp.run(A, B)

    # ---- timed region: device events on the launching stream, max over ranks
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            e0.record(stream)
            for k in range(args.steps):
                step_ev[k][0].record(stream)
                step()
                step_ev[k][1].record(stream)
            e1.record(stream)
        stream.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    step_ms = sorted(a.elapsed_time(b) for a, b in step_ev)
    if ws > 1:
        t = torch.tensor([ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
        torch.distributed.barrier()
    vec_step = mp.vectors_per_step()
    value = vec_step * ws / (ms * 1e-3)

    # ---- dominant kernel: the final pass's correlation (32 px, 75%), timed alone
    p = mp.passes[-1]
    Lx = mp.Lx
    o = p["out"]
    nbytes = mp.scratch.numel()          # as in the step: the 3-point fits run in the record kernel
    import ctypes

    def corr_launch():
        s = ctypes.c_void_p(stream.cuda_stream)
        a = (mp.warped[0].data_ptr(), mp.warped[1].data_ptr(), HW[0] * HW[1], None, HW[0], HW[1], N,
             p["cx"].data_ptr(), p["cy"].data_ptr(), p["ny"], p["nx"], p["weight"].data_ptr(),
             p["weight"].data_ptr(), p["cw"].data_ptr(), 32, 32, 0, 1, 3, 0, o["pk_loc_x"].data_ptr(),
             o["pk_loc_y"].data_ptr(), o["pk_height"].data_ptr(), o["sx"].data_ptr(), o["sy"].data_ptr(),
             o["sxy"].data_ptr(), p["ratio"].data_ptr(), None, mp.scratch.data_ptr(), nbytes)
        if mp.Ld is not None:
            mp.Ld.pivb_dft_xcorr_dev(*a, mp.dft_status.data_ptr(), s)
        else:
            Lx.pivb_xcorr_dev(*a, s)

    with torch.cuda.stream(stream):
        for _ in range(3):
            corr_launch()
        k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k0.record(stream)
        R = 10
        for _ in range(R):
            corr_launch()
        k1.record(stream)
    stream.synchronize()
    kern_ms = k0.elapsed_time(k1) / R
    windows = N * p["ny"] * p["nx"]
    alg_bytes = 2 * N * HW[0] * HW[1] * 4 + 7 * windows * 4 + 2 * 128 * windows   # frames, outputs, records
    hbm_peak, bf16_peak, peak_kind = _peaks()
    achieved = alg_bytes / (kern_ms * 1e-3) / 1e9
    fp32_flops = windows * 80.1e3
    # DRAM traffic of one launch pair (correlation + deferred fits): dram__bytes_read.sum
    # + dram__bytes_write.sum of the same kernels and pass captured by ncu on 8 pairs
    # (xcorr_kernel<32>: 386.7 + 62.8 MB, lm_records_kernel: 65.6 + 4.8 MB, for
    # 512,072 windows; profiles/xcorr_kernel32_pass4_8pairs.md,
    # profiles/lm_records_gauss3_8pairs.md), scaled by windows processed (frames,
    # records and outputs all grow with the pair count).
    traffic = (386.735616e6 + 62.808576e6 + 65.61664e6 + 4.807424e6) / 512072 * windows

    # ---- end to end through host buffers: every step copies its 64 pairs of
    # uint16 frames from pinned memory (chunked, overlapped with compute), converts
    # them on the GPU, runs the passes and reads the final vector fields back
    from pivtools_b200.multipass import HostPipeline

    chunk = args.chunk if (args.chunk > 0 and N % args.chunk == 0) else N
    pipe = HostPipeline(HW, chunk, multipass.MultipassConfig(engine_32=args.engine32, peak_finder=PEAK_FINDER,
                                                           interp_mode=INTERP), device=dev)
    # frames are integer counts in [0, 65535]; every host buffer is page-locked with
    # .pin_memory() (torch.empty_like of a pinned tensor is pageable, which turns the
    # copies synchronous and serialises them with the compute)
    ux_h = torch.empty((N, p["ny"], p["nx"]), dtype=torch.float32).pin_memory()
    uy_h = torch.empty((N, p["ny"], p["nx"]), dtype=torch.float32).pin_memory()
    Ah = A.cpu().to(torch.int32).to(torch.uint16).pin_memory()
    Bh = B.cpu().to(torch.int32).to(torch.uint16).pin_memory()
    if not (Ah.is_pinned() and Bh.is_pinned() and ux_h.is_pinned() and uy_h.is_pinned()):
        raise RuntimeError("host frames are not page-locked")
    e2e_steps = max(2, args.steps)
    with torch.cuda.stream(stream):
        pipe.run(Ah, Bh, ux_h, uy_h)          # warm-up
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    with torch.cuda.stream(stream):
        q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        q0.record(stream)
        for _ in range(e2e_steps):
            pipe.run(Ah, Bh, ux_h, uy_h)
        pipe.finish()                           # every field read back before the end event
        q1.record(stream)
    stream.synchronize()
    e2e_ms = q0.elapsed_time(q1) / e2e_steps
    if ws > 1:
        t = torch.tensor([e2e_ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_val = vec_step * ws / (e2e_ms * 1e-3)
    e2e_launches = pipe.mp.launches_per_step * (N // chunk) + 2 * (N // chunk)
    fin = mp.passes[-1]
    e2e_same = bool(torch.allclose(ux_h, fin["ux"].cpu(), rtol=0, atol=0, equal_nan=True)
                    and torch.allclose(uy_h, fin["uy"].cpu(), rtol=0, atol=0, equal_nan=True))

    accuracy = pipe_ref = None
    if rank == 0 and ws == 1 and not args.no_accuracy:
        with torch.cuda.stream(stream):
            mp.run(A, B)                        # the resident buffers hold this run's passes
        stream.synchronize()
        accuracy = _rms_vs_fp64(mp, A, B)
        pipe_ref = _pipeline_vs_reference(mp, A, B)
    cpu = None
    if rank == 0 and ws == 1 and os.environ.get("PIVB_SKIP_CPU") != "1":
        cpu = _cpu_baseline(args.cpu_pairs)
    served = None
    if rank == 0 and ws == 1 and not args.no_serve:
        del pipe, Ah, Bh
        torch.cuda.empty_cache()
        served = _serve_leg(dev, args.rate, args.duration)

    tensor_core = None
    if rank == 0 and ws == 1 and not args.no_dft_leg:
        # the tensor-core workload (200k 64^2 + 200k 32^2 windows on the split-BF16
        # DFT-as-GEMM path, each size also on the FP32 FFT path) as a sub-object
        tensor_core = run_dft(args, emit=False)

    if rank == 0:
        fp32_tflops = fp32_flops / (kern_ms * 1e-3) / 1e12
        if mp.Ld is not None:
            roof = {"bound": "tensor", "achieved": windows * 1.769e6 / (kern_ms * 1e-3) / 1e12,
                    "peak": bf16_peak, "unit": "TFLOP/s",
                    "frac": windows * 1.769e6 / (kern_ms * 1e-3) / 1e12 / bf16_peak, "traffic": None,
                    "peak_kind": peak_kind, "tensor_flops_per_window": 1.769e6,
                    "kernel": "dft32 tcgen05 kernel + lm_records_kernel (final pass, 4.1M windows)",
                    "kernel_ms": kern_ms, "hbm_view": {"achieved_gbs": achieved, "frac": achieved / hbm_peak}}
        else:
            roof = {"bound": "fp32", "achieved": fp32_tflops, "peak": FP32_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                    "frac": fp32_tflops / FP32_NOMINAL_TFLOPS, "traffic": traffic,
                    "traffic_unit": "bytes per launch (DRAM read + write)",
                    "peak_kind": "nominal FP32 (148 SMs x 128 lanes x 2 x 1.965 GHz; no measured FP32 figure)",
                    "flops_per_window": 80.1e3, "flops_per_launch": fp32_flops,
                    "kernel": "xcorr_kernel<32> + " + ("lm_records_kernel" if PEAK_FINDER == 3 else "lm_fit_kernel") +
                              " (final pass, 4.1M windows)",
                    "kernel_ms": kern_ms,
                    "hbm_view": {"algorithmic_bytes": alg_bytes, "achieved_gbs": achieved, "peak_gbs": hbm_peak,
                                 "frac": achieved / hbm_peak, "peak_kind": peak_kind}}
        line = {
            "metric": METRIC, "value": value, "unit": "vectors/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": _workload_config(N, ws, vec_step, mp.windows_per_step()),
            "impl_detail": {"cuda_graph": graph is not None,
                            "engine_32px": ("tensor-core DFT-as-GEMM (split BF16 x3)" if args.engine32 == "dft"
                                            else "FP32 FFT"),
                            "infill": f"{mp.cfg.infill} least squares (FP64 CG on the GPU)"},
            "step_ms": {"p50": step_ms[len(step_ms) // 2], "max": step_ms[-1]},
            "roofline": roof,
            "e2e": {"value": e2e_val, "unit": "vectors/s", "h2d_bytes_per_step": 2 * N * HW[0] * HW[1] * 2,
                    "d2h_bytes_per_step": 2 * N * p["ny"] * p["nx"] * 4, "frames": "uint16",
                    "chunk_pairs": chunk, "gpu_launches_per_step": e2e_launches, "host_frames_pinned": True,
                    "matches_resident_run": e2e_same},
            "gpu_launches": mp.launches_per_step * args.steps,
            "clocks": clk.summary(),
        }
        if tuned is not None:
            line["autotune"] = {"settings": tuned["settings"], "step_ms_default": tuned["step_ms_default"],
                                "step_ms_tuned": tuned["step_ms_tuned"], "trials": tuned["trials"]}
        if served is not None:
            line["latency_ms"] = {"p50": served["latency_ms"]["p50"], "p99": served["latency_ms"]["p99"],
                                  "source": "served leg: request arrival to result in host memory"}
            line["served"] = served
        if tensor_core is not None:
            line["tensor_core"] = {k: tensor_core[k] for k in ("metric", "value", "unit", "ms_per_step", "config",
                                                                "paths_ms", "dft_vs_fft", "roofline", "accuracy")}
        if accuracy is not None:
            line["accuracy"] = {"per_pass": accuracy, "pipeline_vs_reference": pipe_ref,
                                "rms_px_vs_fp64": max(r["rms_px_vs_fp64"] for r in accuracy),
                                "note": "pair 0, each pass against the FP64 oracle (and the reference's compiled "
                                        "correlator) on the frames that pass correlated; the headline is the worst pass"}
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if graph is not None:
        del graph
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def run_ensemble(args):
    """Ensemble pass at the 5000-pair workload's shapes: 1024x1024 frames at 0.02
    ppp with per-particle row-Gaussian displacements, 16 px square windows at 75%
    (64,009 windows), triple accumulation in batches of --pairs pairs, then the
    finalise (correlation background, plane-mean removal, normalisation) and the
    k-space fit of every window.  One step = one batch accumulated; the value is
    pairs/s; the finalise and the fit are timed once after the steps."""
    import torch

    from pivtools_b200 import ensemble, synthetic

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    shape = (1024, 1024)
    P = args.pairs
    frames = [synthetic.particle_pair(shape, seed=5000 + 97 * rank + k, density=0.02, flow="ensemble_rows",
                                      device=dev)[:2] for k in range(P)]
    A = torch.stack([f[0] for f in frames]).contiguous()
    B = torch.stack([f[1] for f in frames]).contiguous()
    del frames
    bg = args.ensemble_bg
    ep = ensemble.EnsemblePIV(shape, (16, 16), 75, "square", background=bg, device=dev)
    two = ep.two_sweep

    def end_means():
        if ws > 1:
            ep.end_means_distributed()           # one all-reduce of the frame sums
        else:
            ep.end_means()

    def sweeps(n):
        """n batches accumulated; the 'image' methods sweep them twice (frame sums,
        then the mean-subtracted correlation)."""
        if two:
            for _ in range(n):
                ep.accumulate_means(A, B)
            end_means()
        for _ in range(n):
            ep.accumulate(A, B)

    stream = torch.cuda.Stream(device=dev)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        sweeps(max(args.warmup, 1))
        ep.finalize()                            # first launches of the finalise and the fit
        ep.fit()                                 # (module loading) stay out of their timings
    stream.synchronize()
    ep.reset()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            e0.record(stream)
            sweeps(args.steps)
            e1.record(stream)
        stream.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    if ws > 1:
        t = torch.tensor([ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    value = P * ws / (ms * 1e-3)
    with torch.cuda.stream(stream):
        f0, f1, f2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        f0.record(stream)
        if ws > 1:
            ep.finalize_distributed()        # one exchange: reduce-scatter of the sums by window block
        else:
            ep.finalize()
        f1.record(stream)
        fit = ep.fit()
        if ws > 1:
            fit = ep.gather_fit(fit)
        f2.record(stream)
    stream.synchronize()
    fin_ms, fit_ms = f0.elapsed_time(f1), f1.elapsed_time(f2)
    st = fit["status"].cpu().numpy()
    # end to end: each step's uint16 frames (integer counts) stream from pinned host
    # memory in 32-pair chunks (one spectral block each), copies overlapped with
    # conversion and accumulation
    Ah = A.round().clamp(0, 65535).to(torch.int32).to(torch.uint16).cpu().pin_memory()
    Bh = B.round().clamp(0, 65535).to(torch.int32).to(torch.uint16).cpu().pin_memory()
    if not (Ah.is_pinned() and Bh.is_pinned()):
        raise RuntimeError("host frames are not page-locked")
    def host_sweeps(n):
        if two:
            ep.reset()
            for _ in range(n):
                ep.accumulate_means_host(Ah, Bh, chunk=32)
            end_means()
        for _ in range(n):
            ep.accumulate_host(Ah, Bh, chunk=32)

    n_e2e = max(2, min(args.steps, 5))
    with torch.cuda.stream(stream):
        host_sweeps(1)                                   # warm the staging buffers
        q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        q0.record(stream)
        host_sweeps(n_e2e)
        q1.record(stream)
    stream.synchronize()
    e2e_ms = q0.elapsed_time(q1) / n_e2e
    if ws > 1:
        t = torch.tensor([e2e_ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
    sweeps_per_step = 2 if two else 1
    h2d_bytes = 2 * P * shape[0] * shape[1] * 2 * sweeps_per_step
    alg_bytes = 2 * P * shape[0] * shape[1] * 4 * sweeps_per_step
    # the dominant kernel alone (accum_kernel<16>, one launch over the batch) into
    # throwaway sums: FP32 work per window-pair = 7 real 2-D transforms (four
    # forward: A and B under the AB and the auto weights; three inverse: AB, AA,
    # BB) x 2.5 n^2 log2(n^2) + 3 complex products x 6 n (n/2 + 1), n = 16: 38,432
    nc = ep.comp_size[0]
    flops_pair = 7 * 2.5 * nc * nc * math.log2(nc * nc) + 3 * 6 * nc * (nc // 2 + 1)
    tmp = torch.zeros_like(ep.sums)
    with torch.cuda.stream(stream):
        s_c = ctypes.c_void_p(stream.cuda_stream)
        PA, PB = ep._prepare(A, B, P, s_c, in_place=False)
        ep._triple(PA, PB, P, ep.mean_subtract, tmp, None, s_c)            # warm
        k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k0.record(stream)
        for _ in range(5):
            ep._triple(PA, PB, P, ep.mean_subtract, tmp, None, s_c)
        k1.record(stream)
    stream.synchronize()
    acc_ms = k0.elapsed_time(k1) / 5
    del tmp
    acc_tflops = flops_pair * ep.n_win * P / (acc_ms * 1e-3) / 1e12
    hbm_peak, _, peak_kind = _peaks()
    cpu = None
    if rank == 0 and ws == 1 and os.environ.get("PIVB_SKIP_CPU") != "1":
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import numpy as np
        import oracle as O

        g = ep.grid
        w = np.ones((16, 16), np.float32)
        npair = 4
        a1, b1 = A[:npair].cpu().numpy(), B[:npair].cpu().numpy()
        m0 = np.zeros((g.n_win_y, g.n_win_x), np.float32)
        ref = O.ref_bulk() is not None
        acc = O.ref_accumulate_triple if ref else O.accumulate_triple
        acc(a1[:1], b1[:1], m0, g.win_ctrs_x, g.win_ctrs_y, (16, 16), w, w, w, w)      # warm
        t0 = time.perf_counter()
        acc(a1, b1, m0, g.win_ctrs_x, g.win_ctrs_y, (16, 16), w, w, w, w)
        dt = time.perf_counter() - t0
        fit_note = ""
        if O.ref_kspace() is not None:
            fin_planes = {k: v.cpu().numpy()[:4096] for k, v in ep.finalize().items() if k != "norm"}
            t1 = time.perf_counter()
            O.ref_kspace_fit(fin_planes["R_AA"], fin_planes["R_BB"], fin_planes["R_AB"], np.zeros(4096, np.uint8),
                             (16, 16), n_threads=os.cpu_count() or 1)
            dk = time.perf_counter() - t1
            fit_note = f"; reference kspace_lm_fit_batch: {4096 / dk:.0f} fits/s on the same threads"
        cpu = {"value": npair / dt, "unit": "pairs/s", "cores": os.cpu_count() or 1,
               "kind": "reference" if ref else "port",
               "sample": f"{npair} pairs through the {'reference' if ref else 'oracle-port'} "
                         f"bulkxcorr2d_accumulate_triple, OpenMP on all host threads; {dt:.2f} s{fit_note}"}
    if rank == 0:
        line = {
            "metric": "ensemble pairs/s (triple accumulation) on 1 B200", "value": value, "unit": "pairs/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "ensemble pass, 1024x1024 pairs at 0.02 ppp, 16 px square windows at 75% "
                                   f"(64,009 windows), {bg} background"
                                   f"{' (two sweeps per batch)' if two else ''}, k-space fit (flat floor)",
                       "pairs_per_step_per_gpu": P, "l2": f"{P} distinct pairs cycled ({2 * P * 4} MB > L2)",
                       "parallelism": f"dp{ws} (pairs)"},
            "finalize_ms": fin_ms, "fit_ms": fit_ms, "fit_windows_per_s": ep.n_win / (fit_ms * 1e-3),
            "multi_gpu": "pairs sharded; sums reduce-scattered by window block, fits all-gathered" if ws > 1 else None,
            "fit_status_counts": {str(int(k)): int((st == k).sum()) for k in sorted(set(st.tolist()))},
            "projected_5000_pairs_s": 5000 / value + (fin_ms + fit_ms) * 1e-3,
            "roofline": {"bound": "fp32", "achieved": acc_tflops, "peak": FP32_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                         "frac": acc_tflops / FP32_NOMINAL_TFLOPS, "traffic": None,
                         "peak_kind": "nominal FP32 (148 SMs x 128 lanes x 2 x 1.965 GHz; no measured FP32 figure)",
                         "kernel": f"accum_kernel<{nc}> (one launch over the batch)", "kernel_ms": acc_ms,
                         "flops_per_window_pair": flops_pair, "windows": ep.n_win,
                         "hbm_view": {"kernels": "accum_kernel + frame sums" + (" + mean-image subtraction" if two
                                                                                else ""),
                                      "algorithmic_bytes": alg_bytes,
                                      "achieved_gbs": alg_bytes / (ms * 1e-3) / 1e9, "peak_gbs": hbm_peak,
                                      "frac": alg_bytes / (ms * 1e-3) / 1e9 / hbm_peak, "peak_kind": peak_kind}},
            "e2e": {"value": P * ws / (e2e_ms * 1e-3), "unit": "pairs/s", "h2d_bytes_per_step": h2d_bytes,
                    "d2h_bytes_per_step": 0, "frames": "uint16", "chunk_pairs": 32},
            "gpu_launches": (5 * args.steps + 2) if two else 3 * args.steps,
            "clocks": clk.summary(),
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def _mosaic(n_frames, win, side, seed, dev):
    """Frames of 0%-overlap windows of `win` px, each window of frame B shifted
    by its own uniform random (dy, dx) in [-4, 4]^2 px: particle images at
    0.05 ppp (sigma 0.6 px, intensities U[1000, 4000], Poisson noise on a 100
    count background).  Returns A, B (n, side, side) float32 on `dev` and the
    shifts (n, side/win, side/win, 2)."""
    import numpy as np
    import torch

    from pivtools_b200 import synthetic

    nw = side // win
    rng = np.random.default_rng(seed)
    A = torch.empty((n_frames, side, side), dtype=torch.float32, device=dev)
    B = torch.empty_like(A)
    shifts = rng.uniform(-4.0, 4.0, (n_frames, nw, nw, 2))
    n = int(round(0.05 * side * side))
    for k in range(n_frames):
        xs = rng.uniform(-8.0, side + 8.0, n)
        ys = rng.uniform(-8.0, side + 8.0, n)
        amp = rng.uniform(1000.0, 4000.0, n)
        wi = np.clip((ys // win).astype(np.int64), 0, nw - 1)
        wj = np.clip((xs // win).astype(np.int64), 0, nw - 1)
        dy, dx = shifts[k, wi, wj, 0], shifts[k, wi, wj, 1]
        g = torch.Generator(device=dev).manual_seed(int(seed) * 131 + k)
        ia = synthetic._render_torch((side, side), xs, ys, amp, 0.6, dev)
        ib = synthetic._render_torch((side, side), xs + dx, ys + dy, amp, 0.6, dev)
        A[k] = torch.clamp(torch.poisson(ia + 100.0, generator=g), 0, 65535).float()
        B[k] = torch.clamp(torch.poisson(ib + 100.0, generator=g), 0, 65535).float()
    return A, B, shifts


def run_dft(args, emit=True):
    """Tensor-core workload: 200k independent 64x64 and 200k 32x32 windows cut
    from particle images with uniform random shifts in [-4, 4]^2 px, packed as
    mosaics of 0%-overlap windows in 4096 x 4096 frames (49 frames of 4,096
    windows of 64 px, 13 frames of 16,384 windows of 32 px), gauss3 fits.  Both
    window sizes run on the split-BF16 tensor-core DFT-as-GEMM path (the step);
    each size also runs on the FP32 FFT path for the comparison.  Value:
    windows/s of the whole 400k-window step; each path's plane error and
    displacement RMS against the FP64 oracle on a sample frame are in the line."""
    import ctypes

    import numpy as np
    import torch

    from pivtools_b200 import _lib, geometry

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    side = 4096
    sets = {64: args.dft_frames[0], 32: args.dft_frames[1]}
    Lx, Ld = _lib.bulkxcorr2d_lib(), _lib.dft_lib()
    data = {}
    for n, nf in sets.items():
        A, B, sh = _mosaic(nf, n, side, seed=4000 + n + 97 * rank, dev=dev)
        g = geometry.compute_window_centers((side, side), (n, n), 0)
        w = torch.tensor(geometry.window_weight((n, n), "gaussian"), device=dev)
        cw = torch.empty_like(w)
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        assert Lx.pivb_correl_weight_dev(w.data_ptr(), n, n, cw.data_ptr(), st) == 0
        total = nf * g.n_win_y * g.n_win_x
        out = {k: torch.zeros((nf, 1, g.n_win_y, g.n_win_x), device=dev) for k in ("x", "y", "h", "sx", "sy", "sxy")}
        rat = torch.zeros((nf, g.n_win_y, g.n_win_x), device=dev)
        nb = int(Lx.pivb_xcorr_record_bytes(total))
        data[n] = dict(A=A, B=B, shifts=sh, g=g, w=w, cw=cw, out=out, rat=rat, total=total, nf=nf,
                       cx=torch.tensor(g.win_ctrs_x, device=dev), cy=torch.tensor(g.win_ctrs_y, device=dev),
                       scr=torch.empty(nb, dtype=torch.uint8, device=dev), nb=nb)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)

    def launch(n, engine, planes=None, nf=None):
        d = data[n]
        o = d["out"]
        st = ctypes.c_void_p(stream.cuda_stream)
        a = (d["A"].data_ptr(), d["B"].data_ptr(), side * side, None, side, side, d["nf"] if nf is None else nf,
             d["cx"].data_ptr(), d["cy"].data_ptr(), d["g"].n_win_y, d["g"].n_win_x, d["w"].data_ptr(),
             d["w"].data_ptr(), d["cw"].data_ptr(), n, n, 0, 1, 3, 0, o["x"].data_ptr(), o["y"].data_ptr(),
             o["h"].data_ptr(), o["sx"].data_ptr(), o["sy"].data_ptr(), o["sxy"].data_ptr(), d["rat"].data_ptr(),
             None if planes is None else planes.data_ptr(), d["scr"].data_ptr(), d["nb"])
        if engine == "dft":
            code = Ld.pivb_dft_xcorr_dev(*a, status.data_ptr(), st)
        else:
            code = Lx.pivb_xcorr_dev(*a, st)
        if code != 0:
            raise RuntimeError(f"{engine} correlation failed ({code})")

    def timed(fn, reps):
        with torch.cuda.stream(stream):
            for _ in range(max(args.warmup, 1)):
                fn()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
        stream.synchronize()
        return e0.elapsed_time(e1) / reps

    with ClockSampler(local) as clk:
        ms_step = timed(lambda: (launch(64, "dft"), launch(32, "dft")), args.steps)
        ms_dft32 = timed(lambda: launch(32, "dft"), args.steps)
        ms_dft64 = timed(lambda: launch(64, "dft"), args.steps)
        ms_fft32 = timed(lambda: launch(32, "fft"), args.steps)
        ms_fft64 = timed(lambda: launch(64, "fft"), args.steps)
    if int(status.item()) != 0:
        raise RuntimeError("tensor-core MMA completion not observed")
    windows = data[64]["total"] + data[32]["total"]
    value = windows / (ms_step * 1e-3)
    if ws > 1:
        t = torch.tensor([ms_step], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_step = float(t.item())
        value = windows * ws / (ms_step * 1e-3)

    acc = {}
    if rank == 0 and not args.no_accuracy:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        for n, engine in ((32, "dft"), (32, "fft"), (64, "dft"), (64, "fft")):
            d = data[n]
            g = d["g"]
            planes = torch.zeros((g.n_win_y * g.n_win_x, n, n), device=dev)
            launch(n, engine, planes=planes, nf=1)
            stream.synchronize()
            gx, gy = d["out"]["x"][0, 0].cpu().numpy(), d["out"]["y"][0, 0].cpu().numpy()
            fa, fb = d["A"][0].cpu().numpy(), d["B"][0].cpu().numpy()
            wn = d["w"].cpu().numpy()
            o = O.bulkxcorr2d(fa, fb, np.zeros((g.n_win_y, g.n_win_x), np.float32), g.win_ctrs_x, g.win_ctrs_y,
                              (n, n), wn, wn, peak_finder=3, want_f64=True)
            R = o["planes_f64"].reshape(-1, n, n)
            P = planes.cpu().numpy()
            rel = np.abs(P - R).reshape(len(R), -1).max(axis=1) / np.abs(R).reshape(len(R), -1).max(axis=1)
            ox, oy = o["pk_x"][0, 0], o["pk_y"][0, 0]
            both = np.isfinite(gx) & np.isfinite(ox)
            true = d["shifts"][0]
            acc[f"{engine}{n}"] = {
                "windows": int(gx.size), "plane_rel_err_max": float(rel.max()),
                "rms_px_vs_fp64": float(np.sqrt(np.mean((gx - ox)[both] ** 2 + (gy - oy)[both] ** 2))),
                "nan_flips_vs_fp64": int((np.isnan(gx) != np.isnan(ox)).sum()),
                "rms_px_vs_true_shift": float(np.sqrt(np.nanmean((gx - true[..., 1]) ** 2 + (gy - true[..., 0]) ** 2)))}
    if rank == 0:
        _, bf16_peak, peak_kind = _peaks()
        n32, n64 = data[32]["total"], data[64]["total"]
        # tensor flops per window (split BF16, three products): 54 n^3
        tf32, tf64 = 54.0 * 32 ** 3, 54.0 * 64 ** 3
        tflops = (n32 * tf32 + n64 * tf64) / (ms_step * 1e-3) / 1e12
        line = {
            "metric": "windows/s, split-BF16 tensor-core DFT-as-GEMM path (64 px + 32 px windows) on 1 B200",
            "value": value, "unit": "windows/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16x3", "data": "synthetic",
            "config": {"workload": "200k 64x64 + 200k 32x32 independent windows, uniform shifts in [-4, 4] px, "
                                   "mosaics of 0%-overlap windows in 4096^2 frames (49 + 13 frames), gauss3"
                                   if tuple(args.dft_frames) == (49, 13) else
                                   f"{n64} 64x64 + {n32} 32x32 independent windows (reduced case)",
                       "windows_64": n64, "windows_32": n32,
                       "l2": f"inputs {sum(sets.values()) * 2 * side * side * 4 / 1e9:.1f} GB > L2"},
            "paths_ms": {"dft32": ms_dft32, "dft64": ms_dft64, "fft32": ms_fft32, "fft64": ms_fft64},
            "dft_vs_fft": {"32": ms_fft32 / ms_dft32, "64": ms_fft64 / ms_dft64,
                           "step": (ms_fft32 + ms_fft64) / ms_step, "target": 5.0},
            "roofline": {"bound": "tensor", "achieved": tflops, "peak": bf16_peak, "unit": "TFLOP/s",
                         "frac": tflops / bf16_peak, "traffic": None, "peak_kind": peak_kind,
                         "kernel": "dft64 + dft32 tcgen05 kernels + lm_records_kernel",
                         "tensor_flops_per_window": {"32": tf32, "64": tf64},
                         "per_path_tflops": {"dft32": n32 * tf32 / (ms_dft32 * 1e-3) / 1e12,
                                             "dft64": n64 * tf64 / (ms_dft64 * 1e-3) / 1e12}},
            "accuracy": acc, "clocks": clk.summary(),
            "e2e": None, "gpu_launches": 2 * args.steps * 2,
        }
        if not emit:
            del data
            torch.cuda.empty_cache()
            return line
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def _im7_bytes(frames, pack):
    """An Image_Header_7 file of uint16 frames (F, H, W): pack 0 (uncompressed) or
    pack 2 (one zlib block per row), with an intensity-scale record."""
    import struct
    import zlib

    import numpy as np

    F, H, W = frames.shape
    head = struct.pack("<hhhh iiii hhh", 0, pack, -4, 0, W, H, 1, F, 0, 0, 0)
    head += bytes(256 - len(head))
    if pack == 0:
        body = frames.astype("<u2").tobytes()
    else:
        body = b"".join(struct.pack("<i", len(z)) + z for z in
                        (zlib.compress(frames[k, r].astype("<u2").tobytes(), 1) for k in range(F) for r in range(H)))
    rec = b"2 10\x00counts\x00\x00"
    attrs = struct.pack("<ii", 4, len(rec)) + rec + struct.pack("<i", 0)
    return head + body + attrs


def run_ingest(args):
    """Frame ingest: LaVision .im7 camera pairs (2048 x 2048 uint16, pack 0
    uncompressed and pack 2 zlib rows) read from local files, decoded natively
    into page-locked memory, copied and unpacked on the GPU into float32 frames
    with the intensity scale (lavision.read_im7_camera); host threads take files
    in parallel.  Value: pairs/s delivered to the device (wall clock around the
    whole batch, device synchronised)."""
    import tempfile
    import time
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np
    import torch

    from pivtools_b200 import lavision

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(5)
    n_files, H, W = 16, 2048, 2048
    results, cpu_legs = {}, {}
    with tempfile.TemporaryDirectory() as td:
        for pack in (0, 2):
            paths = []
            for k in range(n_files):
                fr = rng.integers(90, 4000, (2, H, W), dtype=np.uint16)
                fr[:, ::7] = 100                       # some structure for the zlib stream
                p = os.path.join(td, f"p{pack}_{k}.im7")
                with open(p, "wb") as f:
                    f.write(_im7_bytes(fr, pack))
                paths.append(p)
            outs = [torch.empty((2, H, W), dtype=torch.float32, device=dev) for _ in paths]

            def one(k):
                lavision.read_im7_camera(paths[k], camera_no=1, frames_per_camera=2, out=outs[k], device=dev)

            for threads in (1, 8):
                with ThreadPoolExecutor(threads) as ex:
                    list(ex.map(one, range(n_files)))          # warm-up (page cache, staging)
                    torch.cuda.synchronize()
                    reps = max(args.steps // 3, 2)
                    t0 = time.perf_counter()
                    for _ in range(reps):
                        list(ex.map(one, range(n_files)))
                    torch.cuda.synchronize()
                    dt = (time.perf_counter() - t0) / reps
                nbytes = sum(os.path.getsize(p) for p in paths)
                results[f"pack{pack}_threads{threads}"] = {
                    "pairs_per_s": n_files / dt, "ms_per_pair": dt / n_files * 1e3,
                    "file_mb_per_s": nbytes / dt / 1e6}
            if os.environ.get("PIVB_SKIP_CPU") != "1":
                # the oracle's restatement of the reference reader (numpy + zlib,
                # float32 frames in host memory) on the same files, one thread and
                # every host thread
                sys.path.insert(0, os.path.join(ROOT, "oracle"))
                import lavision_oracle as LO

                def host(k):
                    return LO.read_im7_camera_host(paths[k], 1, 2)

                host(0)
                for threads in (1, os.cpu_count() or 1):
                    with ThreadPoolExecutor(threads) as ex:
                        t0 = time.perf_counter()
                        list(ex.map(host, range(n_files)))
                        dt = time.perf_counter() - t0
                    cpu_legs[f"pack{pack}_threads{threads}"] = {"pairs_per_s": n_files / dt,
                                                                "ms_per_pair": dt / n_files * 1e3}
    best = max(v["pairs_per_s"] for v in results.values())
    line = {"metric": "LaVision .im7 camera pairs ingested to float32 device frames per second",
            "value": best, "unit": "pairs/s", "n_gpus": 1, "steps": args.steps, "warmup": 1,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16->f32",
            "data": "synthetic", "config": {"workload": "16 .im7 files of 2 frames 2048x2048 uint16, pack 0 and "
                                                        "pack 2 (zlib rows), from the page cache"},
            "legs": results,
            "e2e": {"value": best, "unit": "pairs/s", "note": "the value is end to end: file bytes to float32 "
                                                              "device frames, wall clock, device synchronised",
                    "h2d_bytes_per_step": 2 * H * W * 2, "d2h_bytes_per_step": 0},
            "gpu_launches": "one unpack launch per camera read (2 frames)"}
    if cpu_legs:
        cb = max(cpu_legs.items(), key=lambda kv: kv[1]["pairs_per_s"])
        line["cpu_baseline"] = {"value": cb[1]["pairs_per_s"], "unit": "pairs/s",
                                "cores": int(cb[0].rsplit("threads", 1)[1]), "kind": "port",
                                "sample": "the oracle's restatement of the reference's read_im7_camera (numpy + "
                                          "zlib, float32 frames in host memory) over the same 16 files per pack",
                                "legs": cpu_legs}
    print(json.dumps(line), flush=True)


def _serve_leg(dev, rate, duration, seed_base=0, packed=False):
    """Serving mix: Poisson arrivals at `rate` pairs/s for `duration` s; each
    request is one uint16 pair of a size drawn from {512^2, 1024^2, 2048^2,
    2048x4096} with a schedule drawn from {32; 64-32; 128-64-32-16 px} at 50%
    overlap, particle images of the single-pair workload's particle and flow model
    (uniform (3.3, -1.7) px plus a Gaussian random field of 0.5 px std and 40 px
    correlation length; a small pool per size, cycled), frames in pinned host
    memory, a 120 GB device budget.  Returns the served statistics: vectors/s
    over the run and request latency (arrival to result in host memory)."""
    import numpy as np
    import torch

    from pivtools_b200 import serving, synthetic

    sizes = [(512, 512), (1024, 1024), (2048, 2048), (2048, 4096)]
    scheds = [(32,), (64, 32), (128, 64, 32, 16)]
    pool = {}
    for si, shp in enumerate(sizes):
        pool[shp] = []
        for k in range(2):
            A, B, _ = synthetic.particle_pair(shp, seed=7000 + 10 * si + k + 1000 * seed_base, flow="uniform_grf",
                                              device=dev)
            pool[shp].append((A.to(torch.int32).to(torch.uint16).cpu().pin_memory(),
                              B.to(torch.int32).to(torch.uint16).cpu().pin_memory()))
    srv = serving.PivServer(device=dev, max_batch=4, hbm_budget_bytes=120e9, packed=packed)
    for shp in sizes:                           # build every engine, warm it, pin output buffers
        for sch in scheds:
            srv.reserve_outputs(shp, sch, 64)
            for _ in range(2):
                srv.submit(*pool[shp][0], sch)
            for r in srv.drain():
                srv.release(r)
    torch.cuda.synchronize()
    arr = serving.poisson_arrivals(rate, duration, seed=11 + seed_base)
    rng = np.random.default_rng(12 + seed_base)
    picks = [(sizes[rng.integers(4)], scheds[rng.integers(3)], int(rng.integers(2))) for _ in arr]
    reqs = []
    vec = 0
    d2h = []
    import gc

    gc.disable()                                # no collector pauses inside the served window
    try:
        t0 = time.perf_counter()
        i = 0
        while i < len(arr) or not srv.idle():
            now = time.perf_counter() - t0
            while i < len(arr) and arr[i] <= now:
                shp, sch, k = picks[i]
                reqs.append(srv.submit(*pool[shp][k], sch, arrival=t0 + arr[i]))
                i += 1
            for r in srv.poll():
                vec += int(r.ux.numel())
                d2h.append(r.ux.numel() * 8)
                srv.release(r)
            time.sleep(5e-5)
        t1 = time.perf_counter()
    finally:
        gc.enable()
    lat = np.array([r.done - r.arrival for r in reqs]) * 1e3
    wall = t1 - t0
    by_sched = {}
    for (shp, sch, _), l in zip(picks, lat):
        by_sched.setdefault("-".join(map(str, sch)), []).append(l)
    out = {"vectors_per_s": vec / wall, "wall_s": wall, "requests": len(reqs), "offered_pairs_per_s": rate,
           "served_pairs_per_s": len(reqs) / wall, "duration_s": duration,
           "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "max": float(lat.max()),
                          "by_schedule": {k: {"p50": float(np.percentile(v, 50)), "p99": float(np.percentile(v, 99)),
                                              "n": len(v)} for k, v in sorted(by_sched.items())}},
           "h2d_bytes_per_request": float(np.mean([2 * p[0][0] * p[0][1] * 2 for p in picks])),
           "d2h_bytes_per_request": float(np.mean(d2h)),
           "max_batch": srv.max_batch, "hbm_budget_gb": 120, "engines": len(srv.engines),
           "engine_bytes_gb": srv.used_bytes / 1e9, "packed": packed,
           "pack_stats": dict(srv.pack_stats) if packed else None,
           "workload": f"Poisson {rate:g} pairs/s for {duration:g} s; sizes 512^2, 1024^2, 2048^2, 2048x4096 "
                       "uint16; schedules 32 / 64-32 / 128-64-32-16 px at 50%; flow (3.3, -1.7) px + GRF 0.5 px"}
    del srv, pool
    torch.cuda.empty_cache()
    return out


def run_serve(args):
    """The serving mix alone (see _serve_leg) as its own JSON line."""
    import torch

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        torch.distributed.barrier()
    with ClockSampler(local) as clk:
        st = _serve_leg(dev, args.rate, args.duration, seed_base=rank, packed=args.packed)
    wall = st["wall_s"]
    vec_total = st["vectors_per_s"] * wall
    if ws > 1:
        t = torch.tensor([wall, vec_total], device=dev, dtype=torch.float64)
        w = t.clone()
        torch.distributed.all_reduce(w, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM)
        wall, vec_total = float(w[0].item()), float(t[1].item())
    if rank == 0:
        line = {
            "metric": "served vectors/s with p50/p99 pair latency on 1 B200", "value": vec_total / wall,
            "unit": "vectors/s", "n_gpus": ws, "steps": st["requests"], "warmup": 24,
            "ms_per_step": wall * 1e3 / max(st["requests"], 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": st["workload"], "max_batch": st["max_batch"], "hbm_budget_gb": 120,
                       "packed": st["packed"], "pack_stats": st["pack_stats"],
                       "engines": st["engines"], "engine_bytes_gb": st["engine_bytes_gb"]},
            "latency_ms": st["latency_ms"], "offered_pairs_per_s": st["offered_pairs_per_s"],
            "served_pairs_per_s": st["served_pairs_per_s"],
            "e2e": {"value": vec_total / wall, "unit": "vectors/s", "h2d_bytes_per_step": st["h2d_bytes_per_request"],
                    "d2h_bytes_per_step": st["d2h_bytes_per_request"]},
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def main():
    global PEAK_FINDER, INTERP
    args = _args()
    PEAK_FINDER = args.peak_finder
    INTERP = 1 if args.interp == "lanczos" else 0
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "ensemble":
        run_ensemble(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.workload == "dft":
        run_dft(args)
    elif args.workload == "ingest":
        run_ingest(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
