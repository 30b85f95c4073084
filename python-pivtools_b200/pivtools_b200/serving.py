"""Request loop for instantaneous PIV with continuous batching on one GPU.

Requests (one image pair as pinned uint16 host frames plus a pass schedule)
arrive at any time.  Each (frame shape, schedule) class owns an engine: a
resident MultipassPIV with room for `max_batch` pairs, uint16 staging buffers and
its own CUDA stream, so batches of different classes run concurrently on the
device.  `poll()` is one scheduling round:

  retire   batches whose completion event has fired hand their fields (already
           copied to each request's pinned output) back and free the engine;
  admit    every idle engine with waiting requests takes up to `max_batch` of
           them (oldest first) -- requests that arrived while other work was on
           the GPU join the next free engine of their class -- and enqueues
           H2D of the frames, uint16 -> float32, the passes and the D2H of the
           final field on its stream, then records a completion event.

Engines are created on first use while the estimated device memory stays within
the budget; a request whose engine does not fit waits until one can be made.
Every pair's result is independent of what it is batched with (the kernels work
per pair and per window), so a request's field is the same alone and in a mix.

Packed mode (`packed=True`) runs the waiting requests of every idle class
together as one round on one stream (up to two rounds in flight on two
streams): a round advances all its engines pass by pass, and each pass's
correlations of one window size -- requests of different frame sizes and
schedules -- go into one packed launch (pivb_xcorr_jobs_dev: a work list of
per-request jobs in one grid, plus one launch of the fit kernel), so a round
issues one correlation launch per window size and pass instead of one per
engine.  Requests arriving during a round join a later one.
"""

from __future__ import annotations

import ctypes
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import _lib, multipass


@dataclass
class Request:
    A: object                    # pinned uint16 (H, W) host tensor
    B: object
    schedule: tuple              # window sizes of the passes, e.g. (64, 32)
    arrival: float = 0.0         # host clock (time.perf_counter) at submission
    done: float = 0.0            # host clock when the result was seen complete
    ux: object = None            # pinned float32 (ny, nx) host tensors
    uy: object = None
    finished: bool = False
    rid: int = 0


@dataclass
class _Engine:
    key: tuple
    mp: object
    stream: object
    u16: list
    f32: list
    n_bytes: int
    busy: list = field(default_factory=list)   # requests of the batch in flight
    event: object = None


def schedule_config(schedule, overlap=50):
    ws = [(int(w), int(w)) for w in schedule]
    return multipass.MultipassConfig(window_sizes=ws, overlaps=[overlap] * len(ws))


class PivServer:
    def __init__(self, device=None, max_batch=4, hbm_budget_bytes=120e9, overlap=50, packed=False):
        import torch

        self.torch = torch
        self.packed = packed
        self.device = torch.device("cuda" if device is None else device)
        self.max_batch = max_batch
        self.budget = float(hbm_budget_bytes)
        self.overlap = overlap
        self.engines: dict = {}
        self.used_bytes = 0
        self.waiting: dict = {}
        self.n_submitted = 0
        self.Lp = _lib.pass_lib()
        self.Lx = _lib.bulkxcorr2d_lib()
        self._free: dict = {}          # (ny, nx) -> reusable pinned output pairs
        # packed mode: up to `packed_rounds` rounds in flight, each on its own
        # stream with its own fit records; an engine belongs to one round at a time
        self.packed_rounds = 2
        self._pack_streams = [torch.cuda.Stream(device=self.device) for _ in range(self.packed_rounds)] if packed else []
        self._rounds = []              # in flight: (requests, event, engines, stream index)
        self._records = [None] * self.packed_rounds
        self.pack_stats = {"rounds": 0, "packed_launches": 0, "jobs": 0, "single_launches": 0}

    # ------------------------------------------------------------------ #
    @staticmethod
    def _engine_bytes(shape, schedule, max_batch):
        H, W = shape
        frame = H * W
        # float32 frames A, B + warped A, B + uint16 staging A, B, plus the
        # per-pass grids, outputs and work buffers (small; 10% margin)
        return int(max_batch * frame * (4 * 4 + 2 * 2) * 1.1) + (64 << 20)

    def _engine(self, shape, schedule):
        key = (tuple(shape), tuple(schedule))
        e = self.engines.get(key)
        if e is not None:
            return e
        nb = self._engine_bytes(shape, schedule, self.max_batch)
        if self.used_bytes + nb > self.budget:
            return None
        torch = self.torch
        dev = self.device
        mp = multipass.MultipassPIV(shape, self.max_batch, schedule_config(schedule, self.overlap), device=dev)
        H, W = shape
        u16 = [torch.empty((self.max_batch, H, W), dtype=torch.uint16, device=dev) for _ in range(2)]
        f32 = [torch.empty((self.max_batch, H, W), dtype=torch.float32, device=dev) for _ in range(2)]
        e = _Engine(key=key, mp=mp, stream=torch.cuda.Stream(device=dev), u16=u16, f32=f32, n_bytes=nb)
        self.engines[key] = e
        self.used_bytes += nb
        return e

    def output_shape(self, shape, schedule):
        key = (tuple(shape), int(schedule[-1]))
        cache = self.__dict__.setdefault("_oshape", {})
        if key not in cache:
            from . import geometry

            g = geometry.compute_window_centers(shape, (schedule[-1], schedule[-1]), self.overlap)
            cache[key] = (g.n_win_y, g.n_win_x)
        return cache[key]

    def _outputs(self, ny, nx):
        free = self._free.setdefault((ny, nx), [])
        if free:
            return free.pop()
        torch = self.torch
        return (torch.empty((ny, nx), dtype=torch.float32).pin_memory(),
                torch.empty((ny, nx), dtype=torch.float32).pin_memory())

    def reserve_outputs(self, shape, schedule, count):
        """Pin `count` output pairs for this shape and schedule ahead of time
        (pinned allocations are slow and must stay out of the request path)."""
        ny, nx = self.output_shape(shape, schedule)
        free = self._free.setdefault((ny, nx), [])
        while len(free) < count:
            torch = self.torch
            free.append((torch.empty((ny, nx), dtype=torch.float32).pin_memory(),
                         torch.empty((ny, nx), dtype=torch.float32).pin_memory()))

    def release(self, r):
        """Hand a finished request's output buffers back for reuse."""
        if r.finished and r.ux is not None:
            self._free.setdefault(tuple(r.ux.shape), []).append((r.ux, r.uy))
            r.ux = r.uy = None

    def submit(self, A, B, schedule, arrival=None):
        """Queue one pair (pinned uint16 host tensors of one shape)."""
        shape = tuple(A.shape)
        ny, nx = self.output_shape(shape, schedule)
        ux, uy = self._outputs(ny, nx)
        r = Request(A=A, B=B, schedule=tuple(schedule), arrival=time.perf_counter() if arrival is None else arrival,
                    ux=ux, uy=uy, rid=self.n_submitted)
        self.n_submitted += 1
        self.waiting.setdefault((shape, tuple(schedule)), deque()).append(r)
        return r

    def _launch(self, e, batch):
        torch = self.torch
        k = len(batch)
        with torch.cuda.stream(e.stream):
            for i, r in enumerate(batch):
                e.u16[0][i].copy_(r.A, non_blocking=True)
                e.u16[1][i].copy_(r.B, non_blocking=True)
            st = ctypes.c_void_p(e.stream.cuda_stream)
            n = k * e.u16[0].shape[1] * e.u16[0].shape[2]
            for j in range(2):
                if self.Lp.pivb_u16_to_f32_dev(e.u16[j].data_ptr(), e.f32[j].data_ptr(), n, st) != 0:
                    raise RuntimeError("u16 -> f32 conversion failed")
            ux, uy = e.mp.run(e.f32[0], e.f32[1], n=k)
            for i, r in enumerate(batch):
                r.ux.copy_(ux[i], non_blocking=True)
                r.uy.copy_(uy[i], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(e.stream)
        e.busy = batch
        e.event = ev

    def _records_buffer(self, si, nbytes):
        torch = self.torch
        if self._records[si] is None or self._records[si].numel() < nbytes:
            self._records[si] = torch.empty(max(int(nbytes), 1 << 20), dtype=torch.uint8, device=self.device)
        return self._records[si]

    def _launch_packed(self, work, si):
        """One packed round on stream `si`: `work` is a list of (engine, batch)."""
        torch = self.torch
        stream = self._pack_streams[si]
        st = ctypes.c_void_p(stream.cuda_stream)
        jmax = int(self.Lx.pivb_xcorr_jobs_max())
        with torch.cuda.stream(stream):
            for e, batch in work:
                for i, r in enumerate(batch):
                    e.u16[0][i].copy_(r.A, non_blocking=True)
                    e.u16[1][i].copy_(r.B, non_blocking=True)
                n = len(batch) * e.u16[0].shape[1] * e.u16[0].shape[2]
                for j in range(2):
                    if self.Lp.pivb_u16_to_f32_dev(e.u16[j].data_ptr(), e.f32[j].data_ptr(), n, st) != 0:
                        raise RuntimeError("u16 -> f32 conversion failed")
            n_pass = max(len(e.mp.passes) for e, _ in work)
            for k in range(n_pass):
                act = [(e, b) for e, b in work if k < len(e.mp.passes)]
                frames = [e.mp.stage_pre(k, e.f32[0], e.f32[1], len(b)) for e, b in act]
                groups: dict = {}
                for (e, b), fr in zip(act, frames):
                    if e.mp.packable(k):
                        key = (e.mp.passes[k]["win_h"], e.mp.cfg.peak_finder, e.mp.cfg.peakfit_impl)
                        groups.setdefault(key, []).append(e.mp.job(k, fr[0], fr[1], len(b)))
                    else:
                        e.mp._correlate(k, fr[0], fr[1], len(b))
                        self.pack_stats["single_launches"] += 1
                for (win, finder, impl), jobs in groups.items():
                    for c0 in range(0, len(jobs), jmax):
                        chunk = jobs[c0:c0 + jmax]
                        arr = (_lib.XcorrJob * len(chunk))(*chunk)
                        nb = int(self.Lx.pivb_xcorr_jobs_record_bytes(arr, len(chunk), win))
                        rec = self._records_buffer(si, nb)
                        code = self.Lx.pivb_xcorr_jobs_dev(arr, len(chunk), win, finder, impl, rec.data_ptr(),
                                                           rec.numel(), st)
                        if code != 0:
                            raise RuntimeError(f"packed correlation failed with code {code}")
                        self.pack_stats["packed_launches"] += 1
                        self.pack_stats["jobs"] += len(chunk)
                for e, b in act:
                    e.mp.stage_post(k, len(b))
            for e, batch in work:
                last = e.mp.passes[-1]
                for i, r in enumerate(batch):
                    r.ux.copy_(last["ux"][i], non_blocking=True)
                    r.uy.copy_(last["uy"][i], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
        self.pack_stats["rounds"] += 1
        for e, b in work:
            e.busy = b
        self._rounds.append(([r for _, b in work for r in b], ev, [e for e, _ in work], si))

    def _poll_packed(self):
        finished = []
        now = None
        for rd in list(self._rounds):
            reqs, ev, engines, _ = rd
            if ev.query():
                now = time.perf_counter() if now is None else now
                for r in reqs:
                    r.done = now
                    r.finished = True
                finished.extend(reqs)
                for e in engines:
                    e.busy = []
                self._rounds = [x for x in self._rounds if x is not rd]
        if len(self._rounds) < self.packed_rounds:
            work = []
            for key, q in self.waiting.items():
                if not q:
                    continue
                e = self._engine(*key)
                if e is None or e.busy:
                    continue
                work.append((e, [q.popleft() for _ in range(min(self.max_batch, len(q)))]))
            if work:
                used = {rd[3] for rd in self._rounds}
                si = next(i for i in range(self.packed_rounds) if i not in used)
                self._launch_packed(work, si)
        return finished

    def poll(self):
        """One scheduling round; returns the requests finished in it."""
        if self.packed:
            return self._poll_packed()
        finished = []
        now = None
        for e in self.engines.values():
            if e.busy and e.event.query():
                now = time.perf_counter() if now is None else now
                for r in e.busy:
                    r.done = now
                    r.finished = True
                finished.extend(e.busy)
                e.busy = []
                e.event = None
        for key, q in self.waiting.items():
            if not q:
                continue
            e = self._engine(*key)
            if e is None or e.busy:
                continue
            batch = [q.popleft() for _ in range(min(self.max_batch, len(q)))]
            self._launch(e, batch)
        return finished

    def idle(self):
        return (not self._rounds and all(not e.busy for e in self.engines.values())
                and all(not q for q in self.waiting.values()))

    def drain(self, timeout_s=120.0):
        t0 = time.perf_counter()
        out = []
        while not self.idle():
            out.extend(self.poll())
            if time.perf_counter() - t0 > timeout_s:
                raise TimeoutError("requests still in flight")
            time.sleep(1e-4)
        return out


def poisson_arrivals(rate, duration, seed):
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return np.array(out)
        out.append(t)
