"""The allocation-free correlation entry point (pivb_xcorr_dev_noalloc).

It exists for callers that cannot allocate device memory -- a host whose GPU
memory belongs to another allocator, a stream under CUDA-graph capture, or a
latency-bound pipeline that cannot take the device synchronisation of cudaFree.
Its LM scratch is a fixed 16 MiB device array inside the library.  Through the
C-ABI, on two calls in a row, it must reproduce the scratch-taking entry point
(pivb_xcorr_dev) exactly, and it must refuse a call that needs more scratch than
the array holds.  Collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.
"""

import ctypes

import numpy as np
import pytest

from pivtools_b200 import _lib, geometry, synthetic

pytestmark = pytest.mark.gpu

KEYS = ("pk_x", "pk_y", "pk_h", "sx", "sy", "sxy", "ratio")


def _setup(torch, dev, seed, n, finder):
    A, B, _ = synthetic.particle_pair((192, 224), seed=seed)
    g = geometry.compute_window_centers(A.shape, (n, n), 50)
    w = torch.tensor(geometry.window_weight((n, n), "gaussian"), device=dev)
    L = _lib.bulkxcorr2d_lib()
    cw = torch.empty_like(w)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.pivb_correl_weight_dev(w.data_ptr(), n, n, cw.data_ptr(), s) == 0
    return dict(A=torch.tensor(A[None], device=dev), B=torch.tensor(B[None], device=dev), g=g, w=w, cw=cw, n=n,
                finder=finder, cx=torch.tensor(g.win_ctrs_x, device=dev), cy=torch.tensor(g.win_ctrs_y, device=dev))


def _outputs(torch, dev, case):
    g = case["g"]
    shape = (1, 1, g.n_win_y, g.n_win_x)
    return {k: torch.full(shape, -7.0, device=dev) for k in KEYS}


def _args(case, out):
    g = case["g"]
    A, B = case["A"], case["B"]
    return [A.data_ptr(), B.data_ptr(), A.stride(0), None, A.shape[1], A.shape[2], 1, case["cx"].data_ptr(),
            case["cy"].data_ptr(), g.n_win_y, g.n_win_x, case["w"].data_ptr(), case["w"].data_ptr(),
            case["cw"].data_ptr(), case["n"], case["n"], 0, 1, case["finder"], 0] + \
        [out[k].data_ptr() for k in KEYS] + [None]


def test_no_alloc_matches_scratch_entry_point(cuda):
    import torch

    L = _lib.bulkxcorr2d_lib()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for seed, n, finder in ((11, 32, 6), (12, 16, 4)):    # two calls in a row, different data
        case = _setup(torch, cuda, seed, n, finder)
        ref = _outputs(torch, cuda, case)
        got = _outputs(torch, cuda, case)
        total = case["g"].n_win_y * case["g"].n_win_x
        nbytes = int(L.pivb_xcorr_scratch_bytes(total, 1, finder))
        scratch = torch.empty(nbytes, dtype=torch.uint8, device=cuda)
        assert L.pivb_xcorr_dev(*_args(case, ref), scratch.data_ptr(), nbytes, s) == 0
        assert L.pivb_xcorr_dev_noalloc(*_args(case, got), s) == 0
        torch.cuda.synchronize()
        for k in KEYS:
            a, b = got[k].cpu().numpy(), ref[k].cpu().numpy()
            assert np.array_equal(a, b, equal_nan=True), k
        assert np.isfinite(got["pk_x"].cpu().numpy()).mean() > 0.5


def test_no_alloc_refuses_oversized_call(cuda):
    import torch

    L = _lib.bulkxcorr2d_lib()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    case = _setup(torch, cuda, 13, 32, 5)
    out = _outputs(torch, cuda, case)
    args = _args(case, out)
    # claim 200000 image pairs of this grid: far beyond the 131072-window array
    # (refused on the host before any launch; the frames are never read)
    args[6] = 200000 // (case["g"].n_win_y * case["g"].n_win_x) + 1
    assert L.pivb_xcorr_dev_noalloc(*args, s) == 1
