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


def _skipped_grid_args(torch, dev, n_win_y, n_win_x, out):
    """A call whose every window lies outside a 64 x 64 frame: the correlation
    kernel writes only each window's record flag, so a full-size call stays cheap."""
    A = torch.zeros((1, 64, 64), device=dev)
    w = torch.ones((32, 32), device=dev)
    cx = torch.full((n_win_x,), -1000.0, device=dev)
    cy = torch.full((n_win_y,), -1000.0, device=dev)
    keep = (A, w, cx, cy)
    args = [A.data_ptr(), A.data_ptr(), A.stride(0), None, 64, 64, 1, cx.data_ptr(), cy.data_ptr(), n_win_y,
            n_win_x, w.data_ptr(), w.data_ptr(), w.data_ptr(), 32, 32, 0, 1, 4, 0] + \
        [out[k].data_ptr() for k in KEYS] + [None]
    return args, keep


def test_no_alloc_limit_is_exactly_131072_windows(cuda):
    """131072 LM windows (256 x 512, one pair) fill the array exactly and are
    accepted; one more window row-pair (131073 windows as 1 x 131073) is refused."""
    import torch

    L = _lib.bulkxcorr2d_lib()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = {k: torch.full((256 * 512,), -7.0, device=cuda) for k in KEYS}
    args, keep = _skipped_grid_args(torch, cuda, 256, 512, out)
    assert L.pivb_xcorr_dev_noalloc(*args, s) == 0
    torch.cuda.synchronize()
    for k in KEYS:
        assert bool((out[k] == -7.0).all()), k          # every window skipped, outputs untouched
    big = {k: torch.full((131073,), -7.0, device=cuda) for k in KEYS}
    args, keep = _skipped_grid_args(torch, cuda, 1, 131073, big)
    assert L.pivb_xcorr_dev_noalloc(*args, s) == 1      # refused on the host, nothing launched
    torch.cuda.synchronize()
    assert bool((big["pk_x"] == -7.0).all())


@pytest.mark.parametrize("finder,n_peaks", [(3, 1), (3, 3), (6, 2)])
def test_no_alloc_without_lm_records_matches(cuda, finder, n_peaks):
    """Calls that need no LM records (3-point fits, several peaks) equal the
    scratch-taking entry point too."""
    import torch

    L = _lib.bulkxcorr2d_lib()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    case = _setup(torch, cuda, 21 + finder + n_peaks, 32, finder)
    g = case["g"]
    shape = (1, n_peaks, g.n_win_y, g.n_win_x)
    ref = {k: torch.full(shape if k != "ratio" else (1, g.n_win_y, g.n_win_x), -7.0, device=cuda) for k in KEYS}
    got = {k: torch.full_like(v, -7.0) for k, v in ref.items()}
    ra, ga = _args(case, ref), _args(case, got)
    ra[17] = ga[17] = n_peaks
    total = g.n_win_y * g.n_win_x
    nbytes = max(int(L.pivb_xcorr_scratch_bytes(total, n_peaks, finder)), int(L.pivb_xcorr_record_bytes(total)))
    scratch = torch.empty(nbytes, dtype=torch.uint8, device=cuda)
    assert L.pivb_xcorr_dev(*ra, scratch.data_ptr(), nbytes, s) == 0
    assert L.pivb_xcorr_dev_noalloc(*ga, s) == 0
    torch.cuda.synchronize()
    for k in KEYS:
        assert np.array_equal(got[k].cpu().numpy(), ref[k].cpu().numpy(), equal_nan=True), k
