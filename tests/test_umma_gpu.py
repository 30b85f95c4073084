"""The tensor-core (tcgen05) layer of libpivb_dft: operand layout, descriptors,
accumulation over K-steps and tensor-memory read-back, checked on products with
a known answer (BF16 products are exact in FP32; only the FP32 sums round)."""

import numpy as np
import pytest

from pivtools_b200 import _lib

pytestmark = pytest.mark.gpu


def _bf16(rng, shape):
    """Random float32 values exactly representable in bfloat16, and their bits."""
    x = rng.standard_normal(shape).astype(np.float32)
    bits = (x.view(np.uint32) >> 16).astype(np.uint16)
    return (bits.astype(np.uint32) << 16).view(np.float32), bits


@pytest.mark.parametrize("a_mn", [0, 1])
@pytest.mark.parametrize("N,K", [(16, 16), (32, 32), (64, 32), (64, 64), (128, 48)])
def test_umma_product(cuda, N, K, a_mn):
    import ctypes

    import torch

    L = _lib.dft_lib()
    rng = np.random.default_rng(N * 100 + K + 7 * a_mn)
    a, abits = _bf16(rng, (128, K))
    b, bbits = _bf16(rng, (N, K))
    dA = torch.tensor(abits.view(np.int16), device=cuda)
    dB = torch.tensor(bbits.view(np.int16), device=cuda)
    dD = torch.full((128, N), float("nan"), device=cuda)
    st = torch.zeros(1, dtype=torch.int32, device=cuda)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.pivb_umma_selftest(dA.data_ptr(), dB.data_ptr(), dD.data_ptr(), N, K, a_mn, st.data_ptr(), s) == 0
    torch.cuda.synchronize()
    assert st.item() == 0
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    bound = np.abs(a).astype(np.float64) @ np.abs(b).astype(np.float64).T
    got = dD.cpu().numpy()
    assert np.all(np.abs(got - ref) <= 1e-6 * bound + 1e-30), float(np.max(np.abs(got - ref) / bound))


def test_umma_rejects_bad_shapes(cuda):
    L = _lib.dft_lib()
    assert L.pivb_umma_selftest(1, 1, 1, 24, 32, 0, 1, None) == 1
    assert L.pivb_umma_selftest(1, 1, 1, 32, 8, 0, 1, None) == 1


def test_bounded_wait_times_out_and_context_survives(cuda):
    """A wait that nothing completes ends after its poll limit, reports through
    the status word, frees its tensor memory, and the context stays usable."""
    import ctypes

    import torch

    L = _lib.dft_lib()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = torch.zeros(1, dtype=torch.int32, device=cuda)
    assert L.pivb_wait_timeout_selftest(st.data_ptr(), 2048, s) == 0
    torch.cuda.synchronize()
    assert st.item() == 4                       # every warp saw its wait run out
    test_umma_product(cuda, 32, 32, 0)          # tensor memory was released
    assert L.pivb_wait_timeout_selftest(None, 10, s) == 1
