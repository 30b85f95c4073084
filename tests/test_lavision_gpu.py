"""LaVision frames on the GPU: read_im7_camera (native codecs -> page-locked
memory -> pivb_unpack_pixels_dev) equals the reference reader's float32 camera
frames bit for bit, on every pack type and on LaVision's own lvpyio fixtures;
every .set decoder and codec through decode_set_entry equals the reference's
decoded pixels with the intensity scale applied in float32."""

import ctypes
import json
import os

import numpy as np
import pytest

from pivtools_b200 import _lib
from pivtools_b200 import lavision as LV

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "lavision_ref.npz")


@pytest.fixture(scope="module")
def gold():
    z = np.load(GOLD)
    return z, json.loads(str(z["meta"]))


def test_read_im7_camera_equals_reference(gold, cuda, tmp_path):
    z, meta = gold
    n_checked = 0
    for case in meta["im7"]:
        name = case["name"]
        p = tmp_path / f"{name}.im7"
        p.write_bytes(z[name + "_file"].tobytes())
        for i, (cam, fpc, nfr) in enumerate(case["cams"]):
            got = LV.read_im7_camera(p, camera_no=cam, frames_per_camera=fpc, frames=nfr, device=cuda)
            ref = z[f"{name}_cam{i}"]
            assert got.dtype.is_floating_point and tuple(got.shape) == ref.shape, (name, i)
            assert np.array_equal(got.cpu().numpy(), ref), (name, i)
            n_checked += 1
    assert n_checked >= 14


def test_read_im7_camera_lvpyio_fixtures(gold, cuda, tmp_path):
    import torch

    z, meta = gold
    for name in meta["lvpyio"]:
        p = tmp_path / f"{name}.im7"
        p.write_bytes(z[f"lv_{name}_file"].tobytes())
        lv = z[f"lv_{name}_lvpyio"]
        lv = lv.reshape((-1,) + lv.shape[-2:])
        _, _, sc = LV.read_im7(p)                       # the file's intensity scale
        out = torch.empty((1,) + lv.shape[1:], dtype=torch.float32, device=cuda)
        for k in range(lv.shape[0]):
            got = LV.read_im7_camera(p, camera_no=k + 1, frames_per_camera=1, out=out, device=cuda)
            assert got.data_ptr() == out.data_ptr()
            exp = lv[k].astype(np.float32)
            if sc.slope != 1.0:
                exp *= sc.slope
            if sc.offset != 0.0:
                exp += sc.offset
            assert np.array_equal(got.cpu().numpy()[0], exp), (name, k)


@pytest.mark.parametrize("codec", ["", "Zlib", "LZ4", "IMX"])
def test_set_entries_every_decoder(gold, cuda, codec):
    z, meta = gold
    for case in meta["set"]:
        dec, W, H = case["decoder"], case["width"], case["height"]
        stored = z[f"set_{dec}_{codec or 'none'}_stored"].tobytes()
        ref = z[f"set_{dec}_pixels"].astype(np.float32)
        got = LV.decode_set_entry(stored, codec, dec, W, H, device=cuda)
        assert np.array_equal(got.cpu().numpy(), ref), (dec, codec)
        slope, offset = 0.37, -12.5
        got = LV.decode_set_entry(stored, codec, dec, W, H, slope=slope, offset=offset, device=cuda)
        exp = ref.copy()
        exp *= slope
        exp += offset
        assert np.array_equal(got.cpu().numpy(), exp), (dec, codec)


def test_unpack_batch_with_strides(cuda):
    """Several mono-12p payloads at a padded stride into padded output frames."""
    import torch

    L = _lib.pass_lib()
    rng = np.random.default_rng(3)
    W, H, n = 24, 10, 3
    pb = int(L.pivb_payload_bytes(W * H, 2))
    assert pb == W * H * 3 // 2
    stride = pb + 17
    raw = rng.integers(0, 256, (n, stride), dtype=np.uint8)
    dev_raw = torch.tensor(raw, device=cuda)
    out = torch.full((n, W * H + 5), -1.0, device=cuda)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.pivb_unpack_pixels_dev(dev_raw.data_ptr(), stride, n, W * H, 2, 0, 1.0, 0, 0.0, out.data_ptr(),
                                    W * H + 5, s) == 0
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    for k in range(n):
        b = raw[k, :pb].astype(np.uint32).reshape(-1, 3)
        p0 = b[:, 0] | ((b[:, 1] & 0xF) << 8)
        p1 = (b[:, 1] >> 4) | (b[:, 2] << 4)
        exp = np.stack([p0, p1], 1).ravel().astype(np.float32)
        assert np.array_equal(o[k, :W * H], exp)
        assert np.all(o[k, W * H:] == -1.0)
    # bad arguments: an odd pixel count for a 2-in-3 packing, a short stride
    assert L.pivb_unpack_pixels_dev(dev_raw.data_ptr(), stride, n, W * H - 1, 2, 0, 1.0, 0, 0.0, out.data_ptr(),
                                    W * H + 5, s) == 1
    assert L.pivb_unpack_pixels_dev(dev_raw.data_ptr(), pb - 1, n, W * H, 2, 0, 1.0, 0, 0.0, out.data_ptr(),
                                    W * H + 5, s) == 1
