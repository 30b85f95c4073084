"""Camera payload decode on the GPU (pivb_decode_frames_dev) against the
reference's own decode (fixture), and the container reader end to end."""

import ctypes
import json
import os

import numpy as np
import pytest

from pivtools_b200 import _lib, ingest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
ROTS = {"none": 0, "cw90": 3, "ccw90": 1, "180": 2}


def test_decode_matches_reference_fixture(cuda):
    import torch

    g = np.load(os.path.join(GOLD, "ingest_ref.npz"))
    W, H, n = int(g["W"]), int(g["H"]), int(g["n"])
    L = _lib.pass_lib()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for fi, fmt in enumerate(("Mono12p", "BayerRG8")):
        raw = torch.tensor(g[f"{fmt}_raw"], device=cuda)
        dark = torch.tensor(g[f"{fmt}_dark"], device=cuda)
        stride = int(g[f"{fmt}_stride"])
        for view, rot in ROTS.items():
            for with_dark in (0, 1):
                ref = g[f"{fmt}_{view}_{with_dark}"]
                out = torch.full(ref.shape, -1.0, device=cuda)
                assert L.pivb_decode_frames_dev(raw.data_ptr(), stride, n, 1, W, H, fi,
                                                dark.data_ptr() if with_dark else None, stride, 2, rot,
                                                out.data_ptr(), ref.shape[1] * ref.shape[2], s) == 0
                torch.cuda.synchronize()
                assert np.array_equal(out.cpu().numpy(), ref), (fmt, view, with_dark)
    # frames 2..4 alone: the dark role follows the 1-based file index
    g2 = g["Mono12p_none_1"]
    raw = torch.tensor(g["Mono12p_raw"][int(g["Mono12p_stride"]):], device=cuda)
    out = torch.empty((n - 1, H, W), device=cuda)
    assert L.pivb_decode_frames_dev(raw.data_ptr(), int(g["Mono12p_stride"]), n - 1, 2, W, H, 0,
                                    torch.tensor(g["Mono12p_dark"], device=cuda).data_ptr(),
                                    int(g["Mono12p_stride"]), 2, 0, out.data_ptr(), H * W, s) == 0
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), g2[1:])
    assert L.pivb_decode_frames_dev(raw.data_ptr(), 10, 1, 1, 3, 3, 0, None, 0, 1, 0, out.data_ptr(), 9, s) == 1


def test_container_reader(cuda, tmp_path):
    g = np.load(os.path.join(GOLD, "ingest_ref.npz"))
    W, H, n = int(g["W"]), int(g["H"]), int(g["n"])
    stride = int(g["BayerRG8_stride"])
    p = tmp_path / "Camera1.pivraw"
    d = tmp_path / "dark.pivraw"
    g["BayerRG8_raw"].tofile(p)
    g["BayerRG8_dark"].tofile(d)
    for q, nf in ((p, n), (d, 2)):
        with open(str(q) + ".json", "w") as f:
            json.dump({"width": W, "height": H, "pixel_format": "BayerRG8", "bytes_per_frame": W * H,
                       "frame_stride": stride, "n_frames": nf}, f)
    dec = ingest.PivrawDecoder(p, dark_path=d, view_rotation="cw90", device=cuda)
    got = dec.read(2, 3).cpu().numpy()
    assert np.array_equal(got, g["BayerRG8_cw90_1"][1:])
