"""Camera frames straight to the GPU.

PIVTOOLs Acquisition run containers (``.pivraw``: frames back to back at a fixed
stride, a JSON sidecar with the geometry) are read as raw bytes into page-locked
host memory, copied to the device and decoded there (`pivb_decode_frames_dev`:
Mono12p unpack or BayerRG8 superpixel sum, in-run dark, view rotation) into the
float32 frames the correlation consumes.  The container's validation and the
run alignment across cameras stay with the reference's reader
(pivtools_core/image_handling/readers/pivraw_reader.py); this module moves the
pixels.
"""

from __future__ import annotations

import ctypes
import json
import os

import numpy as np

from . import _lib

FORMATS = {"Mono12p": 0, "BayerRG8": 1}
ROTATIONS = {"none": 0, "ccw90": 1, "180": 2, "cw90": 3}   # np.rot90 turns


def read_sidecar(path):
    with open(str(path) + ".json") as f:
        return json.load(f)


class PivrawDecoder:
    """Decode frames of one camera container on one GPU."""

    def __init__(self, path, dark_path=None, view_rotation="none", device=None):
        import torch

        self.torch = torch
        self.device = torch.device("cuda" if device is None else device)
        self.path = str(path)
        h = read_sidecar(path)
        self.width, self.height = int(h["width"]), int(h["height"])
        self.fmt = FORMATS[h["pixel_format"]]
        self.bytes_per_frame, self.stride = int(h["bytes_per_frame"]), int(h["frame_stride"])
        self.n_frames = int(h["n_frames"])
        self.rot = ROTATIONS[view_rotation]
        dh, dw = (self.height // 2, self.width // 2) if self.fmt == 1 else (self.height, self.width)
        self.shape = (dw, dh) if self.rot % 2 else (dh, dw)
        self.dark = None
        self.dark_frames = 1
        if dark_path is not None:
            dh_ = read_sidecar(dark_path)
            self.dark_frames = int(dh_["n_frames"])
            raw = np.fromfile(str(dark_path), dtype=np.uint8, count=self.dark_frames * self.stride)
            self.dark = torch.tensor(raw, device=self.device)
        self.Lp = _lib.pass_lib()

    def read(self, first_index, count, out=None):
        """Frames first_index .. first_index + count - 1 (1-based) as a (count, H, W)
        float32 device tensor."""
        torch = self.torch
        if first_index < 1 or first_index + count - 1 > self.n_frames:
            raise ValueError(f"frames {first_index}..{first_index + count - 1} outside 1..{self.n_frames}")
        nbytes = count * self.stride
        host = torch.from_numpy(np.fromfile(self.path, dtype=np.uint8, count=nbytes,
                                            offset=(first_index - 1) * self.stride)).pin_memory()
        dev = host.to(self.device, non_blocking=True)
        if out is None:
            out = torch.empty((count,) + self.shape, dtype=torch.float32, device=self.device)
        s = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        rc = self.Lp.pivb_decode_frames_dev(dev.data_ptr(), self.stride, count, first_index, self.width,
                                            self.height, self.fmt, None if self.dark is None else self.dark.data_ptr(),
                                            self.stride, self.dark_frames, self.rot, out.data_ptr(),
                                            self.shape[0] * self.shape[1], s)
        if rc != 0:
            raise RuntimeError("frame decode failed")
        return out
