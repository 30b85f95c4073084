"""LaVision DaVis frames straight to the GPU: .im7 files and .set entries.

The containers' byte-serial codecs (the DaVis token stream of .im7 pack 1 and
IMX .set entries, LZ4 blocks of .im7 pack 20 and LZ4 .set entries, zlib blocks of
.im7 pack 2 and Zlib .set entries) are decoded by the host library
libpivb_lavision.so straight into page-locked memory; the payloads are copied to
the device and unpacked there (`pivb_unpack_pixels_dev`: the packed 10/12-bit
.set encodings, 8/16-bit words, .im7 FLOAT buffers) into float32 frames with the
intensity scale applied, as the correlation consumes them.  The container
walking (headers, frame tables, attribute records, the version-1 mask trailer)
mirrors pivtools_core/image_handling/readers/im7_reader.py and the entry decode
of set_reader.py:1482-1669; the .set directory, manifest and camera logic stay
with the reference's reader, which hands this module an entry's stored bytes.

No CPU fallback: the pixel unpack needs libpivb_pass on a GPU.
"""

from __future__ import annotations

import ctypes
import os
import struct
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
from pathlib import Path
from typing import Optional, Union

import numpy as np

from . import _lib

# Image_Header_7 (im7_reader.py:33-118)
BUFFER_FORMAT_FLOAT = -3
BUFFER_FORMAT_WORD = -4
PACK_UNCOMPRESSED, PACK_RLE, PACK_ZLIB, PACK_FIXED_12BIT, PACK_LZ4 = 0, 1, 2, 3, 20
IM7_VERSION_BUFFER, IM7_VERSION_PER_FRAME = 0, 1
IM7_CAMERA_PLANES = 1
IM7_FOOTER_SIZE = 256
FOOTER_ATTRIBUTES, FOOTER_FRAME_TABLE, FOOTER_MASK_TABLE = 0, 1, 7
DAVIS_MASK_VALID = 1
IEH_END, IEH_SCALE_I, IEH_TYPE_MAX = 0, 4, 13
HEADER_SIZE = 256
HEADER_FORMAT = "<hhhh iiii hhh"
PACK1_PREAMBLE_BYTES = 3
_INT64 = struct.Struct("<q")
_MASK_BLOCK_HEAD = struct.Struct("<iq")
_FOOTER_SLOTS = struct.Struct("<8q")

# pixel encodings of pivb_unpack_pixels_dev; the .set decoder ids of
# set_reader.py:1171-1180 (rgb-24 is refused there too)
ENC_WORD, ENC_RAW8, ENC_FLOAT = 0, 1, 7
SET_DECODERS = {"raw-16-bit": 0, "raw-8-bit": 1, "mono-12p": 2, "mono-12pmsb": 3, "mono-12packed": 4,
                "mono-10p": 5, "mono-10pmsb": 6}
_SET_BITS = {"mono-10p": 10, "mono-10pmsb": 10, "mono-12p": 12, "mono-12packed": 12, "mono-12pmsb": 12,
             "raw-16-bit": 16, "raw-8-bit": 8, "rgb-24": 24}
SET_CODECS = ("", "Uncompressed", "Zlib", "LZ4", "IMX")


class TokenStreamError(IOError):
    """A DaVis token stream that does not decode (davis_tokens.py:130-147)."""


class TruncatedTokenStreamError(TokenStreamError):
    pass


class TokenRunOverrunError(TokenStreamError):
    pass


class TokenValueRangeError(TokenStreamError):
    pass


class TrailingTokenBytesError(TokenStreamError):
    pass


_TOKEN_ERRORS = {
    1: (TruncatedTokenStreamError, "the token stream ended inside a token (truncated file or unknown token)"),
    2: (TokenRunOverrunError, "a 0x7f run of absolutes runs past the values requested"),
    3: (TokenValueRangeError, "the running value left the uint16 range 0..65535"),
}


@dataclass
class IM7Header:
    version: int
    pack_type: int
    buffer_format: int
    is_sparse: int
    size_x: int
    size_y: int
    size_z: int
    size_f: int
    scalar_n: int
    vector_grid: int
    extra_flags: int


@dataclass
class IM7Scales:
    """Intensity scale: physical value = raw * slope + offset."""
    slope: float = 1.0
    offset: float = 0.0
    description: str = ""
    unit: str = ""


# ---------------------------------------------------------------------------
# codecs (libpivb_lavision)
# ---------------------------------------------------------------------------

def _ptr(buf) -> int:
    """Address of a contiguous numpy array or torch tensor."""
    if isinstance(buf, np.ndarray):
        return buf.ctypes.data
    return buf.data_ptr()


def decode_tokens(data: np.ndarray, off: int, out, npix: int, prev: int, where: str):
    """Decode npix token-coded values from data[off:] into out (uint16, numpy or a
    pinned tensor view); returns (off, prev) after the last value.  Raises the
    named TokenStreamError of davis_tokens.py on a stream that does not decode."""
    L = _lib.lavision_lib()
    o, p, w = ctypes.c_longlong(off), ctypes.c_longlong(prev), ctypes.c_longlong(0)
    st = L.pivb_davis_tokens_decode(data.ctypes.data, data.size, ctypes.byref(o), ctypes.byref(p), _ptr(out), npix,
                                    ctypes.byref(w))
    if st < 0:
        raise ValueError(f"{where}: bad token-decoder arguments")
    if st:
        cls, text = _TOKEN_ERRORS[st]
        raise cls(f"{where}: {text} (byte {o.value}, value {w.value} of {npix})")
    return o.value, p.value


def lz4_block_decompress_into(src, dst, expected: int) -> None:
    """Decode one raw LZ4 block (bytes or uint8 array) into dst (expected bytes)."""
    L = _lib.lavision_lib()
    a = np.frombuffer(src, np.uint8) if isinstance(src, (bytes, bytearray, memoryview)) else src
    rc = L.pivb_lz4_block_decode(a.ctypes.data if a.size else 1, a.size, _ptr(dst), expected)
    if rc == 1:
        raise IOError("corrupt LZ4 block")
    if rc == 2:
        raise IOError(f"LZ4 pixel buffer decompressed to fewer than the expected {expected} bytes")
    if rc:
        raise ValueError("bad LZ4 decoder arguments")


def lz4_block_decompress(src, expected: int) -> bytes:
    out = np.empty(expected, np.uint8)
    lz4_block_decompress_into(src, out, expected)
    return out.tobytes()


_ZLIB_ERRORS = {
    1: "the zlib stream does not decompress",
    2: "the zlib stream decompresses to more than the {n} bytes needed",
    3: "the zlib stream ends before its end marker: truncated",
    4: "the zlib stream decompresses to fewer than the {n} bytes needed",
    5: "bytes follow the end of the zlib stream",
}


def zlib_inflate_into(src, dst, expected: int, where: str) -> None:
    L = _lib.lavision_lib()
    a = np.frombuffer(src, np.uint8) if isinstance(src, (bytes, bytearray, memoryview)) else src
    rc = L.pivb_zlib_inflate_exact(a.ctypes.data if a.size else 1, a.size, _ptr(dst), expected)
    if rc:
        raise IOError(f"{where}: " + _ZLIB_ERRORS.get(rc, "bad zlib arguments").format(n=expected))


def _zlib_prefix(src: bytes, cap: int) -> int:
    L = _lib.lavision_lib()
    a = np.frombuffer(src, np.uint8)
    out = np.empty(max(cap, 1), np.uint8)
    got = L.pivb_zlib_inflate_prefix(a.ctypes.data if a.size else 1, a.size, out.ctypes.data, cap)
    if got < 0:
        raise IOError("the first zlib block does not decompress")
    return int(got)


# ---------------------------------------------------------------------------
# .im7 container (im7_reader.py:149-1153)
# ---------------------------------------------------------------------------

def parse_header(raw: bytes, source: str) -> IM7Header:
    """Unpack and check the 256-byte Image_Header_7 (im7_reader.py:149-213)."""
    if len(raw) != HEADER_SIZE:
        raise ValueError(f"Header must be {HEADER_SIZE} bytes, got {len(raw)}")
    v = struct.unpack_from(HEADER_FORMAT, raw, 0)
    dims = dict(zip(("size_x", "size_y", "size_z", "size_f"), v[4:8]))
    bad = {k: x for k, x in dims.items() if x < 1}
    if bad:
        raise ValueError("Damaged .im7 header: every dimension must be at least 1, got "
                         + ", ".join(f"{k}={x}" for k, x in bad.items()))
    if v[0] not in (IM7_VERSION_BUFFER, IM7_VERSION_PER_FRAME):
        raise ValueError(f"{source}: .im7 header version {v[0]} is not read. Known versions are "
                         f"{IM7_VERSION_BUFFER} (every pack type) and {IM7_VERSION_PER_FRAME} (pack_type "
                         f"{PACK_LZ4}, one LZ4 block per frame).")
    if v[0] == IM7_VERSION_PER_FRAME and v[1] != PACK_LZ4:
        raise ValueError(f"{source}: .im7 header version {v[0]} with pack_type {v[1]} is not read: version "
                         f"{v[0]} has only been seen with pack_type {PACK_LZ4}.")
    return IM7Header(*v)


def _itemsize(h: IM7Header) -> int:
    if h.buffer_format == BUFFER_FORMAT_FLOAT:
        return 4
    if h.buffer_format == BUFFER_FORMAT_WORD:
        return 2
    raise ValueError(f"Unsupported buffer_format: {h.buffer_format}. Expected {BUFFER_FORMAT_FLOAT} (FLOAT) or "
                     f"{BUFFER_FORMAT_WORD} (WORD/uint16).")


def _frame_bytes(h: IM7Header) -> int:
    return h.size_x * h.size_y * h.size_z * _itemsize(h)


def _unsupported_pack(h: IM7Header, source: str) -> ValueError:
    if h.pack_type == PACK_FIXED_12BIT:
        return ValueError(f"{source}: pack_type 3 (fixed 12-bit packed) is not read: no real DaVis file of this "
                          f"type has been found to check a decoder against.")
    return ValueError(f"{source}: unsupported pack_type {h.pack_type}. Expected 0 (uncompressed), 1 (token "
                      f"stream), 2 (zlib) or 20 (LZ4).")


def _pool() -> ThreadPoolExecutor:
    global _POOL
    if _POOL is None:
        _POOL = ThreadPoolExecutor(max_workers=max(1, min(16, os.cpu_count() or 1)))
    return _POOL


_POOL: Optional[ThreadPoolExecutor] = None


def _read_uncompressed(f, h, start, end, dst):
    fb = _frame_bytes(h)
    f.seek(HEADER_SIZE + start * fb)
    for k in range(end - start):
        if f.readinto(memoryview(dst[k])) != fb:
            raise IOError("Unexpected EOF reading frame data")
    f.seek(HEADER_SIZE + h.size_f * fb)


def _read_pack1(f, h, source, start, end, dst):
    if h.buffer_format != BUFFER_FORMAT_WORD:
        raise ValueError(f"{source}: pack_type 1 with buffer_format {h.buffer_format} is not read: the token "
                         f"stream codes 16-bit values.")
    npix = h.size_x * h.size_y * h.size_z
    base = f.tell()
    remaining = os.fstat(f.fileno()).st_size - base
    data = np.empty(remaining, np.uint8)
    if f.readinto(memoryview(data)) != remaining:
        raise IOError(f"{source}: short read after the header")
    off, prev = PACK1_PREAMBLE_BYTES, 0
    scratch = None
    for fi in range(h.size_f):
        if start <= fi < end:
            out = dst[fi - start].view(np.uint16)
        else:
            if scratch is None:
                scratch = np.empty(npix, np.uint16)
            out = scratch
        off, prev = decode_tokens(data, off, out, npix, prev, f"{source}: pack-1 frame {fi} of {h.size_f}")
    f.seek(base + off)


def _zlib_block_bytes(f, h) -> int:
    row = h.size_x * _itemsize(h)
    frame = row * h.size_y * h.size_z
    pos = f.tell()
    raw = f.read(4)
    if len(raw) < 4:
        raise IOError("Unexpected EOF reading compressed size")
    n = struct.unpack("<i", raw)[0]
    if n <= 0:
        raise IOError(f"invalid zlib block size: {n}")
    head = _zlib_prefix(f.read(n), row + 1)
    f.seek(pos)
    if head > row:
        return frame
    if head == row:
        return row
    raise IOError(f"First zlib block inflated to {head} bytes; expected one row ({row}) or one frame ({frame})")


def _read_zlib(f, h, source, start, end, dst):
    """Pack 2: every block's size prefix walked and the kept frames' blocks
    inflated in parallel by one native call; f is left at the attribute records."""
    fb = _frame_bytes(h)
    bb = _zlib_block_bytes(f, h)
    per = fb // bb
    base = f.tell()
    rest = np.empty(os.fstat(f.fileno()).st_size - base, np.uint8)
    if f.readinto(memoryview(rest)) != rest.size:
        raise IOError(f"{source}: short read of the zlib blocks")
    L = _lib.lavision_lib()
    consumed, err = ctypes.c_longlong(0), ctypes.c_longlong(-1)
    rc = L.pivb_zlib_blocks_decode(rest.ctypes.data if rest.size else 1, rest.size, start * per, (end - start) * per,
                                   (h.size_f - end) * per, _ptr(dst), bb, max(1, min(16, os.cpu_count() or 1)),
                                   ctypes.byref(consumed), ctypes.byref(err))
    if rc == -2:
        raise IOError(f"{source}: zlib block {err.value}: unexpected EOF or invalid size prefix")
    if rc in (11, 12, 14):
        raise IOError(f"{source}: zlib block {err.value} did not inflate to {bb} bytes")
    if rc in (13, 15):
        raise IOError(f"{source}: zlib block {err.value} does not end at its declared size")
    if rc:
        raise IOError(f"{source}: zlib blocks could not be decoded ({rc})")
    f.seek(base + consumed.value)


def _read_lz4(f, h, source, start, end, dst):
    fb = _frame_bytes(h)
    if h.version == IM7_VERSION_PER_FRAME:
        file_size = os.fstat(f.fileno()).st_size
        starts, blocks = [], []
        for k in range(h.size_f):
            pos = f.tell()
            starts.append(pos)
            raw = f.read(8)
            if len(raw) != 8:
                raise IOError(f"{source}: version-1 LZ4 frame {k} of {h.size_f} is cut off at byte {pos}")
            n = _INT64.unpack(raw)[0]
            if n <= 0 or n > file_size - pos - 8:
                raise IOError(f"{source}: version-1 LZ4 frame {k} of {h.size_f} declares {n} compressed bytes at "
                              f"byte {pos}")
            if start <= k < end:
                blocks.append((k, f.read(n)))
            else:
                f.seek(n, 1)

        def one(item):
            k, comp = item
            try:
                lz4_block_decompress_into(comp, dst[k - start], fb)
            except IOError as exc:
                raise IOError(f"{source}: version-1 LZ4 frame {k} of {h.size_f}: {exc}") from exc

        list(_pool().map(one, blocks))
        pos = f.tell()
        table_raw = f.read(8 * h.size_f)
        if len(table_raw) != 8 * h.size_f:
            raise IOError(f"{source}: the version-1 frame-offset table at byte {pos} is truncated")
        if list(struct.unpack(f"<{h.size_f}q", table_raw)) != starts:
            raise IOError(f"{source}: the version-1 frame-offset table at byte {pos} does not list the frame "
                          f"starts {starts}")
        return
    n = _INT64.unpack(f.read(8))[0]
    if n <= 0:
        raise IOError(f"invalid LZ4 compressed size: {n}")
    comp = f.read(n)
    if len(comp) != n:
        raise IOError(f"Expected {n} bytes of LZ4 data, got {len(comp)}. File may be truncated.")
    if start == 0 and end == h.size_f:
        lz4_block_decompress_into(comp, dst, fb * h.size_f)
    else:
        whole = np.empty(fb * h.size_f, np.uint8)
        lz4_block_decompress_into(comp, whole, whole.size)
        dst[:] = whole.reshape(h.size_f, fb)[start:end]


def _parse_scale_record(data: bytes, sc: IM7Scales) -> None:
    parts = data.split(b"\x00")
    vals = parts[0].decode("utf-8", errors="replace").strip()
    tok = vals.split()
    try:
        if len(tok) >= 2:
            sc.slope, sc.offset = float(tok[0]), float(tok[1])
        elif len(tok) == 1:
            sc.slope = float(tok[0])
    except ValueError:
        pass
    if len(parts) > 1:
        sc.unit = parts[1].decode("utf-8", errors="replace").strip()
    sc.description = vals


def _read_attributes(f, source: str, pack_type: int) -> IM7Scales:
    """The attribute record chain after the pixels; also the check that the pixel
    decode stopped at the right byte (im7_reader.py:747-834)."""
    def fail(pos, why):
        return IOError(f"{source}: pixel data (pack_type {pack_type}) does not end where the attribute records "
                       f"begin ({why} at byte {pos}).")

    sc = IM7Scales()
    first = True
    while True:
        pos = f.tell()
        t = f.read(4)
        if len(t) == 0:
            break
        if len(t) < 4:
            raise fail(pos, f"{len(t)} stray trailing bytes")
        typ = struct.unpack("<i", t)[0]
        if typ == IEH_END:
            if first:
                raise fail(pos, "an empty record list")
            break
        if not 1 <= typ <= IEH_TYPE_MAX:
            raise fail(pos, f"record type {typ}")
        sz = f.read(4)
        if len(sz) < 4:
            raise fail(pos, f"record type {typ} with no size field")
        n = struct.unpack("<i", sz)[0]
        if n < 0:
            raise fail(pos, f"record type {typ} of size {n}")
        data = f.read(n)
        if len(data) != n:
            raise fail(pos, f"record type {typ} of size {n} past end of file")
        if typ == IEH_SCALE_I:
            _parse_scale_record(data, sc)
        first = False
    return sc


def _check_masks_per_frame(f, h: IM7Header, source: str, attr_at: int) -> None:
    """A version-1 file's mask planes must all be valid (1) and its trailer
    consistent (im7_reader.py:432-531); the planes decode in parallel."""
    n = h.size_f
    mask_bytes = h.size_x * h.size_y
    file_size = os.fstat(f.fileno()).st_size

    def damaged(pos, what):
        return IOError(f"{source}: version-1 trailer {what} at byte {pos}. The file is truncated, damaged, or "
                       f"uses a layout this reader does not know.")

    pos = f.tell()
    e = f.read(4)
    if len(e) != 4:
        raise damaged(pos, "ends after the attribute records, with no mask planes")
    if struct.unpack("<i", e)[0] != 0:
        raise damaged(pos, "has an IEH_END record whose size is not 0")
    starts, comps = [], []
    for k in range(n):
        pos = f.tell()
        starts.append(pos)
        head = f.read(_MASK_BLOCK_HEAD.size)
        if len(head) != _MASK_BLOCK_HEAD.size:
            raise damaged(pos, f"cuts off mask {k} of {n}")
        tag, cs = _MASK_BLOCK_HEAD.unpack(head)
        if tag != PACK_LZ4:
            raise damaged(pos, f"gives mask {k} of {n} compression {tag}, not {PACK_LZ4}")
        if not 0 < cs <= file_size - pos - _MASK_BLOCK_HEAD.size:
            raise damaged(pos, f"gives mask {k} of {n} {cs} compressed bytes")
        comps.append(f.read(cs))

    def one(k):
        m = np.empty(mask_bytes, np.uint8)
        try:
            lz4_block_decompress_into(comps[k], m, mask_bytes)
        except IOError as exc:
            raise IOError(f"{source}: version-1 mask {k} of {n}: {exc}") from exc
        if m.min() != DAVIS_MASK_VALID or m.max() != DAVIS_MASK_VALID:
            masked = mask_bytes - int(np.count_nonzero(m == DAVIS_MASK_VALID))
            raise ValueError(f"{source}: frame {k} of {n} carries a DaVis mask with {masked} of {mask_bytes} "
                             f"pixels masked. DaVis masks inside .im7 are not applied.")

    list(_pool().map(one, range(n)))
    pos = f.tell()
    raw = f.read(8 * n)
    if len(raw) != 8 * n:
        raise damaged(pos, "cuts off the mask-offset table")
    if list(struct.unpack(f"<{n}q", raw)) != starts:
        raise damaged(pos, f"has a mask-offset table that does not list the masks at {starts}")
    pos = f.tell()
    footer = f.read()
    if len(footer) != IM7_FOOTER_SIZE:
        raise damaged(pos, f"has a footer of {len(footer)} bytes, not {IM7_FOOTER_SIZE}")
    got = list(_FOOTER_SLOTS.unpack_from(footer))
    want = [0] * len(got)
    want[FOOTER_ATTRIBUTES] = attr_at
    want[FOOTER_FRAME_TABLE] = attr_at - 8 * n
    want[FOOTER_MASK_TABLE] = pos - 8 * n
    if got != want or any(footer[_FOOTER_SLOTS.size:]):
        raise damaged(pos, f"has a footer reading {got}, but the tables give {want}")


def _read_frames(path: Path, start: Optional[int], end: Optional[int], dst_factory):
    """Decode frames [start, end) of an .im7 file into the uint8 (n, frame_bytes)
    buffer dst_factory(header, n) returns, then read the trailer."""
    with open(path, "rb") as f:
        raw = f.read(HEADER_SIZE)
        if len(raw) != HEADER_SIZE:
            raise IOError(f"File too small for header ({len(raw)} < {HEADER_SIZE})")
        h = parse_header(raw, path.name)
        s = 0 if start is None else start
        e = h.size_f if end is None else end
        dst = dst_factory(h, e - s)
        if h.pack_type == PACK_UNCOMPRESSED:
            _itemsize(h)
            _read_uncompressed(f, h, s, e, dst)
        elif h.pack_type == PACK_RLE:
            _read_pack1(f, h, path.name, s, e, dst)
        elif h.pack_type == PACK_ZLIB:
            _read_zlib(f, h, path.name, s, e, dst)
        elif h.pack_type == PACK_LZ4:
            _read_lz4(f, h, path.name, s, e, dst)
        else:
            raise _unsupported_pack(h, path.name)
        attr_at = f.tell()
        sc = _read_attributes(f, path.name, h.pack_type)
        if h.version == IM7_VERSION_PER_FRAME:
            _check_masks_per_frame(f, h, path.name, attr_at)
    return h, dst, sc


def read_im7(filepath: Union[str, Path]):
    """(header, pixels, scales) of an .im7 file, pixels as the reference returns
    them (uint16 or float32; (H, W), (Z, H, W), (F, H, W) or (F, Z, H, W);
    im7_reader.py:911-948), decoded by the native codecs."""
    path = Path(filepath)
    if not path.exists():
        raise FileNotFoundError(f"File not found: {path}")

    def alloc(h, n):
        return np.empty((n, _frame_bytes(h)), np.uint8)

    h, buf, sc = _read_frames(path, None, None, alloc)
    dt = np.dtype("<f4") if h.buffer_format == BUFFER_FORMAT_FLOAT else np.dtype("<u2")
    px = buf.view(dt).reshape(h.size_f, h.size_z, h.size_y, h.size_x)
    if px.shape[0] == 1 and h.size_z == 1:
        px = px[0, 0]
    elif px.shape[0] == 1:
        px = px[0]
    elif h.size_z == 1:
        px = px[:, 0]
    return h, px, sc


def get_im7_frame_count(filepath) -> int:
    path = Path(filepath)
    with open(path, "rb") as f:
        return parse_header(f.read(HEADER_SIZE), path.name).size_f


def get_im7_frame_shape(filepath) -> tuple:
    path = Path(filepath)
    with open(path, "rb") as f:
        h = parse_header(f.read(HEADER_SIZE), path.name)
    return (h.size_y, h.size_x)


# ---------------------------------------------------------------------------
# device path: page-locked staging, copy, unpack on the GPU
# ---------------------------------------------------------------------------

class _Staging:
    """One growing page-locked buffer per device and host thread; a call waits for
    the previous call's copy out of it (an event) before decoding into it again.
    `lock` is held by a call from its decode into the buffer until its copy is
    enqueued."""

    def __init__(self, torch, device):
        import threading

        self.torch, self.device = torch, device
        self.buf = None
        self.done = None
        self.lock = threading.Lock()

    def get(self, nbytes: int):
        torch = self.torch
        if self.done is not None:
            self.done.synchronize()
        if self.buf is None or self.buf.numel() < nbytes:
            self.buf = torch.empty(max(nbytes, 1 << 20), dtype=torch.uint8, pin_memory=True)
        return self.buf[:nbytes]


_STAGING: dict = {}
_STAGING_LOCK = __import__("threading").Lock()


def _staging(torch, device) -> _Staging:
    import threading

    # one buffer per device and host thread, so threads decoding different
    # files overlap
    key = (device.type, device.index, threading.get_ident())
    with _STAGING_LOCK:
        if key not in _STAGING:
            _STAGING[key] = _Staging(torch, device)
        return _STAGING[key]


def _to_device_unpack(torch, device, st: _Staging, host, n_frames: int, payload_bytes: int, npix: int, enc: int,
                      slope: float, offset: float, out):
    """Copy n_frames payloads (page-locked) to the device and unpack them into
    the float32 (n_frames, npix...) tensor out on the current stream."""
    stream = torch.cuda.current_stream(device)
    dev = torch.empty(n_frames * payload_bytes, dtype=torch.uint8, device=device)
    dev.copy_(host, non_blocking=True)
    ev = torch.cuda.Event()
    ev.record(stream)
    st.done = ev
    L = _lib.pass_lib()
    use_slope, use_offset = slope != 1.0, offset != 0.0
    rc = L.pivb_unpack_pixels_dev(dev.data_ptr(), payload_bytes, n_frames, npix, enc, int(use_slope),
                                  float(np.float32(slope)), int(use_offset), float(np.float32(offset)),
                                  out.data_ptr(), npix, ctypes.c_void_p(stream.cuda_stream))
    if rc != 0:
        raise RuntimeError("pivb_unpack_pixels_dev failed")
    return out


def _device(torch, device):
    dev = torch.device("cuda" if device is None else device)
    if dev.type != "cuda":
        raise ValueError("the LaVision frames are decoded on a CUDA device")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    return dev


def read_im7_camera(filepath: Union[str, Path], camera_no: int = 1, frames_per_camera: int = 2,
                    frames: Optional[int] = None, out=None, device=None):
    """One camera's frames of an .im7 file as a float32 (n, H, W) device tensor
    with the intensity scale applied: the frames of read_im7_camera
    (im7_reader.py:982-1153), decoded natively into page-locked memory and
    unpacked on the GPU.  out: optional float32 (n, H, W) device tensor."""
    import torch

    path = Path(filepath)
    if not path.exists():
        raise FileNotFoundError(f"File not found: {path}")
    with open(path, "rb") as f:
        h = parse_header(f.read(HEADER_SIZE), path.name)
    if h.size_z != IM7_CAMERA_PLANES:
        raise ValueError(f"{path.name}: header size_z (planes per frame) is {h.size_z}; a camera image has "
                         f"{IM7_CAMERA_PLANES} plane per frame.")
    if frames is not None and frames < 1:
        raise ValueError(f"frames must be >= 1, got {frames}")
    start = (camera_no - 1) * frames_per_camera
    wanted = frames_per_camera if frames is None else min(frames, frames_per_camera)
    if start >= h.size_f:
        raise ValueError(f"Camera {camera_no} with {frames_per_camera} frames/camera requires frame index {start}, "
                         f"but file only has {h.size_f} frames.")
    end = min(start + wanted, h.size_f)
    n = end - start
    dev = _device(torch, device)
    shape = (n, h.size_y, h.size_x)
    if out is None:
        out = torch.empty(shape, dtype=torch.float32, device=dev)
    else:
        if out.ndim == 3 and out.shape[0] != n:
            raise ValueError(f"{path.name} holds {n} frame(s) for camera {camera_no} (asked for {wanted}), but a "
                             f"{tuple(out.shape)} buffer was supplied.")
        if tuple(out.shape) != shape or out.dtype != torch.float32 or not out.is_contiguous() \
                or out.device != dev:
            raise ValueError(f"read_im7_camera: out must be a contiguous float32 {shape} tensor on {dev}")
    fb = _frame_bytes(h)
    st = _staging(torch, dev)
    holder = {}

    def alloc(hh, nn):
        host = st.get(nn * fb)
        holder["host"] = host
        return host.numpy().reshape(nn, fb)

    with st.lock:
        h, _, sc = _read_frames(path, start, end, alloc)
        enc = ENC_FLOAT if h.buffer_format == BUFFER_FORMAT_FLOAT else ENC_WORD
        with torch.cuda.device(dev):
            return _to_device_unpack(torch, dev, st, holder["host"], n, fb, h.size_x * h.size_y, enc, sc.slope,
                                     sc.offset, out)


# ---------------------------------------------------------------------------
# .set entries (set_reader.py:1482-1669)
# ---------------------------------------------------------------------------

def set_payload_bytes(decoder: str, width: int, height: int) -> int:
    """Packed bytes of one frame in a .set encoding; refuses unknown and
    unimplemented ids as set_reader.py:1482-1513 does."""
    implemented = ", ".join(SET_DECODERS)
    if decoder not in _SET_BITS:
        raise ValueError(f"Unknown .set pixel encoding '{decoder}'. PIVTOOLs decodes: {implemented}.")
    if decoder not in SET_DECODERS:
        raise ValueError(f"PIVTOOLs cannot decode this .set: pixel encoding '{decoder}' is a recognised DaVis "
                         f"encoding but is not implemented. PIVTOOLs decodes: {implemented}.")
    npix = width * height
    if decoder.startswith("mono-10") and npix % 4:
        raise ValueError(f"{decoder} packs four pixels into five bytes, so a frame must hold a multiple of four "
                         f"pixels; {width}x{height} is {npix}.")
    if decoder.startswith("mono-12") and npix % 2:
        raise ValueError(f"{decoder} packs two pixels into three bytes, so a frame must hold an even number of "
                         f"pixels; {width}x{height} is {npix}.")
    return (npix * _SET_BITS[decoder]) // 8


def set_entry_payload(stored: bytes, codec: str, expected: int, where: str = "entry", out=None):
    """The packed payload (uint8, `expected` bytes) of one entry's stored bytes
    under the index codec ('', 'Uncompressed', 'Zlib', 'LZ4' or 'IMX';
    set_reader.py:1552-1669), decoded natively into out (or a new array)."""
    if codec not in SET_CODECS:
        raise ValueError(f"{where}: unknown codec {codec!r}")
    dst = np.empty(expected, np.uint8) if out is None else out
    if codec in ("", "Uncompressed"):
        if len(stored) != expected:
            raise ValueError(f"Pixel data size mismatch: entry holds {len(stored)} bytes but the frame needs "
                             f"{expected}.")
        np.copyto(dst if isinstance(dst, np.ndarray) else dst.numpy(), np.frombuffer(stored, np.uint8))
    elif codec == "Zlib":
        zlib_inflate_into(stored, dst, expected, f"{where}, stored with 'Zlib' compression")
    elif codec == "LZ4":
        try:
            lz4_block_decompress_into(stored, dst, expected)
        except OSError as exc:
            raise IOError(f"{where}: the LZ4 block does not decompress to the {expected} bytes the frame's "
                          f"geometry and encoding need ({exc})") from exc
    else:
        if expected % 2:
            raise ValueError(f"{where}: IMX codes the packed payload as 16-bit words, but this frame packs into "
                             f"{expected} bytes, an odd count.")
        data = np.frombuffer(stored, np.uint8).copy()
        words = (dst if isinstance(dst, np.ndarray) else dst.numpy()).view(np.uint16)
        off, _ = decode_tokens(data, 0, words, expected // 2, 0, f"{where}: IMX entry")
        if off != data.size:
            raise TrailingTokenBytesError(f"{where}: IMX entry: tokens end at byte {off}, entry holds {data.size}")
    return dst


def decode_set_entry(stored: bytes, codec: str, decoder: str, width: int, height: int, slope: float = 1.0,
                     offset: float = 0.0, out=None, device=None):
    """One .set entry as a float32 (height, width) device tensor: the codec on the
    host into page-locked memory, the pixel decoder and the intensity scale on the
    GPU.  The stream's transformers (corrections, geometry) are not applied: the
    caller's stream must declare none."""
    import torch

    expected = set_payload_bytes(decoder, width, height)
    dev = _device(torch, device)
    st = _staging(torch, dev)
    if out is None:
        out = torch.empty((height, width), dtype=torch.float32, device=dev)
    elif tuple(out.shape) != (height, width) or out.dtype != torch.float32 or not out.is_contiguous():
        raise ValueError(f"decode_set_entry: out must be a contiguous float32 ({height}, {width}) tensor")
    with st.lock:
        host = st.get(expected)
        set_entry_payload(stored, codec, expected, out=host.numpy())
        with torch.cuda.device(dev):
            return _to_device_unpack(torch, dev, st, host, 1, expected, width * height, SET_DECODERS[decoder],
                                     slope, offset, out)
