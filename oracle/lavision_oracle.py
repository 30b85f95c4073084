"""LaVision container oracle.  TEST INFRASTRUCTURE ONLY: nothing here is shipped
or called by the product path (pivtools_b200.lavision decodes with the native
libpivb_lavision codecs and the GPU unpack).

* A pure-Python LZ4 block decoder and a greedy LZ4 block encoder, written from
  the published LZ4 block format.  The reference reads LZ4 through the
  third-party python-lz4 package (`lz4.block`, pinned by the reference's
  pyproject; im7_reader.py:270-291), which is absent here: the decoder stands in
  for `lz4.block.decompress` when tests/golden/make_golden.py imports the
  reference's readers, and the encoder writes the pack-20 and LZ4 .set fixtures.
  Parity of the native decoder is anchored on lvpyio's decode of the reference's
  own version-1 pack-20 fixture (unit-tests/fixtures/im7_v1_pack20).
* A DaVis token-stream encoder exercising every token kind of the grammar in
  davis_tokens.py:1-24 (int8 deltas, 0x80 absolute, 0x7f absolute runs, 0x81
  nibble runs ended by a low nibble 8 or by the value count).
* Writers of Image_Header_7 files (im7_reader.py:33-118, 722-869) for packs 0, 1,
  2 and 20 (versions 0 and 1, with the version-1 mask trailer).
* A host reader of camera frames for packs 0 and 2 (version 0), restating the
  reference's read_im7_camera (im7_reader.py:982-1160: header, per-frame reads or
  per-row / per-frame zlib blocks with exact ends, the attribute walk for the
  SCALE_I record, float32 frames with the scale applied in place): the CPU
  baseline of the ingest measurement and a checker of the fixtures.
"""

from __future__ import annotations

import struct
import zlib

import numpy as np


# ---------------------------------------------------------------------------
# LZ4 block format
# ---------------------------------------------------------------------------

def lz4_decode(src: bytes, expected: int) -> bytes:
    """Decode one LZ4 block to exactly `expected` bytes (IOError otherwise)."""
    src = bytes(src)
    out = bytearray()
    i, n = 0, len(src)
    if n == 0:
        if expected:
            raise IOError("empty LZ4 block")
        return b""
    while True:
        if i >= n:
            raise IOError("LZ4 block cut off")
        tok = src[i]
        i += 1
        lit = tok >> 4
        if lit == 15:
            while True:
                if i >= n:
                    raise IOError("LZ4 block cut off")
                s = src[i]
                i += 1
                lit += s
                if s != 255:
                    break
        if i + lit > n or len(out) + lit > expected:
            raise IOError("LZ4 literals overrun")
        out += src[i:i + lit]
        i += lit
        if i == n:
            break
        if n - i < 2:
            raise IOError("LZ4 block cut off")
        off = src[i] | (src[i + 1] << 8)
        i += 2
        if off == 0 or off > len(out):
            raise IOError("LZ4 match offset out of range")
        ml = tok & 15
        if ml == 15:
            while True:
                if i >= n:
                    raise IOError("LZ4 block cut off")
                s = src[i]
                i += 1
                ml += s
                if s != 255:
                    break
        ml += 4
        if len(out) + ml > expected:
            raise IOError("LZ4 match overrun")
        for _ in range(ml):
            out.append(out[-off])
    if len(out) != expected:
        raise IOError(f"LZ4 block decoded to {len(out)} bytes, expected {expected}")
    return bytes(out)


def _lz4_len(v: int) -> bytes:
    b = bytearray()
    while v >= 255:
        b.append(255)
        v -= 255
    b.append(v)
    return bytes(b)


def lz4_encode(data: bytes) -> bytes:
    """Greedy LZ4 block encoder (4-byte hash matches; the last 5 bytes and any
    match within 12 bytes of the end stay literals, as the format requires)."""
    data = bytes(data)
    n = len(data)
    out = bytearray()
    table = {}
    anchor = 0
    i = 0
    limit = n - 12
    while i < limit:
        key = data[i:i + 4]
        cand = table.get(key)
        table[key] = i
        if cand is not None and i - cand <= 65535:
            m = 4
            while i + m < n - 5 and data[cand + m] == data[i + m]:
                m += 1
            lit = i - anchor
            tok_l = min(lit, 15)
            tok_m = min(m - 4, 15)
            out.append((tok_l << 4) | tok_m)
            if lit >= 15:
                out += _lz4_len(lit - 15)
            out += data[anchor:i]
            out += struct.pack("<H", i - cand)
            if m - 4 >= 15:
                out += _lz4_len(m - 4 - 15)
            i += m
            anchor = i
        else:
            i += 1
    lit = n - anchor
    out.append(min(lit, 15) << 4)
    if lit >= 15:
        out += _lz4_len(lit - 15)
    out += data[anchor:]
    return bytes(out)


class _Lz4Block:
    """Stand-in for python-lz4's `lz4.block` module (decompress only)."""

    class LZ4BlockError(Exception):
        pass

    @staticmethod
    def decompress(src, uncompressed_size):
        try:
            return lz4_decode(src, uncompressed_size)
        except IOError as exc:
            raise _Lz4Block.LZ4BlockError(str(exc)) from exc


def install_lz4_stub():
    """Make `import lz4.block` resolve to the oracle decoder (only where python-lz4
    is absent)."""
    import sys
    import types

    try:
        import lz4.block  # noqa: F401
        return
    except ImportError:
        pass
    mod = types.ModuleType("lz4")
    blk = types.ModuleType("lz4.block")
    blk.decompress = _Lz4Block.decompress
    blk.LZ4BlockError = _Lz4Block.LZ4BlockError
    mod.block = blk
    sys.modules["lz4"] = mod
    sys.modules["lz4.block"] = blk


# ---------------------------------------------------------------------------
# DaVis token stream
# ---------------------------------------------------------------------------

def tokens_encode(values, prev: int = 0, rng=None) -> tuple[bytes, int]:
    """Code uint16 values as DaVis tokens starting from running value prev, mixing
    every token kind (chosen by rng where several apply); returns (bytes, prev).
    A nibble run holds an odd number of deltas: pairs (high, low) and a last byte
    whose low nibble 8 ends the run; a low-nibble delta is never -8."""
    rng = np.random.default_rng(0) if rng is None else rng
    v = [int(x) for x in values]
    out = bytearray()
    i = 0
    while i < len(v):
        d = v[i] - prev
        kind = int(rng.integers(0, 4))
        if kind == 0 and -8 <= d <= 7:
            run, p, j = [d], v[i], i + 1
            while j < len(v) and len(run) < 11:
                dd = v[j] - p
                if not -8 <= dd <= 7 or (len(run) % 2 == 1 and dd == -8):
                    break
                run.append(dd)
                p = v[j]
                j += 1
            if len(run) % 2 == 0:
                run.pop()
            out.append(0x81)
            for k in range(0, len(run) - 1, 2):
                out.append(((run[k] & 0xF) << 4) | (run[k + 1] & 0xF))
            out.append(((run[-1] & 0xF) << 4) | 0x8)
            i += len(run)
            prev = v[i - 1]
            continue
        if kind == 1 and -128 <= d <= 127 and (d & 0xFF) not in (0x7F, 0x80, 0x81):
            out.append(d & 0xFF)
            prev = v[i]
            i += 1
            continue
        if kind == 2:
            cnt = int(min(len(v) - i, rng.integers(1, 6)))
            out.append(0x7F)
            out.append(cnt)
            for k in range(cnt):
                out += struct.pack("<H", v[i + k])
            prev = v[i + cnt - 1]
            i += cnt
            continue
        out.append(0x80)
        out += struct.pack("<H", v[i])
        prev = v[i]
        i += 1
    return bytes(out), prev


# ---------------------------------------------------------------------------
# Image_Header_7 files
# ---------------------------------------------------------------------------

def im7_header(version, pack, buffer_format, nx, ny, nz, nf) -> bytes:
    head = struct.pack("<hhhh iiii hhh", version, pack, buffer_format, 0, nx, ny, nz, nf, 0, 0, 0)
    return head + bytes(256 - len(head))


def im7_attributes(slope=None, offset=None, unit="counts", extra=True) -> bytes:
    """Attribute records: a SCALE_X record, an optional SCALE_I (intensity) record,
    a comment, then IEH_END."""
    recs = bytearray()

    def rec(t, data):
        recs.extend(struct.pack("<ii", t, len(data)))
        recs.extend(data)

    rec(1, b"1 0\x00mm\x00\x00")
    if slope is not None:
        txt = f"{slope!r}" if offset is None else f"{slope!r} {offset!r}"
        rec(4, txt.encode() + b"\x00" + unit.encode() + b"\x00\x00\x00")
    if extra:
        rec(6, b"Camera=synthetic")
    recs.extend(struct.pack("<i", 0))
    return bytes(recs)


def im7_pack0(frames: np.ndarray, attrs: bytes) -> bytes:
    """frames (F, Z, H, W) uint16 or float32."""
    F, Z, H, W = frames.shape
    fmt = -3 if frames.dtype == np.float32 else -4
    return im7_header(0, 0, fmt, W, H, Z, F) + frames.astype(frames.dtype.newbyteorder("<")).tobytes() + attrs


def im7_pack1(frames: np.ndarray, attrs: bytes, rng=None) -> bytes:
    """frames (F, Z, H, W) uint16; the 3-byte preamble, running value carried
    across frames, each frame's tokens self-contained."""
    F, Z, H, W = frames.shape
    body = bytearray(b"\x01\x01\x00")
    prev = 0
    for k in range(F):
        b, prev = tokens_encode(frames[k].ravel(), prev, rng)
        body += b
    return im7_header(0, 1, -4, W, H, Z, F) + bytes(body) + attrs


def im7_pack2(frames: np.ndarray, attrs: bytes, per_row: bool) -> bytes:
    F, Z, H, W = frames.shape
    fmt = -3 if frames.dtype == np.float32 else -4
    body = bytearray()
    for k in range(F):
        raw = frames[k].tobytes()
        chunks = [raw[i:i + W * frames.itemsize] for i in range(0, len(raw), W * frames.itemsize)] if per_row \
            else [raw]
        for c in chunks:
            z = zlib.compress(c, 6)
            body += struct.pack("<i", len(z)) + z
    return im7_header(0, 2, fmt, W, H, Z, F) + bytes(body) + attrs


def im7_pack20_v0(frames: np.ndarray, attrs: bytes) -> bytes:
    F, Z, H, W = frames.shape
    fmt = -3 if frames.dtype == np.float32 else -4
    z = lz4_encode(frames.tobytes())
    return im7_header(0, 20, fmt, W, H, Z, F) + struct.pack("<q", len(z)) + z + attrs


def im7_pack20_v1(frames: np.ndarray, attrs: bytes, masks=None) -> bytes:
    """Version 1: per frame an int64 size and an LZ4 block, the frame-offset
    table, the attribute records, per frame an int32 20, an int64 size and an LZ4
    block of the H x W uint8 mask, the mask-offset table and the 256-byte footer."""
    F, Z, H, W = frames.shape
    fmt = -3 if frames.dtype == np.float32 else -4
    buf = bytearray(im7_header(1, 20, fmt, W, H, Z, F))
    starts = []
    for k in range(F):
        starts.append(len(buf))
        z = lz4_encode(frames[k].tobytes())
        buf += struct.pack("<q", len(z)) + z
    buf += struct.pack(f"<{F}q", *starts)
    attr_at = len(buf)
    buf += attrs + struct.pack("<i", 0)          # IEH_END's size field
    mstarts = []
    for k in range(F):
        mstarts.append(len(buf))
        m = np.ones((H, W), np.uint8) if masks is None else masks[k]
        z = lz4_encode(m.tobytes())
        buf += struct.pack("<iq", 20, len(z)) + z
    mtab = len(buf)
    buf += struct.pack(f"<{F}q", *mstarts)
    slots = [0] * 8
    slots[0], slots[1], slots[7] = attr_at, attr_at - 8 * F, mtab
    buf += struct.pack("<8q", *slots) + bytes(256 - 64)
    return bytes(buf)


# ---------------------------------------------------------------------------
# Host reader (packs 0 and 2, version 0)
# ---------------------------------------------------------------------------

def _intensity_scale(f):
    """(slope, offset) from the attribute records at f's position (im7_reader.py:
    747-868): records of int32 type, int32 size and data up to IEH_END or EOF;
    type 4 holds 'slope offset\\0unit\\0'."""
    slope, offset, first = 1.0, 0.0, True
    while True:
        t = f.read(4)
        if not t:
            break
        if len(t) < 4:
            raise IOError("stray bytes after the pixel data")
        typ = struct.unpack("<i", t)[0]
        if typ == 0:
            if first:
                raise IOError("empty record list after the pixel data")
            break
        if not 1 <= typ <= 13:
            raise IOError(f"record type {typ} after the pixel data")
        size = struct.unpack("<i", f.read(4))[0]
        data = f.read(size)
        if size < 0 or len(data) != size:
            raise IOError("attribute record past the end of the file")
        if typ == 4:
            words = data.split(b"\x00")[0].decode("utf-8", "replace").split()
            try:
                if len(words) >= 1:
                    slope = float(words[0])
                if len(words) >= 2:
                    offset = float(words[1])
            except ValueError:
                pass
        first = False
    return slope, offset


def _zlib_exact(comp: bytes, want: int) -> bytes:
    d = zlib.decompressobj()
    out = d.decompress(comp)
    if not d.eof or d.unused_data or len(out) != want:
        raise IOError("zlib block does not inflate to its block size at its declared end")
    return out


def read_im7_camera_host(path, camera_no: int = 1, frames_per_camera: int = 2, frames=None) -> np.ndarray:
    """Float32 frames (n, H, W) of one camera of a pack-0 or pack-2 version-0
    file, scale applied as result *= slope; result += offset."""
    with open(path, "rb") as f:
        head = f.read(256)
        ver, pack, fmt, _, W, H, Z, F = struct.unpack_from("<hhhh iiii", head, 0)
        if ver != 0 or pack not in (0, 2) or min(W, H, Z, F) < 1:
            raise ValueError(f"host reader: version {ver} pack {pack} not restated")
        dt = np.dtype("<u2") if fmt == -4 else np.dtype("<f4")
        row = W * dt.itemsize
        fb = row * H * Z
        start = (camera_no - 1) * frames_per_camera
        if start >= F:
            raise ValueError("camera beyond the file's frames")
        n = min(frames_per_camera if frames is None else min(frames, frames_per_camera), F - start)
        out = np.empty((n, H, W), np.float32)
        if pack == 0:
            f.seek(256 + start * fb)
            for i in range(n):
                raw = f.read(fb)
                if len(raw) != fb:
                    raise IOError("truncated frame")
                out[i] = np.frombuffer(raw, dt).reshape(Z, H, W)[0]
            f.seek(256 + F * fb)
        else:
            pos = f.tell()
            c0 = struct.unpack("<i", f.read(4))[0]
            probe = zlib.decompressobj().decompress(f.read(c0), row + 1)
            f.seek(pos)
            block = fb if len(probe) > row else row
            if len(probe) < row:
                raise IOError("first zlib block is shorter than a row")
            per_frame = fb // block

            def skip(k):
                for _ in range(k):
                    c = struct.unpack("<i", f.read(4))[0]
                    f.seek(c, 1)

            skip(start * per_frame)
            for i in range(n):
                parts = []
                for _ in range(per_frame):
                    c = struct.unpack("<i", f.read(4))[0]
                    if c <= 0:
                        raise IOError("invalid zlib block size")
                    parts.append(_zlib_exact(f.read(c), block))
                out[i] = np.frombuffer(b"".join(parts), dt).reshape(Z, H, W)[0]
            skip((F - start - n) * per_frame)
        slope, offset = _intensity_scale(f)
    if slope != 1.0:
        out *= slope
    if offset != 0.0:
        out += offset
    return out
