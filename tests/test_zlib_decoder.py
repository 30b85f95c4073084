"""The codec library's Deflate decoder (pivb_zlib_inflate_exact) against zlib.

The reference's readers inflate .im7 pack-2 blocks and .set "Zlib" entries with
zlib and check where the stream ends (im7_reader.py:569-594,
set_reader.py:1601-1633).  The library decodes them with its own decoder; this
test drives it and the system zlib's inflate() (through ctypes, into exactly
the expected bytes and then one spare byte) over seeded streams of every block
type (stored, fixed and dynamic Huffman: levels 0-9, the five zlib strategies,
window sizes 2^9-2^15) and over damaged forms of them (truncations, bit flips,
trailing bytes, a wrong expected size), and requires the same bytes and the
same status code: 0 ok, 1 not a valid stream, 2 more than the expected bytes,
3 truncated, 4 fewer than the expected bytes, 5 bytes after the end marker.
"""

import ctypes
import zlib

import numpy as np
import pytest


class _ZStream(ctypes.Structure):
    _fields_ = [("next_in", ctypes.c_void_p), ("avail_in", ctypes.c_uint), ("total_in", ctypes.c_ulong),
                ("next_out", ctypes.c_void_p), ("avail_out", ctypes.c_uint), ("total_out", ctypes.c_ulong),
                ("msg", ctypes.c_char_p), ("state", ctypes.c_void_p), ("zalloc", ctypes.c_void_p),
                ("zfree", ctypes.c_void_p), ("opaque", ctypes.c_void_p), ("data_type", ctypes.c_int),
                ("adler", ctypes.c_ulong), ("reserved", ctypes.c_ulong)]


_Z_OK, _Z_STREAM_END, _Z_NEED_DICT, _Z_STREAM_ERROR, _Z_DATA_ERROR, _Z_MEM_ERROR = 0, 1, 2, -2, -3, -4
_Z_FINISH = 4


@pytest.fixture(scope="module")
def zlib_status():
    """The status code of a stream under the system zlib's inflate(), driven
    with Z_FINISH into exactly `expected` bytes and then one spare byte (what
    tells "longer" from "ends here"), and the bytes it produced."""
    import ctypes.util

    Z = ctypes.CDLL(ctypes.util.find_library("z") or "libz.so.1")
    Z.inflateInit_.argtypes = [ctypes.POINTER(_ZStream), ctypes.c_char_p, ctypes.c_int]
    Z.inflate.argtypes = [ctypes.POINTER(_ZStream), ctypes.c_int]
    Z.inflateEnd.argtypes = [ctypes.POINTER(_ZStream)]
    version = Z.zlibVersion
    version.restype = ctypes.c_char_p
    ver = version()

    def status(z: bytes, expected: int):
        src = ctypes.create_string_buffer(z, len(z) + 1)
        dst = ctypes.create_string_buffer(expected + 1)
        zs = _ZStream()
        assert Z.inflateInit_(ctypes.byref(zs), ver, ctypes.sizeof(_ZStream)) == _Z_OK
        zs.next_in = ctypes.cast(src, ctypes.c_void_p)
        zs.avail_in = len(z)
        zs.next_out = ctypes.cast(dst, ctypes.c_void_p)
        zs.avail_out = expected
        rc = Z.inflate(ctypes.byref(zs), _Z_FINISH)
        if rc == _Z_STREAM_END:
            r = 4 if zs.total_out != expected else (5 if zs.avail_in else 0)
        elif rc in (_Z_DATA_ERROR, _Z_NEED_DICT, _Z_STREAM_ERROR, _Z_MEM_ERROR):
            r = 1
        elif zs.avail_out == 0:
            zs.next_out = ctypes.cast(ctypes.addressof(dst) + expected, ctypes.c_void_p)
            zs.avail_out = 1
            rc = Z.inflate(ctypes.byref(zs), _Z_FINISH)
            if zs.total_out > expected:
                r = 2
            elif rc == _Z_STREAM_END:
                r = 5 if zs.avail_in else 0
            elif rc in (_Z_DATA_ERROR, _Z_NEED_DICT, _Z_STREAM_ERROR):
                r = 1
            else:
                r = 3
        else:
            r = 3
        Z.inflateEnd(ctypes.byref(zs))
        return r, (dst.raw[:expected] if r == 0 else None)

    return status


@pytest.fixture(scope="module")
def inflate():
    from pivtools_b200 import _lib

    L = _lib.lavision_lib()

    def run(z: bytes, expected: int):
        src = np.frombuffer(z, np.uint8).copy() if z else np.zeros(1, np.uint8)
        dst = np.full(expected + 32, 0xA5, np.uint8)
        rc = L.pivb_zlib_inflate_exact(src.ctypes.data, len(z), dst.ctypes.data, expected)
        assert bytes(dst[expected:]) == b"\xa5" * 32, "wrote past the expected size"
        return rc, dst[:expected].tobytes()

    return run


def _payload(rng, kind, n):
    if kind == 0:
        return rng.integers(0, 256, n, dtype=np.uint8).tobytes()
    if kind == 1:
        return rng.integers(0, 4, n, dtype=np.uint8).tobytes()
    if kind == 2:
        return (b"abcabcabd" * (n // 9 + 1))[:n]
    if kind == 3:
        return bytes(n)
    if kind == 4:      # camera-like 16-bit counts: a noisy low byte, a mostly-zero high byte
        return np.clip(rng.normal(120, 40, n // 2 + 1), 0, 65535).astype(np.uint16).tobytes()[:n]
    if kind == 5:      # runs (distance 1) and short periods
        out = bytearray()
        while len(out) < n:
            out += bytes([int(rng.integers(0, 256))]) * int(rng.integers(1, 40))
            out += rng.integers(0, 256, int(rng.integers(0, 8)), dtype=np.uint8).tobytes()
        return bytes(out[:n])
    base = rng.integers(0, 256, 40000, dtype=np.uint8).tobytes()   # far, long matches
    out = bytearray()
    while len(out) < n:
        s = int(rng.integers(0, 39000))
        out += base[s:s + int(rng.integers(3, 600))]
    return bytes(out[:n])


def _check(inflate, zlib_status, z, expected, raw=None):
    want, wbytes = zlib_status(z, expected)
    rc, got = inflate(z, expected)
    assert rc == want, (rc, want, len(z), expected)
    if rc == 0:
        assert got == wbytes
        if raw is not None:
            assert got == raw


@pytest.mark.parametrize("seed", range(4))
def test_decoder_matches_zlib(inflate, zlib_status, seed):
    rng = np.random.default_rng(1000 + seed)
    strategies = [zlib.Z_DEFAULT_STRATEGY, zlib.Z_FILTERED, zlib.Z_HUFFMAN_ONLY, zlib.Z_RLE, zlib.Z_FIXED]
    seen = set()
    for _ in range(150):
        raw = _payload(rng, int(rng.integers(0, 7)), int(rng.choice([0, 1, 2, 7, 100, 1000, 4096, 20000, 70000])))
        c = zlib.compressobj(int(rng.integers(0, 10)), zlib.DEFLATED, int(rng.integers(9, 16)), 9,
                             strategies[int(rng.integers(0, 5))])
        z = c.compress(raw) + c.flush()
        _check(inflate, zlib_status, z, len(raw), raw)
        for e in (len(raw) - 1, len(raw) + 1, len(raw) - int(rng.integers(1, 300)), len(raw) + 300):
            if e >= 0:
                _check(inflate, zlib_status, z, e)
        for cut in {len(z) - 1, len(z) - 4, len(z) - 5, int(rng.integers(0, len(z))), 0, 1, 2, 3}:
            if 0 <= cut < len(z):
                _check(inflate, zlib_status, z[:cut], len(raw))
        _check(inflate, zlib_status, z + b"\x00\x01", len(raw))
        for _ in range(3):
            zz = bytearray(z)
            zz[int(rng.integers(0, len(zz)))] ^= 1 << int(rng.integers(0, 8))
            _check(inflate, zlib_status, bytes(zz), len(raw))
        seen.add(zlib_status(z, len(raw))[0])
    assert seen == {0}


def test_decoder_header_and_block_errors(inflate, zlib_status):
    raw = b"particle image rows " * 50
    z = zlib.compress(raw)
    cases = [
        bytes([z[0], z[1] ^ 1]) + z[2:],          # header check (mod 31) fails
        bytes([0x79, 0x9C]) + z[2:],              # compression method 9
        bytes([0x88, 0x98]) + z[2:],              # window size 2^16
        bytes([0x78, 0xBB]) + z[2:],              # preset dictionary
        z[:2] + bytes([0x07]) + z[3:],            # block type 3
        z[:-4] + bytes([z[-4] ^ 0x80]) + z[-3:],  # wrong Adler-32
        b"\x78\x01\x01\x05\x00\xfb\xff" + b"abcde" + zlib.adler32(b"abcde").to_bytes(4, "big"),   # stored, LEN/NLEN agree
        b"\x78\x01\x01\x05\x00\xfa\xff" + b"abcde" + zlib.adler32(b"abcde").to_bytes(4, "big"),   # stored, NLEN wrong
    ]
    for c in cases:
        _check(inflate, zlib_status, c, len(raw) if c[2:3] != b"\x01" else 5)


def test_row_blocks_in_parallel(zlib_status):
    """pivb_zlib_blocks_decode: a pack-2 style run of size-prefixed row streams,
    inflated on several threads, equals zlib row by row; the first damaged block
    by index is the one reported; a bad size prefix is reported as such."""
    import struct

    from pivtools_b200 import _lib

    L = _lib.lavision_lib()
    rng = np.random.default_rng(7)
    rows = [np.clip(rng.normal(120, 40, 512), 0, 65535).astype(np.uint16).tobytes() for _ in range(96)]
    comp = [zlib.compress(r, int(rng.integers(1, 10))) for r in rows]

    def run(blocks, skip_before, n_blocks, skip_after, threads):
        body = b"".join(struct.pack("<i", len(c)) + c for c in blocks)
        buf = np.frombuffer(body, np.uint8).copy()
        dst = np.zeros(max(1, n_blocks) * 1024, np.uint8)
        used, err = ctypes.c_longlong(0), ctypes.c_longlong(-1)
        rc = L.pivb_zlib_blocks_decode(buf.ctypes.data, buf.size, skip_before, n_blocks, skip_after, dst.ctypes.data,
                                       1024, threads, ctypes.byref(used), ctypes.byref(err))
        return rc, dst, used.value, err.value, len(body)

    for threads in (1, 4, 16):
        rc, dst, used, err, total = run(comp, 8, 80, 8, threads)
        assert rc == 0 and used == total
        assert dst.tobytes() == b"".join(rows[8:88])
    bad = list(comp)
    for k in (30, 50):
        z = bytearray(bad[k])
        z[len(z) // 2] ^= 0x10
        bad[k] = bytes(z)
    want = [zlib_status(bad[k], 1024)[0] for k in (30, 50)]
    assert any(want), "the flipped bits left both streams valid"
    rc, _, _, err, _ = run(bad, 8, 80, 8, 8)
    first = 30 if want[0] else 50
    assert rc == 10 + zlib_status(bad[first], 1024)[0] and err == first - 8
    # a size prefix that runs past the buffer
    body = b"".join(struct.pack("<i", len(c)) + c for c in comp[:40]) + struct.pack("<i", 10 ** 6) + comp[40]
    buf = np.frombuffer(body, np.uint8).copy()
    dst = np.zeros(96 * 1024, np.uint8)
    used, err = ctypes.c_longlong(0), ctypes.c_longlong(-1)
    rc = L.pivb_zlib_blocks_decode(buf.ctypes.data, buf.size, 0, 41, 0, dst.ctypes.data, 1024, 4,
                                   ctypes.byref(used), ctypes.byref(err))
    assert rc == -2 and err.value == 40
