"""LaVision DaVis decode on the host (libpivb_lavision codecs and the container
walk of pivtools_b200.lavision) against the reference reader's results and
LaVision's own lvpyio decodes (tests/golden/lavision_ref.npz, written by
tests/golden/make_golden.py lavision), plus the codecs' error behaviour.  The
GPU unpack is tested in test_lavision_gpu.py."""

import json
import os

import numpy as np
import pytest

from pivtools_b200 import lavision as LV

GOLD = os.path.join(os.path.dirname(__file__), "golden", "lavision_ref.npz")


@pytest.fixture(scope="module")
def gold():
    z = np.load(GOLD)
    return z, json.loads(str(z["meta"]))


def _write(tmp_path, name, arr):
    p = tmp_path / f"{name}.im7"
    p.write_bytes(arr.tobytes())
    return p


def test_read_im7_equals_reference_on_every_pack(gold, tmp_path):
    z, meta = gold
    for case in meta["im7"]:
        name = case["name"]
        p = _write(tmp_path, name, z[name + "_file"])
        _, px, sc = LV.read_im7(p)
        ref = z[name + "_pixels"]
        assert px.dtype == ref.dtype and px.shape == ref.shape, name
        assert np.array_equal(px, ref), name
        assert sc.slope == case["slope"] and sc.offset == case["offset"], name


def test_lvpyio_fixtures(gold, tmp_path):
    """The reference's own pack-1 and version-1 pack-20 files, as LaVision's lvpyio
    decodes them."""
    z, meta = gold
    for name in meta["lvpyio"]:
        p = _write(tmp_path, name, z[f"lv_{name}_file"])
        _, px, _ = LV.read_im7(p)
        lv = z[f"lv_{name}_lvpyio"]
        assert np.array_equal(px.reshape(lv.shape), lv), name
        assert np.array_equal(px, z[f"lv_{name}_ref"]), name


def test_set_entry_payloads_every_codec(gold):
    z, meta = gold
    for case in meta["set"]:
        dec = case["decoder"]
        n = LV.set_payload_bytes(dec, case["width"], case["height"])
        payload = z[f"set_{dec}_payload"]
        assert n == payload.size
        for codec in ("", "Zlib", "LZ4", "IMX"):
            stored = z[f"set_{dec}_{codec or 'none'}_stored"].tobytes()
            got = LV.set_entry_payload(stored, codec, n)
            assert np.array_equal(got, payload), (dec, codec)


def test_set_decoder_refusals():
    with pytest.raises(ValueError, match="not implemented"):
        LV.set_payload_bytes("rgb-24", 4, 4)
    with pytest.raises(ValueError, match="Unknown"):
        LV.set_payload_bytes("mono-14p", 4, 4)
    with pytest.raises(ValueError, match="multiple of four"):
        LV.set_payload_bytes("mono-10p", 3, 3)
    with pytest.raises(ValueError, match="even number"):
        LV.set_payload_bytes("mono-12p", 3, 3)
    with pytest.raises(ValueError, match="odd count"):
        LV.set_entry_payload(b"\x00", "IMX", 15)


def _tok(data, npix, prev=0, off=0):
    arr = np.frombuffer(bytes(data), np.uint8).copy()
    out = np.empty(npix, np.uint16)
    off, prev = LV.decode_tokens(arr, off, out, npix, prev, "t")
    return out, off, prev


def test_token_grammar_known_answers():
    # an absolute, int8 deltas, a run of two absolutes, two nibble runs (a high
    # nibble 8 is a delta of -8; only a low nibble 8 ends a run)
    out, off, prev = _tok([0x80, 0x88, 0x13, 0x05, 0xFE, 0x7F, 0x02, 0x10, 0x00, 0x20, 0x00,
                           0x81, 0x12, 0x88, 0x81, 0x8F, 0x78], 11)
    assert out.tolist() == [5000, 5005, 5003, 16, 32, 33, 35, 27, 19, 18, 25]
    assert off == 17 and prev == 25


def test_token_errors():
    with pytest.raises(LV.TruncatedTokenStreamError):
        _tok([0x80, 0x01], 1)
    with pytest.raises(LV.TokenRunOverrunError):
        _tok([0x7F, 0x03, 0, 0, 0, 0, 0, 0], 2)
    with pytest.raises(LV.TokenValueRangeError):
        _tok([0xFF], 1)                      # 0 - 1
    with pytest.raises(LV.TrailingTokenBytesError):
        LV.set_entry_payload(bytes([0x01, 0x01, 0x00]), "IMX", 4)


def test_token_stream_round_trip():
    import lavision_oracle as LO

    rng = np.random.default_rng(5)
    v = np.clip(np.cumsum(rng.integers(-9, 10, 5000)) + 3000, 0, 65535).astype(np.uint16)
    v[::97] = rng.integers(0, 65535, v[::97].size)
    data, last = LO.tokens_encode(v, 0, rng)
    out, off, prev = _tok(data, v.size)
    assert np.array_equal(out, v) and off == len(data) and prev == last


def test_lz4_round_trip_and_overlapping_matches():
    import lavision_oracle as LO

    rng = np.random.default_rng(6)
    for t in range(20):
        n = int(rng.integers(1, 20000))
        base = rng.integers(0, 256, max(1, n // 50)).astype(np.uint8)
        d = np.resize(base, n) if t % 3 else rng.integers(0, 4, n).astype(np.uint8)
        raw = d.tobytes()
        blk = LO.lz4_encode(raw)
        assert LV.lz4_block_decompress(blk, len(raw)) == raw
    # an overlapping match (offset 1, length 20): run-length of one byte
    blk = bytes([0x1F, 0x41, 0x01, 0x00, 0x01, 0x50]) + b"BCDEF"
    out = LV.lz4_block_decompress(blk, 1 + 20 + 5)
    assert out == b"A" * 21 + b"BCDEF"


def test_lz4_errors():
    with pytest.raises(IOError):
        LV.lz4_block_decompress(bytes([0x10, 0x41, 0x05, 0x00]), 10)     # offset beyond the output
    with pytest.raises(IOError):
        LV.lz4_block_decompress(bytes([0x50, 0x41]), 5)                 # literals cut off
    with pytest.raises(IOError):
        LV.lz4_block_decompress(bytes([0x30]) + b"abc", 4)             # short output


def test_zlib_exact_ends():
    import zlib

    raw = bytes(range(200)) * 3
    z = zlib.compress(raw)
    assert LV.set_entry_payload(z, "Zlib", len(raw)).tobytes() == raw
    with pytest.raises(IOError, match="more than"):
        LV.set_entry_payload(z, "Zlib", len(raw) - 1)
    with pytest.raises(IOError, match="fewer"):
        LV.set_entry_payload(z, "Zlib", len(raw) + 1)
    with pytest.raises(IOError, match="truncated"):
        LV.set_entry_payload(z[:-6], "Zlib", len(raw))
    with pytest.raises(IOError, match="follow"):
        LV.set_entry_payload(z + b"\x00", "Zlib", len(raw))


def test_header_refusals(tmp_path):
    import lavision_oracle as LO

    fr = np.zeros((1, 1, 4, 4), np.uint16)
    bad = bytearray(LO.im7_pack0(fr, LO.im7_attributes()))
    bad[0:2] = (2).to_bytes(2, "little")            # version 2
    p = tmp_path / "v2.im7"
    p.write_bytes(bytes(bad))
    with pytest.raises(ValueError, match="version 2"):
        LV.read_im7(p)
    bad = bytearray(LO.im7_pack0(fr, LO.im7_attributes()))
    bad[2:4] = (3).to_bytes(2, "little")            # pack 3
    p.write_bytes(bytes(bad))
    with pytest.raises(ValueError, match="pack_type 3"):
        LV.read_im7(p)
    good = LO.im7_pack0(fr, LO.im7_attributes())
    p.write_bytes(good[:-20])                       # a record cut off: the decode did not end right
    with pytest.raises(IOError, match="attribute records"):
        LV.read_im7(p)


def test_host_reader_restatement_matches_reference(gold, tmp_path):
    """The oracle's host reader (the ingest measurement's CPU baseline) equals the
    reference reader's float32 camera frames on the pack-0 and pack-2 fixtures."""
    import lavision_oracle as LO

    z, meta = gold
    n = 0
    for case in meta["im7"]:
        name = case["name"]
        if not name.startswith(("p0_", "p2_")):
            continue
        p = _write(tmp_path, name, z[name + "_file"])
        for i, (cam, fpc, nfr) in enumerate(case["cams"]):
            got = LO.read_im7_camera_host(p, cam, fpc, nfr)
            assert got.dtype == np.float32 and np.array_equal(got, z[f"{name}_cam{i}"]), (name, i)
            n += 1
    assert n >= 6
