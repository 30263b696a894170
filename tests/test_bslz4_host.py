"""The bitshuffle + LZ4 chunk oracle on the CPU: hand-assembled LZ4 blocks
(overlapping matches, extended lengths), malformed streams rejected, bit
shuffle against an element-by-element statement, and chunk round trips with
full, tail and leftover blocks."""
from __future__ import annotations

import struct

import numpy as np
import pytest

from oracle import bslz4_oracle as bo


def test_lz4_known_blocks():
    # literals "abc", then a 9-byte match at offset 3 (overlapping), then "xyz12"
    blk = bytes([0x35]) + b"abc" + struct.pack("<H", 3) + bytes([0x50]) + b"xyz12"
    assert bo.lz4_decompress(blk, 17) == b"abcabcabcabcxyz12"
    # offset 1 run with an extended match length: 1 literal + (4 + 15 + 300) bytes
    blk = bytes([0x1F, 0x00]) + struct.pack("<H", 1) + bytes([255, 45]) + bytes([0x50]) + b"tail!"
    out = bo.lz4_decompress(blk, 1 + 319 + 5)
    assert out == b"\x00" * 320 + b"tail!"
    # extended literal length (15 + 20 literals), literals only
    lit = bytes(range(35))
    assert bo.lz4_decompress(bytes([0xF0, 20]) + lit, 35) == lit


@pytest.mark.parametrize("bad", [
    bytes([0x35]) + b"abc" + struct.pack("<H", 9) + bytes([0x50]) + b"xyz12",   # offset beyond output
    bytes([0x35]) + b"ab",                                                       # truncated literals
    bytes([0x35]) + b"abc" + struct.pack("<H", 0) + bytes([0x50]) + b"xyz12",   # zero offset
    bytes([0xF0]),                                                               # truncated length
])
def test_lz4_rejects_malformed(bad):
    with pytest.raises(ValueError):
        bo.lz4_decompress(bad, 17)


def test_bitshuffle_layout():
    rng = np.random.default_rng(0)
    v = rng.integers(0, 65536, 64, dtype=np.uint16)
    data = np.frombuffer(bo.bitshuffle(v), np.uint8)
    n = v.size
    for b in range(16):
        for k in range(n // 8):
            byte = 0
            for j in range(8):
                byte |= ((int(v[8 * k + j]) >> b) & 1) << j
            assert data[b * (n // 8) + k] == byte
    np.testing.assert_array_equal(bo.bitunshuffle(bo.bitshuffle(v), n, np.uint16), v)


@pytest.mark.parametrize("shape", [(64, 64), (96, 96), (3, 5), (40, 41), (192, 192)])
def test_chunk_round_trip(shape):
    rng = np.random.default_rng(shape[0] * 1000 + shape[1])
    frame = rng.poisson(0.3, shape).astype(np.uint16)
    frame[rng.random(shape) < 0.01] = rng.integers(0, 65536, int((rng.random(shape) < 0.01).sum()) or 1,
                                                   dtype=np.uint16)[0]
    chunk = bo.encode_chunk(frame)
    assert struct.unpack(">QI", chunk[:12]) == (frame.size * 2, 8192)
    np.testing.assert_array_equal(bo.decode_chunk(chunk).reshape(shape), frame)
    if frame.size >= 4096:
        assert len(chunk) < frame.nbytes // 2  # sparse counts compress
