"""HDF5 bitshuffle + LZ4 chunks in pure Python/numpy (TEST INFRASTRUCTURE).

Restates the chunk format the reference reads and writes
(io/backends/cuda/decoder.py:258-281 and :957-1003, io/load.py:3271-3320 of
bobleesj/quantem.gpu; the HDF5 bitshuffle filter with LZ4, whose third-party
implementation is not vendored in the reference): a 12-byte header
(big-endian uint64 uncompressed bytes, big-endian uint32 block bytes, 8192),
then per block a big-endian uint32 compressed size and an LZ4 block; each
block holds the bit-shuffled elements of `block bytes` (the last block the
rest, rounded down to a multiple of 8 elements); elements beyond the last
multiple of 8 follow uncompressed. Bit shuffle (decoder.py:322-369): within
a block of n elements of `size` bytes, bit plane b (bit b of the element,
least significant first) is n/8 bytes; byte k of plane b holds bit b of
elements 8k..8k+7, element 8k+j in bit j.

LZ4 block format (the published LZ4 specification): sequences of a token
(high nibble literal length, low nibble match length - 4; 15 extends with
bytes summed until one is below 255), the literals, a little-endian 16-bit
offset and the match; the last sequence is literals only.
"""
from __future__ import annotations

import struct

import numpy as np

BLOCK_BYTES = 8192


# ------------------------------------------------------------ bit shuffle
def bitshuffle(values: np.ndarray) -> bytes:
    """Bit-plane transpose of n elements (n a multiple of 8)."""
    v = np.ascontiguousarray(values)
    size = v.dtype.itemsize
    n = v.size
    assert n % 8 == 0
    bits = np.unpackbits(v.view(np.uint8).reshape(n, size), axis=1, bitorder="little")  # [n][8*size]
    planes = bits.T.reshape(8 * size, n)  # plane b = bit b (little-endian byte order)
    return np.packbits(planes.reshape(8 * size, n // 8, 8), axis=2, bitorder="little").tobytes()


def bitunshuffle(data: bytes, n: int, dtype) -> np.ndarray:
    size = np.dtype(dtype).itemsize
    planes = np.unpackbits(np.frombuffer(data, np.uint8).reshape(8 * size, n // 8, 1), axis=2,
                           bitorder="little").reshape(8 * size, n)
    by = np.packbits(planes.T.reshape(n, size, 8), axis=2, bitorder="little").reshape(n * size)
    return by.view(dtype)


# -------------------------------------------------------------- LZ4 block
def lz4_decompress(src: bytes, out_size: int) -> bytes:
    """Decode one LZ4 block; raises ValueError on a malformed stream."""
    out = bytearray()
    i = 0
    n = len(src)
    while True:
        if i >= n:
            raise ValueError("truncated token")
        token = src[i]
        i += 1
        lit = token >> 4
        if lit == 15:
            while True:
                if i >= n:
                    raise ValueError("truncated literal length")
                b = src[i]
                i += 1
                lit += b
                if b != 255:
                    break
        if i + lit > n or len(out) + lit > out_size:
            raise ValueError("literal run out of bounds")
        out += src[i:i + lit]
        i += lit
        if i == n:
            break
        if i + 2 > n:
            raise ValueError("truncated offset")
        off = src[i] | (src[i + 1] << 8)
        i += 2
        ml = (token & 15) + 4
        if (token & 15) == 15:
            while True:
                if i >= n:
                    raise ValueError("truncated match length")
                b = src[i]
                i += 1
                ml += b
                if b != 255:
                    break
        if off == 0 or off > len(out) or len(out) + ml > out_size:
            raise ValueError("match out of bounds")
        start = len(out) - off
        for j in range(ml):
            out.append(out[start + j])
    if len(out) != out_size:
        raise ValueError("decoded size mismatch")
    return bytes(out)


def _len_bytes(x: int) -> bytes:
    out = bytearray()
    while x >= 255:
        out.append(255)
        x -= 255
    out.append(x)
    return bytes(out)


def lz4_compress(src: bytes) -> bytes:
    """A greedy LZ4 block compressor (4-byte hash matches, the format's end
    rules: the last 5 bytes are literals, no match starts in the last 12)."""
    n = len(src)
    out = bytearray()
    table: dict[bytes, int] = {}
    anchor = 0
    i = 0
    limit = n - 12
    while i < limit:
        key = src[i:i + 4]
        cand = table.get(key)
        table[key] = i
        if cand is not None and i - cand <= 0xFFFF:
            m = 4
            while i + m < n - 5 and src[cand + m] == src[i + m]:
                m += 1
            lit = i - anchor
            tok_l = min(lit, 15)
            tok_m = min(m - 4, 15)
            out.append((tok_l << 4) | tok_m)
            if lit >= 15:
                out += _len_bytes(lit - 15)
            out += src[anchor:i]
            out += struct.pack("<H", i - cand)
            if m - 4 >= 15:
                out += _len_bytes(m - 4 - 15)
            i += m
            anchor = i
        else:
            i += 1
    lit = n - anchor
    out.append(min(lit, 15) << 4)
    if lit >= 15:
        out += _len_bytes(lit - 15)
    out += src[anchor:]
    return bytes(out)


# ------------------------------------------------------------------ chunks
def encode_chunk(frame: np.ndarray, block_bytes: int = BLOCK_BYTES) -> bytes:
    """One HDF5 bitshuffle+LZ4 chunk of a frame."""
    v = np.ascontiguousarray(frame).reshape(-1)
    size = v.dtype.itemsize
    total = v.size * size
    out = bytearray(struct.pack(">QI", total, block_bytes))
    per_block = block_bytes // size
    n8 = (v.size // 8) * 8
    pos = 0
    while pos < n8:
        cnt = min(per_block, n8 - pos)
        comp = lz4_compress(bitshuffle(v[pos:pos + cnt]))
        out += struct.pack(">I", len(comp)) + comp
        pos += cnt
    out += v[n8:].tobytes()
    return bytes(out)


def decode_chunk(chunk: bytes, dtype=np.uint16) -> np.ndarray:
    total, block_bytes = struct.unpack(">QI", chunk[:12])
    size = np.dtype(dtype).itemsize
    n = total // size
    per_block = block_bytes // size
    n8 = (n // 8) * 8
    out = np.empty(n, dtype)
    pos, i = 0, 12
    while pos < n8:
        cnt = min(per_block, n8 - pos)
        (csz,) = struct.unpack(">I", chunk[i:i + 4])
        raw = lz4_decompress(chunk[i + 4:i + 4 + csz], cnt * size)
        out[pos:pos + cnt] = bitunshuffle(raw, cnt, dtype)
        i += 4 + csz
        pos += cnt
    out[n8:] = np.frombuffer(chunk[i:i + (n - n8) * size], dtype)
    return out


def pack(chunks: list[bytes]) -> tuple[np.ndarray, np.ndarray]:
    """Concatenated chunk bytes (uint8) and each chunk's start (int64)."""
    offsets = np.zeros(len(chunks), np.int64)
    pos = 0
    for i, c in enumerate(chunks):
        offsets[i] = pos
        pos += len(c)
    return np.frombuffer(b"".join(chunks), np.uint8).copy(), offsets
