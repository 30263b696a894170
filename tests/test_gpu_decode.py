"""HDF5 bitshuffle + LZ4 chunks on the GPU (qssb_decode_bslz4_u16,
qssb_encode_bslz4_u16 / qssb_pack_bslz4): round trips over full, tail and
leftover blocks; chunks written by the oracle and by the reference's own
writer kernels decode bit for bit, ours decode with the oracle's and the
reference's readers; malformed chunks are reported per chunk without a
fault; decoded counts reconstruct exactly as the originals."""
from __future__ import annotations

import struct

import numpy as np
import pytest
import torch

from oracle import bslz4_oracle as bo
from oracle.ref_cuda import build_bslz4
from quantem.gpu_b200 import SSB
from quantem.gpu_b200.decode import decode_bslz4, encode_bslz4, from_chunks
from quantem.gpu_b200.synthetic import CONFIGS, generate

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _frames(n, shape, seed=0, dense=False):
    rng = np.random.default_rng(seed)
    f = rng.poisson(0.4, (n, *shape)).astype(np.uint16)
    if dense:
        f = rng.integers(0, 65536, (n, *shape), dtype=np.uint16)
    else:
        hot = rng.random((n, *shape)) < 0.002
        f[hot] = rng.integers(1000, 65536, int(hot.sum()), dtype=np.uint16)
    return f


@pytest.mark.parametrize("shape", [(128, 128), (96, 96), (192, 192), (3, 5), (41, 40), (64, 63)])
@pytest.mark.parametrize("dense", [False, True])
def test_round_trip_and_oracle_interchange(shape, dense):
    frames = _frames(6, shape, seed=shape[0] + shape[1], dense=dense)
    t = torch.as_tensor(frames, device=DEV)
    packed, offsets = encode_bslz4(t)
    np.testing.assert_array_equal(decode_bslz4(packed, offsets, shape).cpu().numpy(), frames)
    # our chunks through the oracle's reader
    host = packed.cpu().numpy().tobytes()
    offs = list(offsets.cpu().numpy()) + [len(host)]
    for i in range(len(frames)):
        np.testing.assert_array_equal(bo.decode_chunk(host[offs[i]:offs[i + 1]]).reshape(shape), frames[i])
    # the oracle's chunks through our reader
    chunks = [bo.encode_chunk(f) for f in frames[:3]]
    np.testing.assert_array_equal(from_chunks(chunks, shape, DEV).cpu().numpy(), frames[:3])


@pytest.mark.skipif(not build_bslz4.available(), reason="reference bitshuffle-LZ4 cubin not built")
@pytest.mark.parametrize("shape", [(128, 128), (192, 192)])
def test_reference_writer_and_reader_interchange(shape):
    from oracle.ref_cuda.bslz4 import ReferenceBslz4

    ref = ReferenceBslz4(DEV)
    frames = _frames(33, shape, seed=7)
    t = torch.as_tensor(frames, device=DEV)
    packed, offsets = ref.encode(t)
    np.testing.assert_array_equal(decode_bslz4(packed, offsets, shape).cpu().numpy(), frames)
    ours, our_offsets = encode_bslz4(t)
    np.testing.assert_array_equal(ref.decode(ours, our_offsets, shape).cpu().numpy(), frames)


def _corrupt(chunk: bytes, kind: str) -> bytes:
    if kind == "header":
        return struct.pack(">QI", 12345, 8192) + chunk[12:]
    if kind == "block_size":
        return chunk[:12] + struct.pack(">I", 0x7fffffff) + chunk[16:]
    if kind == "truncated":
        return chunk[: len(chunk) // 2]
    if kind == "lz4":  # first block replaced by literals 'abc' + a match at offset 9
        bad = bytes([0x35]) + b"abc" + struct.pack("<H", 9) + bytes([0x50]) + b"xyz12"
        (csz,) = struct.unpack(">I", chunk[12:16])
        return chunk[:12] + struct.pack(">I", len(bad)) + bad + chunk[16 + csz:]
    raise ValueError(kind)


@pytest.mark.parametrize("kind,code", [("header", 1), ("block_size", 2), ("truncated", 2), ("lz4", 3)])
def test_malformed_chunks_are_reported(kind, code):
    frames = _frames(3, (96, 96), seed=1)
    chunks = [bo.encode_chunk(f) for f in frames]
    chunks[1] = _corrupt(chunks[1], kind)
    offsets = np.zeros(3, np.int64)
    np.cumsum([len(c) for c in chunks[:-1]], out=offsets[1:])
    data = torch.as_tensor(np.frombuffer(b"".join(chunks), np.uint8).copy(), device=DEV)
    offs = torch.as_tensor(offsets, device=DEV)
    with pytest.raises(ValueError, match="chunk 1"):
        decode_bslz4(data, offs, (96, 96))
    out = decode_bslz4(data, offs, (96, 96), check=False).cpu().numpy()
    np.testing.assert_array_equal(out[0], frames[0])
    np.testing.assert_array_equal(out[2], frames[2])
    # the same call again: the context is intact
    assert torch.cuda.synchronize() is None


def test_decoded_acquisition_reconstructs_identically():
    spec = CONFIGS["plain_128x128_det128"]
    counts = generate(spec, DEV).counts
    packed, offsets = encode_bslz4(counts.reshape(-1, 128, 128))
    decoded = decode_bslz4(packed, offsets, (128, 128)).reshape(counts.shape)
    assert torch.equal(decoded.view(torch.int16), counts.view(torch.int16))
    assert packed.numel() < counts.numel() * 2 // 3  # sparse counts compress
    kw = dict(voltage_kV=spec.voltage_kV, semiangle_mrad=spec.semiangle_mrad,
              scan_sampling_A=spec.scan_step_A, det_sampling=spec.det_sampling_mrad)
    a = SSB.from_array(counts, **kw).reconstruct({"C10": 0.0, "C12": 0.0, "phi12": 0.0})
    b = SSB.from_array(decoded, **kw).reconstruct({"C10": 0.0, "C12": 0.0, "phi12": 0.0})
    assert torch.equal(a.object_wave, b.object_wave)


def test_ssb_from_chunks_matches_from_array():
    spec = CONFIGS["plain_32x32_det64"]
    counts = generate(spec, DEV).counts  # [32, 32, 64, 64] -> padded to 128^2 scans by the session
    kw = dict(voltage_kV=spec.voltage_kV, semiangle_mrad=spec.semiangle_mrad,
              scan_sampling_A=spec.scan_step_A, det_sampling=spec.det_sampling_mrad)
    packed, offsets = encode_bslz4(counts.reshape(-1, 64, 64))
    host = packed.cpu().numpy().tobytes()
    offs = list(offsets.cpu().numpy()) + [len(host)]
    chunks = [host[offs[i]:offs[i + 1]] for i in range(len(offs) - 1)]
    ab = {"C10": 50.0, "C12": 20.0, "phi12": 0.3}
    want = SSB.from_array(counts, **kw).reconstruct(ab).object_wave
    a = SSB.from_chunks(chunks, frame_shape=(64, 64), scan_shape=(32, 32), **kw).reconstruct(ab)
    b = SSB.from_chunks(packed.cpu().pin_memory(), chunk_offsets=offsets.cpu(), frame_shape=(64, 64),
                        scan_shape=(32, 32), **kw).reconstruct(ab)
    assert torch.equal(a.object_wave, want) and torch.equal(b.object_wave, want)
