"""HDF5 bitshuffle + LZ4 chunks of u16 detector frames, decoded on the B200.

The step before the SSB path: the reference loads acquisitions stored one
detector frame per HDF5 chunk with the bitshuffle+LZ4 filter and decodes the
raw chunk bytes on the GPU (io/load.py:3271-3320, io/backends/cuda/
decoder.py:258-403 of bobleesj/quantem.gpu). Reading the chunks out of the
HDF5 container (``h5py``'s ``read_direct_chunk``) is the caller's; these
functions take the raw chunk bytes, decode them with ``qssb_decode_bslz4_u16``
into a u16 device tensor ready for ``SSB.from_array``, and write them with
``qssb_encode_bslz4_u16`` (the reference's save path, io/save.py).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .ops import _call, _ptr, _stream

STATUS = {0: "ok", 1: "bad header", 2: "block runs past the chunk", 3: "malformed LZ4 block"}


def _device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("the B200 SSB engine needs a CUDA device (it has no CPU path)")
    return torch.device("cuda", torch.cuda.current_device())


def decode_bslz4(compressed: torch.Tensor, chunk_offsets: torch.Tensor,
                 frame_shape: tuple[int, int], *, check: bool = True) -> torch.Tensor:
    """Decode chunks (concatenated uint8 CUDA bytes; int64 CUDA chunk starts)
    into a uint16 CUDA tensor [n_chunks, *frame_shape]."""
    if compressed.dtype != torch.uint8 or not compressed.is_cuda or compressed.ndim != 1:
        raise ValueError("compressed must be a 1D uint8 CUDA tensor")
    if chunk_offsets.dtype != torch.int64 or not chunk_offsets.is_cuda:
        raise ValueError("chunk_offsets must be an int64 CUDA tensor")
    n = int(chunk_offsets.numel())
    k0, k1 = (int(x) for x in frame_shape)
    out = torch.empty((n, k0, k1), dtype=torch.uint16, device=compressed.device)
    status = torch.empty(n, dtype=torch.int32, device=compressed.device)
    _call("qssb_decode_bslz4_u16", compressed.device, _ptr(compressed), int(compressed.numel()),
          _ptr(chunk_offsets.contiguous()), n, 2 * k0 * k1, _ptr(out), _ptr(status),
          _stream(compressed))
    if check:
        bad = torch.nonzero(status).flatten()
        if bad.numel():
            first = int(bad[0])
            raise ValueError(f"{bad.numel()} chunk(s) failed to decode; chunk {first}: "
                             f"{STATUS.get(int(status[first]), 'error')}")
    return out


def from_chunks(chunks: list[bytes], frame_shape: tuple[int, int],
                device: torch.device | str | None = None) -> torch.Tensor:
    """Upload raw chunk bytes (e.g. from ``read_direct_chunk``) and decode them."""
    dev = torch.device(device) if device is not None else _device()
    offsets = np.zeros(len(chunks), np.int64)
    np.cumsum([len(c) for c in chunks[:-1]], out=offsets[1:])
    data = torch.as_tensor(np.frombuffer(b"".join(chunks), np.uint8).copy()).to(dev)
    return decode_bslz4(data, torch.as_tensor(offsets, device=dev), frame_shape)


def encode_bslz4(frames: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    """Compress uint16 CUDA frames [n, K0, K1] into (packed uint8 CUDA bytes,
    int64 CUDA chunk starts), one chunk per frame."""
    if frames.dtype != torch.uint16 or not frames.is_cuda or frames.ndim != 3:
        raise ValueError("frames must be a uint16 CUDA tensor [n, K0, K1]")
    frames = frames.contiguous()
    n = int(frames.shape[0])
    chunk_bytes = 2 * int(frames.shape[1]) * int(frames.shape[2])
    nbytes = ctypes.c_size_t(0)
    _lib.check(_lib.load().qssb_encode_bslz4_scratch_bytes(n, chunk_bytes, ctypes.byref(nbytes)))
    scratch = torch.empty(int(nbytes.value), dtype=torch.uint8, device=frames.device)
    sizes = torch.empty(n, dtype=torch.int64, device=frames.device)
    _call("qssb_encode_bslz4_u16", frames.device, _ptr(frames), n, chunk_bytes, _ptr(scratch),
          _ptr(sizes), _stream(frames))
    offsets = torch.zeros(n, dtype=torch.int64, device=frames.device)
    offsets[1:] = torch.cumsum(sizes[:-1], dim=0)
    total = int(offsets[-1] + sizes[-1])
    packed = torch.empty(total, dtype=torch.uint8, device=frames.device)
    _call("qssb_pack_bslz4", frames.device, _ptr(scratch), _ptr(frames), n, chunk_bytes,
          _ptr(offsets), _ptr(packed), _stream(frames))
    return packed, offsets
