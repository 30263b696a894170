"""Launch the reference's own bitshuffle + LZ4 kernels (checker and baseline).

Test infrastructure: imported only by tests/ and bench.py's baseline legs.
The kernels come from ``oracle/_ref/bslz4.cubin`` (built by
``build_bslz4.py`` from the reference's source). This file holds the launch
sequences of the reference's writer (io/save.py:166-200, 285-365: forward bit
shuffle, per-block LZ4, chunk packing) and reader (io/load.py:3271-3320: LZ4
blocks, then the u16 unshuffle), for frames whose byte size is a multiple of
the 8192-byte block.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from .build_bslz4 import CUBIN, available

BLOCK = 8192
MAX_OUT = 2 * BLOCK  # lz4_compress_kernel's per-block output stride


def _check(res):
    err = res[0] if isinstance(res, tuple) else res
    if int(err) != 0:
        raise RuntimeError(f"CUDA driver call failed: {err}")
    return res[1:] if isinstance(res, tuple) and len(res) > 1 else None


class ReferenceBslz4:
    def __init__(self, device: torch.device | str = "cuda:0"):
        if not available():
            raise FileNotFoundError(f"{CUBIN} is missing: run python -m oracle.ref_cuda.build_bslz4")
        from cuda.bindings import driver as cu

        self.cu = cu
        self.device = torch.device(device)
        torch.cuda.set_device(self.device)
        torch.zeros(1, device=self.device)
        (self.module,) = _check(cu.cuModuleLoad(str(CUBIN).encode()))
        self.fn = {}
        for name in ("bitshuffle_fwd_8192_16", "lz4_compress_kernel", "pack_h5_chunks_kernel",
                     "h5lz4dc_batched", "shuf_8192_16_batched"):
            (self.fn[name],) = _check(cu.cuModuleGetFunction(self.module, name.encode()))

    def _launch(self, name, grid, block, args):
        stream = self.cu.CUstream(torch.cuda.current_stream(self.device).cuda_stream)
        values = tuple(a[0] for a in args)
        types = tuple(a[1] for a in args)
        _check(self.cu.cuLaunchKernel(self.fn[name], *grid, *block, 0, stream, (values, types), 0))

    def encode(self, frames: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
        """uint16 CUDA frames [n, K0, K1] -> (packed uint8 CUDA, int64 CUDA chunk starts)."""
        P, U32, U64 = ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint64
        n = int(frames.shape[0])
        frame_bytes = 2 * int(frames[0].numel())
        assert frame_bytes % BLOCK == 0 and n < 65536
        n_8kb = frame_bytes // BLOCK
        n_blocks = n * n_8kb
        frames = frames.contiguous()
        shuffled = torch.empty(n * frame_bytes, dtype=torch.uint8, device=self.device)
        self._launch("bitshuffle_fwd_8192_16", (n_8kb, 16, n), (256, 1, 1),
                     [(frames.data_ptr(), P), (shuffled.data_ptr(), P), (frame_bytes, U32)])
        comp = torch.empty(n_blocks * MAX_OUT, dtype=torch.uint8, device=self.device)
        sizes = torch.empty(n_blocks, dtype=torch.int32, device=self.device)
        self._launch("lz4_compress_kernel", (n_blocks, 1, 1), (32, 1, 1),
                     [(shuffled.data_ptr(), P), (comp.data_ptr(), P), (sizes.data_ptr(), P),
                      (BLOCK, U32), (n_blocks, U32)])
        chunk = sizes.view(n, n_8kb).to(torch.int64).sum(dim=1) + 12 + 4 * n_8kb
        starts = torch.zeros(n + 1, dtype=torch.int64, device=self.device)
        starts[1:] = torch.cumsum(chunk, dim=0)
        packed = torch.empty(int(starts[-1]), dtype=torch.uint8, device=self.device)
        self._launch("pack_h5_chunks_kernel", (n, 1, 1), (256, 1, 1),
                     [(comp.data_ptr(), P), (sizes.data_ptr(), P), (starts.data_ptr(), P),
                      (packed.data_ptr(), P), (n, U32), (n_8kb, U32), (MAX_OUT, U32),
                      (frame_bytes, U64), (BLOCK, U32)])
        torch.cuda.synchronize(self.device)
        return packed, starts[:-1].clone()

    def decode(self, packed: torch.Tensor, offsets: torch.Tensor, frame_shape) -> torch.Tensor:
        """The reference reader: block starts walked on the host (as load.py
        does from the chunk headers), LZ4 blocks, then the u16 unshuffle."""
        run, out = self.prepare_decode(packed, offsets, frame_shape)
        run()
        torch.cuda.synchronize(self.device)
        return out

    def prepare_decode(self, packed: torch.Tensor, offsets: torch.Tensor, frame_shape):
        """Host walk and uploads once; returns (launch the two kernels, output)."""
        P, U32 = ctypes.c_void_p, ctypes.c_uint
        n = int(offsets.numel())
        frame_bytes = 2 * int(frame_shape[0]) * int(frame_shape[1])
        assert frame_bytes % BLOCK == 0 and n < 65536
        n_8kb = frame_bytes // BLOCK
        host = packed.cpu().numpy()
        offs = offsets.cpu().numpy()
        starts = np.empty(n * n_8kb, np.uint32)
        for c in range(n):
            pos = 12
            for b in range(n_8kb):
                starts[c * n_8kb + b] = pos
                pos += 4 + int.from_bytes(host[offs[c] + pos:offs[c] + pos + 4].tobytes(), "big")
        d = self.device
        chunk_offsets = torch.as_tensor(offs.astype(np.uint64).view(np.int64), device=d)
        block_starts = torch.as_tensor(starts.view(np.int32), device=d)
        counts = torch.full((n,), n_8kb, dtype=torch.int32, device=d)
        block_offsets = torch.arange(0, n * n_8kb, n_8kb, dtype=torch.int32, device=d)
        lz = torch.empty(n * frame_bytes, dtype=torch.uint8, device=d)
        out = torch.empty((n, *frame_shape), dtype=torch.uint16, device=d)
        keep = (chunk_offsets, block_starts, counts, block_offsets, lz)

        def run():
            _ = keep
            self._launch("h5lz4dc_batched", ((n_8kb + 1) // 2, 1, n), (32, 2, 1),
                         [(packed.data_ptr(), P), (chunk_offsets.data_ptr(), P),
                          (block_starts.data_ptr(), P), (counts.data_ptr(), P),
                          (block_offsets.data_ptr(), P), (BLOCK, U32), (frame_bytes, U32),
                          (lz.data_ptr(), P)])
            self._launch("shuf_8192_16_batched", (n_8kb, 1, n), (256, 1, 1),
                         [(lz.data_ptr(), P), (out.data_ptr(), P), (frame_bytes, U32)])

        return run, out
