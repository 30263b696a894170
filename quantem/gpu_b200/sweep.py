"""Batched aberration sweeps over several scans in one CUDA-graph launch.

The reference scores candidates scan by scan, one CuPy launch sequence (and
host sync) per batch (backend.py:1261-1374, engine.py:2120-2295). Here the
prepared scans (each a resident ``B200SSBBackend``, uneven sizes padded by the
reference's rule to 128^2 or 256^2) get fixed device buffers for their
candidates, losses and workspaces; every scan's loss launches (at 128^2 the
chi-phase table and the pair kernel, which folds in its last CTA; at 256^2 the
set-up, one persistent kernel for the row and column passes over every
L2-sized BF chunk, and the fold) are
captured once into one CUDA graph, and a sweep step is: copy the candidates
in, replay the graph, read the losses out. ``launches_per_replay`` is the
library's own count of the kernels captured (``qssb_kernel_launches``).
The work partition of each scan's loss kernel is chosen by the autotuner
(``autotune.tune_loss``) before capture. By default (``persistent=True``)
each 256^2 scan's row and column passes run as one persistent launch
(``QSSB_FLAG_PERSISTENT``): four kernels for that scan instead of two per BF
chunk, the same losses to float32 rounding, and faster with C30 candidates;
``persistent=False`` keeps the launch sequence.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib, autotune, ops
from ._lib import QSSB_FLAG_PERSISTENT, QSSB_FLAG_QUADRATIC


class MultiScanSweep:
    """Scores ``n_cand`` candidates (C10, C12, phi12, C30) per scan, all scans
    in one graph replay."""

    def __init__(self, backends, n_cand: int | list[int], *, quadratic: bool = False,
                 tune: bool = True, persistent: bool = True):
        if not backends:
            raise ValueError("at least one prepared scan is needed")
        self.backends = list(backends)
        counts = [n_cand] * len(self.backends) if isinstance(n_cand, int) else list(n_cand)
        if len(counts) != len(self.backends) or min(counts) < 1:
            raise ValueError("n_cand must be a positive count per scan")
        for be in self.backends:
            be._require_loss_size()
        self.device = self.backends[0].device
        self.quadratic = bool(quadratic)
        self._slots = []
        for be, n in zip(self.backends, counts):
            cal = be._calibration()
            flags = (be._flags | (QSSB_FLAG_QUADRATIC if quadratic else 0)
                     | (QSSB_FLAG_PERSISTENT if persistent else 0))
            cands = torch.zeros((n, 4), dtype=torch.float32, device=self.device)
            cands[:, 0] = torch.linspace(-100.0, 100.0, n, device=self.device)
            ws = ops.Workspace(self.device)
            overlap = be._overlap_table()  # 128x128 scans: the table-driven pair kernel
            chunks = 0
            if tune:
                chunks = autotune.tune_loss(be.G_qk, be._geom_dev, be._q_row, be._q_col, cal,
                                            cands, flags, ws, overlap=overlap)
            flags |= _lib.flag_chunks(chunks)
            ws.get(ops.loss_workspace_bytes(cal, n, flags))
            out = torch.empty(n, dtype=torch.float32, device=self.device)
            self._slots.append(dict(be=be, cal=cal, flags=flags, cands=cands, ws=ws, out=out,
                                    chunks=chunks, overlap=overlap))
        self.host_cands = [torch.empty((s["cands"].shape[0], 4), dtype=torch.float32).pin_memory()
                           for s in self._slots]
        self.host_out = [torch.empty(s["out"].shape[0], dtype=torch.float32).pin_memory()
                         for s in self._slots]
        self._graph = None
        self.launches_per_replay = 0

    def _launch_all(self) -> None:
        for s in self._slots:
            be = s["be"]
            ops.loss_batch(be.G_qk, be._geom_dev, be._q_row, be._q_col, s["cal"], s["cands"],
                           flags=s["flags"], workspace=s["ws"], out=s["out"],
                           overlap=s["overlap"])

    def capture(self) -> None:
        """Record every scan's loss launches into one CUDA graph."""
        self._launch_all()  # warm-up outside capture: attributes, workspaces
        torch.cuda.synchronize(self.device)
        before = ops.LAUNCH_COUNT
        g = torch.cuda.CUDAGraph()
        stream = torch.cuda.Stream(self.device)
        stream.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.graph(g, stream=stream, capture_error_mode="relaxed"):
            self._launch_all()
        torch.cuda.synchronize(self.device)
        self.launches_per_replay = ops.LAUNCH_COUNT - before
        self._graph = g

    def set_candidates(self, candidates) -> None:
        """Host arrays [n_i, 4] (C10, C12, phi12, C30 in the reference's units)."""
        if len(candidates) != len(self._slots):
            raise ValueError("one candidate array per scan")
        for s, h, c in zip(self._slots, self.host_cands, candidates):
            c = np.asarray(c, dtype=np.float32)
            if c.shape != tuple(s["cands"].shape):
                raise ValueError(f"candidates must have shape {tuple(s['cands'].shape)}")
            if self.quadratic and np.any(c[:, 3]):
                raise ValueError("a quadratic sweep takes C30 == 0 candidates only")
            h.numpy()[:] = c
            s["cands"].copy_(h, non_blocking=True)

    def replay(self) -> None:
        """Score the current candidates of every scan (one graph launch)."""
        if self._graph is None:
            self.capture()
        self._graph.replay()

    def losses(self) -> list[np.ndarray]:
        for s, h in zip(self._slots, self.host_out):
            h.copy_(s["out"], non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        return [h.numpy().copy() for h in self.host_out]

    def __call__(self, candidates) -> list[np.ndarray]:
        self.set_candidates(candidates)
        self.replay()
        return self.losses()
