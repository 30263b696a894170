"""Error behaviour of the backend that callers rely on (backend.py:808-816,
:1078-1086, :1347-1354 of the reference): a device allocation failure during
a reconstruction or an optimisation surfaces as an actionable
``MemoryError``, and the grid search retries a failed batch in halves.

The allocation failure is made on the host (a stand-in that raises torch's
``OutOfMemoryError``); no device memory is exhausted.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from quantem.gpu_b200 import B200SSBBackend
from quantem.gpu_b200.synthetic import CONFIGS, generate

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _oom(*args, **kwargs):
    raise torch.cuda.OutOfMemoryError("CUDA out of memory (simulated on the host)")


@pytest.fixture()
def backend():
    counts = generate(CONFIGS["plain_32x32_det64"], device=DEV).counts
    be = B200SSBBackend(counts, semiangle=20.0, scan_sampling=0.5, det_sampling=20.0 / 12.0,
                        voltage_kV=300, device=DEV)
    yield be
    be.close()


def test_reconstruction_oom_becomes_memory_error(backend, monkeypatch):
    monkeypatch.setattr(backend, "reconstruct_object", _oom)
    with pytest.raises(MemoryError, match=r"during SSB reconstruction \(437 BF pixels"):
        backend.result(compute_loss=False)


def test_optimization_oom_becomes_memory_error(backend, monkeypatch):
    monkeypatch.setattr(backend, "_evaluate", _oom)
    with pytest.raises(MemoryError, match="during SSB optimization"):
        backend.optimize(n_trials=16, verbose=False)
    with pytest.raises(MemoryError, match="bf_radius=<smaller>"):
        backend.refine(verbose=False)


def test_grid_search_retries_failed_batches_in_halves(backend, monkeypatch):
    ref = B200SSBBackend.grid_search(backend, window={"C10_nm": 40}, verbose=False)
    want = dict(ref.aberrations), ref._best_loss
    real = backend._evaluate
    sizes = []

    def flaky(x):
        sizes.append(len(x))
        if len(x) > 100:
            _oom()
        return real(x)

    backend.aberrations.update(C10=0.0, C12=0.0, phi12=0.0)
    monkeypatch.setattr(backend, "_evaluate", flaky)
    backend.grid_search(window={"C10_nm": 40}, verbose=False)
    # 3003 grid points: 256-candidate batches fail, their 128-halves fail, the
    # 64-quarters run; the last 187-candidate batch runs as 94 + 93
    assert max(sizes) == 256 and 64 in sizes and 94 in sizes and 93 in sizes
    assert backend._best_loss == pytest.approx(want[1], rel=1e-6)
    for k in ("C10", "C12", "phi12"):
        assert backend.aberrations[k] == pytest.approx(want[0][k], abs=1e-9)
    # a single candidate that still fails is not retried forever
    monkeypatch.setattr(backend, "_evaluate", _oom)
    with pytest.raises(MemoryError, match="during SSB grid search"):
        backend.grid_search(window={"C10_nm": 40}, verbose=False)
    assert np.isfinite(backend._best_loss)
