"""qssb_object_noalloc: the object entry point for callers that cannot allocate.

Some callers of this library cannot allocate device memory where they call
it: a host application whose own memory pool already owns the whole GPU, a
real-time acquisition loop that must not enter the CUDA allocator (an
allocation can synchronise the device and stall the stream), or a plugin
host that forbids third-party allocations. ``qssb_object_noalloc`` serves
them by keeping its scratch in a fixed 16 MiB array inside the library. These
tests call it through the C ABI and check it against ``qssb_object`` (caller
workspace) with the tolerance the other object tests use, on two calls in a
row, since every call reuses the same array.

The file sorts last so that a run stopping at the first failure has already
run every other test; it builds its own inputs and passes in a fresh process.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import pytest

from quantem.gpu_b200 import _lib


def _calibration(n: int, n_bf: int) -> _lib.Calibration:
    return _lib.Calibration(
        n_bf=n_bf, scan_rows=n, scan_cols=n, reserved=0, wavelength_A=0.019687489006849,
        semiangle_rad=0.0214, det_sampling_row_rad=1e-3, det_sampling_col_rad=1e-3,
        scan_sampling_row_A=0.5, scan_sampling_col_A=0.5, dc_re=1.0, dc_im=0.0)


def test_noalloc_rejects_requests_beyond_its_fixed_scratch():
    """Oversized requests fail before touching the device (no GPU needed)."""
    lib = _lib.load()
    cal = _calibration(256, 20000)
    need = ctypes.c_size_t()
    assert lib.qssb_object_workspace_bytes(ctypes.byref(cal), 0, ctypes.byref(need)) == 0
    assert need.value > _lib.QSSB_NOALLOC_SCRATCH_BYTES
    ab = _lib.Aberrations(0.0, 0.0, 0.0, 0.0)
    rc = lib.qssb_object_noalloc(None, None, None, None, ctypes.byref(cal), ctypes.byref(ab), 0,
                                 None, None, None)
    assert rc == _lib.QSSB_ERR_WORKSPACE
    assert b"16 MiB" in lib.qssb_last_error()


@pytest.mark.gpu
def test_noalloc_object_matches_workspace_object_twice():
    import torch

    from quantem.gpu_b200 import ops
    from quantem.gpu_b200.calibration import bf_geometry, scan_frequencies

    dev = torch.device("cuda:0")
    rng = np.random.default_rng(2024)
    n, det = 128, 32
    yy, xx = np.mgrid[:det, :det]
    disk = (yy - 15.5) ** 2 + (xx - 16.5) ** 2 <= 9.0 ** 2
    rows, cols = (a.astype(np.int32) for a in np.nonzero(disk))
    n_bf = rows.size
    images = rng.poisson(30.0, size=(n_bf, n, n)).astype(np.float64)
    g_half = np.fft.rfft2(images).astype(np.complex64)
    dc = float(images.sum(axis=(1, 2)).mean())
    geo = bf_geometry(rows, cols, (15.5, 16.5), (det, det), (0.6, 0.6), 0.019687489006849,
                      21.4, (1.0, 1.0), 0.1)
    q_row, q_col = scan_frequencies((n, n), (0.5, 0.5))
    cal = _calibration(n, n_bf)
    cal.dc_re = dc
    g = torch.as_tensor(g_half, device=dev)
    geom = torch.as_tensor(geo.stacked(), device=dev)
    qr = torch.as_tensor(q_row, device=dev)
    qc = torch.as_tensor(q_col, device=dev)
    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    for ab in (_lib.Aberrations(-80.0, 25.0, math.radians(20.0), 0.0),
               _lib.Aberrations(35.0, 0.0, 0.0, 1.5e5)):
        ref_obj, ref_ph = ops.object_wave(g, geom, qr, qc, cal, ab)
        for _ in range(2):
            obj = torch.full((n, n), float("nan"), dtype=torch.complex64, device=dev)
            ph = torch.full((n, n), float("nan"), dtype=torch.float32, device=dev)
            rc = lib.qssb_object_noalloc(
                ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(geom.data_ptr()),
                ctypes.c_void_p(qr.data_ptr()), ctypes.c_void_p(qc.data_ptr()), ctypes.byref(cal),
                ctypes.byref(ab), 0, ctypes.c_void_p(obj.data_ptr()), ctypes.c_void_p(ph.data_ptr()),
                stream)
            _lib.check(rc)
            torch.cuda.synchronize(dev)
            a = obj.cpu().numpy()
            b = ref_obj.cpu().numpy()
            assert np.abs(a - b).max() <= 2e-6 * np.abs(b).max()
            err = np.angle(np.exp(1j * (ph.cpu().numpy().astype(np.float64) - ref_ph.cpu().numpy())))
            assert np.abs(err).max() < 2e-4
