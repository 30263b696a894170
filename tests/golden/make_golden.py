"""Generate golden SSB fixtures by running the reference's own Python code.

Run in the development container only (it reads the reference checkout):

    python tests/golden/make_golden.py [--reference PATH]

The reference (bobleesj/quantem.gpu 0.0.1rc6) is CUDA-only: its SSB backend
imports CuPy at module level and its kernels are NVRTC strings. CuPy is not
installed here, so this script installs a small stand-in module named
``cupy`` that maps the array API the reference's *host* code uses onto numpy
(``ndarray.get``/``set``, ``asnumpy``, ``fft``, reductions as 0-d arrays) and
turns every kernel constructor into an inert object. With it the reference
executes, unmodified:

* ``CudaSSBBackend.__init__`` - scan padding (backend.py:229-269), wavelength,
  sampling, ``_compute_bf_mask`` (u64 mean DP, BF selection, backend.py:
  420-518) and ``_extract_gqk`` (gather, FFT, Hermitian half, dc;
  backend.py:520-589);
* ``SSBEngine.cache_rotation`` (engine.py:784-928) - BF geometry;
* ``tests/test_ssb_cuda_128.py::_reference_phase_loss`` - the reference's own
  vectorised float32 restatement of the kernels (pk, Gamma, normalisation,
  DC override, per-BF ifft2, mean phase, loss); the per-BF inverse FFTs it
  computes are captured to form the object wave ``mean_b ifft2(C_b)``.

Array arithmetic is numpy's (pocketfft in complex64 for the FFTs, numpy's
pairwise float32 reductions), so the fixtures pin the reference's algorithm
and float32 decisions; they are not bit-identical to CuPy/cuFFT on a GPU.

Fixtures written to ``tests/golden/`` (small .npz files) are consumed by
``tests/test_oracle_golden.py``.
"""
from __future__ import annotations

import argparse
import hashlib
import importlib.util
import math
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

from oracle.ref_cuda.build_ref import reference_root  # noqa: E402


# ---------------------------------------------------------------------------
# numpy-backed stand-in for the parts of CuPy the reference host code uses
# ---------------------------------------------------------------------------

class ShimArray(np.ndarray):
    """ndarray with CuPy's ``get``/``set`` and 0-d (not scalar) reductions."""

    def get(self, out=None):
        host = np.asarray(self).view(np.ndarray)
        if out is not None:
            out[...] = host
            return out
        return host.copy()

    def set(self, arr):
        self[...] = np.asarray(arr)

    def __array_wrap__(self, obj, context=None, return_scalar=False):
        return np.ndarray.__array_wrap__(self, obj, context, False)


def _view(x):
    if isinstance(x, np.ndarray) and not isinstance(x, ShimArray):
        return x.view(ShimArray)
    if isinstance(x, tuple):
        return tuple(_view(v) for v in x)
    if isinstance(x, list):
        return [_view(v) for v in x]
    return x


def _wrap(fn):
    def inner(*args, **kwargs):
        return _view(fn(*args, **kwargs))
    inner.__name__ = getattr(fn, "__name__", "wrapped")
    return inner


class _InertKernel:
    """Stands in for RawKernel / ElementwiseKernel / RawModule functions."""

    def __init__(self, *args, **kwargs):
        self.max_dynamic_shared_size_bytes = 0

    def __call__(self, *args, **kwargs):
        raise RuntimeError("reference CUDA kernels cannot execute without a GPU")

    def get_function(self, name):
        return _InertKernel()

    def get_global(self, name):
        return bytearray(1 << 16)


class _Pool:
    def free_all_blocks(self):
        return None


FFT_CAPTURE: list[np.ndarray] = []


def _capturing_ifft2(x, *args, **kwargs):
    out = np.fft.ifft2(np.asarray(x), *args, **kwargs)
    FFT_CAPTURE.append(out)
    return _view(out)


def build_cupy_shim() -> types.ModuleType:
    cp = types.ModuleType("cupy")
    for name in (
        "uint8", "uint16", "uint32", "uint64", "int32", "int64", "float32",
        "float64", "complex64", "complex128", "bool_", "pi", "dtype",
        "issubdtype", "integer", "floating",
    ):
        setattr(cp, name, getattr(np, name))
    for name in (
        "asarray", "ascontiguousarray", "empty", "zeros", "ones", "full",
        "arange", "meshgrid", "nonzero", "sqrt", "arctan2", "cos", "sin",
        "clip", "broadcast_to", "conj", "where", "angle", "mean", "abs",
        "maximum", "minimum", "exp", "divide", "percentile", "zeros_like",
        "empty_like", "concatenate", "stack", "linspace", "round", "floor",
    ):
        setattr(cp, name, _wrap(getattr(np, name)))
    cp.ndarray = ShimArray
    cp.asnumpy = lambda x, *a, **k: np.asarray(x).view(np.ndarray).copy()
    fft = types.ModuleType("cupy.fft")
    fft.fft2 = _wrap(np.fft.fft2)
    fft.ifft2 = _capturing_ifft2
    fft.fftfreq = _wrap(np.fft.fftfreq)
    fft.fftshift = _wrap(np.fft.fftshift)
    cp.fft = fft
    cp.RawKernel = _InertKernel
    cp.ElementwiseKernel = _InertKernel
    cp.RawModule = _InertKernel
    cp.get_default_memory_pool = lambda: _Pool()
    cp.get_default_pinned_memory_pool = lambda: _Pool()
    cuda = types.ModuleType("cupy.cuda")

    class _Device:
        def __init__(self, *a):
            pass

        def synchronize(self):
            return None

        def use(self):
            return None

    cuda.Device = _Device
    runtime = types.SimpleNamespace(memGetInfo=lambda: (64 << 30, 80 << 30))
    cuda.runtime = runtime
    cuda.memory = types.SimpleNamespace(OutOfMemoryError=MemoryError)
    cp.cuda = cuda
    testing = types.ModuleType("cupy.testing")
    testing.assert_allclose = np.testing.assert_allclose
    cp.testing = testing
    return cp


def install(reference: Path):
    sys.modules["cupy"] = build_cupy_shim()
    sys.modules["cupy.fft"] = sys.modules["cupy"].fft
    sys.modules["cupy.cuda"] = sys.modules["cupy"].cuda
    sys.path.insert(0, str(reference / "src"))
    sys.path.insert(0, str(reference))
    from quantem.gpu.ssb.compute.cuda.backend import CudaSSBBackend  # noqa: E402
    spec = importlib.util.spec_from_file_location(
        "ref_test_ssb_cuda_128", reference / "tests" / "test_ssb_cuda_128.py"
    )
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return CudaSSBBackend, mod


sys.path.insert(0, str(HERE))
from recipes import digest, disk_input, synthetic_plain_32  # noqa: E402


def run_case(CudaSSBBackend, refmod, name: str, data: np.ndarray, kwargs: dict,
             aberrations: tuple[float, float, float], store_full_g: bool):
    cp = sys.modules["cupy"]
    backend = CudaSSBBackend(cp.asarray(data).view(ShimArray), **kwargs)
    accel = backend._get_accelerator()
    accel.cache_rotation(math.radians(kwargs.get("rotation_angle_deg", 0.0)))
    c = accel._cache
    FFT_CAPTURE.clear()
    phase, loss = refmod._reference_phase_loss(accel, *aberrations)
    obj = FFT_CAPTURE[-1].mean(axis=0).astype(np.complex64)
    g = np.asarray(backend.G_qk)
    out = {
        "input_sha256": np.asarray(digest(data)),
        "input_shape": np.asarray(data.shape),
        "rows": np.asarray(backend.bf_inds_row).astype(np.int32),
        "cols": np.asarray(backend.bf_inds_col).astype(np.int32),
        "center": np.asarray(backend.bf_center, dtype=np.float64),
        "dc": np.asarray(backend.dc_value, dtype=np.complex128),
        "wavelength": np.asarray(backend.wavelength),
        "sampling": np.asarray(backend.sampling, dtype=np.float64),
        "scan_shape": np.asarray(backend.scan_shape),
        "g_shape": np.asarray(g.shape),
        "g_corner": g[:, :4, :4].astype(np.complex64),
        "g_abs2_per_bf": (np.abs(g.astype(np.complex128)) ** 2).sum(axis=(1, 2)),
        "kx_bf": np.asarray(c["kx_bf"]), "ky_bf": np.asarray(c["ky_bf"]),
        "alpha_k2": np.asarray(c["alpha_k2_1d"]),
        "cos2phi_k": np.asarray(c["cos2phi_k_1d"]),
        "sin2phi_k": np.asarray(c["sin2phi_k_1d"]),
        "aperture_k": np.asarray(c["aperture_k_1d"]),
        "qx_1d": np.asarray(c["qx_1d"]), "qy_1d": np.asarray(c["qy_1d"]),
        "aberrations": np.asarray(aberrations, dtype=np.float64),
        "mean_phase": np.asarray(phase, dtype=np.float32),
        "loss": np.asarray(loss, dtype=np.float64),
        "object": obj,
    }
    if store_full_g:
        out["g_half_first3"] = g[:3].astype(np.complex64)
        out.update(run_spec(accel, g, aberrations))
    for key in ("semiangle", "scan_sampling", "det_sampling", "voltage_kV", "bf_radius"):
        if kwargs.get(key) is not None:
            out["kw_" + key] = np.asarray(kwargs[key], dtype=np.float64)
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(f"{name}: B={out['rows'].size} center={tuple(out['center'])} loss={loss:.6g}")


def run_spec(accel, g_half: np.ndarray, aberrations) -> dict:
    """Execute the reference's executable specification (docs/kernels/ssb.md).

    The first eight ``python`` blocks of the page (imports, select_bright_field,
    scan_fft, probe/corrected_object, phase_variance_loss, evaluate_candidate,
    best_tpe_candidate, final_object) are executed as written on CPU torch,
    fed with the reference engine's own cached geometry.
    """
    import re

    import torch

    text = (REFERENCE / "docs" / "kernels" / "ssb.md").read_text()
    blocks = re.findall(r"```python\n(.*?)```", text, re.S)[:8]
    ns: dict = {}
    for block in blocks:
        exec(compile(block, "docs/kernels/ssb.md", "exec"), ns)
    c = accel._cache
    f64 = torch.float64
    qx = torch.as_tensor(np.asarray(c["qx_1d"]), dtype=f64)[None, :, None]
    qy = torch.as_tensor(np.asarray(c["qy_1d"]), dtype=f64)[None, None, :]
    kx = torch.as_tensor(np.asarray(c["kx_bf"]), dtype=f64)[:, None, None]
    ky = torch.as_tensor(np.asarray(c["ky_bf"]), dtype=f64)[:, None, None]
    lam = float(c["wavelength"])
    semi = float(c["semiangle_rad"])
    ang_r = float(c["ang_y_rad"])
    ang_c = float(c["ang_x_rad"])

    def polar(dx, dy):
        r2 = dx * dx + dy * dy
        r = torch.sqrt(r2)
        alpha = r * lam
        denom = torch.sqrt((dx * ang_r) ** 2 + (dy * ang_c) ** 2) / torch.where(r > 0, r, torch.ones_like(r))
        edge = torch.where(denom > 0, (semi - alpha) / torch.where(denom > 0, denom, torch.ones_like(denom)) + 0.5,
                           torch.ones_like(denom))
        return alpha * alpha, torch.atan2(dy, dx), torch.clamp(edge, 0.0, 1.0)

    k_polar = (
        torch.as_tensor(np.asarray(c["alpha_k2_1d"]), dtype=f64),
        torch.atan2(ky[:, 0, 0], kx[:, 0, 0]),
        torch.as_tensor(np.asarray(c["aperture_k_1d"]), dtype=f64),
    )
    geometry = ns["SSBGeometry"](k=k_polar, k_minus_nu=polar(kx - qx, ky - qy), k_plus_nu=polar(kx + qx, ky + qy))
    full = np.empty((g_half.shape[0], g_half.shape[1], qy.shape[-1]), dtype=np.complex128)
    n = qy.shape[-1]
    full[:, :, : g_half.shape[2]] = g_half
    full[:, :, g_half.shape[2]:] = np.conj(g_half[:, (-np.arange(g_half.shape[1])) % g_half.shape[1]][:, :, n - np.arange(g_half.shape[2], n)])
    theta = tuple(torch.tensor(v, dtype=f64) for v in aberrations)
    obj_b = ns["corrected_object"](torch.as_tensor(full), geometry, theta, torch.tensor(lam, dtype=f64),
                                   torch.tensor(complex(accel._dc_value_host), dtype=torch.complex128))
    loss = ns["phase_variance_loss"](obj_b)
    obj, _amp, phi = ns["final_object"](obj_b)
    return {"spec_loss": np.asarray(float(loss)), "spec_object": obj.numpy().astype(np.complex128),
            "spec_phase": phi.numpy()}


REFERENCE = reference_root()


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default=None,
                        help="reference checkout (default: $QSSB_REFERENCE, else the build "
                             "container's checkout)")
    args = parser.parse_args()
    global REFERENCE
    REFERENCE = reference_root(args.reference)
    CudaSSBBackend, refmod = install(REFERENCE)

    ab = (-120.0, 55.0, math.radians(17.0))
    # 1. The reference test's own end-to-end case (explicit bf_radius=3).
    run_case(
        CudaSSBBackend, refmod, "ref_disk128_bfr3", disk_input(123),
        dict(voltage_kV=300, semiangle=21.4, scan_sampling=0.5, det_sampling=1.0, bf_radius=3),
        ab, store_full_g=True,
    )
    # 2. Uneven 96x96 scan: the reference pads it to 128 with the truncated mean DP.
    run_case(
        CudaSSBBackend, refmod, "ref_disk96_padded", disk_input(124, scan=(96, 96)),
        dict(voltage_kV=300, semiangle=21.4, scan_sampling=0.5, det_sampling=1.0, bf_radius=3),
        ab, store_full_g=False,
    )
    # 3. The CPU-runnable plain workload with automatic probe detection
    #    (bf_radius=None: mean+std probe, centroid, sqrt(count/pi) radius);
    #    the reference pads the 32x32 scan to 128x128.
    run_case(
        CudaSSBBackend, refmod, "ref_plain32_auto", synthetic_plain_32(),
        dict(voltage_kV=300, semiangle=20.0, scan_sampling=0.5, det_sampling=20.0 / 12.0),
        (50.0, 20.0, 0.3), store_full_g=False,
    )
    # 4. Hermitian extraction on arange counts (test_ssb_cuda_128.py:513-534).
    cp = sys.modules["cupy"]
    data = np.arange(8 * 8 * 6 * 6, dtype=np.uint16).reshape(8, 8, 6, 6)
    rows = np.asarray([2, 2, 3, 3], dtype=np.int32)
    cols = np.asarray([2, 3, 2, 3], dtype=np.int32)
    g, dc = CudaSSBBackend._extract_gqk(
        cp.asarray(data).view(ShimArray), cp.asarray(rows), cp.asarray(cols), (8, 8), (6, 6)
    )
    np.savez_compressed(
        HERE / "ref_arange_hermitian.npz",
        g_half=np.asarray(g).astype(np.complex64), dc=np.asarray(dc), rows=rows, cols=cols,
    )
    print("ref_arange_hermitian: written")


if __name__ == "__main__":
    main()
