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

    @property
    def device(self):  # CuPy's array.device (numpy's own is the string "cpu")
        return types.SimpleNamespace(id=0)

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


class _GatherTransposeShim:
    """Stands in for the one RawKernel whose effect the fixtures need: the BF
    companion writer's ``gather_transpose`` (engine.py:620-660). Its
    documented effect, for the chunk's BF pixels ``ob < num_bf`` and frames
    ``s < num_scan``: ``output[ob * num_scan + s] = (out type)
    input[s * detector_pixels + bf_linear[bf_offset + ob]]``. Everything
    around it (dtype rule, narrowing on the whole block, file naming, chunk
    order, writer thread) is the reference's own code."""

    def __call__(self, grid, block, args):
        inp, bf_linear, out, num_scan, bf_offset, num_bf, det = args
        src = np.asarray(inp).reshape(int(num_scan), int(det))
        idx = np.asarray(bf_linear)[int(bf_offset):int(bf_offset) + int(num_bf)]
        dst = np.asarray(out).reshape(-1)
        n = int(num_bf) * int(num_scan)
        dst[:n] = src[:, idx].T.astype(dst.dtype).reshape(-1)


def _raw_kernel(code=None, name=None, *args, **kwargs):
    if name == "gather_transpose":
        return _GatherTransposeShim()
    return _InertKernel(code, name, *args, **kwargs)


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
        "empty_like", "concatenate", "stack", "linspace", "round", "floor", "max",
        "nanmax", "any", "rint", "ones_like", "pad", "convolve",
    ):
        setattr(cp, name, _wrap(getattr(np, name)))
    cp.add = np.add  # the ufunc: probe.py's radial profile uses cp.add.at
    cp.ndarray = ShimArray
    cp.asnumpy = lambda x, *a, **k: np.asarray(x).view(np.ndarray).copy()
    fft = types.ModuleType("cupy.fft")
    fft.fft2 = _wrap(np.fft.fft2)
    fft.ifft2 = _capturing_ifft2
    fft.fftfreq = _wrap(np.fft.fftfreq)
    fft.fftshift = _wrap(np.fft.fftshift)
    cp.fft = fft
    cp.RawKernel = _raw_kernel
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
    # quantem.gpu.detector's __init__ imports the HDF5 reader (h5py, absent
    # here); the BF-radius detection needs only its compute/cuda/probe module,
    # whose own package inits import nothing, so register the package bare
    detector = types.ModuleType("quantem.gpu.detector")
    detector.__path__ = [str(reference / "src" / "quantem" / "gpu" / "detector")]
    sys.modules.setdefault("quantem.gpu.detector", detector)
    from quantem.gpu.ssb.compute.cuda.backend import CudaSSBBackend  # noqa: E402
    spec = importlib.util.spec_from_file_location(
        "ref_test_ssb_cuda_128", reference / "tests" / "test_ssb_cuda_128.py"
    )
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return CudaSSBBackend, mod


sys.path.insert(0, str(HERE))
from recipes import digest, disk_input, export_cases, synthetic_plain_32  # noqa: E402


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
    if kwargs.get("det_sampling") is None:
        # detected from the mean DP: det_sampling = 2 * semiangle / radius (backend.py:276-285)
        out["angular_sampling"] = np.asarray(backend.angular_sampling, dtype=np.float64)
    for key in ("semiangle", "scan_sampling", "det_sampling", "voltage_kV", "bf_radius"):
        if kwargs.get(key) is not None:
            out["kw_" + key] = np.asarray(kwargs[key], dtype=np.float64)
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(f"{name}: B={out['rows'].size} center={tuple(out['center'])} loss={loss:.6g}")


def run_export_cases(CudaSSBBackend) -> None:
    """The reference's exact BF companion writer (engine.py:577-701) on three
    blocks: u16 counts that fit u8, the same with one hot pixel outside the
    disk, and u8 counts. Stores the file suffix, size and SHA-256."""
    import tempfile

    cp = sys.modules["cupy"]
    kwargs = dict(voltage_kV=300, semiangle=21.4, scan_sampling=0.5, det_sampling=1.0, bf_radius=3)
    backend = CudaSSBBackend(cp.asarray(disk_input(123)).view(ShimArray), **kwargs)
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, data in export_cases().items():
            path, seconds = backend.export_brightfield(cp.asarray(data).view(ShimArray),
                                                       Path(tmp) / name)
            raw = Path(path).read_bytes()
            out[name + "_suffix"] = np.asarray(Path(path).suffix)
            out[name + "_bytes"] = np.asarray(len(raw))
            out[name + "_sha256"] = np.asarray(hashlib.sha256(raw).hexdigest())
            out[name + "_input_sha256"] = np.asarray(digest(data))
            print(f"export {name}: {Path(path).suffix} {len(raw)} bytes")
    np.savez_compressed(HERE / "ref_bf_export.npz", **out)


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
    parser.add_argument("--only", choices=["export", "detect"], default=None,
                        help="write only the named fixture group")
    args = parser.parse_args()
    global REFERENCE
    REFERENCE = reference_root(args.reference)
    CudaSSBBackend, refmod = install(REFERENCE)
    if args.only in (None, "export"):
        run_export_cases(CudaSSBBackend)
    if args.only in (None, "detect"):
        # det_sampling=None: the reference detects the BF radius from the mean DP
        # (detector/compute/cuda/probe.py:12-119) and sets det_sampling = 2 alpha / r
        run_case(
            CudaSSBBackend, refmod, "ref_plain32_detect", synthetic_plain_32(),
            dict(voltage_kV=300, semiangle=20.0, scan_sampling=0.5, det_sampling=None),
            (50.0, 20.0, 0.3), store_full_g=False,
        )
        run_case(
            CudaSSBBackend, refmod, "ref_disk128_detect", disk_input(123),
            dict(voltage_kV=300, semiangle=21.4, scan_sampling=0.5, det_sampling=None, bf_radius=3),
            (-120.0, 55.0, math.radians(17.0)), store_full_g=False,
        )
    if args.only is not None:
        return

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
