"""Compile the reference's 128x128 SSB CUDA module into oracle/_ref/.

Run in the build container, where the reference tree exists:

    python -m oracle.ref_cuda.build_ref [--reference PATH]

The reference checkout is found by ``reference_root()``: ``--reference``,
else the ``QSSB_REFERENCE`` environment variable, else the build container's
checkout location.

Reads the CUDA source strings of
``src/quantem/gpu/ssb/compute/cuda/kernels/common.py`` (``_DEVICE_FUNCTIONS_CUDA``)
and ``.../fft128.py`` (``_TWIDDLE_DECL``, ``_FFT128_KERNELS``) with ``ast``
(the modules import CuPy, so they are not imported), assembles them as
``build_cuda_code`` does (common.py:620-622) in a temporary directory, and
compiles with the reference's NVRTC options (common.py:708: c++11, fast math,
96 registers, -dlcm=ca) for sm_100a. Only the cubin and a manifest are written
under ``oracle/_ref/``; no reference source is kept.
"""
from __future__ import annotations

import argparse
import ast
import hashlib
import json
import os
import shutil
import subprocess
import tempfile
from pathlib import Path

ORACLE = Path(__file__).resolve().parents[1]
OUT_DIR = ORACLE / "_ref"
CUBIN = OUT_DIR / "ssb_fft128.cubin"
MANIFEST = OUT_DIR / "ssb_fft128.json"
KERNELS_REL = Path("src/quantem/gpu/ssb/compute/cuda/kernels")
# where the build container keeps the reference checkout (read-only); the one
# place a recipe names it - everything else asks reference_root()
_BUILD_CONTAINER_CHECKOUT = "/root/reference"


def reference_root(override: str | Path | None = None) -> Path:
    """The reference checkout to read: ``override``, else ``$QSSB_REFERENCE``,
    else the build container's checkout. It may not exist (GPU boxes)."""
    if override:
        return Path(override)
    return Path(os.environ.get("QSSB_REFERENCE", _BUILD_CONTAINER_CHECKOUT))


DEFAULT_REFERENCE = reference_root()
KERNEL_NAMES = ("ifft128_rows_fused_pk_t32_mr8_packed", "ifft128_cols_t32_mr8")
# the batched phase-variance loss of variance_loss_batch (engine.py:2120-2295):
# rows + gamma + pk into the staging planes (K12), column IFFTs + atan2 +
# sum / sum of squares (K13), both in the same module (fft128.py:152-351, 466-549)
LOSS_KERNEL_NAMES = ("ifft128_rows_fused_pk_batch_t32_mr8_transpose_packed_b4",
                     "ifft128_rows_var_g32_t32_mr1_batch")
TWIDDLE_NAME = "TWIDDLE_128"
# ... and the per-candidate loss from the sums (K14), a RawKernel string of
# engine.py:96-137, compiled on its own (CuPy's RawKernel defaults: no fast math)
SUMS_CUBIN = OUT_DIR / "ssb_loss_sums.cubin"
SUMS_MANIFEST = OUT_DIR / "ssb_loss_sums.json"
SUMS_KERNEL = "loss_from_sums_batch"
ENGINE_REL = Path("src/quantem/gpu/ssb/compute/cuda/engine.py")


def _string_constants(path: Path, names: set[str]) -> dict[str, str]:
    tree = ast.parse(path.read_text())
    found = {}
    for node in tree.body:
        if isinstance(node, ast.Assign) and len(node.targets) == 1:
            tgt = node.targets[0]
            if isinstance(tgt, ast.Name) and tgt.id in names and isinstance(node.value, ast.Constant) \
                    and isinstance(node.value.value, str):
                found[tgt.id] = node.value.value
    missing = names - set(found)
    if missing:
        raise RuntimeError(f"{path}: string constants not found: {sorted(missing)}")
    return found


# Our probe kernel (not reference code): evaluates the reference's own device
# functions chi_full and gamma_mul_pk_onthefly_full (common.py:410-532)
# element-wise, so the 14-term chi convention can be checked on a GPU.
FULL_PROBE_NAME = "qref_full_chi_probe"
FULL_PROBE_SOURCE = """
__global__ void qref_full_chi_probe(
    const float* qx, const float* qy, const float* kx, const float* ky, int n,
    float wavelength, float semiangle_rad, float ang_y_rad, float ang_x_rad,
    const float* mag_scaled, const float* cm, const float* sm, const float* pk,
    const float* g, float* chi_qmk, float* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    chi_qmk[i] = chi_full(qx[i] - kx[i], qy[i] - ky[i], wavelength, mag_scaled, cm, sm);
    const float2 v = gamma_mul_pk_onthefly_full(
        qx[i], qy[i], kx[i], ky[i], wavelength, semiangle_rad, ang_y_rad, ang_x_rad,
        mag_scaled, cm, sm, pk[2 * i], pk[2 * i + 1], make_float2(g[2 * i], g[2 * i + 1]));
    out[2 * i] = v.x;
    out[2 * i + 1] = v.y;
}
"""


def _raw_kernel_sources(path: Path, names: set[str]) -> dict[str, str]:
    """The source strings of module-level ``NAME = cp.RawKernel(r'''...''', ...)``
    assignments (their first argument)."""
    tree = ast.parse(path.read_text())
    found = {}
    for node in tree.body:
        if isinstance(node, ast.Assign) and len(node.targets) == 1:
            tgt = node.targets[0]
            if isinstance(tgt, ast.Name) and tgt.id in names and isinstance(node.value, ast.Call) \
                    and node.value.args and isinstance(node.value.args[0], ast.Constant):
                found[tgt.id] = node.value.args[0].value
    missing = names - set(found)
    if missing:
        raise RuntimeError(f"{path}: RawKernel sources not found: {sorted(missing)}")
    return found


def sums_available() -> bool:
    return SUMS_CUBIN.exists() and SUMS_MANIFEST.exists()


def build_sums(reference: Path = DEFAULT_REFERENCE, force: bool = False, verbose: bool = False
               ) -> Path | None:
    """Compile the reference's loss_from_sums_batch kernel into its own cubin."""
    engine = reference / ENGINE_REL
    if not engine.exists():
        return SUMS_CUBIN if sums_available() else None
    src = _raw_kernel_sources(engine, {"_loss_from_sums_batch_kernel"})["_loss_from_sums_batch_kernel"]
    digest = hashlib.sha256(src.encode()).hexdigest()
    if not force and sums_available():
        if json.loads(SUMS_MANIFEST.read_text()).get("source_sha256") == digest:
            return SUMS_CUBIN
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    with tempfile.TemporaryDirectory() as td:
        cu = Path(td) / "ssb_loss_sums.cu"
        cu.write_text(src)
        cmd = [nvcc, "-cubin", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++11",
               "-o", str(SUMS_CUBIN) + ".tmp", str(cu)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    Path(str(SUMS_CUBIN) + ".tmp").replace(SUMS_CUBIN)
    SUMS_MANIFEST.write_text(json.dumps({
        "source_sha256": digest, "reference_files": [str(ENGINE_REL)],
        "options": "nvcc -cubin sm_100a -std=c++11", "kernels": [SUMS_KERNEL]}, indent=1))
    return SUMS_CUBIN


def module_source(reference: Path) -> str:
    """The CUDA module text the reference's CustomFFT128 hands to NVRTC, plus
    the element-wise probe of its 14-term chi functions."""
    kdir = reference / KERNELS_REL
    common = _string_constants(kdir / "common.py", {"_DEVICE_FUNCTIONS_CUDA"})
    fft = _string_constants(kdir / "fft128.py", {"_TWIDDLE_DECL", "_FFT128_KERNELS"})
    return ('extern "C" {\n' + fft["_TWIDDLE_DECL"] + "\n" + common["_DEVICE_FUNCTIONS_CUDA"]
            + "\n" + fft["_FFT128_KERNELS"] + "\n" + FULL_PROBE_SOURCE + "\n}")


def available() -> bool:
    return CUBIN.exists() and MANIFEST.exists()


def build(reference: Path = DEFAULT_REFERENCE, force: bool = False, verbose: bool = False) -> Path | None:
    """Compile the cubin; returns its path, or None when the reference tree is absent."""
    if not (reference / KERNELS_REL / "fft128.py").exists():
        return CUBIN if available() else None
    src = module_source(reference)
    digest = hashlib.sha256(src.encode()).hexdigest()
    if not force and available():
        if json.loads(MANIFEST.read_text()).get("source_sha256") == digest:
            return CUBIN
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    with tempfile.TemporaryDirectory() as td:
        cu = Path(td) / "ssb_fft128.cu"
        cu.write_text(src)
        cmd = [nvcc, "-cubin", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++11",
               "--use_fast_math", "-maxrregcount=96", "-Xptxas", "-dlcm=ca",
               "-o", str(CUBIN) + ".tmp", str(cu)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    Path(str(CUBIN) + ".tmp").replace(CUBIN)
    MANIFEST.write_text(json.dumps({
        "source_sha256": digest,
        "reference_files": [str(KERNELS_REL / "common.py"), str(KERNELS_REL / "fft128.py")],
        "options": "nvcc -cubin sm_100a -std=c++11 --use_fast_math -maxrregcount=96 -Xptxas -dlcm=ca",
        "kernels": list(KERNEL_NAMES) + list(LOSS_KERNEL_NAMES) + [FULL_PROBE_NAME],
        "twiddle": TWIDDLE_NAME,
    }, indent=1))
    return CUBIN


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", type=Path, default=DEFAULT_REFERENCE)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.reference, force=a.force, verbose=True))
    print(build_sums(a.reference, force=a.force, verbose=True))
