"""Compile the reference's bitshuffle + LZ4 CUDA module into oracle/_ref/.

Run in the build container, where the reference tree exists:

    python -m oracle.ref_cuda.build_bslz4 [--reference PATH]

(the checkout is found as in ``build_ref.reference_root()``)

Reads the CUDA source string ``_CUDA_LZ4_SOURCE`` of
``src/quantem/gpu/io/backends/cuda/decoder.py`` with ``ast`` (the module
imports CuPy) and compiles it with NVRTC, as the reference's CuPy RawModule
does, with its options (decoder.py:1147: c++11, warnings off) for sm_100a
(NVRTC, not nvcc: the source declares its own fixed-width integer types,
which clash with the system headers nvcc includes). Only the cubin and a
manifest are kept under ``oracle/_ref/``.
"""
from __future__ import annotations

import argparse
import hashlib
import json
from pathlib import Path

from .build_ref import DEFAULT_REFERENCE, OUT_DIR, _string_constants

CUBIN = OUT_DIR / "bslz4.cubin"
MANIFEST = OUT_DIR / "bslz4.json"
DECODER_REL = Path("src/quantem/gpu/io/backends/cuda/decoder.py")


def available() -> bool:
    return CUBIN.exists() and MANIFEST.exists()


def build(reference: Path = DEFAULT_REFERENCE, force: bool = False, verbose: bool = False) -> Path | None:
    path = reference / DECODER_REL
    if not path.exists():
        return CUBIN if available() else None
    src = _string_constants(path, {"_CUDA_LZ4_SOURCE"})["_CUDA_LZ4_SOURCE"]
    digest = hashlib.sha256(src.encode()).hexdigest()
    if not force and available() and json.loads(MANIFEST.read_text()).get("source_sha256") == digest:
        return CUBIN
    from cuda.bindings import nvrtc

    opts = [b"-std=c++11", b"-w", b"-arch=sm_100a"]
    err, prog = nvrtc.nvrtcCreateProgram(src.encode(), b"bslz4.cu", 0, [], [])
    if int(err) != 0:
        raise RuntimeError(f"nvrtcCreateProgram: {err}")
    (err,) = nvrtc.nvrtcCompileProgram(prog, len(opts), opts)
    if int(err) != 0:
        _, n = nvrtc.nvrtcGetProgramLogSize(prog)
        log = b" " * n
        nvrtc.nvrtcGetProgramLog(prog, log)
        raise RuntimeError(f"NVRTC failed: {log.decode(errors='replace')}")
    _, size = nvrtc.nvrtcGetCUBINSize(prog)
    cubin = b" " * size
    nvrtc.nvrtcGetCUBIN(prog, cubin)
    nvrtc.nvrtcDestroyProgram(prog)
    if verbose:
        print("nvrtc", " ".join(o.decode() for o in opts))
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    Path(str(CUBIN) + ".tmp").write_bytes(cubin)
    Path(str(CUBIN) + ".tmp").replace(CUBIN)
    MANIFEST.write_text(json.dumps({
        "source_sha256": digest, "reference_file": str(DECODER_REL),
        "options": "nvrtc -arch=sm_100a -std=c++11 -w",
        "kernels": ["bitshuffle_fwd_8192_16", "lz4_compress_kernel", "pack_h5_chunks_kernel",
                    "h5lz4dc_batched", "shuf_8192_16_batched"],
    }, indent=1))
    return CUBIN


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", type=Path, default=DEFAULT_REFERENCE)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.reference, force=a.force, verbose=True))
