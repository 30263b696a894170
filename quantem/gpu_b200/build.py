"""Build ``libqssb.so`` in-tree with nvcc for sm_100a (B200).

    python -m quantem.gpu_b200.build

Cross-compiles without a GPU. The library lands next to this file so it
travels with the source tree.
"""
from __future__ import annotations

import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "libqssb.so"
SOURCES = ["qssb_errors.cu", "qssb_prepare.cu", "qssb_select.cu", "qssb_object.cu", "qssb_loss.cu", "qssb_features.cu", "qssb_mlp.cu",
           "qssb_temporal.cu", "qssb_decode.cu", "qssb_export.cu", "qssb_box.cu", "qssb_gemm_tc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found; the SSB engine needs the CUDA toolkit to build")
    return exe


def sources() -> list[Path]:
    return [CSRC / s for s in SOURCES]


def needs_build() -> bool:
    if not OUT.exists():
        return True
    mtime = OUT.stat().st_mtime
    deps = sources() + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h"))
    deps.append(PKG.parent.parent / "include" / "qssb.h")
    return any(p.stat().st_mtime > mtime for p in deps if p.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every CUDA source into ``libqssb.so`` (skips if up to date)."""
    if not force and not needs_build():
        return OUT
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, *FLAGS, "-o", str(tmp), *map(str, sources())]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    proc = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError(f"nvcc failed with exit code {proc.returncode}")
    if verbose:
        sys.stderr.write(proc.stderr)
    tmp.replace(OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
