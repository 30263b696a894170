"""Deterministic input recipes shared by the golden generator and the tests.

Each recipe regenerates its input exactly; the fixtures store a SHA-256 of
the bytes so a drifting recipe fails loudly instead of comparing garbage.
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent.parent.parent


def disk_input(seed: int, scan=(128, 128)) -> np.ndarray:
    """The reference test's end-to-end input (tests/test_ssb_cuda_128.py:587-697
    of bobleesj/quantem.gpu): Poisson(4) counts on a 16x16 detector plus 80
    counts on a radius-4 disk centred at (8, 8)."""
    rng = np.random.default_rng(seed)
    data = rng.poisson(4.0, size=tuple(scan) + (16, 16)).astype(np.uint16)
    yy, xx = np.ogrid[:16, :16]
    bf = (yy - 8) ** 2 + (xx - 8) ** 2 <= 4 ** 2
    data[..., bf] += 80
    return data


def export_cases() -> dict[str, np.ndarray]:
    """Inputs of the exact BF companion fixtures (the disk case above, 128x128
    scan x 16x16 detector, bf_radius=3): u16 counts that fit u8, the same with
    one hot pixel outside the BF disk, and the counts as u8."""
    base = disk_input(123)
    hot = base.copy()
    hot[5, 7, 0, 0] = 300  # outside the BF disk: the block no longer fits u8
    return {"u16_fits_u8": base, "u16_hot_pixel_outside_bf": hot, "u8": base.astype(np.uint8)}


def synthetic_plain_32() -> np.ndarray:
    """The CPU-runnable plain workload (32x32 scan, 64x64 detector, u16)."""
    if str(REPO) not in sys.path:
        sys.path.insert(0, str(REPO))
    from quantem.gpu_b200.synthetic import CONFIGS, generate

    return generate(CONFIGS["plain_32x32_det64"], device="cpu").counts.numpy()


def digest(a: np.ndarray) -> str:
    """SHA-256 of an array's bytes (C order)."""
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
