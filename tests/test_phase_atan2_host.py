"""The loss kernels' atan2 (``phase_atan2`` in qssb_device.cuh): its
coefficients are the ones the committed fit produces, and a float32
emulation of the whole function with an exactly rounded divide stays within
the polynomial's 2.4e-7 rad (the GPU's fast divide adds up to 2 ulp of t;
its bound, 4e-7 rad, is checked on the GPU). CPU only."""
import importlib.util
import re
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "quantem" / "gpu_b200" / "csrc"


def _fit_module():
    spec = importlib.util.spec_from_file_location("phase_atan2_fit",
                                                  Path(__file__).resolve().parent / "phase_atan2_fit.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _header_coefficients() -> np.ndarray:
    src = (CSRC / "qssb_device.cuh").read_text()
    body = src[src.index("float phase_atan2(float y, float x)"):]
    body = body[:body.index("float r = t * p;")]
    vals = [float(v) for v in re.findall(r"([-+]?\d\.\d+e[-+]\d+)f", body)]
    vals += [1.0]  # the last fma adds 1.0f
    return np.array(vals[::-1], np.float32)  # constant term first


def test_coefficients_match_the_fit():
    mod = _fit_module()
    fitted = mod.fit(mod.N_TERMS)
    np.testing.assert_allclose(_header_coefficients(), fitted, rtol=2e-7, atol=0)


def test_emulated_error_bound_and_special_values():
    mod = _fit_module()
    c = _header_coefficients()
    rng = np.random.default_rng(7)
    n = 400_000
    y = rng.standard_normal(n) * 10.0 ** rng.uniform(-4, 8, n)
    x = rng.standard_normal(n) * 10.0 ** rng.uniform(-4, 8, n)
    got = mod.phase_atan2_f32(y, x, c).astype(np.float64)
    want = np.arctan2(y.astype(np.float32), x.astype(np.float32)).astype(np.float64)
    assert np.max(np.abs(got - want)) <= 2.4e-7
    # axes, diagonals and signed zeros follow IEEE atan2
    ys = np.array([0.0, -0.0, 0.0, -0.0, 1.0, -1.0, 1.0, -1.0, 3.0, 0.0], np.float32)
    xs = np.array([0.0, 0.0, -0.0, -0.0, 0.0, 0.0, 1.0, -1.0, 3.0, -2.0], np.float32)
    got = mod.phase_atan2_f32(ys, xs, c)
    want = np.arctan2(ys, xs)
    assert np.all(np.abs(got.astype(np.float64) - want) <= 2.4e-7)
    assert np.array_equal(np.signbit(got), np.signbit(want))
