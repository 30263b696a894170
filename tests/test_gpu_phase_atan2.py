"""qssb_phase_atan2 (the loss kernels' phase function) against IEEE atan2
on the GPU: error bound over twelve decades of magnitude, exact signed
zeros and axes, NaN propagation."""
import numpy as np
import pytest
import torch

from quantem.gpu_b200 import ops

pytestmark = pytest.mark.gpu


def test_phase_atan2_error_bound():
    rng = np.random.default_rng(11)
    n = 1 << 22
    y = (rng.standard_normal(n) * 10.0 ** rng.uniform(-4, 8, n)).astype(np.float32)
    x = (rng.standard_normal(n) * 10.0 ** rng.uniform(-4, 8, n)).astype(np.float32)
    got = ops.phase_atan2(torch.from_numpy(y).cuda(), torch.from_numpy(x).cuda()).cpu().numpy()
    err = np.abs(got.astype(np.float64) - np.arctan2(y.astype(np.float64), x.astype(np.float64)))
    assert err.max() <= 4e-7, err.max()
    assert np.sqrt(np.mean(err ** 2)) <= 1e-7, np.sqrt(np.mean(err ** 2))


def test_phase_atan2_special_values():
    ys = np.array([0.0, -0.0, 0.0, -0.0, 1.0, -1.0, 2.0, -2.0, 5.0, 0.0, 7.0, np.nan, 1.0],
                  np.float32)
    xs = np.array([0.0, 0.0, -0.0, -0.0, 0.0, 0.0, 2.0, -2.0, -5.0, -3.0, 1e-3, 1.0, np.nan],
                  np.float32)
    got = ops.phase_atan2(torch.from_numpy(ys).cuda(), torch.from_numpy(xs).cuda()).cpu().numpy()
    want = np.arctan2(ys, xs)
    fin = np.isfinite(want)
    assert np.all(np.abs(got[fin].astype(np.float64) - want[fin]) <= 4e-7)
    assert np.array_equal(np.signbit(got[fin]), np.signbit(want[fin]))
    assert np.all(np.isnan(got[~fin]))
    assert got[0] == 0.0 and got[2] == np.float32(np.pi)
