"""The torch FP64 restatement of the oracle (oracle/ssb_torch_fp64.py, the
"FP64 GPU path" of the 256^2 precision study) against the numpy oracle, run
on CPU torch here (the same code runs on the GPU)."""
from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from oracle import ssb_oracle as so
from oracle import ssb_torch_fp64 as tf
from recipes import disk_input, synthetic_plain_32


@pytest.mark.parametrize("case", ["disk_bfr3", "plain32_auto"])
def test_torch_fp64_path_matches_numpy_oracle(case):
    if case == "disk_bfr3":
        data = so.pad_or_crop_scan(disk_input(123))
        kw = dict(voltage_kV=300, semiangle_mrad=21.4, scan_sampling=0.5, det_sampling=1.0,
                  bf_radius=3)
    else:
        data = synthetic_plain_32()
        kw = dict(voltage_kV=300, semiangle_mrad=20.0, scan_sampling=0.5, det_sampling=20.0 / 12.0)
    prep = so.prepare(data, pad=False, **kw)
    pg = tf.prepare(torch.as_tensor(data), **kw)
    np.testing.assert_array_equal(pg.bf.rows, prep.bf.rows)
    assert abs(pg.dc - prep.dc) <= 1e-13 * abs(prep.dc)
    full = so.FullAberrations((-120.0, 55.0, 1500.0, 1000.0, 5.0e4, 3.0e4, 4.0e4, 3.0e6, 2.0e6,
                               2.0e6, 1.0e8, 5.0e7, 5.0e7, 5.0e7),
                              (0.0, 0.3, 0.5, -0.7, 0.0, 1.1, -0.35, 0.17, 1.4, -0.96, 0.0, 0.09,
                               0.79, -1.2))
    for ab in (so.Aberrations(0.0, 0.0, 0.0), so.Aberrations(-120.0, 55.0, math.radians(17.0)),
               so.Aberrations(30.0, 10.0, 0.2, C30=5e4), full):
        o1, p1 = so.reconstruct(prep, ab)
        o2, p2 = tf.reconstruct(pg, ab)
        assert np.abs(o1 - o2.numpy()).max() <= 1e-10 * np.abs(o1).max()
        assert np.abs(so.wrapped_phase_error(p1, p2.numpy())).max() <= 1e-10
        l1, m1 = so.phase_variance_loss(prep.g_half, prep.geo, ab, prep.dc)
        l2, m2 = tf.phase_variance_loss(pg, ab)
        assert abs(l1 - l2) <= 1e-10 * abs(l1)
        assert np.abs(m1 - m2.numpy()).max() <= 1e-10
