"""512^2 and 1024^2 scans (the reference's fft512.py / fft1024.py sizes):
scan FFT, object, loss and the 14-term chi against the FP64 oracle (its
torch restatement, cross-checked against the numpy oracle on CPU), and the
graph pipeline against the backend bit for bit."""
from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from oracle import ssb_oracle as so
from oracle import ssb_torch_fp64 as tf
from quantem.gpu_b200 import B200SSBBackend
from quantem.gpu_b200.pipeline import ColdReconstructor
from recipes import disk_input

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
KW = dict(voltage_kV=300, semiangle_mrad=21.4, scan_sampling=0.5, det_sampling=1.0, bf_radius=3)
FULL = so.FullAberrations((-120.0, 55.0, 1500.0, 1000.0, 5.0e4, 3.0e4, 4.0e4, 3.0e6, 2.0e6, 2.0e6,
                           1.0e8, 5.0e7, 5.0e7, 5.0e7),
                          (0.0, 0.3, 0.5, -0.7, 0.0, 1.1, -0.35, 0.17, 1.4, -0.96, 0.0, 0.09,
                           0.79, -1.2))


def _rms(a, b) -> float:
    err = so.wrapped_phase_error(np.asarray(a, np.float64), np.asarray(b, np.float64))
    return float(np.sqrt(np.mean(err ** 2)))


@pytest.mark.parametrize("scan", [512, 1024])
def test_large_scan_matches_fp64_oracle(scan):
    counts = torch.as_tensor(disk_input(7, scan=(scan, scan)), device=DEV)
    be = B200SSBBackend(counts, semiangle=21.4, scan_sampling=0.5, det_sampling=1.0,
                        voltage_kV=300, bf_radius=3)
    assert be.scan_shape == (scan, scan)
    pg = tf.prepare(counts, **KW)
    np.testing.assert_array_equal(be.bf_inds_row, pg.bf.rows)
    np.testing.assert_array_equal(be.bf_inds_col, pg.bf.cols)
    assert abs(be.dc_value - pg.dc) <= 1e-13 * abs(pg.dc)
    g_ref = pg.g_half
    assert float((be.G_qk.to(torch.complex128) - g_ref).abs().max()) <= 4e-6 * float(g_ref.abs().max())
    ab = so.Aberrations(-120.0, 55.0, math.radians(17.0))
    obj, ph = be.object_and_phase(ab.C10, ab.C12, ab.phi12)
    ref_obj, ref_ph = tf.reconstruct(pg, ab)
    assert _rms(ph.cpu().numpy(), ref_ph.cpu().numpy()) < 1e-5
    assert float((obj.to(torch.complex128) - ref_obj).abs().max()) <= 1e-5 * float(ref_obj.abs().max())
    mp, loss = be.reconstruct_with_loss(ab.C10, ab.C12, ab.phi12)
    ref_loss, ref_mp = tf.phase_variance_loss(pg, ab)
    assert loss == pytest.approx(ref_loss, rel=2e-5)
    assert _rms(mp.cpu().numpy(), ref_mp.cpu().numpy()) < 2e-5
    mp_f, loss_f = be.reconstruct_full_with_loss(np.array(FULL.magnitudes), np.array(FULL.angles))
    ref_loss_f, ref_mp_f = tf.phase_variance_loss(pg, FULL)
    assert loss_f == pytest.approx(ref_loss_f, rel=2e-5)
    assert _rms(mp_f.cpu().numpy(), ref_mp_f.cpu().numpy()) < 2e-5
    be.close()


def test_pipeline_512_matches_backend_bitwise():
    counts = torch.as_tensor(disk_input(7, scan=(512, 512)), device=DEV)
    kw = dict(semiangle=21.4, scan_sampling=0.5, det_sampling=1.0, voltage_kV=300)
    rec = ColdReconstructor(counts.clone(), bf_radius=3, **kw)
    rec.load(counts)
    ph = rec.run().clone()
    be = B200SSBBackend(counts, bf_radius=3, **kw)
    _, want = be.object_and_phase(0.0, 0.0, 0.0)
    assert rec.last_info.n_bf == be.num_bf
    np.testing.assert_array_equal(ph.cpu().numpy(), want.cpu().numpy())
