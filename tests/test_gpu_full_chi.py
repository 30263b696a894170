"""14-term chi on the GPU: the reference's own chi_full /
gamma_mul_pk_onthefly_full (common.py:410-532, compiled from its sources into
oracle/_ref) pin the oracle's restatement; qssb_loss_batch_full is checked
against that oracle at 128^2 and 256^2 (the reference raises at 128,
engine.py:1276-1280, and serves 256 with the same chi)."""
from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from oracle import ssb_oracle as so
from oracle.ref_cuda import build_ref
from quantem.gpu_b200 import B200SSBBackend
from recipes import disk_input

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")

# magnitudes (Angstrom) giving 0.2 - 8 rad per term at the 21.4 mrad aperture edge
MAGS = (-120.0, 55.0, 1500.0, 1000.0, 5.0e4, 3.0e4, 4.0e4, 3.0e6, 2.0e6, 2.0e6,
        1.0e8, 5.0e7, 5.0e7, 5.0e7)
ANGS = tuple(math.radians(a) for a in (0, 17, 30, -40, 0, 65, -20, 10, 80, -55, 0, 5, 45, -70))
FULL = so.FullAberrations(MAGS, ANGS)
KW = dict(voltage_kV=300, semiangle_mrad=21.4, scan_sampling=0.5, det_sampling=1.0, bf_radius=3)


def _case(scan: int, chi_fp64: bool):
    counts = disk_input(123, scan=(scan, scan))
    be = B200SSBBackend(torch.as_tensor(counts, device=DEV), semiangle=21.4, scan_sampling=0.5,
                        det_sampling=1.0, voltage_kV=300, bf_radius=3, chi_fp64=chi_fp64)
    return be, so.prepare(counts, **KW)


@pytest.mark.skipif(not build_ref.available(), reason="reference cubin not built")
def test_reference_chi_full_pins_the_oracle():
    from oracle.ref_cuda.harness import ReferenceObject128

    ref = ReferenceObject128(DEV)
    prep = so.prepare(disk_input(123), **KW)
    geo = prep.geo
    rng = np.random.default_rng(11)
    n = 1 << 16
    b = rng.integers(0, geo.kx.size, n)
    qx = geo.q_row[rng.integers(0, geo.q_row.size, n)].astype(np.float32).astype(np.float64)
    qy = geo.q_col[rng.integers(0, geo.q_col.size, n)].astype(np.float32).astype(np.float64)
    kx = geo.kx[b].astype(np.float32).astype(np.float64)
    ky = geo.ky[b].astype(np.float32).astype(np.float64)
    lam = geo.wavelength
    chi_k = so.chi_full(kx, ky, FULL, lam)
    pk = geo.aperture_k[b] * np.exp(-1j * chi_k)
    g = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=DEV)  # noqa: E731
    chi_ref, out_ref = ref.full_chi_probe(
        t(qx), t(qy), t(kx), t(ky), wavelength=lam, semiangle_rad=geo.semiangle_rad,
        ang_y_rad=geo.ang_row_rad, ang_x_rad=geo.ang_col_rad, magnitudes=MAGS, angles=ANGS,
        pk=t(pk, torch.complex64), g=t(g, torch.complex64))
    chi_ref = chi_ref.cpu().numpy().astype(np.float64)
    chi_o = so.chi_full(qx - kx, qy - ky, FULL, lam)
    inside = np.sqrt((qx - kx) ** 2 + (qy - ky) ** 2) * lam < 0.03
    # float32 fast-math polynomial: a few ulps of the largest term
    assert np.abs(chi_ref - chi_o)[inside].max() <= 2e-5 * (1.0 + np.abs(chi_o[inside]).max())
    # Gamma-hat assembly: compare where |Gamma| is far from the 1e-8 threshold
    _, _, _, am = so._aperture_and_angles(qx - kx, qy - ky, geo)
    _, _, _, ap = so._aperture_and_angles(qx + kx, qy + ky, geo)
    pm = am * np.exp(-1j * chi_o)
    pp = ap * np.exp(-1j * so.chi_full(qx + kx, qy + ky, FULL, lam))
    gam = pm * np.conj(pk) - np.conj(pp) * pk
    ok = np.abs(gam) > 1e-2
    want = g * np.conj(gam / np.abs(np.where(ok, gam, 1.0)))
    got = out_ref.cpu().numpy().astype(np.complex128)
    assert ok.sum() > n // 8
    assert np.abs(got - want)[ok].max() <= 2e-3 * np.abs(g[ok]).max()


@pytest.mark.parametrize("scan", [128, 256])
@pytest.mark.parametrize("chi_fp64", [False, True])
def test_full_chi_loss_and_mean_phase_match_oracle(scan, chi_fp64):
    be, prep = _case(scan, chi_fp64)
    phase, loss = be.reconstruct_full_with_loss(np.array(MAGS), np.array(ANGS))
    ref_loss, ref_mp = so.phase_variance_loss(prep.g_half, prep.geo, FULL, prep.dc)
    err = so.wrapped_phase_error(phase.cpu().numpy(), ref_mp)
    rms = float(np.sqrt(np.mean(err ** 2)))
    assert rms < (2e-6 if chi_fp64 else 2e-5), rms
    assert loss == pytest.approx(ref_loss, rel=2e-5)
    # the flag changes only chi's evaluation precision
    batch = be.variance_loss_batch_full(np.stack([MAGS, np.zeros(14)]),
                                        np.stack([ANGS, np.zeros(14)]))
    assert float(batch[0]) == pytest.approx(loss, rel=1e-6)
    zero_loss, _ = so.phase_variance_loss(prep.g_half, prep.geo, so.full_from_two_term(so.Aberrations()), prep.dc)
    assert float(batch[1]) == pytest.approx(zero_loss, rel=2e-5)
    be.close()


@pytest.mark.parametrize("scan", [128, 256])
def test_full_chi_with_two_terms_matches_the_symmetric_path(scan):
    be, _ = _case(scan, False)
    ab = so.Aberrations(-120.0, 55.0, math.radians(17.0))
    full = so.full_from_two_term(ab)
    ph_f, loss_f = be.reconstruct_full_with_loss(np.array(full.magnitudes), np.array(full.angles))
    ph_s, loss_s = be.reconstruct_with_loss(ab.C10, ab.C12, ab.phi12)
    err = so.wrapped_phase_error(ph_f.cpu().numpy(), ph_s.cpu().numpy())
    assert float(np.sqrt(np.mean(err ** 2))) < 2e-5
    assert loss_f == pytest.approx(loss_s, rel=2e-5)
    be.close()


def test_preview_and_result_route_higher_orders():
    be, prep = _case(128, False)
    ph, loss = be.preview({"C10": 0.0, "C12": 0.0, "phi12": 0.0}, compute_loss=True,
                          higher_order_magnitudes=np.array(MAGS, np.float32),
                          higher_order_angles=np.array(ANGS, np.float32))
    assert ph.dtype == np.float32 and ph.shape == (128, 128)
    ph2, none = be.preview({"C10": 0.0, "C12": 0.0, "phi12": 0.0}, compute_loss=False,
                           higher_order_magnitudes=np.array(MAGS, np.float32),
                           higher_order_angles=np.array(ANGS, np.float32))
    assert none is None
    np.testing.assert_array_equal(ph, ph2)
    # the reference's aberrations-dict format: Cn0 scalars, Cnm_mag + Cnm_angle (deg)
    ab = {"C10": MAGS[0], "C12": MAGS[1], "phi12": ANGS[1]}
    for i, name in enumerate(("C21", "C23", "C30", "C32", "C34", "C41", "C43", "C45", "C50",
                              "C52", "C54", "C56"), start=2):
        if name.endswith("0"):
            ab[name] = MAGS[i]
        else:
            ab[f"{name}_mag"] = MAGS[i]
            ab[f"{name}_angle"] = math.degrees(ANGS[i])
    res = be.reconstruct_result(ab)
    assert res.loss is None
    obj = res.object_wave.cpu().numpy()
    np.testing.assert_allclose(np.abs(obj), 1.0, rtol=1e-6)
    err = so.wrapped_phase_error(np.angle(obj), ph.astype(np.float64))
    assert np.abs(err).max() < 1e-5
    be.close()
