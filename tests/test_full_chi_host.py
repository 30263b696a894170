"""14-term chi on the CPU: the oracle's restatement of chi_full
(common.py:410-471), the polynomial form the kernels evaluate, and the
candidate layout of qssb_full_aberrations_t."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import ssb_oracle as so
from quantem.gpu_b200 import _lib

LAM = so.wavelength_angstrom(300.0)


def _random_full(rng, scale=1.0) -> so.FullAberrations:
    # Angstrom magnitudes of the order met at 300 kV (defocus .. C5)
    typical = np.array([100, 50, 2e3, 1.5e3, 5e4, 1e4, 8e3, 2e5, 1e5, 1e5, 5e6, 1e6, 1e6, 1e6])
    mags = scale * typical * rng.uniform(-1.0, 1.0, 14)
    angs = rng.uniform(-math.pi, math.pi, 14)
    return so.FullAberrations(tuple(mags), tuple(angs))


def _poly_chi(dx, dy, ab: so.FullAberrations, lam: float):
    """The kernels' form (qssb_device.cuh, chi_full_poly): Horner in r2 and in
    z = dx + i dy with K = 2 pi lambda^n C / (n+1) e^{-i m phi}."""
    c0 = np.zeros(3)
    w = np.zeros((6, 3), dtype=complex)
    for (n, m), mag, ang in zip(so.FULL_NM, ab.magnitudes, ab.angles):
        k = 2.0 * math.pi * lam ** n * mag / (n + 1)
        j = (n + 1 - m) // 2
        if m == 0:
            c0[j - 1] += k
        else:
            w[m - 1, j] += k * np.exp(-1j * m * ang)
    z = dx + 1j * dy
    r2 = dx * dx + dy * dy
    s = np.zeros(np.broadcast(dx, dy).shape, dtype=complex)
    for m in range(6, 0, -1):
        s = s * z + (w[m - 1, 0] + r2 * (w[m - 1, 1] + r2 * w[m - 1, 2]))
    return r2 * (c0[0] + r2 * (c0[1] + r2 * c0[2])) + (s * z).real


def test_full_chi_reduces_to_two_term_chi():
    rng = np.random.default_rng(1)
    dx, dy = rng.uniform(-1.5, 1.5, (2, 4096))
    ab = so.Aberrations(-120.0, 55.0, math.radians(17.0), 3.0e4)
    r2 = dx * dx + dy * dy
    ref = so.chi(r2 * LAM * LAM, (dx * dx - dy * dy) / r2, 2 * dx * dy / r2, ab, LAM)
    got = so.chi_full(dx, dy, so.full_from_two_term(ab), LAM)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12)


def test_polynomial_form_matches_the_angle_form():
    rng = np.random.default_rng(2)
    for trial in range(8):
        ab = _random_full(rng)
        dx, dy = rng.uniform(-1.5, 1.5, (2, 2048))
        ref = so.chi_full(dx, dy, ab, LAM)
        got = _poly_chi(dx, dy, ab, LAM)
        np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())


def test_chi_parity_of_odd_and_even_terms():
    """cos(m (phi + pi - a)) = (-1)^m cos(m (phi - a)): odd-m slots are odd in u,
    which is why the full path evaluates every scan frequency."""
    rng = np.random.default_rng(3)
    ab = _random_full(rng)
    dx, dy = rng.uniform(-1.0, 1.0, (2, 512))
    for i, (n, m) in enumerate(so.FULL_NM):
        mags = [0.0] * 14
        mags[i] = ab.magnitudes[i]
        one = so.FullAberrations(tuple(mags), ab.angles)
        a = so.chi_full(dx, dy, one, LAM)
        b = so.chi_full(-dx, -dy, one, LAM)
        np.testing.assert_allclose(b, a if m % 2 == 0 else -a, rtol=1e-9, atol=1e-12)


def test_known_values_at_phi_zero():
    """u along the row axis: chi = (2 pi / lambda) alpha^(n+1) C / (n+1) cos(m a)."""
    u = 0.5
    alpha = LAM * u
    for i, (n, m) in enumerate(so.FULL_NM):
        mags = [0.0] * 14
        angs = [0.0] * 14
        mags[i] = 1.0e4
        angs[i] = 0.3
        got = so.chi_full(np.array([u]), np.array([0.0]), so.FullAberrations(tuple(mags), tuple(angs)), LAM)
        want = 2 * math.pi / LAM * alpha ** (n + 1) * 1.0e4 / (n + 1) * math.cos(m * (0.0 - 0.3))
        assert got[0] == pytest.approx(want, rel=1e-12)


def test_full_oracle_equals_two_term_oracle_on_a_tiny_case():
    from recipes import disk_input

    counts = disk_input(5, scan=(64, 64))
    prep = so.prepare(counts, voltage_kV=300, semiangle_mrad=21.4, scan_sampling=0.5,
                      det_sampling=1.0, bf_radius=2)
    ab = so.Aberrations(-80.0, 30.0, 0.4, 2.0e4)
    l2, mp2 = so.phase_variance_loss(prep.g_half, prep.geo, ab, prep.dc)
    lf, mpf = so.phase_variance_loss(prep.g_half, prep.geo, so.full_from_two_term(ab), prep.dc)
    assert lf == pytest.approx(l2, rel=1e-9)
    assert np.abs(so.wrapped_phase_error(mpf, mp2)).max() < 1e-9


def test_candidate_layout_matches_the_header():
    assert _lib.FULL_TERMS == 14
    assert len(_lib.FULL_TERM_NAMES) == 14
    assert [n for n, _ in so.FULL_NM] == [int(s[1]) for s in _lib.FULL_TERM_NAMES]
    assert [m for _, m in so.FULL_NM] == [int(s[2]) for s in _lib.FULL_TERM_NAMES]
    from pathlib import Path

    header = (Path(__file__).resolve().parent.parent / "include" / "qssb.h").read_text()
    assert "#define QSSB_FULL_TERMS 14" in header
    assert "float magnitude[QSSB_FULL_TERMS];" in header
    assert "float angle_rad[QSSB_FULL_TERMS];" in header
