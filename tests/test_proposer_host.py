"""Host-side pieces of the learned proposer (no GPU): resampling tables,
target canonicalisation, and the sign symmetry of trotter amplitudes that
the canonical targets rely on (checked with the FP64 oracle)."""
from __future__ import annotations

import math

import numpy as np

from oracle import proposer_oracle as po
from oracle import ssb_oracle as so
from quantem.gpu_b200 import proposer as pr


def test_resample_table_rows_are_normalised_tents():
    rng = np.random.default_rng(0)
    kx = rng.uniform(-1, 1, 300)
    ky = rng.uniform(-1, 1, 300)
    off, idx, w = pr.resample_table(kx, ky, 1.05, 0.2, grid=16)
    assert off.size == 16 * 16 + 1 and off[-1] == idx.size == w.size
    for c in range(16 * 16):
        if off[c + 1] > off[c]:
            assert abs(w[off[c]:off[c + 1]].sum() - 1.0) < 1e-5
    # every pixel referenced lies inside its cell's tent support
    step = 2.1 / 16
    for c in (0, 37, 200):
        cx = -1.05 + (c // 16 + 0.5) * step
        cy = -1.05 + (c % 16 + 0.5) * step
        b = idx[off[c]:off[c + 1]]
        assert np.all(np.abs(kx[b] - cx) < 0.2) and np.all(np.abs(ky[b] - cy) < 0.2)


def test_targets_round_trip_and_flip():
    rng = np.random.default_rng(1)
    from quantem.gpu_b200.synthetic import draw_aberrations

    ab = draw_aberrations(rng, 64).astype(np.float64)
    t = pr.canonical_targets(ab)
    dec = pr.decode(t)
    canon = np.where(ab[:, :1] < 0, pr.flipped(ab), ab)
    np.testing.assert_allclose(dec[:, 0], canon[:, 0], rtol=1e-5, atol=1e-3)
    np.testing.assert_allclose(dec[:, 1], canon[:, 1], rtol=1e-4, atol=1e-3)
    d = np.angle(np.exp(2j * (dec[:, 2] - canon[:, 2])))
    assert np.abs(d[canon[:, 1] > 1.0]).max() < 1e-3
    np.testing.assert_allclose(dec[:, 3], canon[:, 3], rtol=1e-5, atol=1e-1)
    np.testing.assert_allclose(pr.flipped(pr.flipped(ab)), np.column_stack(
        [ab[:, 0], ab[:, 1], np.mod(ab[:, 2], np.pi), ab[:, 3]]), atol=1e-9)


def test_trotter_amplitude_is_invariant_under_aberration_sign_flip():
    lam = so.wavelength_angstrom(300)
    lat_rows, lat_cols = np.nonzero(np.ones((9, 9)))
    geo = so.geometry(lat_rows, lat_cols, (4.0, 4.0), (64, 64), (0.5, 0.5), (20 / 12, 20 / 12),
                      lam, 20.0)
    ab = so.Aberrations(230.0, 40.0, 0.7, 3000.0)
    fl = pr.flipped(np.array([[ab.C10, ab.C12, ab.phi12, ab.C30]]))[0]
    g1 = po.gamma(0.25, -0.125, geo.kx, geo.ky, geo.alpha_k2, geo.cos2phi_k, geo.sin2phi_k,
                  geo.aperture_k, ab, geo)
    g2 = po.gamma(0.25, -0.125, geo.kx, geo.ky, geo.alpha_k2, geo.cos2phi_k, geo.sin2phi_k,
                  geo.aperture_k, so.Aberrations(*map(float, fl)), geo)
    np.testing.assert_allclose(np.abs(g1), np.abs(g2), atol=1e-12)
    assert np.abs(g1 - g2).max() > 1e-3  # the phases do differ


class _QuarticLoss:
    """A stand-in backend whose loss is a convex quadratic plus a quartic in
    the scaled search coordinates, minimum at ``truth``."""

    def __init__(self, truth, widths, seed=1):
        self.t = pr.to_x(np.asarray(truth, np.float64)[None])[0]
        a = np.random.default_rng(seed).normal(size=(4, 4))
        self.h = a @ a.T / 4 + np.eye(4)
        self.w = np.asarray(widths, np.float64)
        self.calls = 0

    def variance_loss_batch(self, c10, c12, phi12, c30):
        import torch

        x = pr.to_x(np.stack([c10, c12, phi12, c30], axis=1))
        u = (x - self.t) / self.w
        self.calls += 1
        return torch.tensor(1.0 + np.einsum("ni,ij,nj->n", u, self.h, u) + 0.3 * np.sum(u ** 4, 1),
                            dtype=torch.float32)


def test_surrogate_search_converges_on_a_quartic_bowl():
    """The trust-region quadratic refinement reaches 1e-3 of the search widths
    from a start about 0.7 widths away within 10 rounds of 8 evaluations, one
    loss batch per round."""
    rng = np.random.default_rng(0)
    widths = np.array([120.0, 40.0, 40.0, 5000.0])
    for trial in range(5):
        truth = np.array([rng.uniform(-400, 400), rng.uniform(10, 90), rng.uniform(0, 3),
                          rng.uniform(500, 9000)])
        start = truth + np.array([40.0, 20.0, 0.3, 2000.0]) * rng.normal(size=4)
        start[1] = abs(start[1])
        be = _QuarticLoss(truth, widths)
        tx = pr.to_x(truth[None])[0]

        def done(est):
            return np.linalg.norm((pr.to_x(est[None])[0] - tx) / widths) < 1e-3

        best, evals, rounds = pr.surrogate_search(be, pr.to_x(start[None]), widths, 8, 30,
                                                  np.random.default_rng(2), done=done)
        assert done(best), trial
        assert evals == 8 * rounds and be.calls == rounds
        assert rounds <= 10, (trial, rounds)


def test_surrogate_search_step_stays_in_the_trust_region():
    """The model step of a non-convex quadratic lies on the trust-region
    boundary; a convex one inside it is the Newton step."""
    d = 4
    coef = np.zeros(1 + d + d * (d + 1) // 2)
    coef[1:1 + d] = [1.0, -2.0, 0.5, 0.0]
    k = 1 + d
    diag = [-1.0, 2.0, 3.0, 1.0]
    for i in range(d):
        for j in range(i, d):
            if i == j:
                coef[k] = 0.5 * diag[i]
            k += 1
    u = pr._model_step(coef, d, "full", 0.3)
    assert abs(np.linalg.norm(u) - 0.3) < 1e-6
    coef[1 + d] = 0.5 * 4.0  # h00 = 4: convex
    u = pr._model_step(coef, d, "full", 10.0)
    np.testing.assert_allclose(u, -np.array([1.0, -2.0, 0.5, 0.0]) / np.array([4.0, 2.0, 3.0, 1.0]),
                               rtol=1e-9)
