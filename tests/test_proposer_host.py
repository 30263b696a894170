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


def test_resample_table_equals_the_dense_definition():
    """The sparse build (cells near each pixel only) gives exactly the table of
    the definition: every (cell, pixel) tent weight product, cells beyond the
    radius empty, pixels ascending within a cell, rows normalised."""
    rng = np.random.default_rng(3)
    kx = rng.uniform(-1, 1, 700)
    ky = rng.uniform(-1, 1, 700)
    kmax, h, grid, rad = 1.05, 0.09, 16, 0.9
    off, idx, w = pr.resample_table(kx, ky, kmax, h, grid=grid, cell_radius=rad)
    step = 2 * kmax / grid
    centres = -kmax + (np.arange(grid) + 0.5) * step
    for i in range(grid):
        for j in range(grid):
            c = i * grid + j
            tent = (np.clip(1 - np.abs(kx - centres[i]) / h, 0, None)
                    * np.clip(1 - np.abs(ky - centres[j]) / h, 0, None))
            if centres[i] ** 2 + centres[j] ** 2 > rad ** 2:
                tent[:] = 0
            want = np.nonzero(tent > 0)[0]
            np.testing.assert_array_equal(idx[off[c]:off[c + 1]], want)
            if want.size:
                np.testing.assert_allclose(w[off[c]:off[c + 1]], tent[want] / tent[want].sum(),
                                           rtol=1e-6)


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


def test_heads_loss_gradient_is_the_derivative_of_the_loss():
    """The oracle of ``qssb_mse_heads``: with eps = 0 its gradient is the
    derivative of its loss (central differences, away from winner changes);
    one head is the plain MSE; the losing heads get eps / (heads - 1) of
    their own MSE gradient."""
    rng = np.random.default_rng(3)
    m, n_out, heads = 5, 4, 4
    y = rng.normal(size=(m, 16))
    t = rng.normal(size=(m, n_out))
    w = np.array([1.0, 1.0, 1.0, 0.1])
    loss, dy, win = po.heads_loss_and_grad(y, t, n_out, heads, w, 3, 0.0)
    h = 1e-6
    for r in range(m):
        for c in range(16):
            yp, ym = y.copy(), y.copy()
            yp[r, c] += h
            ym[r, c] -= h
            lp = po.heads_loss_and_grad(yp, t, n_out, heads, w, 3, 0.0)[0]
            lm = po.heads_loss_and_grad(ym, t, n_out, heads, w, 3, 0.0)[0]
            assert abs((lp - lm) / (2 * h) - dy[r, c]) < 1e-6
    l1, dy1, _ = po.heads_loss_and_grad(y, t, n_out, 1)
    np.testing.assert_allclose(l1, np.mean((y[:, :4] - t) ** 2))
    np.testing.assert_allclose(dy1[:, :4], 2 * (y[:, :4] - t) / (m * n_out))
    assert not dy1[:, 4:].any()
    _, dye, _ = po.heads_loss_and_grad(y, t, n_out, heads, w, 3, 0.3)
    for r in range(m):
        for hh in range(heads):
            d = 2 * w * (y[r, 4 * hh:4 * hh + 4] - t[r]) / (m * n_out)
            s = 0.7 if hh == win[r] else 0.1
            np.testing.assert_allclose(dye[r, 4 * hh:4 * hh + 4], s * d, rtol=1e-12)


def test_quadratic_refine_converges_from_a_proposal_in_few_rounds():
    """From the best of eight hypotheses (one within ~15 A of the truth in C1
    and A1, seven decoys) the refinement reaches 0.05 A of the truth of a
    quadratic-plus-quartic bowl within 6 rounds of 8 evaluations, one loss
    batch per round, C3 held at the hypothesis's (true) value."""
    rng = np.random.default_rng(0)
    widths = np.array([20.0, 20.0, 20.0, 3000.0])
    for trial in range(5):
        truth = np.array([rng.uniform(-400, 400), rng.uniform(10, 90), rng.uniform(0, 3),
                          rng.uniform(500, 9000)])
        be = _QuarticLoss(truth, widths, seed=trial)
        tx = pr.to_x(truth[None])[0]
        good = tx + np.append(rng.normal(0.0, 8.0, 3), 0.0)
        decoys = tx + rng.normal(0.0, 1.0, (7, 4)) * np.array([300.0, 80.0, 80.0, 4000.0])
        hyps = np.vstack([decoys[:3], good, decoys[3:]])

        def done(est):
            return np.linalg.norm(pr.to_x(est[None])[0][:3] - tx[:3]) < 0.05

        best, evals, rounds, ok = pr.quadratic_refine(be, hyps, 8.0, 8, 12, done=done)
        assert ok and done(best), trial
        assert evals == 8 * rounds and be.calls == rounds
        assert rounds <= 6, (trial, rounds)
        # without a stopping rule it converges on its own (the step falls below 0.05 A)
        be2 = _QuarticLoss(truth, widths, seed=trial)
        best2, _, _, ok2 = pr.quadratic_refine(be2, hyps, 8.0, 8, 40)
        assert ok2 and np.linalg.norm(pr.to_x(best2[None])[0][:3] - tx[:3]) < 0.5


def test_learned_refine_falls_back_to_the_plain_sweep():
    """When the refinement cannot meet the target within its rounds, the
    plain 64-candidate sweep runs and its evaluations are added."""
    truth = np.array([120.0, 30.0, 0.4, 4000.0])
    be = _QuarticLoss(truth, np.array([20.0, 20.0, 20.0, 3000.0]))
    tx = pr.to_x(truth[None])[0]
    calls = {"n": 0}

    def done(est):  # met only once the plain sweep has scored a few batches
        calls["n"] += 1
        return be.calls > 8 and np.linalg.norm(pr.to_x(est[None])[0][:3] - tx[:3]) < 40.0

    best, evals, rounds, fell_back = pr.learned_refine(be, tx[None] + 200.0, rounds=4, done=done)
    assert fell_back
    assert evals == 8 * 4 + 64 * (be.calls - 4)
    lo, hi = pr.refine_box()
    assert np.all(lo < pr.BOX_LO) and np.all(hi > pr.BOX_HI)
