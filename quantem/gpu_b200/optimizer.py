"""Batched aberration search and Nelder-Mead refinement over the GPU loss.

Every candidate set is scored in one ``qssb_loss_batch`` launch sequence, so
the host loop only proposes points and reads back losses.

* ``batch_nelder_mead`` follows the reference's batched simplex
  (bobleesj/quantem.gpu ``ssb/compute/cuda/optimizer.py:237-396``): standard
  Nelder-Mead coefficients (1, 2, 0.5, 0.5), a 5%-or-0.00025 initial step,
  stable tie ordering, the initial simplex and every shrink evaluated as one
  batch.
* ``batch_sweep`` is the seeded global search that replaces the reference's
  Optuna TPE loop (``optimizer.py:59-191``; Optuna is not a dependency here):
  a scrambled Halton sequence over the same search box, evaluated in large
  batches; the minimum-loss point is kept, never an average.
"""
from __future__ import annotations

import math
from typing import Callable

import numpy as np

EvalBatch = Callable[[np.ndarray], np.ndarray]  # (n, 3) [C10, C12, phi12] -> (n,) losses


def batch_nelder_mead(evaluate: EvalBatch, x0: np.ndarray, xatol: float = 0.1,
                      fatol: float = 1e-8, max_iter: int = 300,
                      flat_fatol: float | None = None) -> tuple[np.ndarray, float, int]:
    """Minimise ``evaluate`` from ``x0`` (3 parameters); returns (x, f, n_evals)."""
    x0 = np.asarray(x0, dtype=np.float64)
    n = x0.size
    simplex = np.empty((n + 1, n), dtype=np.float64)
    simplex[0] = x0
    for i in range(n):
        simplex[i + 1] = x0
        simplex[i + 1, i] += max(abs(x0[i]) * 0.05, 0.00025)
    f = np.asarray(evaluate(simplex), dtype=np.float64)
    n_evals = n + 1
    if flat_fatol is not None and np.ptp(f) <= float(flat_fatol):
        return simplex[0], float(f[0]), n_evals
    alpha, gamma, rho, sigma = 1.0, 2.0, 0.5, 0.5

    def one(x: np.ndarray) -> float:
        return float(np.asarray(evaluate(x[None, :]), dtype=np.float64)[0])

    for _ in range(max_iter):
        order = np.argsort(f, kind="stable")
        simplex = simplex[order]
        f = f[order]
        if np.max(np.abs(simplex[-1] - simplex[0])) < xatol and abs(f[-1] - f[0]) < fatol:
            break
        centroid = simplex[:-1].mean(axis=0)
        xr = centroid + alpha * (centroid - simplex[-1])
        fr = one(xr)
        n_evals += 1
        if f[0] <= fr < f[-2]:
            simplex[-1], f[-1] = xr, fr
            continue
        if fr < f[0]:
            xe = centroid + gamma * (xr - centroid)
            fe = one(xe)
            n_evals += 1
            if fe < fr:
                simplex[-1], f[-1] = xe, fe
            else:
                simplex[-1], f[-1] = xr, fr
            continue
        if fr < f[-1]:
            xc = centroid + rho * (xr - centroid)
            fc = one(xc)
            n_evals += 1
            if fc <= fr:
                simplex[-1], f[-1] = xc, fc
                continue
        else:
            xc = centroid - rho * (centroid - simplex[-1])
            fc = one(xc)
            n_evals += 1
            if fc < f[-1]:
                simplex[-1], f[-1] = xc, fc
                continue
        for i in range(1, n + 1):
            simplex[i] = simplex[0] + sigma * (simplex[i] - simplex[0])
        f[1:] = np.asarray(evaluate(simplex[1:]), dtype=np.float64)
        n_evals += n
    best = int(np.argsort(f, kind="stable")[0])
    return simplex[best], float(f[best]), n_evals


def _radical_inverse(i: np.ndarray, base: int) -> np.ndarray:
    out = np.zeros(i.shape, dtype=np.float64)
    f = 1.0 / base
    i = i.copy()
    while np.any(i > 0):
        out += f * (i % base)
        i //= base
        f /= base
    return out


def halton(n: int, dims: int, seed: int) -> np.ndarray:
    """Scrambled (Cranley-Patterson rotated) Halton points in [0, 1)^dims."""
    primes = [2, 3, 5, 7, 11, 13][:dims]
    idx = np.arange(1, n + 1, dtype=np.int64)
    pts = np.stack([_radical_inverse(idx, p) for p in primes], axis=1)
    shift = np.random.default_rng(seed).random(dims)
    return (pts + shift) % 1.0


def search_box(ranges: dict[str, tuple[float, float] | float], defaults: dict[str, float]
               ) -> tuple[list[str], np.ndarray, np.ndarray]:
    """(free keys, low, high) in internal units (phi12 in radians)."""
    keys = [("C10_nm", "C10", 1.0), ("C12_nm", "C12", 1.0), ("phi12_deg", "phi12", math.pi / 180.0)]
    lo, hi = [], []
    for public, internal, scale in keys:
        spec = ranges.get(public, None)
        if isinstance(spec, tuple):
            lo.append(spec[0] * scale)
            hi.append(spec[1] * scale)
        else:
            v = defaults[internal] if spec is None else spec * scale
            lo.append(v)
            hi.append(v)
    return [k[1] for k in keys], np.asarray(lo), np.asarray(hi)


def batch_sweep(evaluate: EvalBatch, low: np.ndarray, high: np.ndarray, n_trials: int,
                seed: int = 42, batch: int = 64) -> tuple[np.ndarray, float, np.ndarray, np.ndarray]:
    """Seeded quasi-random sweep; returns (best_x, best_f, all_x, all_f)."""
    u = halton(n_trials, 3, seed)
    xs = low[None, :] + u * (high - low)[None, :]
    fs = np.empty(n_trials, dtype=np.float64)
    for s in range(0, n_trials, batch):
        fs[s:s + batch] = evaluate(xs[s:s + batch])
    best = int(np.argsort(fs, kind="stable")[0])
    return xs[best], float(fs[best]), xs, fs
