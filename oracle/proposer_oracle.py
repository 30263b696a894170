"""FP64 CPU restatement of the learned proposer's kernels (TEST INFRASTRUCTURE).

Checks ``qssb_synth_features`` / ``qssb_trotter_features`` (forward model
Gamma(Q, k) as ``ssb_oracle`` evaluates it from kernels/common.py:115-236 of
bobleesj/quantem.gpu, CSR tent resampling, per-Q mean normalisation) and the
MLP's forward pass and gradients (``qssb_gemm_bf16``, ``qssb_gelu_backward``,
``qssb_bias_grad``, ``qssb_mse``, ``qssb_mse_heads``). The reference has no
learned component, so this oracle follows the definitions in
quantem/gpu_b200/proposer.py and the standard back-propagation of a GELU MLP
under a (winner-takes-all) mean-squared error.
"""
from __future__ import annotations

import math

import numpy as np

from . import ssb_oracle as so


def gamma(qx: float, qy: float, kx: np.ndarray, ky: np.ndarray, alpha_k2, cos2_k, sin2_k, ap_k,
          ab: so.Aberrations, geo: so.Geometry) -> np.ndarray:
    """Gamma(Q, k_b) = P(Q-k) conj P(k) - conj P(Q+k) P(k), FP64 (complex [B])."""
    chi_k = so.chi(alpha_k2, cos2_k, sin2_k, ab, geo.wavelength)
    pk = ap_k * np.exp(-1j * chi_k)
    am2, cm, sm, apm = so._aperture_and_angles(qx - kx, qy - ky, geo)
    ap2, cp, sp, app = so._aperture_and_angles(qx + kx, qy + ky, geo)
    pm = apm * np.exp(-1j * so.chi(am2, cm, sm, ab, geo.wavelength))
    pp = app * np.exp(-1j * so.chi(ap2, cp, sp, ab, geo.wavelength))
    return pm * np.conj(pk) - np.conj(pp) * pk


def resample(values: np.ndarray, off: np.ndarray, idx: np.ndarray, w: np.ndarray) -> np.ndarray:
    """values [n_q][B] -> features [n_q][cells], normalised by the mean of covered cells."""
    n_q = values.shape[0]
    cells = off.size - 1
    out = np.zeros((n_q, cells))
    covered = off[1:] > off[:-1]
    for c in range(cells):
        e0, e1 = off[c], off[c + 1]
        if e1 > e0:
            out[:, c] = values[:, idx[e0:e1]] @ w[e0:e1].astype(np.float64)
    mean = out[:, covered].mean(axis=1, keepdims=True)
    return np.where(mean > 0, out / np.where(mean > 0, mean, 1.0), 0.0)


def gelu(x):
    s = math.sqrt(2.0 / math.pi)
    return 0.5 * x * (1.0 + np.tanh(s * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    s = math.sqrt(2.0 / math.pi)
    u = s * (x + 0.044715 * x ** 3)
    t = np.tanh(u)
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * s * (1.0 + 3 * 0.044715 * x * x)


def heads_loss_and_grad(y: np.ndarray, target: np.ndarray, n_out: int, heads: int = 1,
                        out_weight=None, n_select: int | None = None, eps: float = 0.0):
    """Winner-takes-all MSE of ``qssb_mse_heads`` in FP64: row r of y holds
    ``heads`` groups of n_out outputs; the winner has the least squared error
    over the first n_select outputs (ties: lowest index); loss = mean over
    rows of sum_c w_c (y_win,c - t_c)^2 / n_out; dy_h,c = 2 s_h w_c (y_h,c -
    t_c) / (rows n_out), s = 1 - eps for the winner, eps / (heads - 1) for the
    others, 1 with one head. Returns (loss, dy, winners)."""
    y = np.asarray(y, np.float64)
    t = np.asarray(target, np.float64)
    m = y.shape[0]
    n_select = n_out if n_select is None else n_select
    w = np.ones(n_out) if out_weight is None else np.asarray(out_weight, np.float64)
    yh = y[:, :heads * n_out].reshape(m, heads, n_out)
    d = yh - t[:, None, :]
    win = np.argmin(np.sum(d[..., :n_select] ** 2, axis=-1), axis=1)
    dw = d[np.arange(m), win]
    loss = float(np.sum(w * dw * dw) / (m * n_out))
    s = np.full((m, heads), eps / max(1, heads - 1))
    s[np.arange(m), win] = 1.0 - eps if heads > 1 else 1.0
    dy = np.zeros_like(y)
    dy[:, :heads * n_out] = (2.0 * s[:, :, None] * w * d / (m * n_out)).reshape(m, heads * n_out)
    return loss, dy, win


def mlp_loss_and_grads(x: np.ndarray, ws: list, bs: list, target: np.ndarray, n_out: int,
                       heads: int = 1, out_weight=None, n_select: int | None = None,
                       eps: float = 0.0):
    """Winner-takes-all MSE (``heads_loss_and_grad``; plain MSE over the first
    n_out outputs with one head); returns (loss, outputs, [dW], [db]) in FP64."""
    a = [np.asarray(x, np.float64)]
    zs = []
    for i, (w, b) in enumerate(zip(ws, bs)):
        z = a[-1] @ w + b
        zs.append(z)
        if i < len(ws) - 1:
            a.append(gelu(z))
    y = zs[-1]
    loss, dy, _ = heads_loss_and_grad(y, target, n_out, heads, out_weight, n_select, eps)
    dws, dbs = [None] * len(ws), [None] * len(ws)
    g = dy
    for i in range(len(ws) - 1, -1, -1):
        dws[i] = a[i].T @ g
        dbs[i] = g.sum(axis=0)
        if i > 0:
            g = (g @ ws[i].T) * gelu_grad(zs[i - 1])
    return loss, y, dws, dbs
