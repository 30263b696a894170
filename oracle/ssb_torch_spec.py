"""CPU torch restatement of the reference's executable SSB specification.

TEST/BASELINE INFRASTRUCTURE ONLY (see ``oracle/__init__.py``). The reference
has no CPU SSB path (CPU is never a fallback, workflow.py:92-111); its
executable CPU specification is the PyTorch code of ``docs/kernels/ssb.md``
(lines 69-366): ``select_bright_field``, ``scan_fft``, ``probe``,
``corrected_object``, ``phase_variance_loss``, ``final_object``. This module
restates those steps, in float32/complex64 like the spec, with the BF axis
processed in chunks so that a 128^4 workload fits in host memory. It is the
timed CPU baseline of ``bench.py`` (``kind: "port"``), run with every host
thread torch can use.
"""
from __future__ import annotations

import math
import os

import numpy as np
import torch

from . import ssb_oracle as so


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1


def select_bright_field(counts: torch.Tensor, rows: np.ndarray, cols: np.ndarray):
    """Mean DP (float32) and the selected BF columns (R0, R1, B); ssb.md:69-92."""
    mean_k = counts.to(torch.float32).mean(dim=(0, 1))
    selected = counts[:, :, torch.as_tensor(rows, dtype=torch.long), torch.as_tensor(cols, dtype=torch.long)]
    return mean_k, selected


def scan_fft(selected: torch.Tensor) -> torch.Tensor:
    """(B, R0, R1) complex64 scan spectra; ssb.md:105-112."""
    return torch.fft.fft2(selected.permute(2, 0, 1).to(torch.complex64))


def _polar(dx: torch.Tensor, dy: torch.Tensor, lam: float, semi: float, ang_r: float, ang_c: float):
    r2 = dx * dx + dy * dy
    r = torch.sqrt(r2)
    alpha = r * lam
    safe_r = torch.where(r > 0, r, torch.ones_like(r))
    denom = torch.sqrt((dx * ang_r) ** 2 + (dy * ang_c) ** 2) / safe_r
    ok = denom > 0
    edge = torch.where(ok, (semi - alpha) / torch.where(ok, denom, torch.ones_like(denom)) + 0.5,
                       torch.ones_like(denom))
    return alpha * alpha, torch.atan2(dy, dx), torch.clamp(edge, 0.0, 1.0)


def probe(alpha2, azimuth, aperture, theta, wavelength: float) -> torch.Tensor:
    """P = A exp(-i chi), chi = (pi/lambda) alpha^2 (C10 + C12 cos 2(az - phi12)); ssb.md:177-196."""
    c10, c12, phi12 = theta
    chi = (math.pi / wavelength) * alpha2 * (c10 + c12 * torch.cos(2 * (azimuth - phi12)))
    return aperture * torch.exp(-1j * chi)


def corrected_object(g: torch.Tensor, kx: torch.Tensor, ky: torch.Tensor, k_polar, q_row, q_col,
                     theta, cal: dict, dc: complex) -> torch.Tensor:
    """O_b(R) = ifft2(G_b conj(Gamma_hat_b)), DC := dc; ssb.md:197-225."""
    lam, semi, ang_r, ang_c = cal["wavelength"], cal["semi"], cal["ang_r"], cal["ang_c"]
    qx = q_row[None, :, None]
    qy = q_col[None, None, :]
    kxb = kx[:, None, None]
    kyb = ky[:, None, None]
    p_k = probe(*k_polar, theta, lam)[:, None, None]
    p_minus = probe(*_polar(kxb - qx, kyb - qy, lam, semi, ang_r, ang_c), theta, lam)
    p_plus = probe(*_polar(kxb + qx, kyb + qy, lam, semi, ang_r, ang_c), theta, lam)
    gamma = p_minus * p_k.conj() - p_plus.conj() * p_k
    unit = gamma / gamma.abs().clamp_min(1e-8)
    corrected = g * unit.conj()
    corrected[:, 0, 0] = dc
    return torch.fft.ifft2(corrected)


def reconstruct(counts_np: np.ndarray, *, voltage_kV: float, semiangle_mrad: float,
                scan_sampling: float, det_sampling: float, theta=(0.0, 0.0, 0.0),
                bf_stride: int = 1, chunk: int = 128, with_loss: bool = False):
    """u16 counts -> object phase, following the spec on CPU torch.

    ``bf_stride > 1`` evaluates every ``bf_stride``-th BF pixel (a bounded
    sample of the per-BF work); the mean DP pass always covers all data.
    Returns (phase float32 [R0, R1], loss or None, n_bf_evaluated, n_bf).
    """
    torch.set_num_threads(host_threads())
    counts = torch.from_numpy(counts_np)
    lam = so.wavelength_angstrom(voltage_kV)
    mean_k = counts.to(torch.float32).mean(dim=(0, 1))
    bf = so.select_bright_field(mean_k.numpy().astype(np.float32))
    rows, cols = bf.rows[::bf_stride], bf.cols[::bf_stride]
    r0, r1 = int(counts.shape[0]), int(counts.shape[1])
    recip = det_sampling * 1e-3 / lam
    kx = torch.as_tensor((rows - bf.center[0]) * recip, dtype=torch.float32)
    ky = torch.as_tensor((cols - bf.center[1]) * recip, dtype=torch.float32)
    q_row = torch.as_tensor(np.fft.fftfreq(r0, scan_sampling), dtype=torch.float32)
    q_col = torch.as_tensor(np.fft.fftfreq(r1, scan_sampling), dtype=torch.float32)
    cal = dict(wavelength=lam, semi=semiangle_mrad * 1e-3, ang_r=det_sampling * 1e-3,
               ang_c=det_sampling * 1e-3)
    k_polar = _polar(kx, ky, lam, cal["semi"], cal["ang_r"], cal["ang_c"])
    theta_t = tuple(torch.tensor(float(v), dtype=torch.float32) for v in theta)
    flat_rows = torch.as_tensor(rows, dtype=torch.long)
    flat_cols = torch.as_tensor(cols, dtype=torch.long)
    dc = None
    obj_sum = torch.zeros((r0, r1), dtype=torch.complex64)
    s1 = torch.zeros((r0, r1)) if with_loss else None
    s2 = torch.zeros((r0, r1)) if with_loss else None
    gs = []
    for s in range(0, rows.size, chunk):
        sel = counts[:, :, flat_rows[s:s + chunk], flat_cols[s:s + chunk]]
        gs.append(scan_fft(sel))
    g_all = torch.cat(gs)
    dc = complex(g_all[:, 0, 0].mean())
    for s in range(0, rows.size, chunk):
        e = min(rows.size, s + chunk)
        kpol = tuple(t[s:e] for t in k_polar)
        obj_b = corrected_object(g_all[s:e], kx[s:e], ky[s:e], kpol, q_row, q_col, theta_t, cal, dc)
        obj_sum += obj_b.sum(dim=0)
        if with_loss:
            ph = torch.angle(obj_b)
            s1 += ph.sum(dim=0)
            s2 += (ph * ph).sum(dim=0)
    n = rows.size
    obj = obj_sum / n
    loss = None
    if with_loss:
        mean = s1 / n
        loss = float((s2 / n - mean * mean).mean())
    return torch.angle(obj).numpy().astype(np.float32), loss, n, bf.rows.size
