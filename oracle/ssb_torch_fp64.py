"""FP64 GPU restatement of the SSB oracle (TEST INFRASTRUCTURE, never the product).

The numpy oracle (``ssb_oracle.py``) is the FP64 arbiter of parity; at 256^2
scans its scan FFTs and trotter sums take minutes on the host. This module
evaluates the same algorithm, line for line, in torch float64/complex128 on
a GPU: the "FP64 GPU path" the 256^2 precision study compares the float32
kernels with. The host-side decisions (mean pattern, BF selection, geometry)
are the numpy oracle's own functions; only the bulk arithmetic runs on the
device:

* scan FFT - ``ssb_oracle.scan_fft_half`` (backend.py:520-589), as a float64
  ``rfft2`` of the gathered BF images;
* corrected spectra and trotter sum - ``ssb_oracle.corrected_spectra`` /
  ``fourier_sum`` (kernels/common.py:115-236, engine.py:1047-1107);
* object wave - ``ssb_oracle.object_wave`` (engine.py:1109-1151);
* phase-variance loss - ``ssb_oracle.phase_variance_loss`` (engine.py:1464-1514).

Pinned against the numpy oracle in tests/test_fp64_path.py.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import ssb_oracle as so


@dataclass
class PreparedGPU:
    scan_shape: tuple[int, int]
    bf: so.BrightField
    g_half: torch.Tensor      # complex128 [B, R0, R1/2+1]
    dc: complex
    wavelength: float
    geo: so.Geometry
    dev: dict                 # the geometry arrays as float64 device tensors


def prepare(counts: torch.Tensor, *, voltage_kV: float, semiangle_mrad: float,
            scan_sampling: float, det_sampling: float, bf_intensity_threshold: float = 0.0,
            bf_radius: float | None = None, rotation_rad: float = 0.0,
            chunk: int = 128) -> PreparedGPU:
    """``ssb_oracle.prepare`` for a device u16 [R0, R1, K0, K1] (no padding)."""
    r0, r1, k0, k1 = (int(s) for s in counts.shape)
    frames = counts.reshape(-1, k0, k1)
    sums = frames.sum(dim=0, dtype=torch.int64).cpu().numpy().view(np.uint64)
    mean_dp = sums.astype(np.float32) / np.float32(frames.shape[0])
    bf = so.select_bright_field(mean_dp, bf_intensity_threshold, bf_radius)
    rows = torch.as_tensor(bf.rows, device=counts.device, dtype=torch.int64)
    cols = torch.as_tensor(bf.cols, device=counts.device, dtype=torch.int64)
    n_bf = int(rows.numel())
    g = torch.empty((n_bf, r0, r1 // 2 + 1), dtype=torch.complex128, device=counts.device)
    bits = frames.view(torch.int16)
    for s in range(0, n_bf, chunk):
        e = min(n_bf, s + chunk)
        img = (bits[:, rows[s:e], cols[s:e]].to(torch.int32) & 0xFFFF).to(torch.float64)
        g[s:e] = torch.fft.rfft2(img.T.reshape(e - s, r0, r1))
    dc = complex(g[:, 0, 0].mean().item())
    lam = so.wavelength_angstrom(voltage_kV)
    geo = so.geometry(bf.rows, bf.cols, bf.center, (r0, r1), (scan_sampling, scan_sampling),
                      (det_sampling, det_sampling), lam, semiangle_mrad, rotation_rad)
    dev = {k: torch.as_tensor(np.asarray(getattr(geo, k), np.float64), device=counts.device)
           for k in ("kx", "ky", "alpha_k2", "cos2phi_k", "sin2phi_k", "aperture_k", "q_row", "q_col")}
    return PreparedGPU((r0, r1), bf, g, dc, lam, geo, dev)


def _aperture_and_angles(dx, dy, geo: so.Geometry):
    """``ssb_oracle._aperture_and_angles`` in torch float64."""
    r2 = dx * dx + dy * dy
    lam = geo.wavelength
    alpha2 = r2 * lam * lam
    safe = r2 > 1e-300
    inv_r2 = torch.where(safe, 1.0 / torch.where(safe, r2, torch.ones_like(r2)), torch.zeros_like(r2))
    cos2 = (dx * dx - dy * dy) * inv_r2
    sin2 = 2.0 * dx * dy * inv_r2
    r = torch.sqrt(r2)
    inv_r = torch.where(safe, 1.0 / torch.where(safe, r, torch.ones_like(r)), torch.zeros_like(r))
    denom = torch.sqrt((dx * geo.ang_row_rad) ** 2 + (dy * geo.ang_col_rad) ** 2) * inv_r
    ok = denom > 1e-300
    edge = torch.where(ok, (geo.semiangle_rad - r * lam) / torch.where(ok, denom, torch.ones_like(denom))
                       + 0.5, torch.ones_like(denom))
    return alpha2, cos2, sin2, edge.clamp(0.0, 1.0)


def _chi(alpha2, cos2, sin2, ab: so.Aberrations, lam: float):
    factor = math.pi / lam
    out = factor * alpha2 * (ab.C10 + ab.C12 * (cos2 * math.cos(2 * ab.phi12)
                                                  + sin2 * math.sin(2 * ab.phi12)))
    if ab.C30 != 0.0:
        out = out + 0.5 * factor * ab.C30 * alpha2 * alpha2
    return out


def _chi_full(dx, dy, ab: so.FullAberrations, lam: float):
    """``ssb_oracle.chi_full`` in torch float64."""
    alpha = torch.sqrt(dx * dx + dy * dy) * lam
    phi = torch.atan2(dy, dx)
    out = torch.zeros_like(alpha)
    for (n, m), mag, ang in zip(so.FULL_NM, ab.magnitudes, ab.angles):
        if mag != 0.0:
            out = out + alpha ** (n + 1) * (mag / (n + 1)) * torch.cos(m * (phi - ang))
    return (2.0 * math.pi / lam) * out


def _chi_at(dx, dy, alpha2, cos2, sin2, ab, lam: float):
    if isinstance(ab, so.FullAberrations):
        return _chi_full(dx, dy, ab, lam)
    return _chi(alpha2, cos2, sin2, ab, lam)


def _corrected_chunks(prep: PreparedGPU, ab: so.Aberrations, chunk: int):
    """C_b(q) = G_b(q) conj(Gamma_hat_b(q)), full plane, DC := dc, per BF chunk
    (``ssb_oracle.corrected_spectra``)."""
    geo, d = prep.geo, prep.dev
    r0, r1 = prep.scan_shape
    half = r1 // 2 + 1
    n_bf = prep.g_half.shape[0]
    mirror_rows = torch.as_tensor((-np.arange(r0)) % r0, device=prep.g_half.device)
    mirror_cols = torch.as_tensor(r1 - np.arange(half, r1), device=prep.g_half.device)
    qx = d["q_row"][None, :, None]
    qy = d["q_col"][None, None, :]
    for s in range(0, n_bf, chunk):
        e = min(n_bf, s + chunk)
        gh = prep.g_half[s:e]
        g = torch.empty((e - s, r0, r1), dtype=torch.complex128, device=gh.device)
        g[:, :, :half] = gh
        g[:, :, half:] = torch.conj(gh[:, mirror_rows][:, :, mirror_cols])
        kx = d["kx"][s:e, None, None]
        ky = d["ky"][s:e, None, None]
        chi_k = _chi_at(d["kx"][s:e], d["ky"][s:e], d["alpha_k2"][s:e], d["cos2phi_k"][s:e],
                        d["sin2phi_k"][s:e], ab, geo.wavelength)
        pk = (d["aperture_k"][s:e] * torch.exp(-1j * chi_k))[:, None, None]
        am2, cm, sm, apm = _aperture_and_angles(qx - kx, qy - ky, geo)
        ap2, cp, sp, app = _aperture_and_angles(qx + kx, qy + ky, geo)
        pm = apm * torch.exp(-1j * _chi_at(qx - kx, qy - ky, am2, cm, sm, ab, geo.wavelength))
        pp = app * torch.exp(-1j * _chi_at(qx + kx, qy + ky, ap2, cp, sp, ab, geo.wavelength))
        gamma = pm * torch.conj(pk) - torch.conj(pp) * pk
        mag2 = gamma.real ** 2 + gamma.imag ** 2
        big = mag2 > 1e-16
        scale = torch.where(big, 1.0 / torch.sqrt(torch.where(big, mag2, torch.ones_like(mag2))),
                            torch.full_like(mag2, 1e8))
        corrected = g * torch.conj(gamma * scale)
        corrected[:, 0, 0] = prep.dc
        yield corrected


def fourier_sum(prep: PreparedGPU, ab: so.Aberrations, chunk: int = 32) -> torch.Tensor:
    """Sum over BF pixels of C_b(q) on the full plane (complex128)."""
    r0, r1 = prep.scan_shape
    total = torch.zeros((r0, r1), dtype=torch.complex128, device=prep.g_half.device)
    for corrected in _corrected_chunks(prep, ab, chunk):
        total += corrected.sum(dim=0)
    return total


def phase_variance_loss(prep: PreparedGPU, ab: so.Aberrations, chunk: int = 32):
    """``ssb_oracle.phase_variance_loss``: (loss, mean phase [R0, R1])."""
    r0, r1 = prep.scan_shape
    s1 = torch.zeros((r0, r1), dtype=torch.float64, device=prep.g_half.device)
    s2 = torch.zeros_like(s1)
    for corrected in _corrected_chunks(prep, ab, chunk):
        ang = torch.angle(torch.fft.ifft2(corrected))
        s1 += ang.sum(dim=0)
        s2 += (ang * ang).sum(dim=0)
    n_b = prep.g_half.shape[0]
    mean_phase = s1 / n_b
    var = s2 / n_b - mean_phase * mean_phase
    return float(var.mean().item()), mean_phase


def reconstruct(prep: PreparedGPU, ab: so.Aberrations) -> tuple[torch.Tensor, torch.Tensor]:
    """Object wave (complex128) and phase (float64), ``ssb_oracle.reconstruct``."""
    obj = torch.fft.ifft2(fourier_sum(prep, ab) / prep.g_half.shape[0])
    return obj, torch.angle(obj)
