"""Host-side SSB calibration: scan padding rule, BF selection, BF geometry.

These are the reference backend's small control decisions, taken on the
64 KB mean diffraction pattern and the few-thousand BF pixels after the GPU
has done the heavy reduction. Each restates the reference
(bobleesj/quantem.gpu 0.0.1rc6) and keeps its float32 decisions, because
they decide which detector pixels enter the reconstruction:

* ``pad_target`` / padding rule - ``ssb/compute/cuda/backend.py:229-269``;
* ``select_bf`` - ``backend.py:448-518`` (``_compute_bf_mask_from_mean_dp``);
* ``detect_bf_radius`` - ``detector/compute/cuda/probe.py:12-119``;
* ``bf_geometry`` - ``ssb/compute/cuda/engine.py:784-830``
  (``SSBEngine.cache_rotation``), float32 like the reference's CuPy arrays;
* ``scan_frequencies`` - ``backend.py:44-82`` (``spatial_frequencies``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

SUPPORTED_SCAN_SIZES = (128, 256, 512, 1024)


def pad_target(h: int, w: int) -> tuple[int, int] | None:
    """Square scan size the reference pads/crops (h, w) to; None if supported."""
    if (h, w) in {(s, s) for s in SUPPORTED_SCAN_SIZES}:
        return None
    longest = max(h, w)
    t = next((s for s in SUPPORTED_SCAN_SIZES[:-1] if longest <= s), 1024)
    return (t, t)


@dataclass(frozen=True)
class BFSelection:
    rows: np.ndarray           # int32 [B], row-major nonzero order
    cols: np.ndarray           # int32 [B]
    center: tuple[float, float]
    radius: float


def select_bf(mean_dp: np.ndarray, threshold: float = 0.0,
              bf_radius: float | None = None) -> BFSelection:
    """BF pixels from the float32 mean diffraction pattern (reference rule)."""
    dp = np.asarray(mean_dp, dtype=np.float32)
    mask = dp > dp.max() * np.float32(threshold)
    rows, cols = np.nonzero(mask)
    rows = rows.astype(np.int32)
    cols = cols.astype(np.int32)
    if rows.size == 0:
        raise ValueError(
            f"No bright-field pixels found with threshold {threshold:.2f}. Check that "
            "the data contains a visible BF disk, or lower the threshold."
        )
    if bf_radius is None:
        probe_mask = dp > dp.mean() + dp.std()
        total = int(probe_mask.sum())
        if total > 0:
            probe = probe_mask.astype(np.float32)
            rc = np.arange(dp.shape[0], dtype=np.float32).reshape(-1, 1)
            cc = np.arange(dp.shape[1], dtype=np.float32).reshape(1, -1)
            center = (float((rc * probe).sum() / total), float((cc * probe).sum() / total))
            radius = math.sqrt(total / math.pi)
        else:
            center = (dp.shape[0] / 2.0, dp.shape[1] / 2.0)
            radius = min(dp.shape) * 0.25
    else:
        weights = dp[rows, cols].astype(np.float32)
        wsum = float(weights.sum())
        if wsum > 0:
            center = (float((rows.astype(np.float32) * weights).sum() / wsum),
                      float((cols.astype(np.float32) * weights).sum() / wsum))
        else:
            center = (float(rows.mean()), float(cols.mean()))
        radius = float(bf_radius)
    d2 = (rows.astype(np.float32) - center[0]) ** 2 + (cols.astype(np.float32) - center[1]) ** 2
    keep = d2 <= radius ** 2
    rows, cols = rows[keep], cols[keep]
    if rows.size == 0:
        raise ValueError(
            f"No bright-field pixels within bf_radius={radius}. Increase bf_radius or "
            "check detector geometry."
        )
    return BFSelection(rows=rows, cols=cols, center=center, radius=radius)


def detect_bf_radius(mean_dp: np.ndarray, threshold_ratio: float = 0.1
                     ) -> tuple[tuple[int, int], int]:
    """BF disk centre and half-max radius of the smoothed radial profile
    (detector/compute/cuda/probe.py:12-119), on the host copy of the 64 KB
    mean pattern; the backend sets det_sampling = 2 alpha / r from it
    (backend.py:276-285)."""
    dp = np.asarray(mean_dp, dtype=np.float32)
    if dp.ndim != 2 or 0 in dp.shape:
        raise ValueError(f"Expected a non-empty 2D diffraction pattern, got {dp.shape}")
    dp_max = float(np.nanmax(dp))
    if not np.isfinite(dp_max) or dp_max <= 0:
        raise ValueError("Diffraction pattern has no positive finite values.")
    mask = dp > threshold_ratio * dp_max
    if not mask.any():
        raise ValueError(
            f"No pixels above threshold ({threshold_ratio:.0%} of max intensity). "
            "The diffraction pattern may be too noisy or empty.")
    mask_f = mask.astype(np.float32)
    total = float(mask_f.sum())
    n0, n1 = dp.shape
    rc = np.arange(n0, dtype=np.float32).reshape(-1, 1)
    cc = np.arange(n1, dtype=np.float32).reshape(1, -1)
    r0 = max(0, min(int(round(float((rc * mask_f).sum() / total))), n0 - 1))
    c0 = max(0, min(int(round(float((cc * mask_f).sum() / total))), n1 - 1))
    dr = np.arange(n0, dtype=np.float32) - r0
    dcol = np.arange(n1, dtype=np.float32) - c0
    rr = np.sqrt(dr[:, None] ** 2 + dcol[None, :] ** 2)
    max_r = min(r0, c0, n0 - r0, n1 - c0)
    if max_r < 2:
        return (r0, c0), max(1, min(n0, n1) // 4)
    r_int = np.rint(rr).astype(np.int32).ravel()
    flat = dp.ravel()
    valid = r_int < max_r
    profile = np.zeros(max_r, dtype=np.float32)
    counts = np.zeros(max_r, dtype=np.float32)
    np.add.at(profile, r_int[valid], flat[valid])
    np.add.at(counts, r_int[valid], 1.0)
    nz = counts > 0
    profile[nz] /= counts[nz]
    if profile.size > 5:
        sigma = 2.0
        ksize = int(6 * sigma + 1) | 1
        x = np.arange(ksize, dtype=np.float32) - ksize // 2
        kernel = np.exp(-0.5 * (x / sigma) ** 2).astype(np.float32)
        kernel /= kernel.sum()
        padded = np.pad(profile, ksize // 2, mode="edge")
        smooth = np.convolve(padded, kernel, mode="valid")[: profile.size]
        half = float(smooth[:5].mean()) * 0.5
        below = np.nonzero(smooth < half)[0]
        radius = int(below[0]) if below.size else int(profile.size) // 2
    else:
        radius = min(n0, n1) // 4
    return (r0, c0), max(1, radius)


@dataclass(frozen=True)
class BFGeometry:
    """Rotation-dependent per-BF arrays (float32, reference cache names)."""

    kx_bf: np.ndarray
    ky_bf: np.ndarray
    alpha_k2: np.ndarray
    cos2phi_k: np.ndarray
    sin2phi_k: np.ndarray
    aperture_k: np.ndarray
    kx_lo: np.ndarray           # FP64 residual: kx_fp64 = kx_bf + kx_lo
    ky_lo: np.ndarray

    def stacked(self) -> np.ndarray:
        """[8, B] float32 in the order the C ABI's ``bf_geom`` expects."""
        return np.stack([self.kx_bf, self.ky_bf, self.alpha_k2, self.cos2phi_k,
                         self.sin2phi_k, self.aperture_k, self.kx_lo, self.ky_lo]).astype(np.float32)


def bf_geometry(rows: np.ndarray, cols: np.ndarray, center: tuple[float, float],
                detector_shape: tuple[int, int], sampling: tuple[float, float],
                wavelength: float, semiangle_mrad: float,
                angular_sampling: tuple[float, float], rotation_rad: float) -> BFGeometry:
    """Per-BF k-vector, alpha^2, cos/sin 2phi and soft aperture (float32)."""
    recip_r = 1.0 / (sampling[0] * detector_shape[0])
    recip_c = 1.0 / (sampling[1] * detector_shape[1])
    iy = np.arange(detector_shape[0], dtype=np.float32) - np.float32(center[0])
    ix = np.arange(detector_shape[1], dtype=np.float32) - np.float32(center[1])
    kxa = iy[:, None] * np.float32(recip_r)
    kya = ix[None, :] * np.float32(recip_c)
    cos_a = math.cos(-rotation_rad)
    sin_a = math.sin(-rotation_rad)
    kxr = kxa * np.float32(cos_a) + kya * np.float32(sin_a)
    kyr = -kxa * np.float32(sin_a) + kya * np.float32(cos_a)
    kx = kxr[rows, cols].astype(np.float32)
    ky = kyr[rows, cols].astype(np.float32)
    k_mag = np.sqrt(kx * kx + ky * ky)
    phi = np.arctan2(ky, kx)
    alpha = k_mag * np.float32(wavelength)
    cphi = np.cos(phi)
    sphi = np.sin(phi)
    semi = semiangle_mrad * 1e-3
    ang_r, ang_c = angular_sampling
    denom = np.sqrt((cphi * np.float32(ang_r * 1e-3)) ** 2 + (sphi * np.float32(ang_c * 1e-3)) ** 2)
    aperture = np.clip((np.float32(semi) - alpha) / denom + np.float32(0.5), 0, 1).astype(np.float32)
    # the same k in FP64 (carried as a float32 residual for near-tied overlaps)
    kr64 = (rows.astype(np.float64) - center[0]) * recip_r
    kc64 = (cols.astype(np.float64) - center[1]) * recip_c
    kx64 = kr64 * cos_a + kc64 * sin_a
    ky64 = -kr64 * sin_a + kc64 * cos_a
    return BFGeometry(
        kx_bf=kx, ky_bf=ky,
        alpha_k2=(alpha ** 2).astype(np.float32),
        cos2phi_k=(cphi * cphi - sphi * sphi).astype(np.float32),
        sin2phi_k=(np.float32(2.0) * sphi * cphi).astype(np.float32),
        aperture_k=aperture,
        kx_lo=(kx64 - kx.astype(np.float64)).astype(np.float32),
        ky_lo=(ky64 - ky.astype(np.float64)).astype(np.float32),
    )


def scan_frequencies(scan_shape: tuple[int, int], scan_sampling: tuple[float, float]
                     ) -> tuple[np.ndarray, np.ndarray]:
    """fftfreq grids (1/A) of the scan axes, float32."""
    return (np.fft.fftfreq(scan_shape[0], scan_sampling[0]).astype(np.float32),
            np.fft.fftfreq(scan_shape[1], scan_sampling[1]).astype(np.float32))
