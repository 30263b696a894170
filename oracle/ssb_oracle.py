"""FP64 numpy oracle for the SSB ptychography path (test infrastructure only).

Every function restates one step of the reference (bobleesj/quantem.gpu,
version 0.0.1rc6) and cites the file:line it follows. Paths are relative to
the reference project root.

Precision policy: decisions the reference takes in float32 (the mean
diffraction pattern, the bright-field threshold, the centroid and the radius
cut) are reproduced in float32 exactly, because they choose *which* detector
pixels enter the sum. Everything downstream (FFTs, probe phase, overlap
normalisation, sums, inverse FFT, atan2) is evaluated in float64: this is the
"FP64 oracle" every GPU result is compared with.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

# Pre-computed relativistic wavelengths in Angstrom for common voltages.
# Same table values as src/quantem/gpu/optics/physics.py:24-30 (physical
# constants, kept identical so that lambda(300 kV) matches bit for bit).
_COMMON_WAVELENGTHS_A = {
    80: 0.041757160772834,
    120: 0.033492152726724,
    200: 0.025079340450548,
    300: 0.019687489006849,
    400: 0.016439434169908,
}

SUPPORTED_SCAN_SIZES = (128, 256, 512, 1024)


def wavelength_angstrom(voltage_kV: float) -> float:
    """Relativistic electron wavelength in Angstrom.

    Follows ``wavelength_A_from_kV`` (src/quantem/gpu/optics/physics.py:33-86):
    table lookup for integral common voltages, else the relativistic de
    Broglie formula lambda = h / sqrt(2 m e V (1 + e V / (2 m c^2))).
    """
    v_int = int(voltage_kV)
    if v_int == voltage_kV and v_int in _COMMON_WAVELENGTHS_A:
        return _COMMON_WAVELENGTHS_A[v_int]
    h = 6.62607015e-34
    m = 9.1093837015e-31
    e = 1.602176634e-19
    c = 299792458.0
    volts = voltage_kV * 1e3
    gamma = 1.0 + e * volts / (2.0 * m * c * c)
    return h / math.sqrt(2.0 * m * e * volts * gamma) * 1e10


def pad_or_crop_scan(data: np.ndarray) -> np.ndarray:
    """Pad (with the dtype-truncated mean DP) or centre-crop to a supported scan.

    Follows ``CudaSSBBackend.__init__`` (src/quantem/gpu/ssb/compute/cuda/
    backend.py:229-269): shapes other than 128/256/512/1024 squares go to the
    smallest supported square that holds the longest side; oversize axes are
    centre-cropped, undersize axes padded with the mean diffraction pattern,
    which is an integer sum divided in float64 and cast back to the source
    dtype (truncation for integers).
    """
    h, w = int(data.shape[0]), int(data.shape[1])
    if (h, w) in {(s, s) for s in SUPPORTED_SCAN_SIZES}:
        return data
    longest = max(h, w)
    target = next((s for s in SUPPORTED_SCAN_SIZES[:-1] if longest <= s), 1024)
    if h > target or w > target:
        r0 = max(0, (h - target) // 2)
        c0 = max(0, (w - target) // 2)
        data = data[r0:r0 + min(target, h), c0:c0 + min(target, w)]
        h, w = int(data.shape[0]), int(data.shape[1])
    if h < target or w < target:
        pad_top = (target - h) // 2
        pad_left = (target - w) // 2
        det = data.shape[2:]
        flat = data.reshape(-1, det[0] * det[1])
        if np.issubdtype(data.dtype, np.integer):
            acc = flat.astype(np.int64).sum(axis=0)
        else:
            acc = flat.astype(np.float64).sum(axis=0)
        mean_dp = (acc.reshape(det).astype(np.float64) / flat.shape[0]).astype(data.dtype)
        padded = np.broadcast_to(mean_dp[None, None], (target, target) + tuple(det)).copy()
        padded[pad_top:pad_top + h, pad_left:pad_left + w] = data
        data = padded
    return data


def mean_dp_u64(data: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Exact u64 detector sums and the float32 mean diffraction pattern.

    Follows ``CudaSSBBackend._compute_bf_mask`` (backend.py:432-441):
    ``frames.sum(axis=0, dtype=uint64).astype(float32) / N``.
    Returns (sums u64 [K0, K1], mean_dp f32 [K0, K1]).
    """
    frames = data.reshape(-1, data.shape[-2], data.shape[-1])
    sums = frames.sum(axis=0, dtype=np.uint64)
    mean_dp = sums.astype(np.float32) / int(frames.shape[0])
    return sums, mean_dp.astype(np.float32, copy=False)


@dataclass(frozen=True)
class BrightField:
    """Selected BF pixels in row-major ``nonzero`` order plus the disk fit."""

    rows: np.ndarray
    cols: np.ndarray
    center: tuple[float, float]
    radius: float


def select_bright_field(
    mean_dp: np.ndarray,
    threshold: float = 0.0,
    bf_radius: float | None = None,
) -> BrightField:
    """Bright-field mask from the mean DP, reproducing float32 decisions.

    Follows ``CudaSSBBackend._compute_bf_mask_from_mean_dp``
    (backend.py:448-518): threshold at ``max * thr``; with ``bf_radius=None``
    the probe is ``mean_dp > mean + std``, its centroid the disk centre and
    ``sqrt(count / pi)`` the radius; with an explicit radius the centre is the
    intensity-weighted centroid of the thresholded pixels. Pixels with
    float32 ``dist^2 <= r^2`` are kept.
    """
    mean_dp = np.asarray(mean_dp, dtype=np.float32)
    mask = mean_dp > mean_dp.max() * np.float32(threshold)
    rows, cols = np.nonzero(mask)
    rows = rows.astype(np.int32)
    cols = cols.astype(np.int32)
    if rows.size == 0:
        raise ValueError(
            f"No bright-field pixels found with threshold {threshold:.2f}."
        )
    if bf_radius is None:
        probe_mask = mean_dp > mean_dp.mean() + mean_dp.std()
        probe_total = int(probe_mask.sum())
        if probe_total > 0:
            probe = probe_mask.astype(np.float32)
            rc = np.arange(mean_dp.shape[0], dtype=np.float32).reshape(-1, 1)
            cc = np.arange(mean_dp.shape[1], dtype=np.float32).reshape(1, -1)
            center_row = float((rc * probe).sum() / probe_total)
            center_col = float((cc * probe).sum() / probe_total)
            radius = math.sqrt(probe_total / math.pi)
        else:
            center_row = mean_dp.shape[0] / 2.0
            center_col = mean_dp.shape[1] / 2.0
            radius = min(mean_dp.shape) * 0.25
    else:
        weights = mean_dp[rows, cols].astype(np.float32)
        weight_sum = float(weights.sum())
        if weight_sum > 0:
            center_row = float((rows.astype(np.float32) * weights).sum() / weight_sum)
            center_col = float((cols.astype(np.float32) * weights).sum() / weight_sum)
        else:
            center_row = float(rows.mean())
            center_col = float(cols.mean())
        radius = float(bf_radius)
    dist_sq = (rows.astype(np.float32) - center_row) ** 2 + (
        cols.astype(np.float32) - center_col
    ) ** 2
    within = dist_sq <= radius ** 2
    rows = rows[within]
    cols = cols[within]
    if rows.size == 0:
        raise ValueError(f"No bright-field pixels within bf_radius={radius}.")
    return BrightField(rows=rows, cols=cols, center=(center_row, center_col), radius=radius)


def scan_fft_half(
    data: np.ndarray,
    rows: np.ndarray,
    cols: np.ndarray,
) -> tuple[np.ndarray, complex]:
    """Per-BF-pixel scan FFT, Hermitian half-plane, FP64.

    Follows ``CudaSSBBackend._extract_gqk`` (backend.py:520-589): gather the
    BF columns, ``fft2`` over the two scan axes, keep columns ``0..R1/2`` and
    ``dc = mean_b G_b[0, 0]``. Returns (G [B, R0, R1//2+1] complex128, dc).
    """
    r0, r1 = int(data.shape[0]), int(data.shape[1])
    flat = data.reshape(r0 * r1, data.shape[2], data.shape[3])
    b = int(rows.size)
    half = r1 // 2 + 1
    g = np.empty((b, r0, half), dtype=np.complex128)
    chunk = 256
    for s in range(0, b, chunk):
        e = min(b, s + chunk)
        images = flat[:, rows[s:e], cols[s:e]].T.reshape(e - s, r0, r1).astype(np.float64)
        g[s:e] = np.fft.rfft2(images)
    dc = complex(g[:, 0, 0].mean())
    return g, dc


def expand_hermitian(half: np.ndarray, ncols: int) -> np.ndarray:
    """Full-plane spectrum from the half plane: G[r, c] = conj(G[-r, N - c]).

    Follows ``ld_gqk_maybe_herm`` (kernels/common.py:65-84).
    """
    n_b, n_r, stored = half.shape
    full = np.empty((n_b, n_r, ncols), dtype=half.dtype)
    full[:, :, :stored] = half
    mirror_rows = (-np.arange(n_r)) % n_r
    mirror_cols = ncols - np.arange(stored, ncols)
    full[:, :, stored:] = np.conj(half[:, mirror_rows][:, :, mirror_cols])
    return full


@dataclass(frozen=True)
class Geometry:
    """Rotation-dependent BF geometry and scan frequencies (float64)."""

    kx: np.ndarray          # [B] row component of k_b, 1/A
    ky: np.ndarray          # [B] col component of k_b, 1/A
    alpha_k2: np.ndarray    # [B]
    cos2phi_k: np.ndarray   # [B]
    sin2phi_k: np.ndarray   # [B]
    aperture_k: np.ndarray  # [B]
    q_row: np.ndarray       # [R0] fftfreq(R0, d=scan_sampling_row)
    q_col: np.ndarray       # [R1]
    wavelength: float
    semiangle_rad: float
    ang_row_rad: float
    ang_col_rad: float


def geometry(
    rows: np.ndarray,
    cols: np.ndarray,
    center: tuple[float, float],
    scan_shape: tuple[int, int],
    scan_sampling: tuple[float, float],
    det_sampling_mrad: tuple[float, float],
    wavelength: float,
    semiangle_mrad: float,
    rotation_rad: float = 0.0,
) -> Geometry:
    """BF k-vectors, probe geometry at k_b and scan frequencies, FP64.

    Follows ``SSBEngine.cache_rotation`` (engine.py:784-830):
    ``k = (i - centre) * (det_sampling * 1e-3 / lambda)`` per axis, passive
    rotation by ``-theta``, ``alpha = lambda |k|``, ``phi = atan2(k_col, k_row)``
    and the soft aperture ``clip((alpha_max - alpha)/denom + 0.5, 0, 1)`` with
    ``denom = sqrt((cos(phi) d_row)^2 + (sin(phi) d_col)^2)``. Scan
    frequencies follow ``spatial_frequencies`` (backend.py:44-82).
    """
    recip_r = det_sampling_mrad[0] * 1e-3 / wavelength
    recip_c = det_sampling_mrad[1] * 1e-3 / wavelength
    kr = (rows.astype(np.float64) - center[0]) * recip_r
    kc = (cols.astype(np.float64) - center[1]) * recip_c
    cos_a = math.cos(-rotation_rad)
    sin_a = math.sin(-rotation_rad)
    kx = kr * cos_a + kc * sin_a
    ky = -kr * sin_a + kc * cos_a
    k_mag = np.sqrt(kx * kx + ky * ky)
    phi = np.arctan2(ky, kx)
    alpha = k_mag * wavelength
    ang_r = det_sampling_mrad[0] * 1e-3
    ang_c = det_sampling_mrad[1] * 1e-3
    semi = semiangle_mrad * 1e-3
    denom = np.sqrt((np.cos(phi) * ang_r) ** 2 + (np.sin(phi) * ang_c) ** 2)
    aperture = np.clip((semi - alpha) / denom + 0.5, 0.0, 1.0)
    return Geometry(
        kx=kx,
        ky=ky,
        alpha_k2=alpha * alpha,
        cos2phi_k=np.cos(2.0 * phi),
        sin2phi_k=np.sin(2.0 * phi),
        aperture_k=aperture,
        q_row=np.fft.fftfreq(scan_shape[0], scan_sampling[0]),
        q_col=np.fft.fftfreq(scan_shape[1], scan_sampling[1]),
        wavelength=float(wavelength),
        semiangle_rad=semi,
        ang_row_rad=ang_r,
        ang_col_rad=ang_c,
    )


def _aperture_and_angles(dx, dy, geo: Geometry):
    """alpha^2, cos 2phi, sin 2phi and soft aperture at displacement (dx, dy).

    Follows ``compute_geometry`` (kernels/common.py:115-157) in FP64, with the
    same conventions at |u| = 0 (cos 2phi = sin 2phi = 0, aperture 1 when
    the aperture edge is outside the origin).
    """
    r2 = dx * dx + dy * dy
    lam = geo.wavelength
    alpha2 = r2 * lam * lam
    safe = r2 > 1e-300
    inv_r2 = np.where(safe, 1.0 / np.where(safe, r2, 1.0), 0.0)
    cos2 = (dx * dx - dy * dy) * inv_r2
    sin2 = 2.0 * dx * dy * inv_r2
    r = np.sqrt(r2)
    alpha = r * lam
    inv_r = np.where(safe, 1.0 / np.where(safe, r, 1.0), 0.0)
    denom = np.sqrt((dx * geo.ang_row_rad) ** 2 + (dy * geo.ang_col_rad) ** 2) * inv_r
    ok = denom > 1e-300
    edge = np.where(ok, (geo.semiangle_rad - alpha) / np.where(ok, denom, 1.0) + 0.5, 1.0)
    aperture = np.clip(edge, 0.0, 1.0)
    return alpha2, cos2, sin2, aperture


@dataclass(frozen=True)
class Aberrations:
    """Two-term aberrations in the reference's numeric convention.

    ``C10`` and ``C12`` enter chi numerically in Angstrom (the reference labels
    them nm but never converts: engine.py:456 and common.py:201-205), ``phi12``
    in radians. ``C30`` (spherical aberration, same numeric length unit) is an
    optional extension of the reference's 14-term Krivanek chi
    (common.py:410-471, slot 4: ``(2 pi / lambda) C30 alpha^4 / 4``).
    """

    C10: float = 0.0
    C12: float = 0.0
    phi12: float = 0.0
    C30: float = 0.0


def chi(alpha2, cos2phi, sin2phi, ab: Aberrations, wavelength: float):
    """chi = (pi/lambda) alpha^2 (C10 + C12 cos 2(phi - phi12)) + (pi/2lambda) C30 alpha^4.

    Follows ``_pk_kernel`` (engine.py:217-231) and ``gamma_mul_pk_onthefly``
    (kernels/common.py:173-205); the C30 term follows ``chi_full``
    (common.py:410-471).
    """
    factor = math.pi / wavelength
    cos_term = cos2phi * math.cos(2.0 * ab.phi12) + sin2phi * math.sin(2.0 * ab.phi12)
    out = factor * alpha2 * (ab.C10 + ab.C12 * cos_term)
    if ab.C30 != 0.0:
        out = out + 0.5 * factor * ab.C30 * alpha2 * alpha2
    return out


# Slot layout of the 14-term chi (aberration.py:63 of the reference):
# (n, m) of C10, C12, C21, C23, C30, C32, C34, C41, C43, C45, C50, C52, C54, C56.
FULL_NM = ((1, 0), (1, 2), (2, 1), (2, 3), (3, 0), (3, 2), (3, 4),
           (4, 1), (4, 3), (4, 5), (5, 0), (5, 2), (5, 4), (5, 6))


@dataclass(frozen=True)
class FullAberrations:
    """The 14 Krivanek coefficients: magnitudes (length unit of C10) and
    angles phi_nm in radians, slot order ``FULL_NM`` (engine.py:1244-1262)."""

    magnitudes: tuple
    angles: tuple


def chi_full(dx, dy, ab: FullAberrations, wavelength: float):
    """chi = (2 pi / lambda) sum_i alpha^(n_i+1) C_i / (n_i+1) cos(m_i (phi - phi_i)).

    Follows ``chi_full`` and ``pack_aberration_coefs`` (kernels/common.py:
    410-471, 646-674) in FP64, with alpha = lambda |u| and phi = atan2(dy, dx)
    evaluated directly (the reference reaches cos(m phi) by a Chebyshev
    recurrence from dx / |u|; at |u| = 0 both give chi = 0).
    """
    r = np.sqrt(dx * dx + dy * dy)
    alpha = r * wavelength
    phi = np.arctan2(dy, dx)
    out = np.zeros(np.broadcast(dx, dy).shape)
    for (n, m), mag, ang in zip(FULL_NM, ab.magnitudes, ab.angles):
        if mag == 0.0:
            continue
        out = out + alpha ** (n + 1) * (mag / (n + 1)) * np.cos(m * (phi - ang))
    return (2.0 * math.pi / wavelength) * out


def full_from_two_term(ab: Aberrations) -> FullAberrations:
    """The same chi as ``ab`` in the 14-slot layout."""
    mags = [0.0] * 14
    angs = [0.0] * 14
    mags[0], mags[1], angs[1], mags[4] = ab.C10, ab.C12, ab.phi12, ab.C30
    return FullAberrations(tuple(mags), tuple(angs))


def _chi_at(dx, dy, alpha2, cos2, sin2, ab, wavelength: float):
    if isinstance(ab, FullAberrations):
        return chi_full(dx, dy, ab, wavelength)
    return chi(alpha2, cos2, sin2, ab, wavelength)


def corrected_spectra(
    g_half: np.ndarray,
    geo: Geometry,
    ab: Aberrations,
    dc: complex,
    bf: slice,
) -> np.ndarray:
    """C_b(q) = G_b(q) conj(Gamma_hat_b(q)) over the full plane, DC := dc.

    Follows ``gamma_mul_pk_onthefly`` (kernels/common.py:173-236) and the DC
    override of ``ifft128_rows_fused_pk_t32_mr8_packed`` (kernels/fft128.py:
    98-100): Gamma = P(q-k) conj(P(k)) - conj(P(q+k)) P(k) with
    P = A exp(-i chi); Gamma_hat = Gamma / |Gamma| when |Gamma|^2 > 1e-16,
    else Gamma * 1e8.
    """
    n_r = geo.q_row.size
    n_c = geo.q_col.size
    g = expand_hermitian(g_half[bf], n_c)
    kx = geo.kx[bf][:, None, None]
    ky = geo.ky[bf][:, None, None]
    qx = geo.q_row[None, :, None]
    qy = geo.q_col[None, None, :]
    chi_k = _chi_at(geo.kx[bf], geo.ky[bf], geo.alpha_k2[bf], geo.cos2phi_k[bf],
                    geo.sin2phi_k[bf], ab, geo.wavelength)
    pk = (geo.aperture_k[bf] * np.exp(-1j * chi_k))[:, None, None]
    am2, cm, sm, apm = _aperture_and_angles(qx - kx, qy - ky, geo)
    ap2, cp_, sp, app = _aperture_and_angles(qx + kx, qy + ky, geo)
    pm = apm * np.exp(-1j * _chi_at(qx - kx, qy - ky, am2, cm, sm, ab, geo.wavelength))
    pp = app * np.exp(-1j * _chi_at(qx + kx, qy + ky, ap2, cp_, sp, ab, geo.wavelength))
    gamma = pm * np.conj(pk) - np.conj(pp) * pk
    mag2 = gamma.real ** 2 + gamma.imag ** 2
    scale = np.where(mag2 > 1e-16, 1.0 / np.sqrt(np.where(mag2 > 1e-16, mag2, 1.0)), 1e8)
    corrected = g * np.conj(gamma * scale)
    corrected[:, 0, 0] = dc
    assert corrected.shape[1:] == (n_r, n_c)
    return corrected


def fourier_sum(
    g_half: np.ndarray,
    geo: Geometry,
    ab: Aberrations,
    dc: complex,
    chunk: int = 128,
) -> np.ndarray:
    """S(q) = sum_b C_b(q) (the trotter sum), full plane, FP64."""
    n_b = g_half.shape[0]
    total = np.zeros((geo.q_row.size, geo.q_col.size), dtype=np.complex128)
    for s in range(0, n_b, chunk):
        total += corrected_spectra(g_half, geo, ab, dc, slice(s, min(n_b, s + chunk))).sum(axis=0)
    return total


def object_wave(
    g_half: np.ndarray,
    geo: Geometry,
    ab: Aberrations,
    dc: complex,
) -> np.ndarray:
    """O = (1/B) sum_b ifft2(C_b) = ifft2((1/B) sum_b C_b), FP64.

    Follows ``SSBEngine.reconstruct_object`` (engine.py:1109-1151) and the
    Fourier-sum path ``_reconstruct_object_fourier_sum`` (engine.py:1047-1107);
    B counts every selected BF pixel, including aperture-0 ones.
    """
    n_b = g_half.shape[0]
    return np.fft.ifft2(fourier_sum(g_half, geo, ab, dc) / n_b)


def phase(obj: np.ndarray) -> np.ndarray:
    """Object phase ``angle(O)`` (results.py:117-122)."""
    return np.angle(obj)


def phase_moments(
    g_half: np.ndarray,
    geo: Geometry,
    ab: Aberrations,
    dc: complex,
    chunk: int = 128,
) -> tuple[np.ndarray, np.ndarray]:
    """Per-pixel sum_b phi_b and sum_b phi_b^2 with phi_b = angle(ifft2(C_b)).

    Follows ``reconstruct_with_loss`` + ``_sum_sumsq_phase_kernel``
    (engine.py:49-73, 1464-1514).
    """
    n_b = g_half.shape[0]
    s1 = np.zeros((geo.q_row.size, geo.q_col.size))
    s2 = np.zeros_like(s1)
    for s in range(0, n_b, chunk):
        ang = np.angle(np.fft.ifft2(corrected_spectra(g_half, geo, ab, dc, slice(s, min(n_b, s + chunk)))))
        s1 += ang.sum(axis=0)
        s2 += (ang * ang).sum(axis=0)
    return s1, s2


def phase_variance_loss(
    g_half: np.ndarray,
    geo: Geometry,
    ab: Aberrations,
    dc: complex,
) -> tuple[float, np.ndarray]:
    """L = mean_R[(1/B) sum phi_b^2 - ((1/B) sum phi_b)^2] and mean phase.

    Follows the reference objective (docs/kernels/ssb.md:256-266;
    engine.py:1503-1514). Returns (loss, mean_phase [R0, R1]).
    """
    n_b = g_half.shape[0]
    s1, s2 = phase_moments(g_half, geo, ab, dc)
    mean_phase = s1 / n_b
    var = s2 / n_b - mean_phase * mean_phase
    return float(var.mean()), mean_phase


@dataclass
class Prepared:
    """Everything the reference prepares once per dataset (a1-a8)."""

    scan_shape: tuple[int, int]
    detector_shape: tuple[int, int]
    sums: np.ndarray
    mean_dp: np.ndarray
    bf: BrightField
    g_half: np.ndarray
    dc: complex
    wavelength: float
    sampling: tuple[float, float]
    geo: Geometry


def detect_bf_radius(mean_dp: np.ndarray, threshold_ratio: float = 0.1
                     ) -> tuple[tuple[int, int], int]:
    """BF disk centre and half-maximum radius of the mean DP
    (detector/compute/cuda/probe.py:12-119): centre of mass of the pixels
    above ``threshold_ratio`` of the maximum, rounded; mean intensity per
    integer-rounded radius out to the nearest edge; that profile smoothed by a
    normalised 13-tap Gaussian (sigma 2, edge-padded); the radius is the first
    bin below half the mean of the first five smoothed bins. Profile sums are
    taken in FP64 and rounded once (the reference adds float32 atomically, in
    no fixed order)."""
    dp = np.asarray(mean_dp, dtype=np.float32)
    if dp.ndim != 2 or 0 in dp.shape:
        raise ValueError(f"Expected a non-empty 2D diffraction pattern, got shape {dp.shape}")
    peak = float(np.nanmax(dp))
    if not np.isfinite(peak) or peak <= 0:
        raise ValueError("Diffraction pattern has no positive finite values")
    above = dp > np.float32(threshold_ratio * peak)
    if not above.any():
        raise ValueError("No pixels above threshold")
    n0, n1 = dp.shape
    rr, cc = np.nonzero(above)
    r0 = min(max(int(round(float(np.float32(rr.mean())))), 0), n0 - 1)
    c0 = min(max(int(round(float(np.float32(cc.mean())))), 0), n1 - 1)
    edge = min(r0, c0, n0 - r0, n1 - c0)
    if edge < 2:
        return (r0, c0), max(1, min(n0, n1) // 4)
    dist = np.sqrt(np.add.outer((np.arange(n0) - r0) ** 2, (np.arange(n1) - c0) ** 2).astype(np.float32))
    ring = np.rint(dist).astype(np.int64).ravel()
    keep = ring < edge
    total = np.bincount(ring[keep], weights=dp.ravel()[keep].astype(np.float64), minlength=edge)
    count = np.bincount(ring[keep], minlength=edge)
    prof = np.where(count > 0, total / np.maximum(count, 1), total).astype(np.float32)
    if prof.size <= 5:
        return (r0, c0), max(1, min(n0, n1) // 4)
    taps = np.exp(-0.5 * ((np.arange(13, dtype=np.float32) - 6) / np.float32(2.0)) ** 2)
    taps = (taps / taps.sum()).astype(np.float32)
    ext = np.concatenate([np.full(6, prof[0]), prof, np.full(6, prof[-1])]).astype(np.float32)
    smooth = np.array([np.dot(ext[i:i + 13].astype(np.float64), taps[::-1].astype(np.float64))
                       for i in range(prof.size)], dtype=np.float32)
    half = 0.5 * float(smooth[:5].mean())
    low = np.nonzero(smooth < half)[0]
    radius = int(low[0]) if low.size else prof.size // 2
    return (r0, c0), max(1, radius)


def prepare(
    data: np.ndarray,
    *,
    voltage_kV: float,
    semiangle_mrad: float,
    scan_sampling: float | tuple[float, float],
    det_sampling: float | tuple[float, float] | None,
    bf_intensity_threshold: float = 0.0,
    bf_radius: float | None = None,
    rotation_rad: float = 0.0,
    pad: bool = True,
) -> Prepared:
    """u16 4D data -> resident SSB state, reference semantics (a1-a8).

    ``pad=False`` keeps a native (non-power-of-two) scan: the reference always
    pads (backend.py:229-269); the native variant exists only to check the
    GPU path's native-size mode.
    """
    if data.ndim != 4:
        raise ValueError("data must be 4D (R0, R1, K0, K1)")
    if pad:
        data = pad_or_crop_scan(data)
    if isinstance(scan_sampling, (int, float)):
        scan_sampling = (float(scan_sampling), float(scan_sampling))
    lam = wavelength_angstrom(voltage_kV)
    det = (int(data.shape[2]), int(data.shape[3]))
    sums, mean_dp = mean_dp_u64(data)
    if det_sampling is None:
        # backend.py:276-285: det_sampling = 2 alpha / r from the detected radius
        _, radius = detect_bf_radius(mean_dp)
        det_sampling = (2.0 * semiangle_mrad) / radius
    if isinstance(det_sampling, (int, float)):
        det_sampling = (float(det_sampling), float(det_sampling))
    bf = select_bright_field(mean_dp, bf_intensity_threshold, bf_radius)
    g_half, dc = scan_fft_half(data, bf.rows, bf.cols)
    recip = (det_sampling[0] * 1e-3 / lam, det_sampling[1] * 1e-3 / lam)
    sampling = (1.0 / (recip[0] * det[0]), 1.0 / (recip[1] * det[1]))
    scan_shape = (int(data.shape[0]), int(data.shape[1]))
    geo = geometry(
        bf.rows, bf.cols, bf.center, scan_shape, tuple(scan_sampling),
        tuple(det_sampling), lam, semiangle_mrad, rotation_rad,
    )
    return Prepared(
        scan_shape=scan_shape,
        detector_shape=det,
        sums=sums,
        mean_dp=mean_dp,
        bf=bf,
        g_half=g_half,
        dc=dc,
        wavelength=lam,
        sampling=sampling,
        geo=geo,
    )


def reconstruct(prep: Prepared, ab: Aberrations) -> tuple[np.ndarray, np.ndarray]:
    """Object wave (complex128) and phase (float64) at fixed aberrations."""
    obj = object_wave(prep.g_half, prep.geo, ab, prep.dc)
    return obj, phase(obj)


def wrapped_phase_error(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Phase difference wrapped to (-pi, pi], compared as unit phasors.

    Mirrors the unit-phasor comparison of
    tests/test_ssb_mps_cuda_reference.py:2016-2027.
    """
    return np.angle(np.exp(1j * (np.asarray(a, np.float64) - np.asarray(b, np.float64))))


def bf_companion(data: np.ndarray, rows: np.ndarray, cols: np.ndarray) -> tuple[str, bytes]:
    """The exact bright-field companion file (engine.py:577-701): suffix and
    bytes of the selected BF pixels' counts, BF-major ``[bf, scan]``.

    u8/u16 counts only (``TypeError`` otherwise, engine.py:598-602); u16 is
    narrowed to u8 only when the largest count of the whole block is at most
    255 (engine.py:603-604); BF order is the selection's (row-major).
    """
    data = np.asarray(data)
    if data.dtype not in (np.uint8, np.uint16):
        raise TypeError(f"Exact CUDA BF-source export supports uint8 or uint16 counts; got {data.dtype}.")
    out_dtype = np.uint8 if int(data.max()) <= 255 else np.uint16
    plane = data.shape[0] * data.shape[1]
    flat = data.reshape(plane, data.shape[2] * data.shape[3])
    lin = np.asarray(rows, np.int64) * data.shape[3] + np.asarray(cols, np.int64)
    cols_bf = np.ascontiguousarray(flat[:, lin].T).astype(out_dtype)
    return (".u8" if out_dtype == np.uint8 else ".u16"), cols_bf.tobytes()
