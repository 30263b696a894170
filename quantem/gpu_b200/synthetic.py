"""Seeded synthetic 4D-STEM data from a weak-phase forward model.

The reference's own benchmarks run on private acquisitions, so every workload
here is synthesised with the shapes, sizes and value distributions those
acquisitions have: a weak-phase object of Gaussian atoms (sigma 0.3 A, peak
0.3 rad) on a 4 A square lattice with 5% vacancies, probed at 300 kV with a
20 mrad soft aperture; intensities are |FFT(probe * exp(i phi))|^2 scaled to a
mean dose per probe position and Poisson-sampled into uint16.

Conventions match the SSB model of the reference (bobleesj/quantem.gpu
``src/quantem/gpu/ssb/compute/cuda/engine.py:784-830`` and
``kernels/common.py:115-236``):

* detector pixel ``i`` sits at frequency ``(i - K/2) * dk``,
  ``dk = det_sampling[mrad] * 1e-3 / lambda`` (1/A);
* the probe is ``P(x) = IFFT[A(k) exp(-i chi(k))]`` with
  ``chi = (pi/lambda) alpha^2 (C10 + C12 cos 2(phi - phi12)) + (pi / 2 lambda) C30 alpha^4``,
  ``alpha = lambda |k|``, in the reference's numeric length unit (Angstrom);
* the scan FFT uses ``exp(-2 pi i q . R)`` with ``q = fftfreq(R, step)``.

With these, the weak-phase scan spectrum is ``G(q, k) ~ i Phi(q) Gamma(q, k)``
with exactly the reference's double-overlap ``Gamma``, so the SSB loss
minimum sits at the true aberrations.

Runs on any torch device; ``device="cuda"`` generates the 537 MB workload in
well under a second. Inputs are plumbing, not the measured path.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from .physics import wavelength_angstrom


@dataclass(frozen=True)
class SyntheticSpec:
    """One synthetic acquisition (physical units; C10/C12/C30 in Angstrom)."""

    scan_shape: tuple[int, int] = (32, 32)
    detector_shape: tuple[int, int] = (64, 64)
    voltage_kV: float = 300.0
    semiangle_mrad: float = 20.0
    scan_step_A: float = 0.5
    det_sampling_mrad: float = 20.0 / 12.0
    dose: float = 1000.0
    C10: float = 0.0
    C12: float = 0.0
    phi12: float = 0.0
    C30: float = 0.0
    atom_sigma_A: float = 0.3
    atom_peak_rad: float = 0.3
    lattice_A: float = 4.0
    vacancy_fraction: float = 0.05
    seed: int = 0
    # False: counts are the expected intensities rounded to integers (no
    # Poisson noise), for studies whose error floor must not be shot noise
    poisson: bool = True

    def aberrations(self) -> dict[str, float]:
        """Aberrations in the reference's numeric convention (Angstrom, rad)."""
        return {"C10": self.C10, "C12": self.C12, "phi12": self.phi12}


# The BASELINE workloads as concrete synthetic inputs. BF radius in pixels is
# semiangle / det_sampling (12 px for the CPU case, 24 px at 128^4).
CONFIGS: dict[str, SyntheticSpec] = {
    "plain_32x32_det64": SyntheticSpec(
        scan_shape=(32, 32), detector_shape=(64, 64), det_sampling_mrad=20.0 / 12.0,
    ),
    "plain_128x128_det128": SyntheticSpec(
        scan_shape=(128, 128), detector_shape=(128, 128), det_sampling_mrad=20.0 / 24.0,
    ),
    "stress_256x256_det128": SyntheticSpec(
        scan_shape=(256, 256), detector_shape=(128, 128), det_sampling_mrad=20.0 / 24.0,
        C10=200.0,
    ),
    # the reference's 512^2 timing shape (512 x 512 x 192 x 192 u16, ~8.9k BF
    # pixels): a 53.3 px BF radius on the 192^2 detector
    "large_512x512_det192": SyntheticSpec(
        scan_shape=(512, 512), detector_shape=(192, 192), det_sampling_mrad=25.0 / 53.3,
        semiangle_mrad=25.0, C10=100.0,
    ),
}


@dataclass
class SyntheticData:
    """Generated counts plus the ground truth used to make them."""

    counts: torch.Tensor                  # uint16 [R0, R1, K0, K1]
    spec: SyntheticSpec
    object_phase: np.ndarray | None = None
    extra: dict = field(default_factory=dict)


def _soft_aperture(kr: torch.Tensor, kc: torch.Tensor, lam: float, semi_rad: float,
                   d_rad: float) -> torch.Tensor:
    """Soft aperture clip((alpha_max - lambda|k|)/d + 0.5, 0, 1) for equal sampling."""
    alpha = lam * torch.sqrt(kr * kr + kc * kc)
    return torch.clamp((semi_rad - alpha) / d_rad + 0.5, 0.0, 1.0)


def probe_spectrum(spec: SyntheticSpec, device: torch.device | str = "cpu") -> torch.Tensor:
    """A(k) exp(-i chi(k)) on the detector grid, fft order, complex128."""
    lam = wavelength_angstrom(spec.voltage_kV)
    k0, k1 = spec.detector_shape
    dk = spec.det_sampling_mrad * 1e-3 / lam
    fr = torch.fft.fftfreq(k0, device=device, dtype=torch.float64) * k0 * dk
    fc = torch.fft.fftfreq(k1, device=device, dtype=torch.float64) * k1 * dk
    kr, kc = torch.meshgrid(fr, fc, indexing="ij")
    a = _soft_aperture(kr, kc, lam, spec.semiangle_mrad * 1e-3, spec.det_sampling_mrad * 1e-3)
    k2 = kr * kr + kc * kc
    alpha2 = lam * lam * k2
    safe = torch.where(k2 > 0, k2, torch.ones_like(k2))
    cos2 = torch.where(k2 > 0, (kr * kr - kc * kc) / safe, torch.zeros_like(k2))
    sin2 = torch.where(k2 > 0, 2 * kr * kc / safe, torch.zeros_like(k2))
    factor = math.pi / lam
    chi = factor * alpha2 * (
        spec.C10 + spec.C12 * (cos2 * math.cos(2 * spec.phi12) + sin2 * math.sin(2 * spec.phi12))
    ) + 0.5 * factor * spec.C30 * alpha2 * alpha2
    return a * torch.exp(-1j * chi)


def object_phase_canvas(spec: SyntheticSpec, canvas: int, dx: float,
                        rng: np.random.Generator) -> np.ndarray:
    """Periodic weak-phase lattice of Gaussian atoms with random vacancies."""
    extent = canvas * dx
    n_sites = int(math.ceil(extent / spec.lattice_A)) + 1
    offset = rng.uniform(0, spec.lattice_A, size=2)
    sites = []
    for i in range(n_sites):
        for j in range(n_sites):
            sites.append((offset[0] + i * spec.lattice_A, offset[1] + j * spec.lattice_A))
    sites = np.asarray(sites)
    keep = rng.random(len(sites)) >= spec.vacancy_fraction
    sites = sites[keep]
    x = np.arange(canvas) * dx
    phase = np.zeros((canvas, canvas))
    two_s2 = 2.0 * spec.atom_sigma_A ** 2
    reach = 5.0 * spec.atom_sigma_A
    for (ar, ac) in sites:
        dr = x - ar
        dc = x - ac
        mr = np.abs(dr) < reach
        mc = np.abs(dc) < reach
        if not mr.any() or not mc.any():
            continue
        gr = np.exp(-dr[mr] ** 2 / two_s2)
        gc = np.exp(-dc[mc] ** 2 / two_s2)
        phase[np.ix_(mr, mc)] += spec.atom_peak_rad * gr[:, None] * gc[None, :]
    return phase


# Above this many detector samples the counts are drawn batch by batch.
_WHOLE_ARRAY_LIMIT = 1 << 31


def generate(spec: SyntheticSpec, device: torch.device | str = "cpu",
             batch: int = 1024) -> SyntheticData:
    """Generate uint16 counts I[R0, R1, K0, K1] for ``spec`` on ``device``."""
    device = torch.device(device)
    lam = wavelength_angstrom(spec.voltage_kV)
    k0, k1 = spec.detector_shape
    if k0 != k1:
        raise ValueError("the synthetic generator uses square detectors")
    r0, r1 = spec.scan_shape
    dk = spec.det_sampling_mrad * 1e-3 / lam
    dx = 1.0 / (k0 * dk)                       # probe-window pixel, Angstrom
    rng = np.random.default_rng(spec.seed)
    span = max(r0, r1) * spec.scan_step_A
    canvas = int(math.ceil(span / dx)) + k0 + 2
    phi = object_phase_canvas(spec, canvas, dx, rng)
    trans = torch.exp(1j * torch.as_tensor(phi, device=device))      # complex128

    pk = probe_spectrum(spec, device)                                  # fft order
    pk = pk / torch.sqrt((pk.abs() ** 2).sum())
    kr = torch.fft.fftfreq(k0, device=device, dtype=torch.float64) * k0 * dk
    kc = torch.fft.fftfreq(k1, device=device, dtype=torch.float64) * k1 * dk

    pos_r = torch.arange(r0, device=device, dtype=torch.float64) * spec.scan_step_A / dx
    pos_c = torch.arange(r1, device=device, dtype=torch.float64) * spec.scan_step_A / dx
    pr, pc = torch.meshgrid(pos_r, pos_c, indexing="ij")
    pr = pr.reshape(-1)
    pc = pc.reshape(-1)
    orr = torch.floor(pr).long()
    occ = torch.floor(pc).long()
    fr = pr - orr
    fc = pc - occ
    ar = torch.arange(k0, device=device)

    def intensities(s: int, e: int) -> torch.Tensor:
        # Sub-pixel probe shift by a Fourier phase ramp, window at integer offset.
        ramp_r = torch.exp(-2j * math.pi * fr[s:e, None] * dx * kr[None, :])
        ramp_c = torch.exp(-2j * math.pi * fc[s:e, None] * dx * kc[None, :])
        probe = torch.fft.ifft2(pk[None] * ramp_r[:, :, None] * ramp_c[:, None, :])
        probe = torch.fft.fftshift(probe, dim=(-2, -1))
        rows = orr[s:e, None, None] + ar[None, :, None]
        cols = occ[s:e, None, None] + ar[None, None, :]
        window = trans[rows, cols]
        psi = torch.fft.fftshift(torch.fft.fft2(probe * window), dim=(-2, -1))
        return (psi.abs() ** 2).to(torch.float32)

    gen = torch.Generator(device=device)
    gen.manual_seed(int(spec.seed) + 7919)
    n_frames = r0 * r1
    if n_frames * k0 * k1 <= _WHOLE_ARRAY_LIMIT:
        intens = torch.empty((n_frames, k0, k1), device=device, dtype=torch.float32)
        for s in range(0, n_frames, batch):
            e = min(n_frames, s + batch)
            intens[s:e] = intensities(s, e)
        scale = spec.dose / intens.sum(dim=(1, 2)).mean()
        intens *= scale
        counts = torch.poisson(intens, generator=gen) if spec.poisson else torch.round(intens)
        counts = torch.clamp(counts, max=65535).to(torch.int32).to(torch.uint16)
    else:
        # large acquisitions: two streaming passes (frame totals, then counts
        # drawn batch by batch straight into the u16 array)
        total = torch.zeros((), device=device, dtype=torch.float64)
        for s in range(0, n_frames, batch):
            total += intensities(s, min(n_frames, s + batch)).sum(dim=(1, 2), dtype=torch.float64).sum()
        scale = spec.dose / (total / n_frames)
        counts = torch.empty((n_frames, k0, k1), device=device, dtype=torch.uint16)
        for s in range(0, n_frames, batch):
            e = min(n_frames, s + batch)
            lam_b = intensities(s, e) * scale.to(torch.float32)
            c = torch.poisson(lam_b, generator=gen) if spec.poisson else torch.round(lam_b)
            counts[s:e] = torch.clamp(c, max=65535).to(torch.int32).to(torch.uint16)
    counts = counts.reshape(r0, r1, k0, k1)
    return SyntheticData(counts=counts, spec=spec, object_phase=phi,
                         extra={"probe_pixel_A": dx, "canvas": canvas})


# Batched-sweep workload: three 128^2-detector scans of uneven size; true
# aberrations and candidates drawn from C1 in [-50, 50] nm, |A1| in [0, 10] nm
# at a random angle, C3 in [0, 1] um - in the reference's numeric convention
# (Angstrom values): C10 in [-500, 500], C12 in [0, 100], C30 in [0, 1e4].
SWEEP_SCANS = ((96, 96), (128, 128), (160, 120))
SWEEP_RANGES = {"C10": (-500.0, 500.0), "C12": (0.0, 100.0), "phi12": (0.0, math.pi),
                "C30": (0.0, 1.0e4)}


def draw_aberrations(rng: np.random.Generator, n: int) -> np.ndarray:
    """[n, 4] float32 (C10, C12, phi12, C30) uniform in SWEEP_RANGES."""
    cols = [rng.uniform(*SWEEP_RANGES[k], size=n) for k in ("C10", "C12", "phi12", "C30")]
    return np.stack(cols, axis=1).astype(np.float32)


def sweep_specs(seed: int = 7, dose: float = 2.0e4) -> list[SyntheticSpec]:
    """The three scans of the batched sweep, each with its own true aberrations."""
    rng = np.random.default_rng(seed)
    truth = draw_aberrations(rng, len(SWEEP_SCANS))
    return [SyntheticSpec(scan_shape=shape, detector_shape=(128, 128),
                          det_sampling_mrad=20.0 / 24.0, dose=dose, C10=float(t[0]),
                          C12=float(t[1]), phi12=float(t[2]), C30=float(t[3]), seed=seed + i)
            for i, (shape, t) in enumerate(zip(SWEEP_SCANS, truth))]
