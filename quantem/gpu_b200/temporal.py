"""Temporal joining of drift-corrected SSB reconstructions on the B200.

Same functions, arguments and results as the reference's temporal helpers
(``quantem.gpu.ssb.temporal``, ssb/temporal.py:1-402 of bobleesj/quantem.gpu):
each frame's complex object wave is shifted by a known scan-coordinate drift
as a Fourier phase ramp, optionally referenced to frame 0's global phase, and
averaged with per-frame weights. The shift and the join run as the
``qssb_fourier_shift`` / ``qssb_join_object_waves`` kernels; arrays are torch
CUDA tensors.
"""
from __future__ import annotations

import math
import time
from collections.abc import Sequence
from dataclasses import dataclass
from typing import Literal

import torch

from . import ops
from .protocol import SSBResult

PhaseReference = Literal["first", "none"]


@dataclass
class SSBTimeSeriesResult:
    """Shared-calibration SSB object-wave time series (temporal.py:25-75)."""

    object_waves: torch.Tensor
    aberrations: dict[str, float]
    rotation_angle_deg: float
    shifts: torch.Tensor
    weights: torch.Tensor
    phase_reference: PhaseReference = "first"
    elapsed: float | None = None
    voltage_kV: float | None = None
    semiangle_mrad: float | None = None
    scan_sampling_A: float | None = None
    mode: str = "shared_calibration_time_series"

    @property
    def phase(self) -> torch.Tensor:
        """Phase stack with shape ``(time, row, col)``."""
        return torch.angle(self.object_waves)

    @property
    def amplitude(self) -> torch.Tensor:
        """Amplitude stack with shape ``(time, row, col)``."""
        return torch.abs(self.object_waves)

    def time_average(self, weights=None) -> SSBResult:
        """A single complex average of the preserved time series."""
        result = join_object_waves(self.object_waves, shifts=None,
                                   weights=self.weights if weights is None else weights,
                                   phase_reference="none")
        result.aberrations = dict(self.aberrations)
        result.rotation_angle_deg = self.rotation_angle_deg
        result.voltage_kV = self.voltage_kV
        result.semiangle_mrad = self.semiangle_mrad
        result.scan_sampling_A = self.scan_sampling_A
        result.join_mode = "shared_calibration_time_series_average"
        return result


def _device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("the B200 SSB engine needs a CUDA device (it has no CPU path)")
    return torch.device("cuda", torch.cuda.current_device())


def _as_stack(object_waves) -> torch.Tensor:
    """(time, row, col) complex64 CUDA stack from a 2D wave, a 3D stack or a
    sequence of 2D waves (temporal.py:110-126)."""
    if isinstance(object_waves, torch.Tensor):
        stack = object_waves
    else:
        try:
            stack = torch.stack([torch.as_tensor(w) for w in object_waves], dim=0)
        except TypeError as exc:
            raise ValueError("object_waves must be a 2D object wave, a 3D stack, or a "
                             "sequence of 2D object waves") from exc
    if stack.ndim == 2:
        stack = stack[None]
    if stack.ndim != 3:
        raise ValueError(f"object_waves must resolve to (time, row, col), got {tuple(stack.shape)}")
    if not stack.is_cuda:
        stack = stack.to(_device())
    if not torch.is_complex(stack):
        stack = stack.to(torch.complex64)
    return stack.to(torch.complex64).contiguous()


def _normalize_shifts(shifts, n_time: int, device) -> torch.Tensor:
    if shifts is None:
        return torch.zeros((n_time, 2), dtype=torch.float32, device=device)
    out = torch.as_tensor(shifts, dtype=torch.float32).to(device)
    if tuple(out.shape) != (n_time, 2):
        raise ValueError(f"shifts must have shape ({n_time}, 2), got {tuple(out.shape)}")
    return out.contiguous()


def _normalize_weights(weights, n_time: int, device) -> torch.Tensor:
    """Non-negative weights scaled to sum 1 (temporal.py:127-140)."""
    if weights is None:
        return torch.full((n_time,), 1.0 / float(n_time), dtype=torch.float32, device=device)
    w = torch.as_tensor(weights, dtype=torch.float32).to(device)
    if tuple(w.shape) != (n_time,):
        raise ValueError(f"weights must have shape ({n_time},), got {tuple(w.shape)}")
    if bool((w < 0).any()):
        raise ValueError("weights must be non-negative")
    total = float(w.sum())
    if not math.isfinite(total) or total <= 0:
        raise ValueError("weights must sum to a positive finite value")
    return (w / total).contiguous()


def fourier_shift_2d(image, shift: Sequence[float]) -> torch.Tensor:
    """Periodic subpixel shift ``(row, col)`` in pixels (temporal.py:77-107):
    positive shifts move content toward larger indices. Complex inputs keep
    complex64; real inputs return the real part in their dtype."""
    arr = torch.as_tensor(image)
    if arr.ndim != 2:
        raise ValueError(f"image must be 2D, got shape {tuple(arr.shape)}")
    dev = arr.device if arr.is_cuda else _device()
    wave = arr.to(dev).to(torch.complex64).contiguous()[None]
    shifts = torch.tensor([[float(shift[0]), float(shift[1])]], dtype=torch.float32, device=dev)
    out = ops.fourier_shift(wave, shifts)[0]
    if torch.is_complex(arr):
        return out
    return out.real.to(arr.dtype)


def _align(stack: torch.Tensor, shifts: torch.Tensor) -> torch.Tensor:
    return ops.fourier_shift(stack, shifts)


def join_object_waves(object_waves, shifts=None, *, weights=None,
                      phase_reference: PhaseReference = "first",
                      return_aligned_stack: bool = False):
    """Join a drift-corrected time series of object waves (temporal.py:183-257)."""
    if phase_reference not in {"first", "none"}:
        raise ValueError("phase_reference must be 'first' or 'none'")
    t0 = time.perf_counter()
    stack = _as_stack(object_waves)
    n_time = int(stack.shape[0])
    shifts_t = _normalize_shifts(shifts, n_time, stack.device)
    weights_t = _normalize_weights(weights, n_time, stack.device)
    aligned = _align(stack, shifts_t)
    joined = ops.join_frames(aligned, weights_t, phase_reference=phase_reference == "first",
                             write_back=return_aligned_stack)
    result = SSBResult(object_wave=joined, backend="cuda", loss=None,
                       elapsed=time.perf_counter() - t0, num_bf=None)
    result.num_frames = n_time
    result.time_shifts = shifts_t
    result.time_weights = weights_t
    result.phase_reference = phase_reference
    result.join_mode = "drift_corrected_complex_mean"
    if return_aligned_stack:
        return result, aligned
    return result


def _reconstruct_objects(ssb_frames, *, aberrations, rotation_angle_deg) -> list[torch.Tensor]:
    objects = []
    for ssb in ssb_frames:
        coefs = dict(ssb.aberrations)
        if aberrations is not None:
            coefs.update(aberrations)
        if rotation_angle_deg is not None:
            ssb.set_rotation(rotation_angle_deg)
        objects.append(torch.as_tensor(ssb.reconstruct(coefs).object_wave))
    return objects


def _scan_sampling(first) -> float | None:
    s = first.scan_sampling_A
    if isinstance(s, tuple):
        return float(s[0])
    return None if s is None else float(s)


def ssb_time_series(ssb_frames, shifts=None, *, weights=None, aberrations=None,
                    rotation_angle_deg: float | None = None,
                    phase_reference: PhaseReference = "first") -> SSBTimeSeriesResult:
    """Shared-calibration object-wave time series (temporal.py:260-335)."""
    if not ssb_frames:
        raise ValueError("ssb_frames must contain at least one SSB frame")
    if phase_reference not in {"first", "none"}:
        raise ValueError("phase_reference must be 'first' or 'none'")
    t0 = time.perf_counter()
    stack = _as_stack(_reconstruct_objects(ssb_frames, aberrations=aberrations,
                                           rotation_angle_deg=rotation_angle_deg))
    n_time = int(stack.shape[0])
    shifts_t = _normalize_shifts(shifts, n_time, stack.device)
    weights_t = _normalize_weights(weights, n_time, stack.device)
    aligned = _align(stack, shifts_t)
    if phase_reference == "first":  # rotate frames t > 0 in place; the mean is not needed
        ops.join_frames(aligned, weights_t, phase_reference=True, write_back=True)
    first = ssb_frames[0]
    return SSBTimeSeriesResult(
        object_waves=aligned, aberrations=dict(aberrations or first.aberrations),
        rotation_angle_deg=(float(rotation_angle_deg) if rotation_angle_deg is not None
                            else float(first.rotation_angle_deg)),
        shifts=shifts_t, weights=weights_t, phase_reference=phase_reference,
        elapsed=time.perf_counter() - t0, voltage_kV=first.voltage_kV,
        semiangle_mrad=first.semiangle_mrad, scan_sampling_A=_scan_sampling(first))


def ssb_time_average(ssb_frames, shifts=None, *, weights=None, aberrations=None,
                     rotation_angle_deg: float | None = None,
                     phase_reference: PhaseReference = "first",
                     return_aligned_stack: bool = False):
    """Reconstruct and join a drift-corrected SSB time series (temporal.py:338-402)."""
    if not ssb_frames:
        raise ValueError("ssb_frames must contain at least one SSB frame")
    objects = _reconstruct_objects(ssb_frames, aberrations=aberrations,
                                   rotation_angle_deg=rotation_angle_deg)
    joined = join_object_waves(objects, shifts, weights=weights, phase_reference=phase_reference,
                               return_aligned_stack=return_aligned_stack)
    result = joined[0] if return_aligned_stack else joined
    first = ssb_frames[0]
    result.aberrations = dict(aberrations or first.aberrations)
    result.rotation_angle_deg = (float(rotation_angle_deg) if rotation_angle_deg is not None
                                 else float(first.rotation_angle_deg))
    result.voltage_kV = first.voltage_kV
    result.semiangle_mrad = first.semiangle_mrad
    result.scan_sampling_A = _scan_sampling(first)
    result.join_mode = "ssb_time_average"
    return joined
