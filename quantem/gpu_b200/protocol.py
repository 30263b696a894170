"""The SSB backend contract, mirrored from the reference.

Same names, fields and semantics as bobleesj/quantem.gpu:

* ``SSBPrecision``, ``SSBExportState``, ``SSBProtocol`` -
  ``src/quantem/gpu/ssb/compute/protocol.py:16-122``;
* ``BrightfieldDisk`` - ``src/quantem/gpu/ssb/bf_selector.py:10-76``;
* ``SSBResult`` - ``src/quantem/gpu/ssb/results.py:42-130``.

They are restated here (not imported) so that the engine runs where the
reference is not installed; a backend satisfying this ``SSBProtocol`` also
satisfies the reference's runtime-checkable protocol (checked in the tests).
"""
from __future__ import annotations

import math
import pathlib
from contextlib import AbstractContextManager
from dataclasses import dataclass, field
from pathlib import Path
from typing import Literal, Protocol, runtime_checkable

import numpy as np


@dataclass(frozen=True)
class SSBPrecision:
    """Numeric storage required from every SSB backend."""

    real_dtype: Literal["float32"] = "float32"
    complex_dtype: Literal["complex64"] = "complex64"


@dataclass(frozen=True)
class BrightfieldDisk:
    """Validated detector coordinates and geometry for one BF selection.

    Coordinates follow the public ``(row, col)`` convention and are stored as
    read-only int32 copies.
    """

    rows: np.ndarray
    cols: np.ndarray
    center_row_col: tuple[float, float]
    radius_px: float
    detected_radius_px: float
    detector_shape: tuple[int, int]

    def __post_init__(self) -> None:
        rows = np.asarray(self.rows, dtype=np.int32).reshape(-1).copy()
        cols = np.asarray(self.cols, dtype=np.int32).reshape(-1).copy()
        if rows.size == 0 or rows.shape != cols.shape:
            raise ValueError("BF rows and columns must be non-empty matching vectors.")
        det = tuple(int(v) for v in self.detector_shape)
        if len(det) != 2 or min(det) < 1:
            raise ValueError("detector_shape must contain two positive (row, col) sizes.")
        if rows.min() < 0 or cols.min() < 0 or rows.max() >= det[0] or cols.max() >= det[1]:
            raise ValueError(f"BF coordinates fall outside detector shape {det}.")
        linear = rows.astype(np.int64) * det[1] + cols
        if np.unique(linear).size != rows.size:
            raise ValueError("BF coordinates must not contain duplicates.")
        center = tuple(float(v) for v in self.center_row_col)
        if len(center) != 2 or not all(math.isfinite(v) for v in center):
            raise ValueError("center_row_col must contain two finite values.")
        radius = float(self.radius_px)
        detected = float(self.detected_radius_px)
        if not math.isfinite(radius) or radius <= 0:
            raise ValueError("radius_px must be a positive finite value.")
        if not math.isfinite(detected) or detected <= 0:
            raise ValueError("detected_radius_px must be a positive finite value.")
        rows.flags.writeable = False
        cols.flags.writeable = False
        object.__setattr__(self, "rows", rows)
        object.__setattr__(self, "cols", cols)
        object.__setattr__(self, "center_row_col", center)
        object.__setattr__(self, "radius_px", radius)
        object.__setattr__(self, "detected_radius_px", detected)
        object.__setattr__(self, "detector_shape", det)

    @property
    def size(self) -> int:
        """Number of selected BF detector pixels."""
        return int(self.rows.size)


@dataclass(frozen=True)
class SSBExportState:
    """Compact host state for browser/widget consumers."""

    backend: Literal["cuda", "mps", "webgpu"]
    scan_shape: tuple[int, int]
    brightfield: BrightfieldDisk
    kx_bf: np.ndarray
    ky_bf: np.ndarray
    qx_1d: np.ndarray
    qy_1d: np.ndarray
    aperture_k: np.ndarray
    alpha_k2: np.ndarray
    cos2phi_k: np.ndarray
    sin2phi_k: np.ndarray
    wavelength_A: float
    semiangle_rad: float
    angular_sampling_rad: tuple[float, float]
    sampling_A: tuple[float, float]
    dc_value: complex
    precision: SSBPrecision = SSBPrecision()
    bf_source_path: pathlib.Path | None = None
    bf_source_dtype: np.dtype | None = None
    bf_source_max_value: int | None = None

    @property
    def num_bf(self) -> int:
        """Number of complete bright-field detector pixels."""
        return self.brightfield.size

    @property
    def active_num_bf(self) -> int:
        """Number of selected BF pixels with nonzero probe aperture weight."""
        return int(np.count_nonzero(np.asarray(self.aperture_k) > 0.0))


def _format_aberrations(aberrations: dict) -> str:
    if not aberrations:
        return "  (none)"
    lines = []
    if "C10" in aberrations:
        lines.append(f"  Defocus (C10)  {aberrations['C10']:.1f} nm")
    if "C12" in aberrations:
        lines.append(f"  Astigmatism    {aberrations['C12']:.1f} nm")
    if "phi12" in aberrations:
        lines.append(f"  Astig. angle   {math.degrees(aberrations['phi12']):.1f}°")
    return "\n".join(lines)


@dataclass
class SSBResult:
    """Result of one SSB reconstruction.

    ``object_wave`` is the complex64 transmission function (a torch CUDA
    tensor from this engine, or a numpy array after persistence); ``phase``
    and ``amplitude`` derive from it.
    """

    object_wave: object
    backend: Literal["cuda", "mps", "webgpu"]
    aberrations: dict[str, float] = field(default_factory=dict)
    rotation_angle_deg: float = 0.0
    loss: float | None = None
    elapsed: float | None = None
    timings: dict[str, float] = field(default_factory=dict)
    n_trials: int | None = None
    num_bf: int | None = None
    refine_method: str | None = None
    refine_nfev: int | None = None
    refine_elapsed: float | None = None
    voltage_kV: float | None = None
    semiangle_mrad: float | None = None
    scan_sampling_A: float | tuple[float, float] | None = None
    source_path: str | None = None
    bf_center: tuple[float, float] | None = None
    bf_radius: float | None = None
    detected_bf_radius: float | None = None
    optuna_trials: list[dict] | None = None
    reused: bool = False
    saved_path: Path | None = None
    metadata: dict[str, object] = field(default_factory=dict)

    def __repr__(self) -> str:
        lines = ["SSB Result", f"  Shape          {tuple(self.object_wave.shape)}"]
        if self.loss is not None:
            lines.append(f"  Loss           {self.loss:.6f}")
        if self.num_bf is not None:
            lines.append(f"  BF pixels      {self.num_bf}")
        if self.n_trials is not None:
            lines.append(f"  Trials         {self.n_trials}")
        lines.append(f"  Rotation       {self.rotation_angle_deg:.1f}°")
        if self.aberrations:
            lines.append(_format_aberrations(self.aberrations))
        if self.elapsed is not None:
            lines.append(f"  Time           {self.elapsed:.2f}s")
        return "\n".join(lines)

    @property
    def phase(self):
        """``angle(object_wave)``."""
        obj = self.object_wave
        if hasattr(obj, "angle") and not isinstance(obj, np.ndarray):
            return obj.angle()
        return np.angle(obj)

    @property
    def amplitude(self):
        """``abs(object_wave)``."""
        obj = self.object_wave
        if hasattr(obj, "abs") and not isinstance(obj, np.ndarray):
            return obj.abs()
        return np.abs(obj)


@runtime_checkable
class SSBProtocol(Protocol):
    """Backend contract (protocol.py:62-122 of the reference)."""

    backend: Literal["cuda", "mps", "webgpu"]
    precision: SSBPrecision

    @property
    def scan_shape(self) -> tuple[int, int]: ...

    @property
    def detector_shape(self) -> tuple[int, int]: ...

    @property
    def num_bf(self) -> int: ...

    def fit(self, *, trials: int, refinement: str | None,
            search_ranges: dict[str, tuple[float, float] | float] | None,
            refine_lock: list[str] | None, seed: int, verbose: bool) -> SSBResult: ...

    def reconstruct_result(self, aberrations: dict[str, float], *,
                           compute_loss: bool = True) -> SSBResult: ...

    def cache_rotation(self, rotation_rad: float) -> None: ...

    def preview(self, aberrations: dict[str, float], *, compute_loss: bool,
                higher_order_magnitudes: np.ndarray | None,
                higher_order_angles: np.ndarray | None) -> tuple[np.ndarray, float | None]: ...

    def preview_context(self, num_bf: int) -> AbstractContextManager | None: ...

    def browser_state(self) -> SSBExportState: ...

    def export_brightfield(self, data, path_stem: str | pathlib.Path
                           ) -> tuple[pathlib.Path, float] | None: ...

    def close(self) -> None: ...


__all__ = [
    "BrightfieldDisk",
    "SSBExportState",
    "SSBPrecision",
    "SSBProtocol",
    "SSBResult",
]
