"""Public ``SSB`` session with the reference's signature, on the B200 engine.

Mirrors ``quantem.gpu.SSB`` (bobleesj/quantem.gpu ``src/quantem/gpu/ssb/
workflow.py:370-1292``): explicit public units, validated C10/C12/phi12
mappings, ``fit`` / ``reconstruct`` / ``preview`` / ``close``, and no CPU
fallback. The backend is always ``B200SSBBackend``; the reference's CuPy
device probe (``device/backend.py:106-125``) is not consulted.

Out of scope here (raise explicitly): ``SSB.open`` (HDF5 decode), saved-result
reuse (``save_to``), series reconstruction, and the MPS/WebGPU backends.
"""
from __future__ import annotations

import math
from contextlib import AbstractContextManager
from pathlib import Path
from typing import Literal

import numpy as np

from .backend import B200SSBBackend
from .protocol import SSBProtocol, SSBResult


def _validate_aberrations(aberrations: dict[str, float] | None) -> dict[str, float]:
    """A complete, owned C10/C12/phi12 mapping (workflow.py:69-89)."""
    if aberrations is None:
        return {"C10": 0.0, "C12": 0.0, "phi12": 0.0}
    required = {"C10", "C12", "phi12"}
    missing = required - aberrations.keys()
    extra = aberrations.keys() - required
    if missing or extra:
        details = []
        if missing:
            details.append(f"missing {sorted(missing)}")
        if extra:
            details.append(f"unknown {sorted(extra)}")
        raise ValueError(
            "SSB aberrations must contain exactly C10, C12, and phi12 (nm, nm, radians); "
            f"{', '.join(details)}."
        )
    return {name: float(aberrations[name]) for name in ("C10", "C12", "phi12")}


def _resolve_backend(backend: str) -> Literal["cuda"]:
    requested = str(backend).lower()
    if requested in {"auto", "cuda"}:
        return "cuda"
    if requested in {"mps", "webgpu"}:
        raise RuntimeError(f"The B200 engine serves CUDA only; backend {backend!r} is not available.")
    raise ValueError(f"Unknown SSB backend {backend!r}. Use 'auto', 'cuda', 'mps', or 'webgpu'.")


class SSB:
    """One SSB session (same parameters and semantics as the reference)."""

    def __init__(self, data: object, *, backend: str = "auto", voltage_kV: float,
                 semiangle_mrad: float, scan_sampling_A: float | tuple[float, float],
                 scan_shape: tuple[int, int] | None = None,
                 det_sampling: float | tuple[float, float] | None = None,
                 aberrations: dict[str, float] | None = None, rotation_angle_deg: float = 0.0,
                 bf_intensity_threshold: float = 0.0, bf_radius: int | None = None,
                 source_path: str | None = None, chi_fp64: bool = False) -> None:
        self.backend = _resolve_backend(backend)
        self._data = data
        self._scan_shape = scan_shape
        self.voltage_kV = float(voltage_kV)
        self.semiangle_mrad = float(semiangle_mrad)
        self.scan_sampling_A = scan_sampling_A
        self.det_sampling = det_sampling
        self._aberrations_explicit = aberrations is not None
        self.aberrations = _validate_aberrations(aberrations)
        self.rotation_angle_deg = float(rotation_angle_deg)
        self.bf_intensity_threshold = float(bf_intensity_threshold)
        self.bf_radius = bf_radius
        self.source_path = source_path
        self.source_dtype = str(getattr(data, "dtype", ""))
        self.source_bytes = int(getattr(data, "nbytes", 0) or 0)
        self._chi_fp64 = bool(chi_fp64)
        self._session: B200SSBBackend | None = None
        self._reconstruction: SSBResult | None = None
        self.best_loss = float("inf")
        self.trial_history: list[dict[str, object]] = []

    @classmethod
    def from_array(cls, data: object, **kwargs) -> "SSB":
        """Create a session from an in-memory uint8/uint16 detector array."""
        return cls(data, **kwargs)

    @classmethod
    def from_chunks(cls, chunks, *, frame_shape: tuple[int, int], scan_shape: tuple[int, int],
                    chunk_offsets=None, **kwargs) -> "SSB":
        """Create a session from an acquisition stored one detector frame per
        HDF5 bitshuffle+LZ4 chunk (the format ``SSB.open`` reads in the
        reference, io/load.py:3271-3320): ``chunks`` is a list of raw chunk
        bytes (e.g. from ``read_direct_chunk``), or a uint8 tensor of packed
        chunks with ``chunk_offsets``; the chunks cross to the GPU compressed
        and are decoded there."""
        import torch

        from .decode import decode_bslz4, from_chunks

        r0, r1 = (int(x) for x in scan_shape)
        k0, k1 = (int(x) for x in frame_shape)
        if chunk_offsets is None:
            counts = from_chunks(list(chunks), (k0, k1))
        else:
            dev = torch.device("cuda", torch.cuda.current_device())
            data = torch.as_tensor(chunks).to(dev, non_blocking=True)
            offs = torch.as_tensor(chunk_offsets, dtype=torch.int64).to(dev, non_blocking=True)
            counts = decode_bslz4(data, offs, (k0, k1))
        if counts.shape[0] != r0 * r1:
            raise ValueError(f"{counts.shape[0]} chunks for a {r0}x{r1} scan")
        return cls(counts.reshape(r0, r1, k0, k1), **kwargs)

    @classmethod
    def open(cls, *args, **kwargs) -> "SSB":
        raise NotImplementedError("SSB.open needs an HDF5 reader (h5py), which this build does "
                                  "not bundle: read the chunks with read_direct_chunk and use "
                                  "SSB.from_chunks, or load counts and use SSB.from_array.")

    def _prepare(self) -> B200SSBBackend:
        if self._session is None:
            self._session = B200SSBBackend(
                self._data, semiangle=self.semiangle_mrad, scan_sampling=self.scan_sampling_A,
                det_sampling=self.det_sampling, voltage_kV=self.voltage_kV,
                scan_shape=self._scan_shape, bf_intensity_threshold=self.bf_intensity_threshold,
                bf_radius=self.bf_radius,
                aberrations=self.aberrations if self._aberrations_explicit else None,
                rotation_angle_deg=self.rotation_angle_deg, chi_fp64=self._chi_fp64,
            )
        return self._session

    @property
    def _backend_protocol(self) -> SSBProtocol:
        backend = self._prepare()
        if not isinstance(backend, SSBProtocol):
            raise TypeError("The B200 implementation does not satisfy SSBProtocol.")
        return backend

    def _accept_result(self, result: SSBResult) -> SSBResult:
        result.source_path = self.source_path
        self.aberrations = dict(result.aberrations)
        self._aberrations_explicit = True
        self.rotation_angle_deg = float(result.rotation_angle_deg)
        self.best_loss = float(result.loss) if result.loss is not None else float("inf")
        self.trial_history = [dict(t) for t in result.optuna_trials or ()]
        self._reconstruction = result
        return result

    def fit(self, *, trials: int = 200, refinement: str | None = "nelder-mead",
            search_ranges: dict[str, tuple[float, float] | float] | None = None,
            refine_lock: list[str] | None = None, seed: int = 42,
            save_to: str | Path | None = None, force: bool = False,
            verbose: bool = True) -> SSBResult:
        """Optimise C10/C12/phi12 and return the final reconstruction."""
        if trials < 0:
            raise ValueError(f"trials must be non-negative, got {trials}.")
        if refinement not in {"nelder-mead", None}:
            raise ValueError("refinement must be 'nelder-mead' or None.")
        if save_to is not None:
            raise NotImplementedError("saved-result reuse is outside the B200 engine's scope.")
        result = self._backend_protocol.fit(trials=int(trials), refinement=refinement,
                                            search_ranges=search_ranges, refine_lock=refine_lock,
                                            seed=int(seed), verbose=verbose)
        return self._accept_result(result)

    def reconstruct(self, aberrations: dict[str, float] | None = None, *,
                    compute_loss: bool = True, save_to: str | Path | None = None,
                    force: bool = False, verbose: bool = False) -> SSBResult:
        """Complex object wave at fixed aberrations."""
        if save_to is not None:
            raise NotImplementedError("saved-result reuse is outside the B200 engine's scope.")
        coefs = self.aberrations if aberrations is None else _validate_aberrations(aberrations)
        if (not force and aberrations is None and self._reconstruction is not None
                and (not compute_loss or self._reconstruction.loss is not None)):
            return self._reconstruction
        result = self._backend_protocol.reconstruct_result(coefs, compute_loss=compute_loss)
        return self._accept_result(result)

    def preview(self, aberrations: dict[str, float], *, compute_loss: bool = True,
                higher_order_magnitudes: np.ndarray | None = None,
                higher_order_angles: np.ndarray | None = None,
                context: AbstractContextManager | None = None) -> tuple[np.ndarray, float | None]:
        """Transient float32 mean-phase image (and optional loss)."""
        coefs = _validate_aberrations(aberrations)
        if (higher_order_magnitudes is None) != (higher_order_angles is None):
            raise ValueError("higher_order_magnitudes and higher_order_angles must be provided together.")
        backend = self._backend_protocol
        kwargs = dict(compute_loss=compute_loss, higher_order_magnitudes=higher_order_magnitudes,
                      higher_order_angles=higher_order_angles)
        if context is None:
            return backend.preview(coefs, **kwargs)
        with context:
            return backend.preview(coefs, **kwargs)

    def preview_context(self, num_bf: int):
        return self._backend_protocol.preview_context(int(num_bf))

    def browser_state(self):
        return self._backend_protocol.browser_state()

    def export_brightfield(self, path_stem: str | Path) -> tuple[str, float] | None:
        written = self._backend_protocol.export_brightfield(self._data, path_stem)
        if written is None:
            return None
        path, elapsed = written
        return str(path), float(elapsed)

    @property
    def scan_shape(self) -> tuple[int, int]:
        return self._backend_protocol.scan_shape

    @property
    def num_bf(self) -> int:
        return self._backend_protocol.num_bf

    def set_rotation(self, rotation_angle_deg: float) -> None:
        self.rotation_angle_deg = float(rotation_angle_deg)
        self._backend_protocol.cache_rotation(math.radians(self.rotation_angle_deg))

    def close(self) -> None:
        if self._session is not None:
            self._session.close()
            self._session = None
        self._data = None

    def __enter__(self) -> "SSB":
        return self

    def __exit__(self, *exc) -> None:
        self.close()


__all__ = ["SSB"]
