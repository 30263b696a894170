"""``B200SSBBackend``: the reference's CUDA SSB backend contract on sm_100a.

Drop-in for ``CudaSSBBackend`` (bobleesj/quantem.gpu
``src/quantem/gpu/ssb/compute/cuda/backend.py:88``) and the engine methods it
delegates to (``engine.py:402``): same constructor keywords, attributes,
``SSBProtocol`` members (``compute/protocol.py:62-122``), units and error
types. The device work runs in ``libqssb.so`` through ``quantem.gpu_b200.ops``:

=========================  ==========================================
reference step             B200 kernel (C ABI)
=========================  ==========================================
u64 mean DP (K1)           qssb_mean_dp_u64
BF gather (K3)             qssb_gather_bf_columns
cuFFT fft2 + slice (K4)    qssb_scan_fft_half
pk + fused IFFT + mean     qssb_object (Fourier-sum, one IFFT)
(K5-K9)
phase-variance loss        qssb_loss_batch (candidate batch, one
(K10-K15)                  launch sequence)
=========================  ==========================================

Unsupported work fails explicitly; nothing falls back to the CPU.
"""
from __future__ import annotations

import math
import time
from contextlib import contextmanager
from pathlib import Path
from typing import Literal

import numpy as np
import torch

from . import _lib, autotune, ops
from ._lib import (
    FULL_TERM_NAMES,
    FULL_TERMS,
    GEOM_ROWS,
    QSSB_FLAG_CHI_FP64,
    QSSB_FLAG_QUADRATIC,
    Aberrations,
    Calibration,
)
from .calibration import (
    BFGeometry,
    bf_geometry,
    detect_bf_radius,
    pad_target,
    scan_frequencies,
    select_bf,
)
from .optimizer import batch_nelder_mead, batch_sweep, search_box
from .physics import electron_wavelength_angstrom
from .protocol import BrightfieldDisk, SSBExportState, SSBPrecision, SSBResult

NATIVE_SCAN_SIZES = (128, 256, 512, 1024)
LOSS_SCAN_SIZES = (128, 256, 512, 1024)


def _as_device_counts(data, device: torch.device) -> torch.Tensor:
    """Counts as a contiguous CUDA uint16 tensor (H2D copy for host input)."""
    if isinstance(data, np.ndarray):
        if data.dtype not in (np.uint8, np.uint16):
            raise TypeError(f"SSB counts must be uint8 or uint16, got {data.dtype}")
        t = torch.from_numpy(np.ascontiguousarray(data))
    elif isinstance(data, torch.Tensor):
        t = data
    else:
        raise TypeError("data must be a numpy array or a torch tensor")
    if t.dtype == torch.uint8:
        t = t.to(device=device).to(torch.uint16)
    elif t.dtype != torch.uint16:
        raise TypeError(f"SSB counts must be uint8 or uint16, got {t.dtype}")
    if not t.is_cuda or t.device != device:
        t = t.to(device, non_blocking=False)
    return t.contiguous()


def _as_device_counts_exact(data, device: torch.device) -> torch.Tensor:
    """Counts on ``device`` in their own u8/u16 type (no widening), as the
    exact BF companion writer needs them (engine.py:591-602)."""
    if isinstance(data, np.ndarray):
        dtype = data.dtype
        t = torch.from_numpy(np.ascontiguousarray(data)) if dtype in (np.uint8, np.uint16) else None
    elif isinstance(data, torch.Tensor):
        dtype, t = data.dtype, data
    else:
        raise TypeError("data must be a numpy array or a torch tensor")
    if t is None or t.dtype not in (torch.uint8, torch.uint16):
        raise TypeError(f"Exact CUDA BF-source export supports uint8 or uint16 counts; got {dtype}.")
    if not t.is_cuda or t.device != device:
        t = t.to(device)
    return t


_FREQ_CACHE: dict = {}


def _device_frequencies(scan_shape, scan_sampling, device) -> tuple[torch.Tensor, torch.Tensor]:
    """Device fftfreq grids of the scan axes, uploaded once per shape/sampling/device."""
    key = (tuple(scan_shape), tuple(float(s) for s in scan_sampling), str(device))
    hit = _FREQ_CACHE.get(key)
    if hit is None:
        q_row, q_col = scan_frequencies(scan_shape, scan_sampling)
        hit = tuple(t.clone() for t in ops.STAGING.upload([q_row, q_col], torch.device(device)))
        _FREQ_CACHE[key] = hit
    return hit


class B200SSBBackend:
    """Single-sideband reconstruction on one B200, reference contract."""

    _DEFAULT_OPTIMIZE_RANGES = {"C10_nm": (-400, 400), "C12_nm": (0, 100), "phi12_deg": (-90, 90)}
    _DEFAULT_GRID_HALF_WIDTHS = {"C10_nm": 50, "C12_nm": 20, "phi12_deg": 30}
    _DEFAULT_GRID_POINTS = {"C10_nm": 21, "C12_nm": 11, "phi12_deg": 13}
    _SWEEP_BATCH = 64
    backend = "cuda"
    precision = SSBPrecision()

    def __init__(
        self,
        data,
        semiangle: float,
        scan_sampling: float | tuple[float, float],
        det_sampling: float | tuple[float, float] | None = None,
        *,
        voltage_kV: float | None = None,
        energy: float | None = None,
        scan_shape: tuple[int, int] | None = None,
        bf_intensity_threshold: float = 0.0,
        bf_radius: int | None = None,
        aberrations: dict[str, float] | None = None,
        rotation_angle_deg: float = 0.0,
        detector_gain=None,
        gqk_storage: Literal["herm"] = "herm",
        device: torch.device | str | None = None,
        chi_fp64: bool = False,
    ):
        t0 = time.perf_counter()
        if voltage_kV is not None and energy is not None:
            raise ValueError("Specify voltage_kV or energy, not both.")
        if voltage_kV is not None:
            energy = voltage_kV * 1e3
        elif energy is None:
            raise ValueError("Specify voltage_kV (kV) or energy (eV).")
        if gqk_storage != "herm":
            raise ValueError(
                "gqk_storage='full' was removed from the SSB runtime path. Use the default "
                "exact Hermitian storage."
            )
        if detector_gain is not None:
            raise NotImplementedError("detector_gain is not supported by the B200 SSB engine yet.")
        if not torch.cuda.is_available():
            raise RuntimeError("The B200 SSB engine requires a CUDA device; there is no CPU path.")
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        counts = _as_device_counts(data, self.device)
        if counts.ndim == 3:
            if scan_shape is None:
                n = int(counts.shape[0])
                side = int(round(n ** 0.5))
                if side * side != n:
                    raise ValueError(
                        f"scan_shape is required: {n} frames is not a perfect square. "
                        "Pass scan_shape=(rows, cols)."
                    )
                scan_shape = (side, side)
            if scan_shape[0] * scan_shape[1] != counts.shape[0]:
                raise ValueError("scan_shape does not match number of frames.")
            counts = counts.reshape(scan_shape[0], scan_shape[1], counts.shape[1], counts.shape[2])
        elif counts.ndim != 4:
            raise ValueError("data must be 3D or 4D.")
        counts = self._pad_or_crop(counts)
        if isinstance(scan_sampling, (int, float)):
            scan_sampling = (float(scan_sampling), float(scan_sampling))
        self.energy = energy
        self.voltage_kV = voltage_kV
        self.semiangle_mrad = semiangle
        self.semiangle_cutoff = semiangle
        self.scan_sampling = tuple(scan_sampling)
        self.bf_intensity_threshold = float(bf_intensity_threshold)
        self.aberrations = dict(aberrations) if aberrations is not None else {"C10": 0.0, "C12": 0.0, "phi12": 0.0}
        self._rotation_angle_rad = math.radians(rotation_angle_deg)
        self.gqk_storage = gqk_storage
        self._flags = QSSB_FLAG_CHI_FP64 if chi_fp64 else 0
        scan_gpts = (int(counts.shape[0]), int(counts.shape[1]))
        det_gpts = (int(counts.shape[2]), int(counts.shape[3]))
        if scan_gpts[0] not in NATIVE_SCAN_SIZES:
            raise NotImplementedError(
                f"The B200 SSB engine supports {NATIVE_SCAN_SIZES} scans after the reference's "
                f"padding rule; got {scan_gpts}."
            )
        self.wavelength = electron_wavelength_angstrom(energy)
        n_frames = scan_gpts[0] * scan_gpts[1]
        # (a3) exact u64 frame sums on the GPU
        sums_dev, _ = ops.mean_dp_u64(counts, want_mean=False)
        self._detected_radius_px = None
        sums_host = None
        if det_sampling is None:
            # (a5) the half-max radius detector runs on the host mean pattern
            sums_host = sums_dev.cpu().numpy().view(np.uint64).reshape(det_gpts)
            _, r = detect_bf_radius(ops.mean_from_sums(sums_host, n_frames))
            self._detected_radius_px = float(r)
            det_sampling = (2 * semiangle) / r
            det_sampling = (det_sampling, det_sampling)
        elif isinstance(det_sampling, (int, float)):
            det_sampling = (float(det_sampling), float(det_sampling))
        self.angular_sampling = tuple(det_sampling)
        recip = (det_sampling[0] * 1e-3 / self.wavelength, det_sampling[1] * 1e-3 / self.wavelength)
        self.sampling = (1.0 / (recip[0] * det_gpts[0]), 1.0 / (recip[1] * det_gpts[1]))
        self.gpts = det_gpts
        self._scan_shape = scan_gpts
        self._bf_rows_host = self._bf_cols_host = None
        self._geometry_host = None
        if sums_host is None and (bf_radius is None or bf_radius > 0):
            # (a4) selection and (a8) geometry on the device; the one host sync
            # of preparation reads the 48-byte selection result
            sel = ops.select_bf(sums_dev, det_gpts, n_frames, self.bf_intensity_threshold, bf_radius)
            geom_buf = ops.bf_geometry(
                sel, det_gpts, self._k_step(), self._rotation_angle_rad, self.wavelength,
                self.semiangle_cutoff * 1e-3,
                (self.angular_sampling[0] * 1e-3, self.angular_sampling[1] * 1e-3))
            info = ops.read_bf_info(sel)
            if info.n_mask == 0:
                raise ValueError(
                    f"No bright-field pixels found with threshold {self.bf_intensity_threshold:.2f}. "
                    "Check that the data contains a visible BF disk, or lower the threshold.")
            if info.n_bf == 0:
                raise ValueError(
                    f"No bright-field pixels within bf_radius={info.radius}. Increase bf_radius or "
                    "check detector geometry.")
            n_bf = int(info.n_bf)
            self._bf_linear = sel.bf_linear[:n_bf]
            self._geom_dev = geom_buf[:GEOM_ROWS * n_bf].view(GEOM_ROWS, n_bf)
            self.bf_center = (float(info.center_row), float(info.center_col))
            self._bf_radius_selected = float(info.radius)
            self.dc_value = complex(float(info.dc_re), float(info.dc_im))
        else:
            if sums_host is None:
                sums_host = sums_dev.cpu().numpy().view(np.uint64).reshape(det_gpts)
            # (a4) BF selection on the host mean pattern (radius-detection path)
            sel = select_bf(ops.mean_from_sums(sums_host, n_frames), self.bf_intensity_threshold,
                            bf_radius)
            self._bf_rows_host, self._bf_cols_host = sel.rows, sel.cols
            self.bf_center = sel.center
            self._bf_radius_selected = sel.radius
            lin_host = (sel.rows.astype(np.int64) * det_gpts[1] + sel.cols).astype(np.int32)
            self.dc_value = complex(float(sums_host.reshape(-1)[lin_host].astype(np.float64).mean()), 0.0)
            geo = bf_geometry(sel.rows, sel.cols, sel.center, det_gpts, self.sampling, self.wavelength,
                              self.semiangle_cutoff, self.angular_sampling, self._rotation_angle_rad)
            self._geometry_host = geo
            self._bf_linear, self._geom_dev = ops.STAGING.upload([lin_host, geo.stacked()], self.device)
        self._q_row_host, self._q_col_host = scan_frequencies(scan_gpts, self.scan_sampling)
        self._q_row, self._q_col = _device_frequencies(scan_gpts, self.scan_sampling, self.device)
        self._cached_rotation = self._rotation_angle_rad
        # (a6) gather + Hermitian scan FFT; dc exact from the integer sums
        columns = ops.gather_bf_columns(counts, self._bf_linear, validate=False)
        self.G_qk = ops.scan_fft_half(columns, scan_gpts)
        del columns
        self._workspace = ops.Workspace(self.device)
        self._subset_stack: list = []
        self._best_loss = float("inf")
        self._elapsed_optimize = 0.0
        self._elapsed_refine = 0.0
        self._elapsed_grid = 0.0
        self._n_trials: int | None = None
        self._refine_method: str | None = None
        self._refine_nfev: int | None = None
        self._optuna_trials: list[dict] = []
        self.timings = {"prepare_s": time.perf_counter() - t0}

    # ------------------------------------------------------------ preparation
    def _pad_or_crop(self, counts: torch.Tensor) -> torch.Tensor:
        """Reference padding rule (backend.py:229-269) on the device."""
        h, w = int(counts.shape[0]), int(counts.shape[1])
        target = pad_target(h, w)
        if target is None:
            return counts
        t = target[0]
        if h > t or w > t:
            r0 = max(0, (h - t) // 2)
            c0 = max(0, (w - t) // 2)
            counts = counts[r0:r0 + min(t, h), c0:c0 + min(t, w)].contiguous()
            h, w = int(counts.shape[0]), int(counts.shape[1])
        if h < t or w < t:
            sums, _ = ops.mean_dp_u64(counts, want_mean=False)
            n = h * w
            fill = (sums.cpu().numpy().view(np.uint64).astype(np.float64) / n).astype(np.uint16)
            padded = torch.as_tensor(fill, device=self.device).expand(t, t, *fill.shape).contiguous()
            top, left = (t - h) // 2, (t - w) // 2
            padded[top:top + h, left:left + w] = counts
            counts = padded
        return counts

    # ---------------------------------------------------------------- helpers
    def _k_step(self) -> tuple[float, float]:
        """Detector pixel pitch in 1/A, as cache_rotation derives it from the sampling."""
        return (1.0 / (self.sampling[0] * self.gpts[0]), 1.0 / (self.sampling[1] * self.gpts[1]))

    def _host_selection(self) -> None:
        if self._bf_rows_host is None:
            lin = self._bf_linear.cpu().numpy().astype(np.int64)
            self._bf_rows_host = (lin // self.gpts[1]).astype(np.int32)
            self._bf_cols_host = (lin % self.gpts[1]).astype(np.int32)

    @property
    def bf_inds_row(self) -> np.ndarray:
        """Selected BF detector rows (int32, row-major order); host copy made on first use."""
        self._host_selection()
        return self._bf_rows_host

    @bf_inds_row.setter
    def bf_inds_row(self, value) -> None:
        self._bf_rows_host = value

    @property
    def bf_inds_col(self) -> np.ndarray:
        """Selected BF detector columns (int32); host copy made on first use."""
        self._host_selection()
        return self._bf_cols_host

    @bf_inds_col.setter
    def bf_inds_col(self, value) -> None:
        self._bf_cols_host = value

    @property
    def _geometry(self) -> BFGeometry:
        """Host copy of the per-BF geometry (reference cache names), made on first use."""
        if self._geometry_host is None:
            g = self._geom_dev.cpu().numpy()
            self._geometry_host = BFGeometry(*[g[i].copy() for i in range(GEOM_ROWS)])
        return self._geometry_host

    @_geometry.setter
    def _geometry(self, value) -> None:
        self._geometry_host = value

    def _object_flags(self, quadratic: bool = True) -> int:
        """Flags of the object kernels: the session's, plus the autotuned work
        partition and trotter tile when cached for this scan size and BF count."""
        return self._flags | autotune.cached_object(self.device, self._scan_shape[0],
                                                    int(self.G_qk.shape[0]), self._flags, quadratic)

    def autotune(self) -> dict:
        """Time the object kernels' work partitions and trotter tiles on this
        dataset and cache the fastest for every later session with the same
        scan size and BF count."""
        bits = autotune.tune_object(self.G_qk, self._geom_dev, self._q_row, self._q_col,
                                    self._calibration(), Aberrations(0.0, 0.0, 0.0, 0.0),
                                    self._flags, self._workspace)
        return {"object_chunks": (bits >> _lib.QSSB_FLAG_CHUNKS_SHIFT) & _lib.QSSB_FLAG_CHUNKS_MAX,
                "object_tile_variant": (bits >> _lib.QSSB_FLAG_VARIANT_SHIFT) & _lib.QSSB_FLAG_VARIANT_MAX}

    def _calibration(self) -> Calibration:
        return Calibration(
            n_bf=int(self.G_qk.shape[0]), scan_rows=self._scan_shape[0], scan_cols=self._scan_shape[1],
            reserved=0, wavelength_A=self.wavelength, semiangle_rad=self.semiangle_cutoff * 1e-3,
            det_sampling_row_rad=self.angular_sampling[0] * 1e-3,
            det_sampling_col_rad=self.angular_sampling[1] * 1e-3,
            scan_sampling_row_A=self.scan_sampling[0], scan_sampling_col_A=self.scan_sampling[1],
            dc_re=self.dc_value.real, dc_im=self.dc_value.imag,
        )

    def _resolve_coefs(self, C10=None, C12=None, phi12=None) -> tuple[float, float, float]:
        a = self.aberrations
        return (a.get("C10", 0.0) if C10 is None else C10,
                a.get("C12", 0.0) if C12 is None else C12,
                a.get("phi12", 0.0) if phi12 is None else phi12)

    def _candidates(self, c10, c12, phi12, c30=None) -> torch.Tensor:
        c10 = np.atleast_1d(np.asarray(c10, dtype=np.float32))
        n = c10.size
        c12 = np.broadcast_to(np.asarray(c12, dtype=np.float32), (n,))
        phi12 = np.broadcast_to(np.asarray(phi12, dtype=np.float32), (n,))
        c30 = np.zeros(n, np.float32) if c30 is None else np.broadcast_to(np.asarray(c30, np.float32), (n,))
        host = np.stack([c10, c12, phi12, c30], axis=1).astype(np.float32)
        return torch.as_tensor(host, device=self.device)



    def _require_loss_size(self) -> None:
        if self._scan_shape[0] not in LOSS_SCAN_SIZES:
            raise NotImplementedError(f"phase-variance loss supports {LOSS_SCAN_SIZES} scans")

    # ------------------------------------------------------------- contract
    @property
    def scan_shape(self) -> tuple[int, int]:
        return tuple(int(v) for v in self._scan_shape)

    @property
    def detector_shape(self) -> tuple[int, int]:
        return tuple(int(v) for v in self.gpts)

    @property
    def num_bf(self) -> int:
        return int(self.G_qk.shape[0])

    def cache_rotation(self, rotation_rad: float) -> None:
        """Per-BF geometry for one scan-to-detector rotation (engine.py:784-830)."""
        self._rotation_angle_rad = float(rotation_rad)
        if self._cached_rotation == self._rotation_angle_rad and self._geom_dev is not None:
            return
        geo = bf_geometry(self.bf_inds_row, self.bf_inds_col, self.bf_center, self.gpts,
                          self.sampling, self.wavelength, self.semiangle_cutoff,
                          self.angular_sampling, self._rotation_angle_rad)
        self._geometry = geo
        self._geom_dev = torch.as_tensor(geo.stacked(), device=self.device).contiguous()
        self._cached_rotation = self._rotation_angle_rad

    def reconstruct_object(self, C10=None, C12=None, phi12=None, rotation_angle_rad=None,
                           *, C30: float = 0.0) -> torch.Tensor:
        """Complex object wave (complex64 [R0, R1], on the GPU)."""
        C10, C12, phi12 = self._resolve_coefs(C10, C12, phi12)
        if rotation_angle_rad is not None:
            self.cache_rotation(rotation_angle_rad)
        obj, _ = ops.object_wave(self.G_qk, self._geom_dev, self._q_row, self._q_col,
                                 self._calibration(), Aberrations(C10, C12, phi12, C30),
                                 flags=self._object_flags(C30 == 0.0), workspace=self._workspace,
                                 want_phase=False)
        return obj

    def object_and_phase(self, C10: float, C12: float, phi12: float, C30: float = 0.0
                         ) -> tuple[torch.Tensor, torch.Tensor]:
        """Object wave and its float32 phase from one launch sequence."""
        return ops.object_wave(self.G_qk, self._geom_dev, self._q_row, self._q_col,
                               self._calibration(), Aberrations(C10, C12, phi12, C30),
                               flags=self._object_flags(C30 == 0.0), workspace=self._workspace)

    # the loss of a square 128..1024 scan evaluates the candidate-independent
    # overlap apertures once per geometry (qssb_overlap_table) instead of once
    # per candidate; the table is float2 per (BF pixel, retained scan
    # frequency), so it is built only while it stays below this share of the
    # free device memory and below OVERLAP_TABLE_MAX_BYTES
    use_overlap_table = True
    OVERLAP_TABLE_MAX_BYTES = 16 << 30
    OVERLAP_TABLE_FREE_SHARE = 0.25

    def _overlap_table(self) -> torch.Tensor | None:
        rows, cols = self._scan_shape
        if not self.use_overlap_table or rows != cols or rows not in (128, 256, 512, 1024):
            return None
        if getattr(self, "_overlap_geom", None) is not self._geom_dev:
            self._overlap = None
            self._overlap_geom = self._geom_dev
            need = ops.overlap_table_bytes(self._calibration())
            free, _ = torch.cuda.mem_get_info(self.device)
            if need <= min(self.OVERLAP_TABLE_MAX_BYTES, self.OVERLAP_TABLE_FREE_SHARE * free):
                self._overlap = ops.overlap_table(self._geom_dev, self._q_row, self._q_col,
                                                  self._calibration())
        return self._overlap

    def variance_loss_batch(self, C10, C12, phi12, C30=None) -> torch.Tensor:
        """Phase-variance losses (float32 CUDA [n]) for a candidate batch."""
        self._require_loss_size()
        cands = self._candidates(C10, C12, phi12, C30)
        quad = C30 is None or not np.any(np.asarray(C30))
        flags = self._flags | (QSSB_FLAG_QUADRATIC if quad else 0)
        losses, _ = ops.loss_batch(self.G_qk, self._geom_dev, self._q_row, self._q_col,
                                   self._calibration(), cands, flags=flags,
                                   workspace=self._workspace, overlap=self._overlap_table())
        return losses

    def variance_loss(self, C10: float, C12: float, phi12: float) -> float:
        return float(self.variance_loss_batch([C10], [C12], [phi12])[0])

    def reconstruct_with_loss(self, C10: float, C12: float, phi12: float):
        """Mean over b of the per-BF phases, and the loss (engine.py:1464-1514)."""
        self._require_loss_size()
        cands = self._candidates([C10], [C12], [phi12])
        losses, mp = ops.loss_batch(self.G_qk, self._geom_dev, self._q_row, self._q_col,
                                    self._calibration(), cands,
                                    flags=self._flags | QSSB_FLAG_QUADRATIC,
                                    workspace=self._workspace, want_mean_phase=True,
                                    overlap=self._overlap_table())
        return mp[0], float(losses[0])

    def reconstruct(self, C10: float, C12: float, phi12: float) -> torch.Tensor:
        """Mean per-BF phase image (engine.py:1153-1190)."""
        return self.reconstruct_with_loss(C10, C12, phi12)[0]

    def reconstruct_phase(self, C10=None, C12=None, phi12=None, rotation_angle_rad=None):
        C10, C12, phi12 = self._resolve_coefs(C10, C12, phi12)
        if rotation_angle_rad is not None:
            self.cache_rotation(rotation_angle_rad)
        return self.reconstruct(C10, C12, phi12)

    # ---------------------------------------------------- 14-term chi
    def _full_candidates(self, mags, angles) -> torch.Tensor:
        """float32 CUDA [n, 28] rows (14 magnitudes, 14 angles) from [14] or [n, 14]."""
        m = np.atleast_2d(np.asarray(mags, dtype=np.float32))
        a = np.atleast_2d(np.asarray(angles, dtype=np.float32))
        if m.shape[-1] != FULL_TERMS or a.shape != m.shape:
            raise ValueError("magnitudes and angles must each have shape (14,) or (n, 14)")
        rows = np.ascontiguousarray(np.concatenate([m, a], axis=1))
        return torch.as_tensor(rows, device=self.device)

    def variance_loss_batch_full(self, mags, angles) -> torch.Tensor:
        """Phase-variance losses (float32 CUDA [n]) with the 14-term chi."""
        self._require_loss_size()
        losses, _ = ops.loss_batch_full(self.G_qk, self._geom_dev, self._q_row, self._q_col,
                                        self._calibration(), self._full_candidates(mags, angles),
                                        flags=self._flags, workspace=self._workspace)
        return losses

    def reconstruct_full_with_loss(self, mags_m, angles_rad):
        """Mean per-BF phase and loss with the 14-term chi (engine.py:1350-1458).

        The reference raises NotImplementedError at 128 (engine.py:1373-1377);
        this path serves 128 and 256.
        """
        self._require_loss_size()
        losses, mp = ops.loss_batch_full(self.G_qk, self._geom_dev, self._q_row, self._q_col,
                                         self._calibration(),
                                         self._full_candidates(mags_m, angles_rad),
                                         flags=self._flags, workspace=self._workspace,
                                         want_mean_phase=True)
        return mp[0], float(losses[0])

    def reconstruct_full(self, mags_m, angles_rad):
        """Mean per-BF phase with the 14-term chi (engine.py:1244-1292)."""
        return self.reconstruct_full_with_loss(mags_m, angles_rad)[0]

    def _higher_order_arrays(self) -> tuple[np.ndarray, np.ndarray, bool]:
        """(magnitudes [14], angles [14] rad, any higher order active) from the
        aberrations dict: C10, C12, phi12 (rad); Cn0 scalars; Cnm_mag with
        Cnm_angle in degrees (backend.py:730-771)."""
        a = self.aberrations
        mags = np.zeros(FULL_TERMS, dtype=np.float32)
        angs = np.zeros(FULL_TERMS, dtype=np.float32)
        mags[0] = a.get("C10", 0.0)
        mags[1] = a.get("C12", 0.0)
        angs[1] = a.get("phi12", 0.0)
        active = False
        for idx, name in enumerate(FULL_TERM_NAMES[2:], start=2):
            if name.endswith("0"):
                mag, ang = float(a.get(name, 0.0)), 0.0
            else:
                mag = float(a.get(f"{name}_mag", 0.0))
                ang = math.radians(float(a.get(f"{name}_angle", 0.0)))
            active = active or mag != 0.0
            mags[idx] = mag
            angs[idx] = ang
        return mags, angs, active

    @staticmethod
    def phase_to_numpy(phase) -> np.ndarray:
        return phase.detach().float().cpu().numpy().astype(np.float32, copy=False)

    def _brightfield(self) -> BrightfieldDisk:
        rows = self.bf_inds_row.astype(np.float64)
        cols = self.bf_inds_col.astype(np.float64)
        radius = float(np.sqrt((rows - self.bf_center[0]) ** 2 + (cols - self.bf_center[1]) ** 2).max()) + 1e-3
        sampling = 0.5 * (float(self.angular_sampling[0]) + float(self.angular_sampling[1]))
        return BrightfieldDisk(rows=self.bf_inds_row, cols=self.bf_inds_col,
                               center_row_col=self.bf_center, radius_px=radius,
                               detected_radius_px=2.0 * float(self.semiangle_cutoff) / sampling,
                               detector_shape=self.detector_shape)

    def result(self, *, compute_loss: bool = True) -> SSBResult:
        C10, C12, phi12 = self._resolve_coefs()
        mags, angs, higher = self._higher_order_arrays()
        if higher:
            # 14-term chi: the mean per-BF phase as a unit-amplitude object
            # and no diagnostic loss (backend.py:795-820)
            phase = self.reconstruct_full(mags, angs)
            obj = torch.polar(torch.ones_like(phase), phase)
        else:
            with self._oom_as_memory_error("reconstruction"):
                obj = self.reconstruct_object(C10, C12, phi12)
        loss = None
        if compute_loss and not higher and self._scan_shape[0] in LOSS_SCAN_SIZES:
            try:
                loss = self.variance_loss(C10, C12, phi12)
            except (ValueError, ZeroDivisionError, FloatingPointError):
                loss = None
            if loss is not None and not math.isfinite(loss):
                loss = None
        elapsed = self._elapsed_optimize + self._elapsed_grid + self._elapsed_refine
        bf = self._brightfield()
        return SSBResult(
            object_wave=obj, backend="cuda", aberrations=dict(self.aberrations),
            rotation_angle_deg=math.degrees(self._rotation_angle_rad), loss=loss,
            elapsed=elapsed if elapsed > 0 else None, timings=dict(self.timings),
            n_trials=self._n_trials, num_bf=self.num_bf, refine_method=self._refine_method,
            refine_nfev=self._refine_nfev,
            refine_elapsed=self._elapsed_refine if self._elapsed_refine > 0 else None,
            voltage_kV=self.voltage_kV, semiangle_mrad=self.semiangle_mrad,
            scan_sampling_A=self.scan_sampling[0], bf_center=bf.center_row_col,
            bf_radius=bf.radius_px, detected_bf_radius=bf.detected_radius_px,
            optuna_trials=self._optuna_trials,
        )

    def reconstruct_result(self, aberrations: dict[str, float], *,
                           compute_loss: bool = True) -> SSBResult:
        self.aberrations.update(aberrations)
        return self.result(compute_loss=compute_loss)

    def preview(self, aberrations: dict[str, float], *, compute_loss: bool,
                higher_order_magnitudes: np.ndarray | None,
                higher_order_angles: np.ndarray | None) -> tuple[np.ndarray, float | None]:
        if higher_order_magnitudes is not None:
            if compute_loss:
                phase, loss = self.reconstruct_full_with_loss(higher_order_magnitudes,
                                                              higher_order_angles)
                return self.phase_to_numpy(phase), float(loss)
            return self.phase_to_numpy(self.reconstruct_full(higher_order_magnitudes,
                                                             higher_order_angles)), None
        if compute_loss:
            phase, loss = self.reconstruct_with_loss(aberrations["C10"], aberrations["C12"],
                                                     aberrations["phi12"])
        else:
            phase, loss = self.reconstruct(aberrations["C10"], aberrations["C12"],
                                           aberrations["phi12"]), None
        return self.phase_to_numpy(phase), None if loss is None else float(loss)

    @contextmanager
    def _bf_subset(self, indices: np.ndarray):
        idx = torch.as_tensor(np.asarray(indices, dtype=np.int64), device=self.device)
        saved = (self.G_qk, self.bf_inds_row, self.bf_inds_col, self._geom_dev, self._geometry,
                 self._bf_linear)
        try:
            self.G_qk = self.G_qk.index_select(0, idx).contiguous()
            self.bf_inds_row = self.bf_inds_row[indices]
            self.bf_inds_col = self.bf_inds_col[indices]
            self._geom_dev = self._geom_dev.index_select(1, idx).contiguous()
            self._bf_linear = self._bf_linear.index_select(0, idx).contiguous()
            yield self
        finally:
            (self.G_qk, self.bf_inds_row, self.bf_inds_col, self._geom_dev, self._geometry,
             self._bf_linear) = saved

    def preview_context(self, num_bf: int):
        """Deterministic reduced-BF context (engine.py:336-360)."""
        full = self.num_bf
        count = max(1, min(int(num_bf), full))
        step = max(1, full // count)
        return self._bf_subset(np.arange(0, full, step)[:count])

    def browser_state(self) -> SSBExportState:
        geo = self._geometry
        return SSBExportState(
            backend="cuda", scan_shape=self.scan_shape, brightfield=self._brightfield(),
            kx_bf=geo.kx_bf.copy(), ky_bf=geo.ky_bf.copy(), qx_1d=self._q_row_host.copy(),
            qy_1d=self._q_col_host.copy(), aperture_k=geo.aperture_k.copy(),
            alpha_k2=geo.alpha_k2.copy(), cos2phi_k=geo.cos2phi_k.copy(),
            sin2phi_k=geo.sin2phi_k.copy(), wavelength_A=float(self.wavelength),
            semiangle_rad=float(self.semiangle_cutoff * 1e-3),
            angular_sampling_rad=(float(self.angular_sampling[0] * 1e-3),
                                  float(self.angular_sampling[1] * 1e-3)),
            sampling_A=(float(self.sampling[0]), float(self.sampling[1])),
            dc_value=complex(self.dc_value),
        )

    _EXPORT_CHUNK_BF = 256  # BF pixels per device chunk (engine.py:662)

    def export_brightfield(self, data, path_stem) -> tuple[Path, float]:
        """Write the exact detector counts of the selected BF pixels, BF-major
        ``[bf, scan]``, to ``path_stem`` + ``.u8`` or ``.u16``; returns the path
        and the seconds it took (backend.py:693-702, engine.py:577-701).

        The rules are the reference's: u8 or u16 counts only (``TypeError``
        otherwise); the data must have the engine's scan shape (``ValueError``);
        u16 is narrowed to u8 only when the largest count of the WHOLE block -
        not just of the BF pixels - is at most 255. The device gathers and
        transposes 256 BF pixels at a time (``qssb_export_bf_columns``) into
        one of two pinned host buffers while a writer thread appends the
        previous chunk to the file.
        """
        from concurrent.futures import ThreadPoolExecutor

        start = time.perf_counter()
        counts = _as_device_counts_exact(data, self.device)
        if counts.ndim != 4 or tuple(int(v) for v in counts.shape[:2]) != self.scan_shape:
            raise ValueError(
                "CUDA BF-source data must match the engine scan shape; "
                f"got {tuple(counts.shape)}, expected {self.scan_shape} + detector.")
        counts = counts.contiguous()
        max_value = int(ops.count_max(counts).cpu()[0]) & 0xFFFFFFFF
        out_dtype = np.dtype(np.uint8 if max_value <= 255 else np.uint16)
        torch_out = torch.uint8 if out_dtype == np.uint8 else torch.uint16
        path = Path(path_stem).with_suffix(".u8" if out_dtype == np.uint8 else ".u16")
        path = path.expanduser().resolve()
        path.parent.mkdir(parents=True, exist_ok=True)
        path.unlink(missing_ok=True)

        num_bf = self.num_bf
        plane = int(self.scan_shape[0] * self.scan_shape[1])
        cap = max(1, min(num_bf, self._EXPORT_CHUNK_BF))
        row_bytes = plane * out_dtype.itemsize
        device_cols = torch.empty((cap, plane), dtype=torch_out, device=self.device)
        host = [torch.empty((cap, row_bytes), dtype=torch.uint8, pin_memory=True) for _ in range(2)]
        pending = [None, None]
        stream = torch.cuda.current_stream(self.device)
        with path.open("wb") as fh, ThreadPoolExecutor(max_workers=1) as writer:
            for chunk, off in enumerate(range(0, num_bf, cap)):
                slot = chunk % 2
                if pending[slot] is not None:
                    pending[slot].result()
                n = min(cap, num_bf - off)
                ops.export_bf_columns(counts, self._bf_linear[off:off + n], device_cols[:n])
                host[slot][:n].copy_(device_cols[:n].view(torch.uint8), non_blocking=True)
                done = torch.cuda.Event()
                done.record(stream)
                done.synchronize()
                pending[slot] = writer.submit(host[slot][:n].numpy().tofile, fh)
            for fut in pending:
                if fut is not None:
                    fut.result()
        self._bf_source = (path, out_dtype, max_value)
        self.bf_source_write_seconds = time.perf_counter() - start
        return path, self.bf_source_write_seconds

    # ------------------------------------------------------------ fitting
    @contextmanager
    def _oom_as_memory_error(self, stage: str):
        """A device allocation failure inside ``stage`` becomes the reference's
        actionable ``MemoryError`` (backend.py:808-816, :1078-1086)."""
        try:
            yield
        except torch.cuda.OutOfMemoryError:
            free_gb = torch.cuda.mem_get_info(self.device)[0] / 1e9
            raise MemoryError(
                f"Out of GPU VRAM during SSB {stage} "
                f"({self.num_bf} BF pixels, {free_gb:.1f} GB free).\n"
                f"Try: SSB(..., bf_radius=<smaller>) to reduce BF pixel count, "
                f"or restart the kernel to free stale GPU memory."
            ) from None

    def _evaluate_retrying(self, x: np.ndarray, verbose: bool = False) -> np.ndarray:
        """Losses of a candidate batch; on a device allocation failure, free the
        loss workspace and the allocator's cached blocks and score the batch
        in halves (the reference halves its BF chunk, backend.py:1347-1354;
        the B200 loss workspace scales with the candidate count instead)."""
        try:
            return self._evaluate(x)
        except torch.cuda.OutOfMemoryError:
            if len(x) <= 1:
                raise
            self._workspace.release()
            torch.cuda.empty_cache()
            half = (len(x) + 1) // 2
            if verbose:
                print(f"  OOM - retrying with {half}-candidate batches")
            return np.concatenate([self._evaluate_retrying(x[:half], verbose),
                                   self._evaluate_retrying(x[half:], verbose)])

    def _evaluate(self, x: np.ndarray) -> np.ndarray:
        x = np.atleast_2d(np.asarray(x, dtype=np.float64))
        return self.variance_loss_batch(x[:, 0], x[:, 1], x[:, 2]).double().cpu().numpy()

    def optimize(self, aberrations=None, rotation_angle_deg=None, n_trials: int = 200,
                 seed: int = 42, verbose: bool = True, bf_subsample: float | None = None,
                 objective_mode: str = "exact"):
        """Seeded batched global search over C10/C12/phi12 (replaces Optuna TPE)."""
        t0 = time.perf_counter()
        if objective_mode not in {"native", "exact"}:
            raise ValueError(f"objective_mode must be 'native' or 'exact'; got {objective_mode!r}.")
        if rotation_angle_deg is not None:
            raise NotImplementedError("rotation search is not supported by the B200 sweep")
        ranges = dict(self._DEFAULT_OPTIMIZE_RANGES) if aberrations is None else dict(aberrations)
        keys, lo, hi = search_box(ranges, self.aberrations)
        with self._oom_as_memory_error("optimization"):
            best_x, best_f, xs, fs = batch_sweep(self._evaluate, lo, hi, int(n_trials), seed=seed,
                                                 batch=self._SWEEP_BATCH)
        self._optuna_trials = [
            {"params": {"C10_nm": float(x[0]), "C12_nm": float(x[1]), "phi12_deg": math.degrees(x[2])},
             "loss": float(f)} for x, f in zip(xs, fs)
        ]
        for k, v in zip(keys, best_x):
            self.aberrations[k] = float(v)
        self._best_loss = best_f
        self._n_trials = int(n_trials)
        self._elapsed_optimize = time.perf_counter() - t0
        if verbose:
            print(f"  Optimize: loss={best_f:.6f} {self.aberrations} {self._elapsed_optimize:.2f}s")
        return self

    def refine(self, verbose: bool = True, xatol: float = 0.1, fatol: float = 1e-8,
               lock: list[str] | None = None, bf_subsample: float | None = None,
               objective_mode: str | None = None):
        """Batched Nelder-Mead from the current aberrations (backend.py:1112-1259)."""
        t0 = time.perf_counter()
        if lock:
            raise ValueError(
                "GPU-only SSB Nelder-Mead does not support locked refinement yet "
                f"(locked: {', '.join(sorted(lock))})."
            )
        x0 = np.array([self.aberrations["C10"], self.aberrations["C12"], self.aberrations["phi12"]])
        with self._oom_as_memory_error("refinement"):
            best_x, best_f, nfev = batch_nelder_mead(self._evaluate, x0, xatol=xatol, fatol=fatol)
        for i, k in enumerate(("C10", "C12", "phi12")):
            self.aberrations[k] = float(best_x[i])
        self._best_loss = best_f
        self._refine_method = "nelder-mead"
        self._refine_nfev = int(nfev)
        self._elapsed_refine = time.perf_counter() - t0
        if verbose:
            print(f"  Refine (nelder-mead, {nfev} evals): loss={best_f:.6f} {self._elapsed_refine:.2f}s")
        return self

    def grid_search(self, window=None, n_points=None, verbose: bool = True):
        """Exhaustive C10 x C12 x phi12 grid around the current aberrations."""
        t0 = time.perf_counter()
        window = window or {}
        n_points = n_points or {}
        hw = {k: window.get(k, v) for k, v in self._DEFAULT_GRID_HALF_WIDTHS.items()}
        npts = {k: n_points.get(k, v) for k, v in self._DEFAULT_GRID_POINTS.items()}
        c10 = np.linspace(self.aberrations["C10"] - hw["C10_nm"], self.aberrations["C10"] + hw["C10_nm"], npts["C10_nm"])
        c12 = np.linspace(max(0, self.aberrations["C12"] - hw["C12_nm"]), self.aberrations["C12"] + hw["C12_nm"], npts["C12_nm"])
        p_deg = math.degrees(self.aberrations["phi12"])
        phi = np.radians(np.linspace(p_deg - hw["phi12_deg"], p_deg + hw["phi12_deg"], npts["phi12_deg"]))
        grid = np.array(np.meshgrid(c10, c12, phi, indexing="ij")).reshape(3, -1).T
        with self._oom_as_memory_error("grid search"):
            losses = np.concatenate([self._evaluate_retrying(grid[s:s + 256], verbose)
                                     for s in range(0, len(grid), 256)])
        best = int(np.argmin(losses))
        self.aberrations.update(C10=float(grid[best, 0]), C12=float(grid[best, 1]), phi12=float(grid[best, 2]))
        self._best_loss = float(losses[best])
        self._elapsed_grid = time.perf_counter() - t0
        if verbose:
            print(f"  Grid ({len(grid)} evals): loss={self._best_loss:.6f}")
        return self

    def fit(self, *, trials: int, refinement: str | None,
            search_ranges: dict[str, tuple[float, float] | float] | None,
            refine_lock: list[str] | None, seed: int, verbose: bool) -> SSBResult:
        if trials:
            self.optimize(aberrations=search_ranges, n_trials=int(trials), seed=int(seed),
                          verbose=verbose)
        if refinement == "nelder-mead":
            self.refine(verbose=verbose, lock=refine_lock)
        return self.result()

    # --------------------------------------------------------------- memory
    def free(self) -> None:
        self.G_qk = None
        self._geom_dev = None
        self._overlap = self._overlap_geom = None
        self._workspace.release()

    def close(self) -> None:
        self.free()


__all__ = ["B200SSBBackend"]
