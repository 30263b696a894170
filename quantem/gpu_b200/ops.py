"""Device operations of the SSB engine, called through the C ABI.

Thin wrappers that check shapes/dtypes on the host, allocate outputs as
torch CUDA tensors (torch is the allocator and stream provider only) and
call ``libqssb.so``. Every computation runs in the native sm_100a kernels;
a CPU tensor is rejected rather than computed elsewhere.
"""
from __future__ import annotations

import contextlib
import ctypes

import torch

from . import _lib
from ._lib import Aberrations, Calibration, check

# Kernel launches each entry point enqueues (the evidence counted by bench.py).
# Kernel launches made through this module, counted by the library itself
# (qssb_kernel_launches before and after each call); graph replays add their
# captured count where they are issued.
LAUNCH_COUNT = 0
_PROFILE: list | None = None


@contextlib.contextmanager
def profile_ops():
    """Record (entry point, start event, end event) around every C-ABI call.

    Events are recorded on the calling stream, so their elapsed time is the
    device time of the kernels that call enqueued.
    """
    global _PROFILE
    prev = _PROFILE
    _PROFILE = []
    try:
        yield _PROFILE
    finally:
        _PROFILE = prev


def _call(name: str, device: torch.device, *args) -> None:
    global LAUNCH_COUNT
    fn = getattr(_lib.load(), name)
    before = int(_lib.load().qssb_kernel_launches())
    if _PROFILE is None:
        check(fn(*args))
    else:
        stream = torch.cuda.current_stream(device)
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        check(fn(*args))
        end.record(stream)
        _PROFILE.append((name, start, end))
    LAUNCH_COUNT += int(_lib.load().qssb_kernel_launches()) - before


def _require_cuda(t: torch.Tensor, name: str, dtype: torch.dtype) -> None:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (the SSB engine has no CPU path)")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


def _stream(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _ptr(t: torch.Tensor | None) -> ctypes.c_void_p:
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


class PinnedStaging:
    """A reusable pinned host buffer for batching small host->device uploads."""

    def __init__(self):
        self._buf: torch.Tensor | None = None

    def upload(self, arrays, device: torch.device) -> list[torch.Tensor]:
        """Copy numpy arrays to ``device`` with one pinned H2D transfer.

        Returns device tensors (views into one allocation) with the arrays'
        dtypes and shapes; each array starts on a 256-byte boundary.
        """
        import numpy as np

        offsets, total = [], 0
        for a in arrays:
            offsets.append(total)
            total += (a.nbytes + 255) & ~255
        self.wait()  # the previous upload must have left the pinned buffer
        if self._buf is None or self._buf.numel() < total:
            self._buf = torch.empty(max(total, 1 << 16), dtype=torch.uint8, pin_memory=True)
        host = self._buf.numpy()
        for a, off in zip(arrays, offsets):
            host[off:off + a.nbytes] = np.ascontiguousarray(a).view(np.uint8).reshape(-1)
        dev = self._buf[:total].to(device, non_blocking=True)
        out = []
        for a, off in zip(arrays, offsets):
            t = dev[off:off + a.nbytes].view(getattr(torch, str(a.dtype)))
            out.append(t.reshape(a.shape))
        # the pinned buffer may be rewritten only after this copy has run
        self._event = torch.cuda.Event()
        self._event.record(torch.cuda.current_stream(device))
        return out

    def wait(self) -> None:
        ev = getattr(self, "_event", None)
        if ev is not None:
            ev.synchronize()


STAGING = PinnedStaging()


class Workspace:
    """A reusable, growing device scratch buffer (256-byte aligned)."""

    def __init__(self, device: torch.device | str = "cuda"):
        self.device = torch.device(device)
        self._buf: torch.Tensor | None = None

    def get(self, nbytes: int) -> torch.Tensor:
        if self._buf is None or self._buf.numel() < nbytes:
            self._buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=self.device)
        return self._buf

    def release(self) -> None:
        self._buf = None


def mean_dp_u64(counts: torch.Tensor, want_mean: bool = True
                ) -> tuple[torch.Tensor, torch.Tensor | None]:
    """Exact u64 detector sums and float32 mean DP of ``counts[..., K0, K1]``.

    Returns (sums as int64 [K0, K1] holding the u64 values, mean_dp f32 [K0, K1]
    or None when ``want_mean`` is False).
    """
    _require_cuda(counts, "counts", torch.uint16)
    k0, k1 = int(counts.shape[-2]), int(counts.shape[-1])
    n_frames = counts.numel() // (k0 * k1)
    sums = torch.empty((k0, k1), dtype=torch.int64, device=counts.device)
    mean = torch.empty((k0, k1), dtype=torch.float32, device=counts.device) if want_mean else None
    _call("qssb_mean_dp_u64", counts.device, _ptr(counts), n_frames, k0 * k1, _ptr(sums),
          _ptr(mean), _stream(counts))
    return sums, mean


def mean_from_sums(sums_u64, n_frames: int):
    """float32(sum) / n_frames with IEEE rounding: the kernel's mean, on the host."""
    import numpy as np

    return np.asarray(sums_u64, dtype=np.uint64).astype(np.float32) / np.float32(n_frames)


BF_INFO_BYTES = ctypes.sizeof(_lib.BFInfo)


class DeviceSelection:
    """Device outputs of :func:`select_bf`: BF indices (capacity K0*K1), the
    ``qssb_bf_info_t`` bytes and the float32 mean pattern (or None)."""

    def __init__(self, bf_linear: torch.Tensor, info: torch.Tensor, mean_dp: torch.Tensor | None):
        self.bf_linear = bf_linear
        self.info = info
        self.mean_dp = mean_dp


def select_bf(sums: torch.Tensor, det_shape: tuple[int, int], n_frames: int,
              threshold: float = 0.0, bf_radius: float | None = None,
              want_mean: bool = False) -> DeviceSelection:
    """BF selection on the device from the exact u64 sums (no host sync)."""
    _require_cuda(sums, "sums", torch.int64)
    k0, k1 = int(det_shape[0]), int(det_shape[1])
    if sums.numel() != k0 * k1:
        raise ValueError("sums must hold det_rows * det_cols entries")
    radius = 0.0 if bf_radius is None else float(bf_radius)
    if bf_radius is not None and not radius > 0:
        raise ValueError("bf_radius must be positive")
    dev = sums.device
    lin = torch.empty(k0 * k1, dtype=torch.int32, device=dev)
    info = torch.empty(BF_INFO_BYTES, dtype=torch.uint8, device=dev)
    mean = torch.empty((k0, k1), dtype=torch.float32, device=dev) if want_mean else None
    _call("qssb_select_bf", dev, _ptr(sums), k0, k1, int(n_frames), float(threshold), radius,
          _ptr(mean), _ptr(lin), _ptr(info), _stream(sums))
    return DeviceSelection(lin, info, mean)


def read_bf_info(sel: DeviceSelection) -> "_lib.BFInfo":
    """Copy the 48-byte selection result to the host (the one sync of a cold
    preparation)."""
    host = torch.empty(BF_INFO_BYTES, dtype=torch.uint8, pin_memory=True)
    host.copy_(sel.info, non_blocking=True)
    torch.cuda.current_stream(sel.info.device).synchronize()
    return _lib.BFInfo.from_buffer_copy(host.numpy().tobytes())


def bf_geometry(sel: DeviceSelection, det_shape: tuple[int, int], k_step: tuple[float, float],
                rotation_rad: float, wavelength_A: float, semiangle_rad: float,
                det_sampling_rad: tuple[float, float]) -> torch.Tensor:
    """Float32 buffer of 8*capacity whose first 8*n_bf floats are the
    ``[8][n_bf]`` geometry of the selected pixels (written on the device)."""
    import math

    k0, k1 = int(det_shape[0]), int(det_shape[1])
    cap = int(sel.bf_linear.numel())
    geom = torch.empty(_lib.GEOM_ROWS * cap, dtype=torch.float32, device=sel.bf_linear.device)
    gp = _lib.GeometryParams(
        k_step_row_inv_A=float(k_step[0]), k_step_col_inv_A=float(k_step[1]),
        rot_cos=math.cos(-rotation_rad), rot_sin=math.sin(-rotation_rad),
        wavelength_A=float(wavelength_A), semiangle_rad=float(semiangle_rad),
        det_sampling_row_rad=float(det_sampling_rad[0]),
        det_sampling_col_rad=float(det_sampling_rad[1]))
    _call("qssb_bf_geometry", sel.bf_linear.device, _ptr(sel.bf_linear), _ptr(sel.info), k0, k1,
          cap, ctypes.byref(gp), _ptr(geom), _stream(geom))
    return geom


BOX_WORDS = 8  # the device box record: r0, r1, c0, c1, width, pixels, valid, unused


def bf_box_estimate(sample_sums: torch.Tensor, det_shape: tuple[int, int], capacity: int,
                    radius_px: float = 0.0, margin: int = 2,
                    out: torch.Tensor | None = None) -> torch.Tensor:
    """Superset box of the BF disk from u64 sums of some frames (device int32[8])."""
    _require_cuda(sample_sums, "sample_sums", torch.int64)
    box = out if out is not None else torch.empty(BOX_WORDS, dtype=torch.int32,
                                                  device=sample_sums.device)
    _call("qssb_bf_box_estimate", sample_sums.device, _ptr(sample_sums), int(det_shape[0]),
          int(det_shape[1]), float(radius_px), int(margin), int(capacity), _ptr(box),
          _stream(sample_sums))
    return box


def mean_dp_u64_box(counts: torch.Tensor, box: torch.Tensor, box_cols: torch.Tensor,
                    sums: torch.Tensor | None = None) -> torch.Tensor:
    """Exact u64 frame sums (int64 [K0, K1]) that also write the box's columns."""
    _require_cuda(counts, "counts", torch.uint16)
    _require_cuda(box, "box", torch.int32)
    _require_cuda(box_cols, "box_cols", torch.uint16)
    k0, k1 = int(counts.shape[-2]), int(counts.shape[-1])
    n_frames = counts.numel() // (k0 * k1)
    if box_cols.ndim != 2 or box_cols.shape[1] != n_frames:
        raise ValueError("box_cols must be [capacity, n_frames]")
    if sums is None:
        sums = torch.empty((k0, k1), dtype=torch.int64, device=counts.device)
    _call("qssb_mean_dp_u64_box", counts.device, _ptr(counts), n_frames, k0, k1, _ptr(sums),
          _ptr(box), int(box_cols.shape[0]), _ptr(box_cols), _stream(counts))
    return sums


def bf_box_map(sel: DeviceSelection, det_shape: tuple[int, int], box: torch.Tensor,
               capacity: int, out: tuple[torch.Tensor, torch.Tensor] | None = None
               ) -> tuple[torch.Tensor, torch.Tensor]:
    """(map int32 [capacity]: BF pixel -> box column, ok int32 [1]); capacity
    is the box columns' row count (the map holds as many entries)."""
    dev = sel.bf_linear.device
    if out is None:
        out = (torch.empty(capacity, dtype=torch.int32, device=dev),
               torch.empty(1, dtype=torch.int32, device=dev))
    bmap, ok = out
    _call("qssb_bf_box_map", dev, _ptr(sel.bf_linear), _ptr(sel.info), int(det_shape[0]),
          int(det_shape[1]), int(min(capacity, bmap.numel())), int(capacity), _ptr(box), _ptr(bmap),
          _ptr(ok), _stream(box))
    return bmap, ok


def scan_fft_half_mapped(box_cols: torch.Tensor, bf_map: torch.Tensor, n_bf: int,
                         scan_shape: tuple[int, int], out: torch.Tensor | None = None
                         ) -> torch.Tensor:
    """Hermitian half-plane scan spectra of BF pixels whose images are box
    columns ``bf_map[b]`` (128x128 scans)."""
    _require_cuda(box_cols, "box_cols", torch.uint16)
    _require_cuda(bf_map, "bf_map", torch.int32)
    r0, r1 = int(scan_shape[0]), int(scan_shape[1])
    if box_cols.shape[1] != r0 * r1 or bf_map.numel() < n_bf:
        raise ValueError("box_cols must be [capacity, R0*R1] and bf_map hold n_bf entries")
    g = out if out is not None else torch.empty((n_bf, r0, r1 // 2 + 1), dtype=torch.complex64,
                                                device=box_cols.device)
    _call("qssb_scan_fft_half_mapped", box_cols.device, _ptr(box_cols), int(box_cols.shape[0]),
          _ptr(bf_map), int(n_bf), r0, r1, _ptr(g), _stream(box_cols))
    return g


def gather_bf_columns(counts: torch.Tensor, bf_linear: torch.Tensor, validate: bool = True,
                      variant: int = 0) -> torch.Tensor:
    """columns[b, f] = counts[f, bf_linear[b]] (u16, BF-major).

    ``validate`` checks the index range on the device (two host syncs); the
    backend passes indices it built itself and skips it. ``variant`` names
    the tile shape (``qssb_gather_bf_columns_2d_ex``; 0 = built-in rule).
    """
    _require_cuda(counts, "counts", torch.uint16)
    _require_cuda(bf_linear, "bf_linear", torch.int32)
    k0, k1 = int(counts.shape[-2]), int(counts.shape[-1])
    n_frames = counts.numel() // (k0 * k1)
    n_bf = int(bf_linear.numel())
    if validate and n_bf and (int(bf_linear.min()) < 0 or int(bf_linear.max()) >= k0 * k1):
        raise ValueError("bf_linear indices must lie in [0, K0*K1)")
    out = torch.empty((n_bf, n_frames), dtype=torch.uint16, device=counts.device)
    _call("qssb_gather_bf_columns_2d_ex", counts.device, _ptr(counts), n_frames, k0, k1,
          _ptr(bf_linear), n_bf, _ptr(out), int(variant), _stream(counts))
    return out


_COUNT_BYTES = {torch.uint8: 1, torch.uint16: 2}


def count_max(counts: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """Largest count of a u8/u16 CUDA block, as a device int32 scalar-like [1]
    tensor holding the u32 result (read it with ``int(t[0])``)."""
    if not isinstance(counts, torch.Tensor) or not counts.is_cuda:
        raise ValueError("counts must be a CUDA tensor (the SSB engine has no CPU path)")
    if counts.dtype not in _COUNT_BYTES:
        raise TypeError(f"counts must be uint8 or uint16, got {counts.dtype}")
    if not counts.is_contiguous():
        raise ValueError("counts must be contiguous")
    if out is None:
        out = torch.empty(1, dtype=torch.int32, device=counts.device)
    _call("qssb_count_max", counts.device, _ptr(counts), _COUNT_BYTES[counts.dtype],
          counts.numel(), _ptr(out), _stream(counts))
    return out


def export_bf_columns(counts: torch.Tensor, bf_linear: torch.Tensor, out: torch.Tensor) -> None:
    """out[b, f] = counts[f, bf_linear[b]] for the ``out.shape[0]`` BF pixels of
    ``bf_linear`` (u8/u16 in, u8/u16 out; narrowing keeps the low byte)."""
    if counts.dtype not in _COUNT_BYTES or out.dtype not in _COUNT_BYTES:
        raise TypeError("counts and out must be uint8 or uint16")
    for t, name in ((counts, "counts"), (out, "out")):
        if not t.is_cuda or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous CUDA tensor")
    _require_cuda(bf_linear, "bf_linear", torch.int32)
    det = int(counts.shape[-2]) * int(counts.shape[-1])
    n_scan = counts.numel() // det
    n_bf = int(out.shape[0])
    if out.ndim != 2 or out.shape[1] != n_scan or bf_linear.numel() < n_bf:
        raise ValueError("out must be [n_bf, n_scan] with n_bf <= len(bf_linear)")
    _call("qssb_export_bf_columns", counts.device, _ptr(counts), _COUNT_BYTES[counts.dtype],
          n_scan, det, _ptr(bf_linear), n_bf, _ptr(out), _COUNT_BYTES[out.dtype], _stream(counts))


def scan_fft_variants(scan_rows: int) -> int:
    """Launch shapes ``qssb_scan_fft_half_ex`` offers at this scan size (1..n)."""
    n = ctypes.c_int32(0)
    check(_lib.load().qssb_scan_fft_variants(int(scan_rows), ctypes.byref(n)))
    return int(n.value)


def scan_fft_half(columns: torch.Tensor, scan_shape: tuple[int, int], variant: int = 0
                  ) -> torch.Tensor:
    """Hermitian half-plane scan spectra G[b, r, c], c in [0, R1/2] (complex64).
    ``variant`` names the launch shape (0 = built-in; every shape gives the
    same bits)."""
    _require_cuda(columns, "columns", torch.uint16)
    r0, r1 = int(scan_shape[0]), int(scan_shape[1])
    n_bf = int(columns.shape[0])
    if columns.shape[1] != r0 * r1:
        raise ValueError("columns must hold R0*R1 frames per BF pixel")
    g = torch.empty((n_bf, r0, r1 // 2 + 1), dtype=torch.complex64, device=columns.device)
    _call("qssb_scan_fft_half_ex", columns.device, _ptr(columns), n_bf, r0, r1, _ptr(g),
          int(variant), _stream(columns))
    return g


def object_workspace_bytes(cal: Calibration, flags: int = 0) -> int:
    n = ctypes.c_size_t(0)
    check(_lib.load().qssb_object_workspace_bytes(ctypes.byref(cal), int(flags), ctypes.byref(n)))
    return int(n.value)


def object_wave(g_half: torch.Tensor, bf_geom: torch.Tensor, q_row: torch.Tensor,
                q_col: torch.Tensor, cal: Calibration, ab: Aberrations, *, flags: int = 0,
                workspace: Workspace | None = None, want_phase: bool = True,
                dc_device: torch.Tensor | None = None, out: tuple | None = None
                ) -> tuple[torch.Tensor, torch.Tensor | None]:
    """Object wave (complex64 [R0, R1]) and its phase (float32) for one candidate."""
    _require_cuda(g_half, "g_half", torch.complex64)
    _require_cuda(bf_geom, "bf_geom", torch.float32)
    _require_cuda(q_row, "q_row", torch.float32)
    _require_cuda(q_col, "q_col", torch.float32)
    r0, r1 = int(cal.scan_rows), int(cal.scan_cols)
    if (tuple(g_half.shape) != (cal.n_bf, r0, r1 // 2 + 1)
            or tuple(bf_geom.shape) != (_lib.GEOM_ROWS, cal.n_bf)):
        raise ValueError("g_half / bf_geom shapes do not match the calibration")
    ws = workspace or Workspace(g_half.device)
    need = object_workspace_bytes(cal, flags)
    buf = ws.get(need)
    if out is not None:
        obj, ph = out
    else:
        obj = torch.empty((r0, r1), dtype=torch.complex64, device=g_half.device)
        ph = torch.empty((r0, r1), dtype=torch.float32, device=g_half.device) if want_phase else None
    if dc_device is None:
        _call("qssb_object", g_half.device, _ptr(g_half), _ptr(bf_geom), _ptr(q_row), _ptr(q_col),
              ctypes.byref(cal), ctypes.byref(ab), int(flags), _ptr(buf), buf.numel(), _ptr(obj),
              _ptr(ph), _stream(g_half))
    else:
        _call("qssb_object_ex", g_half.device, _ptr(g_half), _ptr(bf_geom), _ptr(q_row),
              _ptr(q_col), ctypes.byref(cal), ctypes.byref(ab), int(flags), _ptr(dc_device),
              _ptr(buf), buf.numel(), _ptr(obj), _ptr(ph), _stream(g_half))
    return obj, ph


def loss_workspace_bytes(cal: Calibration, n_cand: int, flags: int = 0) -> int:
    n = ctypes.c_size_t(0)
    check(_lib.load().qssb_loss_workspace_bytes(ctypes.byref(cal), int(n_cand), int(flags),
                                                ctypes.byref(n)))
    return int(n.value)


def loss_full_workspace_bytes(cal: Calibration, n_cand: int, flags: int = 0) -> int:
    n = ctypes.c_size_t(0)
    check(_lib.load().qssb_loss_full_workspace_bytes(ctypes.byref(cal), int(n_cand), int(flags),
                                                     ctypes.byref(n)))
    return int(n.value)


def loss_batch_full(g_half: torch.Tensor, bf_geom: torch.Tensor, q_row: torch.Tensor,
                    q_col: torch.Tensor, cal: Calibration, candidates: torch.Tensor, *,
                    flags: int = 0, workspace: Workspace | None = None,
                    want_mean_phase: bool = False
                    ) -> tuple[torch.Tensor, torch.Tensor | None]:
    """Losses with the 14-term chi: ``candidates`` float32 CUDA [n, 28] holding
    14 magnitudes then 14 angles per row (``qssb_full_aberrations_t``)."""
    _require_cuda(g_half, "g_half", torch.complex64)
    _require_cuda(bf_geom, "bf_geom", torch.float32)
    _require_cuda(candidates, "candidates", torch.float32)
    if candidates.ndim != 2 or candidates.shape[1] != 2 * _lib.FULL_TERMS:
        raise ValueError("candidates must have shape (n, 28): 14 magnitudes, then 14 angles")
    if (tuple(g_half.shape) != (cal.n_bf, int(cal.scan_rows), int(cal.scan_cols) // 2 + 1)
            or tuple(bf_geom.shape) != (_lib.GEOM_ROWS, cal.n_bf)):
        raise ValueError("g_half / bf_geom shapes do not match the calibration")
    n = int(candidates.shape[0])
    r0, r1 = int(cal.scan_rows), int(cal.scan_cols)
    ws = workspace or Workspace(g_half.device)
    buf = ws.get(loss_full_workspace_bytes(cal, n, flags))
    losses = torch.empty(n, dtype=torch.float32, device=g_half.device)
    mp = (torch.empty((n, r0, r1), dtype=torch.float32, device=g_half.device)
          if want_mean_phase else None)
    _call("qssb_loss_batch_full", g_half.device, _ptr(g_half), _ptr(bf_geom), _ptr(q_row),
          _ptr(q_col), ctypes.byref(cal), _ptr(candidates), n, int(flags), _ptr(buf), buf.numel(),
          _ptr(losses), _ptr(mp), _stream(g_half))
    return losses, mp


_CANCEL: torch.Tensor | None = None


def set_cancel_flag(flag: torch.Tensor | None) -> None:
    """Register (or with None clear) the device int32 flag the table-driven
    loss kernel polls between BF-pixel pairs; nonzero stops a batch and its
    losses come back NaN. The tensor is kept referenced while registered."""
    global _CANCEL
    if flag is not None:
        _require_cuda(flag, "flag", torch.int32)
    _CANCEL = flag
    check(_lib.load().qssb_set_cancel(_ptr(flag)))


def overlap_table_bytes(cal: Calibration) -> int:
    """Bytes of the overlap table of a square 128, 256, 512 or 1024 scan."""
    nbytes = ctypes.c_size_t(0)
    check(_lib.load().qssb_overlap_table_bytes(ctypes.byref(cal), ctypes.byref(nbytes)))
    return int(nbytes.value)


def overlap_table(bf_geom: torch.Tensor, q_row: torch.Tensor, q_col: torch.Tensor,
                  cal: Calibration) -> torch.Tensor:
    """The candidate-independent overlap apertures of a square-scan dataset
    (float32 CUDA [n_bf, E, 2]) for ``loss_batch(..., overlap=...)``.

    E is 8383 at 128x128 (the pair kernel's retained-frequency order) and
    (N/2+1)*N + N/2 at N = 256, 512, 1024 (rows 0..N/2 of the scan-frequency
    plane, then the partner (N-r, N/2) of each row r)."""
    _require_cuda(bf_geom, "bf_geom", torch.float32)
    if tuple(bf_geom.shape) != (_lib.GEOM_ROWS, cal.n_bf):
        raise ValueError("bf_geom shape does not match the calibration")
    table = torch.empty(overlap_table_bytes(cal) // 4, dtype=torch.float32, device=bf_geom.device)
    _call("qssb_overlap_table", bf_geom.device, _ptr(bf_geom), _ptr(q_row), _ptr(q_col),
          ctypes.byref(cal), _ptr(table), _stream(bf_geom))
    return table.view(cal.n_bf, -1, 2)


def loss_batch(g_half: torch.Tensor, bf_geom: torch.Tensor, q_row: torch.Tensor,
               q_col: torch.Tensor, cal: Calibration, candidates: torch.Tensor, *,
               flags: int = 0, workspace: Workspace | None = None, want_mean_phase: bool = False,
               out: torch.Tensor | None = None, overlap: torch.Tensor | None = None
               ) -> tuple[torch.Tensor, torch.Tensor | None]:
    """Phase-variance losses for ``candidates`` (float32 CUDA [n, 4]: C10, C12, phi12, C30).

    ``overlap`` (from ``overlap_table``, square 128 .. 1024 scans) supplies
    the candidate-independent apertures: at 128x128 it selects the pair
    kernel (two BF pixels per inverse 2D FFT); at 256 .. 1024 the row pass
    of the quadratic-chi loss reads them instead of evaluating them."""
    _require_cuda(g_half, "g_half", torch.complex64)
    _require_cuda(bf_geom, "bf_geom", torch.float32)
    _require_cuda(candidates, "candidates", torch.float32)
    if candidates.ndim != 2 or candidates.shape[1] != 4:
        raise ValueError("candidates must have shape (n, 4): C10, C12, phi12, C30")
    if (tuple(g_half.shape) != (cal.n_bf, int(cal.scan_rows), int(cal.scan_cols) // 2 + 1)
            or tuple(bf_geom.shape) != (_lib.GEOM_ROWS, cal.n_bf)):
        raise ValueError("g_half / bf_geom shapes do not match the calibration")
    n = int(candidates.shape[0])
    r0, r1 = int(cal.scan_rows), int(cal.scan_cols)
    ws = workspace or Workspace(g_half.device)
    buf = ws.get(loss_workspace_bytes(cal, n, flags))
    if out is not None:
        _require_cuda(out, "out", torch.float32)
        if out.numel() != n:
            raise ValueError("out must hold one loss per candidate")
    losses = out if out is not None else torch.empty(n, dtype=torch.float32, device=g_half.device)
    mp = (torch.empty((n, r0, r1), dtype=torch.float32, device=g_half.device)
          if want_mean_phase else None)
    if overlap is None:
        _call("qssb_loss_batch", g_half.device, _ptr(g_half), _ptr(bf_geom), _ptr(q_row),
              _ptr(q_col), ctypes.byref(cal), _ptr(candidates), n, int(flags), _ptr(buf),
              buf.numel(), _ptr(losses), _ptr(mp), _stream(g_half))
    else:
        _require_cuda(overlap, "overlap", torch.float32)
        if overlap.shape[0] != cal.n_bf or overlap.numel() * 4 != overlap_table_bytes(cal):
            raise ValueError("overlap table does not match the calibration")
        _call("qssb_loss_batch_ex", g_half.device, _ptr(g_half), _ptr(bf_geom), _ptr(q_row),
              _ptr(q_col), ctypes.byref(cal), _ptr(candidates), n, int(flags), _ptr(overlap),
              _ptr(buf), buf.numel(), _ptr(losses), _ptr(mp), _stream(g_half))
    return losses, mp


def phase_atan2(y: torch.Tensor, x: torch.Tensor) -> torch.Tensor:
    """atan2(y, x) by the loss kernels' phase function (float32 CUDA tensors
    of one shape; |error| <= 4e-7 rad against IEEE atan2)."""
    _require_cuda(y, "y", torch.float32)
    _require_cuda(x, "x", torch.float32)
    if y.shape != x.shape:
        raise ValueError("y and x must have the same shape")
    y, x = y.contiguous(), x.contiguous()
    out = torch.empty_like(y)
    _call("qssb_phase_atan2", y.device, _ptr(y), _ptr(x), _ptr(out), y.numel(), _stream(y))
    return out


# ------------------------------------------------------------ time series
def fourier_shift(frames: torch.Tensor, shifts: torch.Tensor, out: torch.Tensor | None = None
                  ) -> torch.Tensor:
    """Fourier-ramp shift of every frame (complex64 CUDA [T, R, C], shifts
    float32 CUDA [T, 2] in pixels); R and C powers of two in 64..1024."""
    _require_cuda(frames, "frames", torch.complex64)
    _require_cuda(shifts, "shifts", torch.float32)
    if frames.ndim != 3 or tuple(shifts.shape) != (frames.shape[0], 2):
        raise ValueError("frames must be (T, R, C) and shifts (T, 2)")
    t, r, c = (int(x) for x in frames.shape)
    if out is None:
        out = torch.empty_like(frames)
    _call("qssb_fourier_shift", frames.device, _ptr(frames), _ptr(out), t, r, c, _ptr(shifts),
          _stream(frames))
    return out


def join_frames(frames: torch.Tensor, weights: torch.Tensor, *, phase_reference: int,
                write_back: bool, workspace: Workspace | None = None) -> torch.Tensor:
    """Weighted complex mean of frames (complex64 CUDA [T, ...]) with optional
    global-phase referencing to frame 0; weights float32 CUDA [T], summing to 1."""
    _require_cuda(frames, "frames", torch.complex64)
    _require_cuda(weights, "weights", torch.float32)
    t = int(frames.shape[0])
    n_pix = frames[0].numel()
    joined = torch.empty(frames.shape[1:], dtype=torch.complex64, device=frames.device)
    buf = None
    if phase_reference:
        n = ctypes.c_size_t(0)
        check(_lib.load().qssb_join_workspace_bytes(t, ctypes.byref(n)))
        buf = (workspace or Workspace(frames.device)).get(int(n.value))
    _call("qssb_join_object_waves", frames.device, _ptr(frames), _ptr(weights), t, n_pix,
          int(phase_reference), _ptr(buf), 0 if buf is None else buf.numel(), _ptr(joined),
          1 if write_back else 0, _stream(frames))
    return joined
