"""Repeated cold reconstructions of same-shaped scans through CUDA graphs.

A cold reconstruction (u16 counts in HBM -> exact frame sums -> BF selection
-> BF geometry -> gather -> scan FFT -> corrected Fourier sum -> inverse FFT
-> phase) launches about a dozen kernels; issuing them from Python costs more
than the first few kernels take on a B200. For a stream of acquisitions of
one shape and calibration (a detector feeding scans, a benchmark loop),
``ColdReconstructor`` records the launch sequence once as two CUDA graphs:

* stage A - memset + frame sums, ``qssb_select_bf``, ``qssb_bf_geometry`` and
  the 48-byte copy of the selection result to pinned host memory;
* stage B - ``qssb_gather_bf_columns_2d``, ``qssb_scan_fft_half`` and
  ``qssb_object_ex`` (dc read from the device selection result), one graph
  per BF count, with buffers sized for it.

With ``use_box`` (128x128 scans, detector columns and frame count multiples
of 8) the counts are read once: stage A first sums the first 512 frames and estimates
a superset box of the BF disk (``qssb_bf_box_estimate``), the frame-sum pass
writes the box's columns as it streams (``qssb_mean_dp_u64_box``), and after
the selection ``qssb_bf_box_map`` maps every BF pixel to its box column;
stage B then transforms straight from the box (``qssb_scan_fft_half_mapped``).
When a BF pixel falls outside the box (the map's ok flag, read with the
selection result) that run takes the gathering stage B instead, so results
never depend on the estimate. Off by default: on a B200 at 128^4 the sum
pass's scattered 16-byte box-column stores (107 MB) add ~50 us, more than the
gather (~60 us) they replace saves once the sample sums, the estimate and the
map are counted (0.374 against 0.330 ms per reconstruction).

With ``tune`` (the default) the first run of a BF count asks the autotuner
for the gather's tile shape, the scan FFT's launch shape and the object's
work partition and trotter tile (timed on the real inputs, then cached), and
stage B is recorded with them.

Every ``run`` recomputes everything from the counts in the input buffer; only
allocation and launch overhead are shared. The one host sync reads the BF
count between the stages (the buffers of stage B depend on it).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import autotune, ops
from ._lib import Aberrations, Calibration
from .backend import _device_frequencies
from .calibration import scan_frequencies  # noqa: F401  (re-exported for callers)
from .physics import electron_wavelength_angstrom


class ColdReconstructor:
    """Cold u16 -> phase reconstructions of one scan shape, graph-launched."""

    def __init__(self, counts: torch.Tensor, *, semiangle: float, scan_sampling: float,
                 det_sampling: float, voltage_kV: float, bf_intensity_threshold: float = 0.0,
                 bf_radius: float | None = None, rotation_angle_deg: float = 0.0,
                 aberrations: tuple = (0.0, 0.0, 0.0, 0.0), use_graphs: bool = True,
                 use_box: bool = False, tune: bool = True):
        if counts.ndim != 4 or counts.dtype != torch.uint16 or not counts.is_cuda:
            raise ValueError("counts must be a CUDA uint16 tensor [R0, R1, K0, K1]")
        r0, r1, k0, k1 = (int(x) for x in counts.shape)
        if r0 != r1 or r0 not in (128, 256, 512, 1024):
            raise NotImplementedError("ColdReconstructor takes native 128^2 .. 1024^2 scans")
        self.device = counts.device
        self.counts = counts  # the input buffer: load() copies new data into it
        self.scan_shape = (r0, r1)
        self.det_shape = (k0, k1)
        self.n_frames = r0 * r1
        self.wavelength = electron_wavelength_angstrom(voltage_kV * 1e3)
        self.semiangle = float(semiangle)
        self.scan_sampling = (float(scan_sampling), float(scan_sampling))
        self.ang = (float(det_sampling), float(det_sampling))
        self.threshold = float(bf_intensity_threshold)
        self.bf_radius = bf_radius
        self.rotation = math.radians(rotation_angle_deg)
        recip = self.ang[0] * 1e-3 / self.wavelength
        self.k_step = (recip, recip)
        self.ab = Aberrations(*(float(a) for a in aberrations))
        self.use_graphs = bool(use_graphs)
        self.tune = bool(tune)
        self.q_row, self.q_col = _device_frequencies(self.scan_shape, self.scan_sampling, self.device)
        self.info_host = torch.empty(ops.BF_INFO_BYTES, dtype=torch.uint8, pin_memory=True)
        # the box path: BF columns written by the frame-sum pass
        self.use_box = (use_box and r0 == 128 and k1 % 8 == 0 and self.n_frames % 8 == 0
                        and counts.data_ptr() % 16 == 0)
        if self.use_box:
            self.box_capacity = max(1, (k0 * k1) // 2)
            self.box_cols = torch.empty((self.box_capacity, self.n_frames), dtype=torch.uint16,
                                        device=self.device)
            self.box = torch.empty(ops.BOX_WORDS, dtype=torch.int32, device=self.device)
            self.box_map = (torch.empty(self.box_capacity, dtype=torch.int32, device=self.device),
                            torch.empty(1, dtype=torch.int32, device=self.device))
            self.ok_host = torch.zeros(1, dtype=torch.int32, pin_memory=True)
        self.box_runs = 0  # runs that used the box columns
        self._graph_a = None
        self._b: dict[int, dict] = {}
        self.last_info = None

    def load(self, data) -> None:
        """Copy a new acquisition (host or device, same shape) into the input buffer."""
        src = torch.as_tensor(data)
        if tuple(src.shape) != tuple(self.counts.shape):
            raise ValueError("new data must have the reconstructor's shape")
        self.counts.copy_(src.view(torch.uint16) if src.dtype == torch.int16 else src,
                          non_blocking=True)

    # ------------------------------------------------------------ stage A
    SAMPLE_FRAMES = 512  # frames whose sums place the box

    def _stage_a(self) -> None:
        if self.use_box:
            frames = self.counts.view(-1, *self.det_shape)
            sample, _ = ops.mean_dp_u64(frames[: min(self.SAMPLE_FRAMES, self.n_frames)],
                                        want_mean=False)
            ops.bf_box_estimate(sample, self.det_shape, self.box_capacity,
                                radius_px=float(self.bf_radius or 0.0), out=self.box)
            sums = ops.mean_dp_u64_box(self.counts, self.box, self.box_cols)
        else:
            sums, _ = ops.mean_dp_u64(self.counts, want_mean=False)
        sel = ops.select_bf(sums, self.det_shape, self.n_frames, self.threshold, self.bf_radius)
        geom = ops.bf_geometry(sel, self.det_shape, self.k_step, self.rotation, self.wavelength,
                               self.semiangle * 1e-3, (self.ang[0] * 1e-3, self.ang[1] * 1e-3))
        if self.use_box:
            ops.bf_box_map(sel, self.det_shape, self.box, self.box_capacity, out=self.box_map)
            self.ok_host.copy_(self.box_map[1], non_blocking=True)
        self.info_host.copy_(sel.info, non_blocking=True)
        self._a = (sums, sel, geom)

    def _calibration(self, n_bf: int) -> Calibration:
        return Calibration(
            n_bf=n_bf, scan_rows=self.scan_shape[0], scan_cols=self.scan_shape[1], reserved=0,
            wavelength_A=self.wavelength, semiangle_rad=self.semiangle * 1e-3,
            det_sampling_row_rad=self.ang[0] * 1e-3, det_sampling_col_rad=self.ang[1] * 1e-3,
            scan_sampling_row_A=self.scan_sampling[0], scan_sampling_col_A=self.scan_sampling[1],
            dc_re=0.0, dc_im=0.0)

    # ------------------------------------------------------------ stage B
    def _make_b(self, n_bf: int, mapped: bool = False) -> dict:
        _, sel, geom_buf = self._a
        lin = sel.bf_linear[:n_bf]
        geom = geom_buf[: 8 * n_bf].view(8, n_bf)
        dc_dev = sel.info[32:48].view(torch.float64)  # qssb_bf_info_t.dc_re, dc_im
        r0, r1 = self.scan_shape
        st = {"cal": self._calibration(n_bf), "ws": ops.Workspace(self.device),
              "obj": torch.empty((r0, r1), dtype=torch.complex64, device=self.device),
              "phase": torch.empty((r0, r1), dtype=torch.float32, device=self.device),
              "gather_variant": 0, "fft_variant": 0, "obj_flags": 0}
        if self.tune:
            # the autotuner's shapes for this detector, scan and BF count
            # (cached after the first search; timed on these very inputs)
            if mapped:
                g = ops.scan_fft_half_mapped(self.box_cols, self.box_map[0], n_bf, self.scan_shape)
            else:
                st["gather_variant"] = autotune.tune_gather(self.counts, lin)
                columns = ops.gather_bf_columns(self.counts, lin, validate=False,
                                                variant=st["gather_variant"])
                st["fft_variant"] = autotune.tune_scan_fft(columns, self.scan_shape)
                g = ops.scan_fft_half(columns, self.scan_shape, variant=st["fft_variant"])
                del columns
            st["obj_flags"] = autotune.tune_object(g, geom, self.q_row, self.q_col, st["cal"],
                                                   self.ab, 0, st["ws"])
            del g
        st["ws"].get(ops.object_workspace_bytes(st["cal"], st["obj_flags"]))

        def launch():
            if mapped:
                columns = None
                g = ops.scan_fft_half_mapped(self.box_cols, self.box_map[0], n_bf, self.scan_shape)
            else:
                columns = ops.gather_bf_columns(self.counts, lin, validate=False,
                                                variant=st["gather_variant"])
                g = ops.scan_fft_half(columns, self.scan_shape, variant=st["fft_variant"])
            ops.object_wave(g, geom, self.q_row, self.q_col, st["cal"], self.ab,
                            flags=st["obj_flags"], workspace=st["ws"], dc_device=dc_dev,
                            out=(st["obj"], st["phase"]))
            st["keep"] = (columns, g)

        st["launch"] = launch
        if self.use_graphs:
            launch()  # warm-up outside capture: attributes, allocations
            torch.cuda.synchronize(self.device)
            g = torch.cuda.CUDAGraph()
            before = ops.LAUNCH_COUNT
            with torch.cuda.graph(g, capture_error_mode="relaxed"):
                launch()
            st["launches"] = ops.LAUNCH_COUNT - before
            ops.LAUNCH_COUNT = before  # capture launched nothing; replays are counted
            st["graph"] = g
        return st

    def run(self) -> torch.Tensor:
        """One cold reconstruction of the current input buffer; returns the phase
        (float32 [R0, R1], on the device, valid until the next run)."""
        if self.use_graphs:
            if self._graph_a is None:
                self._stage_a()  # warm-up outside capture
                torch.cuda.synchronize(self.device)
                g = torch.cuda.CUDAGraph()
                before = ops.LAUNCH_COUNT
                with torch.cuda.graph(g, capture_error_mode="relaxed"):
                    self._stage_a()
                self._launches_a = ops.LAUNCH_COUNT - before
                ops.LAUNCH_COUNT = before
                self._graph_a = g
            self._graph_a.replay()
            ops.LAUNCH_COUNT += self._launches_a
        else:
            self._stage_a()
        torch.cuda.current_stream(self.device).synchronize()
        info = ops._lib.BFInfo.from_buffer_copy(self.info_host.numpy().tobytes())
        self.last_info = info
        if info.n_bf <= 0:
            raise ValueError("No bright-field pixels selected.")
        mapped = bool(self.use_box and int(self.ok_host[0]) == 1)
        self.box_runs += int(mapped)
        key = (int(info.n_bf), mapped)
        st = self._b.get(key)
        if st is None:
            st = self._make_b(int(info.n_bf), mapped)
            self._b[key] = st
        if self.use_graphs:
            st["graph"].replay()
            ops.LAUNCH_COUNT += st["launches"]
        else:
            st["launch"]()
        return st["phase"]
