"""SSB recon/s at 128^4 u16 on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload: plain SSB at production size - scan 128x128, detector 128x128,
uint16 (537 MB), ~1784 bright-field pixels, synthetic weak-phase data
(seeded; the reference's own benchmarks use private acquisitions). One step
is one cold reconstruction: u16 counts resident in HBM -> u64 mean DP -> BF
selection -> BF geometry -> BF gather -> Hermitian scan FFT -> corrected
Fourier sum -> inverse FFT -> float32 object phase, all recomputed each step
by ``ColdReconstructor`` (the C-ABI launch sequence replayed as two CUDA
graphs, one host sync for the BF count); ``cold_backend_recon_per_s`` is the
same through a new ``B200SSBBackend`` per step. Inputs (537 MB per step) are
larger than the 126 MB L2.

``--impl reference`` times the reference's CPU path for the same workload:
the reference has no CPU SSB implementation, so this is the CPU torch
restatement of its executable specification (docs/kernels/ssb.md) from
``oracle/ssb_torch_spec.py``, run with every host thread, rank 0 only.

Multi-GPU: replicas (each rank reconstructs its own scan; no collective on the
data path), ``scaling: weak``, time = max over ranks.
"""
from __future__ import annotations

import argparse
import gc
import json
import math
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np
import torch

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "SSB recon/s at 128^4 u16"
UNIT = "recon/s"
SPEC_NAME = "plain_128x128_det128"
KW = dict(semiangle=20.0, scan_sampling=0.5, det_sampling=20.0 / 24.0, voltage_kV=300)
WORKLOAD = ("plain SSB, scan 128x128 x detector 128x128 uint16 (537 MB), ~1784 BF pixels, "
            "cold u16->object phase per step")


def _config(n_bf: int, world: int) -> dict:
    """The workload dict both arms print (identical keys and values)."""
    return {"workload": WORKLOAD, "n_bf": int(n_bf), "scan": [128, 128], "detector": [128, 128],
            "l2": "inputs larger than L2 (537 MB u16 per step)", "parallelism": f"replicas x{world}"}


def _sig(x, digits: int = 4):
    """Round floats (recursively) to a few significant digits for the summary."""
    if isinstance(x, float):
        return float(f"{x:.{digits}g}")
    if isinstance(x, dict):
        return {k: _sig(v, digits) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [_sig(v, digits) for v in x]
    return x


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return world, rank, local


def _barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def _max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """SM clock, power and throttle reasons sampled during the timed region.

    Polls NVML from a background thread every ~2 ms (the timed region of a
    short run lasts only tens of milliseconds). Without NVML (pynvml missing
    or failing) no clock record is produced. Reads settings only.
    """

    REASONS = {  # NVML clocks-event-reason bits
        "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
        "sw_power_cap": 0x4,
    }

    def __init__(self, index: int):
        self.index = index
        self.samples: list[tuple[float, int]] = []
        self.max_mhz = None
        self._stop = None
        self._thread = None

    def start(self):
        import threading

        try:
            import pynvml

            pynvml.nvmlInit()
            handle = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(handle, pynvml.NVML_CLOCK_SM))
        except Exception:  # noqa: BLE001 - NVML missing: no clock record
            return
        self._stop = threading.Event()

        def poll():
            while not self._stop.is_set():
                try:
                    mhz = pynvml.nvmlDeviceGetClockInfo(handle, pynvml.NVML_CLOCK_SM)
                    reasons = pynvml.nvmlDeviceGetCurrentClocksEventReasons(handle)
                    self.samples.append((float(mhz), int(reasons)))
                except Exception:  # noqa: BLE001
                    pass
                time.sleep(0.002)

        self._thread = threading.Thread(target=poll, daemon=True)
        self._thread.start()

    def stop(self) -> dict | None:
        if self._thread is None:
            return None
        self._stop.set()
        self._thread.join(timeout=2)
        if not self.samples:
            return None
        seen = sorted({name for _, bits in self.samples for name, b in self.REASONS.items() if bits & b})
        return {"sm_mhz": float(np.median([m for m, _ in self.samples])), "sm_max_mhz": self.max_mhz,
                "reasons": seen, "samples": len(self.samples), "source": "nvml"}


def _peaks() -> tuple[float, str]:
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic(kernel: str) -> float | None:
    p = REPO / "profiles" / "traffic.json"
    if p.exists():
        v = json.loads(p.read_text()).get(kernel)
        return None if v is None else float(v)
    return None


def cpu_baseline(counts_host: np.ndarray, budget_s: float = 15.0) -> dict:
    """Reference-spec CPU recon on the host cores, bounded to ~budget_s."""
    from oracle import ssb_torch_spec as spec

    kw = dict(voltage_kV=300, semiangle_mrad=KW["semiangle"], scan_sampling=KW["scan_sampling"],
              det_sampling=KW["det_sampling"])
    spec.reconstruct(counts_host, bf_stride=8, **kw)  # warm-up (allocator, threads)
    t0 = time.perf_counter()
    n = 0
    while True:
        spec.reconstruct(counts_host, **kw)
        n += 1
        if time.perf_counter() - t0 > budget_s or n >= 20:
            break
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": UNIT, "cores": spec.host_threads(), "kind": "port",
            "sample": f"{n} full 128^4 reconstructions (all BF pixels) of the same workload"}


def reference_cuda_baseline(counts: torch.Tensor, be, steps: int, warmup: int) -> dict:
    """The reference's own 128x128 object kernels (built from its CUDA sources
    into oracle/_ref/) timed on this GPU beside ours: warm object redraws from
    the same resident G, and cold reconstructions with its G construction
    replayed through torch's gather/cuFFT (its CuPy steps)."""
    from oracle.ref_cuda import build_ref

    if not build_ref.available():
        return {"unavailable": "oracle/_ref/ssb_fft128.cubin not built (needs the reference tree)"}
    from oracle.ref_cuda.harness import ReferenceObject128, reference_cold_object

    dev = counts.device
    stream = torch.cuda.current_stream(dev)
    ref = ReferenceObject128(dev)
    semi = KW["semiangle"] * 1e-3
    ang = KW["det_sampling"] * 1e-3
    wargs = (be.G_qk, be._geom_dev, be._q_row, be._q_col, be.wavelength, semi, ang, ang)

    def timed(fn, n):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize(dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(n):
            fn()
        e.record(stream)
        torch.cuda.synchronize(dev)
        return s.elapsed_time(e) / n

    warm_ms = timed(lambda: torch.angle(ref.object(*wargs, 10.0, 5.0, 0.1, be.dc_value)), steps)
    cold = dict(wavelength=be.wavelength, semiangle_mrad=KW["semiangle"],
                det_sampling_mrad=KW["det_sampling"], scan_sampling_A=KW["scan_sampling"],
                C10=0.0, C12=0.0, phi12=0.0)
    cold_ms = timed(lambda: reference_cold_object(counts, ref, **cold), max(3, steps // 4))
    ref_obj = ref.object(*wargs, 0.0, 0.0, 0.0, be.dc_value)
    our_obj, _ = be.object_and_phase(0.0, 0.0, 0.0)
    d = torch.angle(our_obj * torch.conj(ref_obj)).double()
    del ref
    loss = {}
    if build_ref.sums_available():
        # the reference's batched loss (variance_loss_batch: K12 + K13 over
        # 1024-pixel BF chunks, K14) on the same G, 64 candidates like ours
        from oracle.ref_cuda.harness import ReferenceLossBatch128

        rl = ReferenceLossBatch128(dev)
        c10 = np.linspace(-50.0, 50.0, 64)
        lfn = lambda: rl.losses(be.G_qk, be._geom_dev, be._q_row, be._q_col,  # noqa: E731
                                be.wavelength, semi, ang, ang, c10, 0.0, 0.0, be.dc_value)
        loss_ms = timed(lfn, 3)
        ours = be.variance_loss_batch(c10, 0.0, 0.0).double()
        rel = ((lfn().double() - ours).abs() / ours.abs()).max()
        loss = {"loss_evals_per_s": 64 * 1e3 / loss_ms, "loss_batch64_ms": loss_ms,
                "loss_max_rel_diff_vs_ours": float(rel)}
        del rl
        torch.cuda.empty_cache()
    return {
        **loss,
        "warm_recon_per_s": 1e3 / warm_ms, "cold_recon_per_s": 1e3 / cold_ms,
        "phase_rms_rad_vs_ours": float(torch.sqrt(torch.mean(d * d))),
        "kind": "reference CUDA kernels ifft128_rows_fused_pk_t32_mr8_packed + ifft128_cols_t32_mr8 "
                "(its sources, its nvrtc options, sm_100a; oracle/_ref) with its gather/cuFFT/mean "
                "steps as torch library calls",
    }


def stress_256(dev: torch.device, steps: int) -> dict:
    """Precision and scale stress: 256^2 scan x 128^2 detector u16 (2.1 GB),
    defocus 20 nm (C10 = 200 A), doses 50 / 1000 / 20000 e per position. Per
    dose: the float32 path (FP32 FFTs, Kahan trotter sum) against the FP64 GPU
    restatement of the oracle at the true aberrations (phase RMS), and the cold
    recon time at 256^2."""
    from dataclasses import replace

    from oracle import ssb_oracle as so
    from oracle import ssb_torch_fp64 as tf
    from quantem.gpu_b200 import B200SSBBackend
    from quantem.gpu_b200.synthetic import CONFIGS, generate

    base = CONFIGS["stress_256x256_det128"]
    out = {"workload": "scan 256x256 x detector 128x128 uint16 (2.1 GB), C10 = 200 A",
           "doses": {}}
    stream = torch.cuda.current_stream(dev)
    for dose in (50.0, 1000.0, 20000.0):
        spec = replace(base, dose=dose)
        counts = generate(spec, dev).counts.contiguous()
        kw = dict(semiangle=spec.semiangle_mrad, scan_sampling=spec.scan_step_A,
                  det_sampling=spec.det_sampling_mrad, voltage_kV=spec.voltage_kV)

        def cold():
            be = B200SSBBackend(counts, device=dev, **kw)
            return be, be.object_and_phase(spec.C10, 0.0, 0.0)[1]

        for _ in range(2):
            be, ph = cold()
        torch.cuda.synchronize(dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(steps):
            be, ph = cold()
        e.record(stream)
        torch.cuda.synchronize(dev)
        prep = tf.prepare(counts, voltage_kV=spec.voltage_kV, semiangle_mrad=spec.semiangle_mrad,
                          scan_sampling=spec.scan_step_A, det_sampling=spec.det_sampling_mrad)
        _, ref = tf.reconstruct(prep, so.Aberrations(spec.C10, 0.0, 0.0))
        err = so.wrapped_phase_error(ph.cpu().numpy(), ref.cpu().numpy())
        out["doses"][str(int(dose))] = {
            "phase_rms_rad_vs_fp64_gpu": float(np.sqrt(np.mean(err ** 2))),
            "phase_max_rad_vs_fp64_gpu": float(np.abs(err).max()),
            "cold_recon_per_s": 1e3 * steps / s.elapsed_time(e), "n_bf": be.num_bf}
        del counts, be, prep
        torch.cuda.empty_cache()
    return out


def large_512(dev: torch.device, steps: int = 5) -> dict:
    """The reference's 512^2 timing shape: 512 x 512 scan x 192 x 192 detector
    u16 (19.3 GB on the device), ~8.9k BF pixels, synthetic. Cold u16 -> phase
    through the graph pipeline; the backend's G construction; then, from the
    resident G, the warm complex object, the exact mean phase, and phase +
    loss - the three figures the reference publishes for this shape."""
    from quantem.gpu_b200 import B200SSBBackend
    from quantem.gpu_b200.pipeline import ColdReconstructor
    from quantem.gpu_b200.synthetic import CONFIGS, generate

    spec = CONFIGS["large_512x512_det192"]
    t0 = time.perf_counter()
    counts = generate(spec, dev).counts
    torch.cuda.synchronize(dev)
    gen_s = time.perf_counter() - t0
    kw = dict(semiangle=spec.semiangle_mrad, scan_sampling=spec.scan_step_A,
              det_sampling=spec.det_sampling_mrad, voltage_kV=spec.voltage_kV)
    stream = torch.cuda.current_stream(dev)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, n):
        fn()
        torch.cuda.synchronize(dev)
        s.record(stream)
        for _ in range(n):
            fn()
        e.record(stream)
        torch.cuda.synchronize(dev)
        return s.elapsed_time(e) / n

    rec = ColdReconstructor(counts, **kw)
    cold_ms = timed(rec.run, steps)
    n_bf = rec.last_info.n_bf
    del rec
    torch.cuda.empty_cache()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    be = B200SSBBackend(counts, device=dev, **kw)
    torch.cuda.synchronize(dev)
    construct_s = time.perf_counter() - t0
    obj_ms = timed(lambda: be.reconstruct_object(spec.C10, 0.0, 0.0), steps)
    phase_ms = timed(lambda: be.reconstruct(spec.C10, 0.0, 0.0), max(2, steps // 2))
    loss_ms = timed(lambda: be.reconstruct_with_loss(spec.C10, 0.0, 0.0), max(2, steps // 2))
    out = {
        "workload": "scan 512x512 x detector 192x192 uint16 (19.3 GB), synthetic, C10 = 100 A",
        "n_bf": n_bf, "generate_s": gen_s,
        "cold_u16_to_phase_ms": cold_ms,
        "backend_construct_s": construct_s,
        "warm_complex_object_ms": obj_ms,
        "exact_mean_phase_ms": phase_ms,
        "exact_phase_plus_loss_ms": loss_ms,
        "reference_published_ms": {
            "gpu": "RTX PRO 6000 Blackwell Max-Q, real data with 8928 BF",
            "complex_object": 13.883, "exact_phase": 32.035, "exact_phase_plus_loss": 32.335,
            "g_construction_s": 0.27},
    }
    del be, counts
    torch.cuda.empty_cache()
    return out


def temporal_join(dev: torch.device, steps: int = 10) -> dict:
    """Time-series join (temporal.py's join_object_waves): T complex64 object
    waves of N^2, subpixel drift correction by a Fourier ramp, phase reference
    to frame 0, weighted mean; device-resident stack. Algorithmic bytes per
    frame: three read+write passes of the shift (48 B/pixel) and the join's
    overlap and mean reads (16 B/pixel) plus the aligned write-back (8 B)."""
    from oracle import temporal_oracle as to
    from quantem.gpu_b200.temporal import join_object_waves

    out = {"workload": "complex64 object-wave stacks, random subpixel drifts, phase reference "
                       "'first', weighted mean, aligned stack returned"}
    stream = torch.cuda.current_stream(dev)
    rng = np.random.default_rng(11)
    for n, t in ((128, 256), (512, 64)):
        g = torch.Generator(device=dev).manual_seed(n)
        stack = torch.polar(1.0 + 0.05 * torch.randn((t, n, n), generator=g, device=dev),
                            0.2 * torch.randn((t, n, n), generator=g, device=dev)).to(torch.complex64)
        shifts = torch.as_tensor(rng.uniform(-4, 4, (t, 2)), dtype=torch.float32, device=dev)
        weights = torch.as_tensor(rng.uniform(0.5, 1.0, t), dtype=torch.float32, device=dev)
        fn = lambda: join_object_waves(stack, shifts=shifts, weights=weights,  # noqa: E731
                                       phase_reference="first", return_aligned_stack=True)
        fn()
        torch.cuda.synchronize(dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(steps):
            fn()
        e.record(stream)
        torch.cuda.synchronize(dev)
        ms = s.elapsed_time(e) / steps
        alg = 72.0 * n * n * t
        # CPU: the FP64 oracle on 4 frames, scaled per frame (one host thread for numpy's FFT)
        host = stack[:4].cpu().numpy()
        t0 = time.perf_counter()
        to.join_object_waves(host, shifts[:4].cpu().numpy(), weights[:4].cpu().numpy(), "first")
        cpu_fps = 4 / (time.perf_counter() - t0)
        out[f"{n}x{n}_T{t}"] = {"ms": ms, "frames_per_s": t * 1e3 / ms,
                                "alg_gbs": alg / ms / 1e6, "cpu_oracle_frames_per_s": cpu_fps}
        del stack
    return out


def bslz4_decode(dev: torch.device, steps: int = 10) -> dict:
    """The acquisition decode before the SSB path: the 128^4 synthetic counts
    as HDF5 bitshuffle+LZ4 chunks (one 32 KB frame each, 16384 chunks, written
    by qssb_encode_bslz4_u16) decoded into the u16 device tensor; beside it
    the reference's own reader kernels on the same bytes (oracle/_ref) and the
    pure-Python format oracle on a sample of frames (one host thread)."""
    from oracle import bslz4_oracle as bo
    from quantem.gpu_b200.decode import decode_bslz4, encode_bslz4
    from quantem.gpu_b200.synthetic import CONFIGS, generate

    counts = generate(CONFIGS[SPEC_NAME], device=dev).counts.reshape(-1, 128, 128)
    packed, offsets = encode_bslz4(counts)
    out_bytes = counts.numel() * 2
    stream = torch.cuda.current_stream(dev)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    decode_bslz4(packed, offsets, (128, 128))
    torch.cuda.synchronize(dev)
    s.record(stream)
    for _ in range(steps):
        decode_bslz4(packed, offsets, (128, 128), check=False)
    e.record(stream)
    torch.cuda.synchronize(dev)
    ms = s.elapsed_time(e) / steps
    res = {"workload": "128^4 synthetic u16 counts as 16384 bitshuffle+LZ4 chunks of 32 KB",
           "compressed_mb": packed.numel() / 1e6, "decoded_mb": out_bytes / 1e6,
           "ratio": out_bytes / packed.numel(), "decode_ms": ms,
           "decoded_gbs": out_bytes / ms / 1e6,
           "compressed_gbs": packed.numel() / ms / 1e6}
    try:
        from oracle.ref_cuda.bslz4 import ReferenceBslz4

        ref = ReferenceBslz4(dev)
        # the reference reader walks block starts on the host first (not timed);
        # its two kernels are timed like ours
        run, got = ref.prepare_decode(packed, offsets, (128, 128))
        run()
        torch.cuda.synchronize(dev)
        s.record(stream)
        for _ in range(steps):
            run()
        e.record(stream)
        torch.cuda.synchronize(dev)
        res["reference_decode_ms"] = s.elapsed_time(e) / steps
        res["speedup_vs_reference_kernels"] = res["reference_decode_ms"] / ms
        res["reference_matches"] = bool(torch.equal(got.view(torch.int16), counts.view(torch.int16)))
    except Exception as exc:  # noqa: BLE001 - the checker is optional on this leg
        res["reference"] = f"unavailable: {exc}"
    host = packed[: int(offsets[8])].cpu().numpy().tobytes()
    offs = list(offsets[:8].cpu().numpy()) + [len(host)]
    t0 = time.perf_counter()
    for i in range(8):
        bo.decode_chunk(host[offs[i]:offs[i + 1]])
    res["cpu_oracle_frames_per_s"] = 8 / (time.perf_counter() - t0)
    res["frames_per_s"] = counts.shape[0] * 1e3 / ms
    return res


def sweep_3scans(dev: torch.device, steps: int) -> dict:
    """Batched aberration sweep: scans of 96^2, 128^2 and 160x120 positions
    (128^2 detector, padded by the reference's rule to 128^2, 128^2, 256^2),
    64 candidates each with C1, A1 and C3, all three scored in one CUDA-graph
    launch with autotuned loss partitions (the 256^2 scan's passes in one
    persistent launch; the launch sequence measured beside it)."""
    from quantem.gpu_b200 import B200SSBBackend
    from quantem.gpu_b200.sweep import MultiScanSweep
    from quantem.gpu_b200.synthetic import draw_aberrations, generate, sweep_specs

    specs = sweep_specs()
    backends = []
    for spec in specs:
        counts = generate(spec, dev).counts
        backends.append(B200SSBBackend(counts, semiangle=spec.semiangle_mrad,
                                       scan_sampling=spec.scan_step_A,
                                       det_sampling=spec.det_sampling_mrad,
                                       voltage_kV=spec.voltage_kV, device=dev))
        del counts
    rng = np.random.default_rng(5)
    cands = [draw_aberrations(rng, 64) for _ in specs]
    for i, spec in enumerate(specs):
        cands[i][17] = (spec.C10, spec.C12, spec.phi12, spec.C30)
    sw = MultiScanSweep(backends, 64)
    losses = sw(cands)
    stream = torch.cuda.current_stream(dev)

    def timed(fn):
        fn()
        torch.cuda.synchronize(dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(steps):
            fn()
        e.record(stream)
        torch.cuda.synchronize(dev)
        return s.elapsed_time(e) / steps

    graph_ms = timed(sw.replay)
    direct_ms = timed(sw._launch_all)
    # the same sweep with the 256^2 scan's row and column launches per BF chunk
    sws = MultiScanSweep(backends, 64, persistent=False)
    ls = sws(cands)
    sequence_ms = timed(sws.replay)
    n = sum(c.shape[0] for c in cands)
    return {
        "workload": "scans 96x96, 128x128, 160x120 (padded to 128, 128, 256) x 128^2 detector, "
                    "64 candidates each (C1 in +-50 nm, |A1| <= 10 nm, C3 <= 1 um)",
        "n_bf": [be.num_bf for be in backends],
        "graph_launch_ms": graph_ms, "evals_per_s_graph": n * 1e3 / graph_ms,
        "evals_per_s_direct": n * 1e3 / direct_ms,
        "kernel_launches_per_graph": sw.launches_per_replay,
        "launch_sequence": {"evals_per_s_graph": n * 1e3 / sequence_ms,
                            "kernel_launches_per_graph": sws.launches_per_replay,
                            "max_rel_diff_vs_persistent": float(max(
                                np.max(np.abs(a - b) / np.abs(b)) for a, b in zip(ls, losses)))},
        "autotuned_chunks_per_candidate": [s["chunks"] for s in sw._slots],
        "truth_ranked_first": [bool(int(np.argmin(l)) == 17) for l in losses],
    }


def learned_fits(dev: torch.device, n_cases: int = 16) -> dict:
    """Learned proposal + 8-candidate refinement vs the plain 64-candidate sweep.

    The proposer is trained here (50k forward-model samples of the 64^2 x 64^2
    lattice, 40 epochs, after a one-epoch warm-up on a throwaway model) with
    the library's own kernels (its large GEMMs on the tcgen05 tensor cores,
    each step replayed as one CUDA graph); train_s includes synthesising the
    samples. Each case is a fully simulated 64^2-scan x
    64^2-detector dataset (padded to 128^2 by the reference rule) with
    aberrations drawn from the sweep ranges at 1e6 e per position:
    ``n_cases`` weak-phase objects (0.03 rad atoms) and ``n_cases // 2`` of
    the configs' 0.3 rad objects. SSB evaluations (candidates scored) are
    counted until the current best estimate's phase is within tau rad RMS
    (1e-4 on the weak-phase objects, 1e-3 on the 0.3 rad ones, whose phase
    moves ten times as much per A of aberration, finer than the float32
    loss resolves at 1e-4) of an FP64-oracle phase:
      * ``..._vs_loss_optimum_...``: the FP64 phase at the loss optimum (the
        minimiser's goal, refined from the truth), which both searches
        converge to, so this measures the search alone;
      * ``..._vs_truth_...``: the FP64 phase at the true aberrations. The loss
        optimum lies 1e-5 .. 1.6e-4 rad from it on the weak-phase objects and
        1e-4 .. 1.6e-3 rad on the 0.3 rad ones (the phase-variance objective,
        not the search, sets that floor; listed per case); a case whose floor
        exceeds tau is reached only by passing through on the way, so it is
        counted, not compared.
    plain = a 64-candidate zoom sweep over the whole range (at most 200
    rounds); learned = the proposal's eight hypotheses (four heads, two
    signs), then ``proposer.learned_refine`` (8 per round; the plain sweep as
    its fallback, evaluations added). Fits/s time the same searches with the
    oracle checks' own time taken out."""
    from oracle import ssb_oracle as so
    from oracle import ssb_torch_fp64 as tf
    from quantem.gpu_b200 import B200SSBBackend
    from quantem.gpu_b200 import proposer as pr
    from quantem.gpu_b200.synthetic import SyntheticSpec, draw_aberrations, generate

    # warm-up (module loading, first launches, graph capture) on a throwaway model
    pr.Proposer(dev, seed=99).train(n_samples=2048, epochs=1)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    prop = pr.Proposer(dev, seed=0)
    info = prop.train(n_samples=50_000, epochs=40)
    torch.cuda.synchronize(dev)
    train_s = time.perf_counter() - t0
    # FLOPs of a training step at batch 256: forward 2 m n k per layer, backward
    # the weight gradients of every layer and the input gradients of layers 2-4
    dims = [pr.N_IN, pr.HIDDEN, pr.HIDDEN, pr.HIDDEN, pr.N_OUT_PAD]
    fwd = sum(2 * 256 * dims[i] * dims[i + 1] for i in range(4))
    bwd = fwd + sum(2 * 256 * dims[i] * dims[i + 1] for i in range(1, 4))
    steps = info["epochs"] * (50_000 // 256)
    val = prop.validate(2048)
    rng = np.random.default_rng(77)
    w0 = np.array([120.0, 40.0, 40.0, 5000.0])
    rows = []
    cases = [(i, 0.03, "weak") for i in range(n_cases)] + \
            [(i, 0.3, "0.3rad") for i in range(n_cases // 2)]
    for i, peak, obj in cases:
        ab = draw_aberrations(rng, 1)[0]
        spec = SyntheticSpec(scan_shape=(64, 64), detector_shape=(64, 64),
                             det_sampling_mrad=20.0 / 12.0, dose=1e6, C10=float(ab[0]),
                             C12=float(ab[1]), phi12=float(ab[2]), C30=float(ab[3]),
                             atom_peak_rad=peak, seed=100 + i)
        counts = generate(spec, dev).counts
        be = B200SSBBackend(counts, semiangle=20.0, scan_sampling=0.5, det_sampling=20.0 / 12.0,
                            voltage_kV=300, device=dev)
        padded = torch.as_tensor(so.pad_or_crop_scan(counts.cpu().numpy()), device=dev)
        prep = tf.prepare(padded, voltage_kV=300, semiangle_mrad=20.0, scan_sampling=0.5,
                          det_sampling=20.0 / 12.0)
        truth = tf.reconstruct(prep, so.Aberrations(*map(float, ab)))[1].cpu().numpy()
        # the objective's own optimum, refined from the truth, and its FP64 phase
        x_opt, _, _ = pr.surrogate_search(be, pr.to_x(ab[None]), w0 / 16, 8, 300,
                                          np.random.default_rng(5), min_radius=1e-7)
        at_opt = tf.reconstruct(prep, so.Aberrations(*map(float, x_opt)))[1].cpu().numpy()
        del padded, prep
        check_s = [0.0]

        def rms(est, ref):
            ph = be.object_and_phase(*map(float, est))[1].cpu().numpy()
            return float(np.sqrt(np.mean(so.wrapped_phase_error(ph, ref) ** 2)))

        def timed(fn):
            check_s[0] = 0.0
            torch.cuda.synchronize(dev)
            t = time.perf_counter()
            out = fn()
            torch.cuda.synchronize(dev)
            return out, time.perf_counter() - t - check_s[0]

        floor = rms(x_opt, truth)
        tau_obj = 1e-4 if obj == "weak" else 1e-3
        for crit, ref in (("opt", at_opt), ("truth", truth)):
            def ok(est, ref=ref):
                torch.cuda.synchronize(dev)
                t = time.perf_counter()
                r = rms(est, ref) <= tau_obj
                check_s[0] += time.perf_counter() - t
                return r

            (bp, pe, _), t_plain = timed(lambda: pr.zoom_search(
                be, None, (pr.BOX_HI - pr.BOX_LO) / 2, 64, 200, 0.75, np.random.default_rng(1),
                done=ok))
            (bl, le, _, fell), t_learned = timed(lambda: pr.learned_refine(
                be, pr.to_x(prop.propose(be)), rng=np.random.default_rng(2), done=ok))
            rows.append({"crit": crit, "obj": obj, "tau": tau_obj, "plain": pe, "learned": le,
                         "plain_done": ok(bp), "learned_done": ok(bl), "fell_back": fell,
                         "plain_s": t_plain, "learned_s": t_learned,
                         "floor": floor if crit == "truth" else 0.0})
        del be, counts

    def summary(crit, obj):
        """Means, the ratio and fits/s over the cases whose loss optimum lies
        within tau of the reference phase (a converging minimiser cannot stay
        inside the target otherwise; those are counted, not compared) and that
        both searches reached (one that ran out of rounds has no count to
        compare); every case is listed as (plain, learned, plain reached,
        learned reached, floor)."""
        rs = [r for r in rows if r["crit"] == crit and r["obj"] == obj]
        ok_floor = [r for r in rs if r["floor"] <= r["tau"]]
        both = [r for r in ok_floor if r["plain_done"] and r["learned_done"]] or ok_floor or rs
        pe = float(np.mean([r["plain"] for r in both]))
        le = float(np.mean([r["learned"] for r in both]))
        return {"mean_evals_plain64": pe, "mean_evals_learned8": le, "evals_ratio": pe / le,
                "ratio_over": "cases with floor <= tau that both reached",
                "both_reached": len(both), "n_cases": len(rs),
                "floor_above_tau": len(rs) - len(ok_floor),
                "plain_reached": sum(r["plain_done"] for r in rs),
                "learned_reached": sum(r["learned_done"] for r in rs),
                "learned_fell_back": sum(r["fell_back"] for r in rs),
                "fits_per_s_plain64": len(both) / sum(r["plain_s"] for r in both),
                "fits_per_s_learned8": len(both) / sum(r["learned_s"] for r in both),
                "cases": [[r["plain"], r["learned"], int(r["plain_done"]), int(r["learned_done"]),
                           float("%.3g" % r["floor"])] for r in rs]}

    return {
        "workload": "64^2 scan x 64^2 detector (padded to 128^2), 1e6 e/position, aberrations "
                    "in the sweep ranges (C1, A1, C3); weak-phase (0.03 rad) and 0.3 rad atoms",
        "train_s": train_s, "train_samples": 50_000, "train_epochs": info["epochs"],
        "train_tflops": (fwd + bwd) * steps / train_s / 1e12,
        "val_best_head_A": {"rmse": [round(v, 1) for v in val["rmse_units"]],
                            "median_abs": [round(v, 1) for v in val["median_abs_units"]],
                            "order": "C1, A1a, A1b, C3"},
        "tau_1e-4_vs_loss_optimum_weak_phase": summary("opt", "weak"),
        "tau_1e-4_vs_truth_weak_phase": summary("truth", "weak"),
        "tau_1e-3_vs_loss_optimum_0.3rad": summary("opt", "0.3rad"),
        "tau_1e-3_vs_truth_0.3rad": summary("truth", "0.3rad"),
    }


def run_reference(args, world, rank) -> None:
    if rank != 0:
        return
    from oracle import ssb_torch_spec as spec
    from quantem.gpu_b200.synthetic import CONFIGS, generate

    dev = "cuda" if torch.cuda.is_available() else "cpu"
    counts = generate(CONFIGS[SPEC_NAME], device=dev).counts.cpu().numpy()
    kw = dict(voltage_kV=300, semiangle_mrad=KW["semiangle"], scan_sampling=KW["scan_sampling"],
              det_sampling=KW["det_sampling"])
    n_bf = 0
    for _ in range(args.warmup):
        n_bf = spec.reconstruct(counts, **kw)[3]
    t0 = time.perf_counter()
    for _ in range(args.steps):
        n_bf = spec.reconstruct(counts, **kw)[3]
    dt = time.perf_counter() - t0
    value = args.steps / dt
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "reference",
        "config": _config(n_bf, args.gpus),
        "reference_path": "CPU torch restatement of the reference's executable specification "
                          "(docs/kernels/ssb.md), every host thread",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": spec.host_threads(), "kind": "port",
                         "sample": "one full 128^4 reconstruction per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_b200(args, world, rank, local) -> None:
    from quantem.gpu_b200 import SSB, B200SSBBackend, ops
    from quantem.gpu_b200._lib import Aberrations
    from quantem.gpu_b200.synthetic import CONFIGS, generate
    from dataclasses import replace

    dev = torch.device("cuda", local)
    spec = replace(CONFIGS[SPEC_NAME], seed=CONFIGS[SPEC_NAME].seed + rank)
    counts = generate(spec, device=dev).counts.contiguous()
    ab = dict(C10=0.0, C12=0.0, phi12=0.0)
    stream = torch.cuda.current_stream(dev)

    from quantem.gpu_b200.pipeline import ColdReconstructor

    def backend_step():
        be = B200SSBBackend(counts, device=dev, **KW)
        obj, ph = be.object_and_phase(ab["C10"], ab["C12"], ab["phi12"])
        return be, ph

    # the headline: graph-launched cold reconstructions of the resident counts
    # (every step recomputes sums, selection, geometry, gather, scan FFT,
    # object and phase; only allocation and launch overhead are shared)
    rec = ColdReconstructor(counts, semiangle=KW["semiangle"], scan_sampling=KW["scan_sampling"],
                            det_sampling=KW["det_sampling"], voltage_kV=KW["voltage_kV"])
    for _ in range(max(3, args.warmup)):
        ph = rec.run()
    be, _ = backend_step()
    torch.cuda.synchronize(dev)
    n_bf = be.num_bf
    clocks = Clocks(dev.index)
    _barrier(world)
    torch.cuda.synchronize(dev)
    clocks.start()
    launches0 = ops.LAUNCH_COUNT
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    box0 = rec.box_runs
    for _ in range(args.steps):
        ph = rec.run()
    end.record(stream)
    torch.cuda.synchronize(dev)
    clock_info = clocks.stop()
    box_steps = rec.box_runs - box0
    launches = ops.LAUNCH_COUNT - launches0
    _barrier(world)
    elapsed_ms = _max_over_ranks(start.elapsed_time(end), world)
    value = world * args.steps / (elapsed_ms / 1e3)
    ph = ph.clone()

    # the same through the backend object per step (the reference-contract path)
    for _ in range(3):
        backend_step()
    torch.cuda.synchronize(dev)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(args.steps):
        be, _ = backend_step()
    s1.record(stream)
    torch.cuda.synchronize(dev)
    backend_cold = 1e3 * args.steps / s0.elapsed_time(s1)

    # a stream of scans: two acquisitions resident (2 x 537 MB), one cold
    # reconstructor per buffer on its own stream, alternating, so that one
    # scan's HBM-bound frame sums run beside the other's compute-bound stages
    counts_b = counts.clone()
    rec_b = ColdReconstructor(counts_b, semiangle=KW["semiangle"], scan_sampling=KW["scan_sampling"],
                              det_sampling=KW["det_sampling"], voltage_kV=KW["voltage_kV"])
    sa, sb = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def two_scans():
        with torch.cuda.stream(sa):
            rec.run()
        with torch.cuda.stream(sb):
            rec_b.run()

    for _ in range(max(3, args.warmup)):
        two_scans()
    torch.cuda.synchronize(dev)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    ev0 = torch.cuda.Event()
    ev0.record(stream)
    sa.wait_event(ev0)
    sb.wait_event(ev0)
    pairs = max(1, args.steps // 2)
    for _ in range(pairs):
        two_scans()
    ea, eb = torch.cuda.Event(), torch.cuda.Event()
    ea.record(sa)
    eb.record(sb)
    stream.wait_event(ea)
    stream.wait_event(eb)
    p1.record(stream)
    torch.cuda.synchronize(dev)
    pipelined = 1e3 * 2 * pairs / p0.elapsed_time(p1)
    del rec_b, counts_b

    # per-stage kernel time: each stage launched back to back between two events,
    # with the tile shapes the cold reconstructor's autotuner chose
    tuned = rec._b.get((n_bf, False), {})
    gv, fv, of = (tuned.get("gather_variant", 0), tuned.get("fft_variant", 0),
                  tuned.get("obj_flags", 0))
    sums, _ = ops.mean_dp_u64(counts, want_mean=False)
    cols = ops.gather_bf_columns(counts, be._bf_linear, validate=False, variant=gv)
    cal = be._calibration()
    ab0 = Aberrations(0.0, 0.0, 0.0, 0.0)
    ws = ops.Workspace(dev)
    # the box path of the headline (ColdReconstructor): sums of the first 512
    # frames + box estimate + frame sums writing the box columns; selection;
    # the scan FFT from the box; the object. The gathering path's stages too.
    frames = counts.view(-1, 128, 128)
    cap = rec.box_capacity if rec.use_box else 8192
    box_cols = rec.box_cols if rec.use_box else None
    box = torch.empty(ops.BOX_WORDS, dtype=torch.int32, device=dev)

    def box_sums():
        sample, _ = ops.mean_dp_u64(frames[:512], want_mean=False)
        ops.bf_box_estimate(sample, (128, 128), cap, out=box)
        return ops.mean_dp_u64_box(counts, box, box_cols)

    stage_fns = {}
    if rec.use_box:
        box_sums()
        bsel = ops.select_bf(sums, (128, 128), 128 * 128)
        bmap, _ = ops.bf_box_map(bsel, (128, 128), box, cap)
        stage_fns["qssb_mean_dp_u64_box"] = box_sums
        stage_fns["qssb_scan_fft_half_mapped"] = lambda: ops.scan_fft_half_mapped(
            box_cols, bmap, n_bf, (128, 128))
    stage_fns.update({
        "qssb_mean_dp_u64": lambda: ops.mean_dp_u64(counts, want_mean=False),
        "qssb_select_bf": lambda: ops.select_bf(sums, (128, 128), 128 * 128),
        "qssb_gather_bf_columns_2d": lambda: ops.gather_bf_columns(counts, be._bf_linear,
                                                                   validate=False, variant=gv),
        "qssb_scan_fft_half": lambda: ops.scan_fft_half(cols, (128, 128), variant=fv),
        "qssb_object": lambda: ops.object_wave(be.G_qk, be._geom_dev, be._q_row, be._q_col, cal,
                                               ab0, flags=of, workspace=ws),
    })
    stage_ms = {}
    for name, fn in stage_fns.items():
        fn()
        torch.cuda.synchronize(dev)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 20
        a0.record(stream)
        for _ in range(reps):
            fn()
        a1.record(stream)
        torch.cuda.synchronize(dev)
        stage_ms[name] = a0.elapsed_time(a1) / reps
    del cols

    # warm redraw (object from resident G) and loss evaluations: secondary figures
    torch.cuda.synchronize(dev)
    for _ in range(5):
        be.object_and_phase(10.0, 5.0, 0.1)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    n_warm = 50
    for i in range(n_warm):
        be.object_and_phase(10.0 + i, 5.0, 0.1)
    e.record(stream)
    torch.cuda.synchronize(dev)
    warm_ms = s.elapsed_time(e) / n_warm
    cands = torch.zeros((64, 4), dtype=torch.float32, device=dev)
    cands[:, 0] = torch.linspace(-50, 50, 64, device=dev)
    be.variance_loss_batch(cands[:, 0].cpu().numpy(), 0.0, 0.0)
    torch.cuda.synchronize(dev)
    s.record(stream)
    for _ in range(3):
        be.variance_loss_batch(cands[:, 0].cpu().numpy(), 0.0, 0.0)
    e.record(stream)
    torch.cuda.synchronize(dev)
    loss_batch_ms = s.elapsed_time(e) / 3
    # the same batch through the table-free kernel (one BF pixel per 2D FFT,
    # apertures evaluated per candidate)
    be.use_overlap_table = False
    be.variance_loss_batch(cands[:, 0].cpu().numpy(), 0.0, 0.0)
    torch.cuda.synchronize(dev)
    s.record(stream)
    for _ in range(3):
        be.variance_loss_batch(cands[:, 0].cpu().numpy(), 0.0, 0.0)
    e.record(stream)
    torch.cuda.synchronize(dev)
    loss_batch_plain_ms = s.elapsed_time(e) / 3
    be.use_overlap_table = True
    # 14-term chi (full plane, per-element polynomial chi): 8-candidate batches
    rng = np.random.default_rng(5)
    fm = np.tile(np.array([10.0, 5.0, 1500.0, 1000.0, 5e4, 3e4, 4e4, 3e6, 2e6, 2e6, 1e8, 5e7, 5e7,
                           5e7], np.float32), (8, 1)) * rng.uniform(0.5, 1.0, (8, 14)).astype(np.float32)
    fa = rng.uniform(-np.pi, np.pi, (8, 14)).astype(np.float32)
    be.variance_loss_batch_full(fm, fa)
    torch.cuda.synchronize(dev)
    s.record(stream)
    for _ in range(3):
        be.variance_loss_batch_full(fm, fa)
    e.record(stream)
    torch.cuda.synchronize(dev)
    loss_full_ms = s.elapsed_time(e) / 3

    # end to end through the public API: pinned host counts -> SSB -> host phase
    host = counts.cpu().pin_memory()
    h2d = host.numel() * host.element_size()
    d2h = 0
    def e2e_step():
        with SSB.from_array(host, voltage_kV=300, semiangle_mrad=KW["semiangle"],
                            scan_sampling_A=KW["scan_sampling"],
                            det_sampling=KW["det_sampling"]) as ssb:
            res = ssb.reconstruct(compute_loss=False)
            return res.phase.cpu()
    for _ in range(2):
        out = e2e_step()
    d2h = out.numel() * out.element_size() + 128 * 128 * (4 + 8)  # phase + mean DP + u64 sums
    torch.cuda.synchronize(dev)
    gc.collect()  # a collection of the earlier legs' garbage stays out of the timed steps
    _barrier(world)
    t0 = time.perf_counter()
    n_e2e = max(3, min(args.steps, 10))
    for _ in range(n_e2e):
        e2e_step()
    torch.cuda.synchronize(dev)
    e2e_s = _max_over_ranks(time.perf_counter() - t0, world)
    e2e_value = world * n_e2e / e2e_s

    # end to end from the acquisition as stored (one bitshuffle+LZ4 chunk per
    # frame, the reference's file format): pinned host chunks -> SSB.from_chunks
    # (decoded on the GPU) -> host phase
    from quantem.gpu_b200.decode import encode_bslz4

    packed_dev, offs_dev = encode_bslz4(counts.reshape(-1, 128, 128))
    packed_host = packed_dev.cpu().pin_memory()
    offs_host = offs_dev.cpu().pin_memory()
    del packed_dev, offs_dev

    def e2e_chunks_step():
        with SSB.from_chunks(packed_host, chunk_offsets=offs_host, frame_shape=(128, 128),
                             scan_shape=(128, 128), voltage_kV=300,
                             semiangle_mrad=KW["semiangle"], scan_sampling_A=KW["scan_sampling"],
                             det_sampling=KW["det_sampling"]) as ssb:
            return ssb.reconstruct(compute_loss=False).phase.cpu()
    for _ in range(2):
        e2e_chunks_step()
    torch.cuda.synchronize(dev)
    gc.collect()
    _barrier(world)
    n_chunks_e2e = 3 * n_e2e  # ~3 ms steps: more of them for a stable wall-clock figure
    t0 = time.perf_counter()
    for _ in range(n_chunks_e2e):
        e2e_chunks_step()
    torch.cuda.synchronize(dev)
    e2e_c_s = _max_over_ranks(time.perf_counter() - t0, world)
    e2e_chunks = {"value": world * n_chunks_e2e / e2e_c_s, "unit": UNIT,
                  "h2d_bytes_per_step": packed_host.numel() + 8 * offs_host.numel(),
                  "d2h_bytes_per_step": d2h,
                  "api": "SSB.from_chunks(pinned host bitshuffle+LZ4 chunks, decoded on the GPU)"
                         ".reconstruct()",
                  "compression_ratio": counts.numel() * 2 / packed_host.numel()}

    if rank != 0:
        return
    peak, peak_kind = _peaks()
    n_r, k2, half = 128 * 128, 128 * 128, 128 * 65
    alg = {  # algorithmic bytes per launch of each entry point
        "qssb_mean_dp_u64_box": (2 * n_r * k2, "k_sum_frames_box"),
        "qssb_mean_dp_u64": (2 * n_r * k2, "k_sum_frames_vec8"),
        "qssb_gather_bf_columns_2d": (4 * n_r * n_bf, "k_gather_bbox"),
        "qssb_scan_fft_half_mapped": (2 * n_r * n_bf + 8 * n_bf * half, "k_scan_fft128p"),
        "qssb_scan_fft_half": (2 * n_r * n_bf + 8 * n_bf * half, "k_scan_fft128p"),
        "qssb_object": (8 * n_bf * half + 12 * 128 * 128, "k_trotter_quad4"),
    }
    rooflines = {}
    for op, (nbytes, kernel) in alg.items():
        if op in stage_ms:
            ach = nbytes / (stage_ms[op] / 1e3) / 1e9
            rooflines[op] = {"achieved": ach, "frac": ach / peak, "alg_bytes_per_launch": nbytes,
                             "avg_launch_ms": stage_ms[op], "kernel": kernel}
    path = (["qssb_mean_dp_u64_box", "qssb_select_bf", "qssb_scan_fft_half_mapped", "qssb_object"]
            if rec.use_box else ["qssb_mean_dp_u64", "qssb_select_bf", "qssb_gather_bf_columns_2d",
                                 "qssb_scan_fft_half", "qssb_object"])
    dominant = max((k for k in rooflines if k in path), key=lambda k: rooflines[k]["avg_launch_ms"])
    dom = rooflines[dominant]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": elapsed_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": _config(n_bf, world),
        "roofline": {"bound": LIMITER.get(dom["kernel"], "hbm"),
                     "model": "algorithmic HBM bytes per launch / CUDA-event time vs measured copy bandwidth",
                     "kernel": f"{dom['kernel']} ({dominant}), the step's longest stage",
                     "achieved": dom["achieved"], "peak": peak, "unit": "GB/s", "frac": dom["frac"],
                     "peak_kind": f"{peak_kind} hbm_gbs", "traffic": _traffic(dom["kernel"]),
                     "alg_bytes_per_launch": dom["alg_bytes_per_launch"],
                     "avg_launch_ms": dom["avg_launch_ms"]},
        "roofline_by_stage": {k: {"kernel": v["kernel"], "achieved_gbs": v["achieved"], "frac": v["frac"],
                                  "traffic": _traffic(v["kernel"])} for k, v in rooflines.items()},
        "stage_ms": stage_ms,
        "autotuned": {"gather_variant": gv, "scan_fft_variant": fv,
                      "object_chunks": (of >> 16) & 0x7FFF, "object_tile_variant": (of >> 8) & 0xF},
        "cold_path": ("BF columns written by the frame-sum pass (box) in "
                      f"{box_steps} of {args.steps} timed steps, gathered in the rest"),
        "cold_backend_recon_per_s": backend_cold,
        "pipelined_two_scans_recon_per_s": pipelined,
        "warm_recon_per_s": 1e3 / warm_ms,
        "loss_evals_per_s_batch64": 64 * 1e3 / loss_batch_ms,
        "loss_evals_per_s_batch64_table_free": 64 * 1e3 / loss_batch_plain_ms,
        "loss_full_chi_evals_per_s_batch8": 8 * 1e3 / loss_full_ms,
        "gpu_launches": launches,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "api": "SSB.from_array(pinned host u16).reconstruct()"},
        "e2e_from_chunks": e2e_chunks,
        "clocks": clock_info,
    }
    if world == 1 and not args.no_reference_cuda:
        rc = reference_cuda_baseline(counts, be, min(args.steps, 20), 3)
        line["reference_cuda"] = rc
        if "cold_recon_per_s" in rc:
            line["speedup_vs_reference_cuda"] = {
                "cold": value / rc["cold_recon_per_s"],
                "warm": line["warm_recon_per_s"] / rc["warm_recon_per_s"]}
            if "loss_evals_per_s" in rc:
                line["speedup_vs_reference_cuda"]["loss_batch64"] = (
                    line["loss_evals_per_s_batch64"] / rc["loss_evals_per_s"])
    if world == 1 and not args.no_stress:
        line["stress_256"] = stress_256(dev, 5)
        if not args.no_large:
            line["large_512"] = large_512(dev)
        line["sweep_3scans"] = sweep_3scans(dev, 5)
        line["temporal_join"] = temporal_join(dev)
        line["bslz4_decode"] = bslz4_decode(dev)
        line["learned_fits"] = learned_fits(dev)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(counts.cpu().numpy())
    if world == 1 and not args.no_oracle:
        from oracle import ssb_oracle as so

        hostc = counts.cpu().numpy()
        prep = so.prepare(hostc, voltage_kV=300, semiangle_mrad=KW["semiangle"],
                          scan_sampling=KW["scan_sampling"], det_sampling=KW["det_sampling"])
        _, ref_ph = so.reconstruct(prep, so.Aberrations(0.0, 0.0, 0.0))
        err = so.wrapped_phase_error(ph.cpu().numpy(), ref_ph)
        line["phase_rms_rad_vs_fp64"] = float(np.sqrt(np.mean(err ** 2)))
    line["headline"] = _headline(line)
    print(json.dumps(line), flush=True)


# Measured limiter of each kernel the roofline can name (ncu: issue active,
# warps active, DRAM throughput; the kernel summaries under profiles/)
LIMITER = {"k_sum_frames_vec8": "hbm", "k_gather_bbox": "hbm", "k_scan_fft128p": "latency",
           "k_trotter_quad4": "issue"}


def _headline(line: dict) -> dict:
    """The claims of the line in one compact object, printed last so that a
    reader who keeps only the end of the output still has them."""
    h = {"cold_recon_per_s": line["value"],
         "pipelined_two_scans_recon_per_s": line.get("pipelined_two_scans_recon_per_s"),
         "warm_recon_per_s": line.get("warm_recon_per_s"),
         "e2e_recon_per_s": line["e2e"]["value"],
         "e2e_from_chunks_recon_per_s": line.get("e2e_from_chunks", {}).get("value"),
         "loss_evals_per_s": line.get("loss_evals_per_s_batch64"),
         "stage_us": {k.replace("qssb_", ""): 1e3 * v for k, v in line.get("stage_ms", {}).items()},
         "roofline": {"kernel": line["roofline"]["kernel"].split(" ")[0],
                      "bound": line["roofline"]["bound"], "hbm_frac": line["roofline"]["frac"]}}
    rc = line.get("reference_cuda", {})
    if "cold_recon_per_s" in rc:
        h["reference_cuda_recon_per_s"] = {"cold": rc["cold_recon_per_s"], "warm": rc["warm_recon_per_s"]}
        h["speedup_vs_reference_cuda"] = line.get("speedup_vs_reference_cuda")
    if "loss_evals_per_s" in rc:
        h["reference_cuda_loss_evals_per_s"] = rc["loss_evals_per_s"]
    if "phase_rms_rad_vs_fp64" in line:
        h["phase_rms_rad_vs_fp64_128"] = line["phase_rms_rad_vs_fp64"]
    st = line.get("stress_256")
    if st:
        h["stress_256_phase_rms_rad"] = {d: v["phase_rms_rad_vs_fp64_gpu"] for d, v in st["doses"].items()}
    lg = line.get("large_512")
    if lg:
        h["large_512_ms"] = {"cold": lg["cold_u16_to_phase_ms"], "warm_object": lg["warm_complex_object_ms"],
                             "phase_plus_loss": lg["exact_phase_plus_loss_ms"]}
    sw = line.get("sweep_3scans")
    if sw:
        h["sweep_3scans"] = {"evals_per_s": sw["evals_per_s_graph"],
                             "launches_per_graph": sw["kernel_launches_per_graph"],
                             "truth_first": sw["truth_ranked_first"],
                             "launch_sequence_evals_per_s":
                                 sw["launch_sequence"]["evals_per_s_graph"],
                             "launch_sequence_launches_per_graph":
                                 sw["launch_sequence"]["kernel_launches_per_graph"]}
    lf = line.get("learned_fits")
    if lf:
        keys = ("tau_1e-4_vs_loss_optimum_weak_phase", "tau_1e-4_vs_truth_weak_phase",
                "tau_1e-3_vs_loss_optimum_0.3rad", "tau_1e-3_vs_truth_0.3rad")
        h["learned_fits"] = {
            k: {q: lf[k][q] for q in ("mean_evals_plain64", "mean_evals_learned8", "evals_ratio",
                                      "both_reached", "floor_above_tau", "learned_fell_back",
                                      "n_cases")}
            for k in keys if k in lf}
        h["learned_fits"]["train_tflops"] = lf.get("train_tflops")
    cb = line.get("cpu_baseline")
    if cb:
        h["cpu_baseline"] = {"recon_per_s": cb["value"], "cores": cb["cores"]}
    return _sig(h, 4)


def run_profile_once(local: int, with_256: bool = False, with_512: str | None = None,
                     with_mlp: bool = False) -> None:
    """One cold reconstruction, one warm object, one loss and one 64-candidate
    loss batch on the 128^4 workload, untimed: the launch sequence the ncu
    summaries under profiles/ are captured from. ``with_mlp``: then two
    training steps of the proposer's MLP at batch 256 on random inputs (its
    first tcgen05 launch is the 256 x 512 x 16384 input layer)."""
    from quantem.gpu_b200 import B200SSBBackend
    from quantem.gpu_b200.synthetic import CONFIGS, generate

    dev = torch.device("cuda", local)
    counts = generate(CONFIGS[SPEC_NAME], device=dev).counts
    torch.cuda.synchronize(dev)
    be = B200SSBBackend(counts, device=dev, **KW)
    be.object_and_phase(10.0, 5.0, 0.1)
    loss = be.variance_loss(10.0, 5.0, 0.1)
    losses = be.variance_loss_batch(np.linspace(-50.0, 50.0, 64), 0.0, 0.0)
    torch.cuda.synchronize(dev)
    out = {"profile_once": True, "n_bf": be.num_bf, "loss": loss, "loss_batch0": float(losses[0])}
    if with_256:
        del be, counts
        spec = CONFIGS["stress_256x256_det128"]
        c256 = generate(spec, device=dev).counts
        be = B200SSBBackend(c256, device=dev, **KW)
        out["loss256"] = float(be.variance_loss_batch([spec.C10], [0.0], [0.0])[0])
        torch.cuda.synchronize(dev)
    if with_512:
        # "full": the 512^2 x 192^2 timing shape (19.3 GB); "small": 512^2 x 48^2
        # (1.2 GB, ~440 BF) for multi-pass captures of the same kernels
        from dataclasses import replace

        del be
        torch.cuda.empty_cache()
        spec = CONFIGS["large_512x512_det192"]
        if with_512 == "small":
            spec = replace(spec, detector_shape=(48, 48), det_sampling_mrad=spec.semiangle_mrad / 20.0)
        c512 = generate(spec, device=dev).counts
        kw = dict(semiangle=spec.semiangle_mrad, scan_sampling=spec.scan_step_A,
                  det_sampling=spec.det_sampling_mrad, voltage_kV=spec.voltage_kV)
        be = B200SSBBackend(c512, device=dev, **kw)
        be.object_and_phase(spec.C10, 0.0, 0.0)
        _, out["loss512"] = be.reconstruct_with_loss(spec.C10, 0.0, 0.0)
        out["n_bf512"] = be.num_bf
        torch.cuda.synchronize(dev)
    if with_mlp:
        from quantem.gpu_b200 import proposer as pr

        mlp = pr.MLP(dev, seed=0)
        g = torch.Generator(device=dev).manual_seed(1)
        x = torch.rand((256, pr.N_IN), generator=g, device=dev).to(torch.bfloat16)
        t = torch.rand((256, pr.N_OUT), generator=g, device=dev)
        for _ in range(2):
            mlp.forward(x)
            loss_t = mlp.backward_and_step(t, 1e-4)
        out["mlp_loss"] = float(loss_t.item())
    print(json.dumps(out))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-oracle", action="store_true")
    ap.add_argument("--with-256", action="store_true",
                    help="--profile-once: also one 256^2 scan loss evaluation")
    ap.add_argument("--with-512", choices=["full", "small"], default=None,
                    help="--profile-once: also one 512^2 cold preparation, object and loss")
    ap.add_argument("--with-mlp", action="store_true",
                    help="--profile-once: also two proposer MLP training steps (batch 256)")
    ap.add_argument("--no-large", action="store_true",
                    help="skip the 512^2 x 192^2 (19.3 GB) leg")
    ap.add_argument("--no-stress", action="store_true",
                    help="skip the 256^2 dose sweep against the FP64 GPU path")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="skip timing the reference's own CUDA object kernels")
    ap.add_argument("--profile-once", action="store_true",
                    help="run the untimed launch sequence used for ncu captures")
    args = ap.parse_args()
    world, rank, local = _dist()
    try:
        if args.profile_once:
            run_profile_once(local, args.with_256, args.with_512, args.with_mlp)
        elif args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_b200(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
