"""Autotuner for the work partition and tile shapes of the SSB kernels.

The loss kernel's CTAs each own one (candidate, BF chunk); with one CTA per
SM resident, the number of chunks per candidate decides how many waves the
batch takes and how full the last one is. The trotter kernel's BF chunk count
trades grid size against the cost of folding the partial sums, and its tile
shape (2, 4 or 8 adjacent frequencies per thread) trades registers against
one sincos per tile. Both go through the flags (``QSSB_FLAG_CHUNKS``, bits
16..30; ``QSSB_FLAG_VARIANT``, bits 8..11). The BF gather's tile shape
(frames x band pixels, bounding-box or pixel-major tiles) and the scan FFT's
launch shape (persistent CTAs per SM; at 256^2 and up the column pass's
strip width and CTAs per SM) are named by the ``_ex`` entry points'
``variant`` argument; every gather and FFT variant gives the same bits.

The tuner times a small set of candidates with CUDA events on the real
inputs, keeps the fastest and caches it per (device, kind, shape) in memory
and in a JSON file (``$QSSB_TUNING_CACHE``, default
``~/.cache/quantem_gpu_b200/tuning.json``) so later processes skip the
search. A cached choice gives identical bits on every call; different
partitions or trotter tiles differ only in float32 rounding.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

import torch

from . import _lib, ops

_CACHE: dict[str, int] | None = None


def _path() -> Path:
    env = os.environ.get("QSSB_TUNING_CACHE")
    return Path(env) if env else Path.home() / ".cache" / "quantem_gpu_b200" / "tuning.json"


def _cache() -> dict[str, int]:
    global _CACHE
    if _CACHE is None:
        try:
            _CACHE = {k: int(v) for k, v in json.loads(_path().read_text()).items()}
        except (OSError, ValueError):
            _CACHE = {}
    return _CACHE


def _store(key: str, value: int) -> None:
    _cache()[key] = int(value)
    try:
        p = _path()
        p.parent.mkdir(parents=True, exist_ok=True)
        tmp = p.with_suffix(".tmp")
        tmp.write_text(json.dumps(_cache(), indent=1, sort_keys=True))
        tmp.replace(p)
    except OSError:
        pass  # a read-only home keeps the in-memory cache only


def _key(kind: str, device: torch.device, *parts) -> str:
    name = torch.cuda.get_device_name(device).replace(" ", "_")
    return ":".join([kind, name] + [str(p) for p in parts])


def _time_ms(fn, device: torch.device, reps: int) -> float:
    stream = torch.cuda.current_stream(device)
    fn()  # warm-up: workspace growth, attributes
    torch.cuda.synchronize(device)
    best = float("inf")
    for _ in range(reps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        fn()
        e.record(stream)
        torch.cuda.synchronize(device)
        best = min(best, s.elapsed_time(e))
    return best


def loss_chunk_options(n_bf: int, n_cand: int, sms: int, scan: int = 128) -> list[int]:
    """Chunks per candidate whose CTA count fills whole waves, plus neighbours.

    At 256^2 and above the knob is the column pass's interleave, whose CTA
    count is (scan / strip width) x chunks x candidates."""
    opts = set()
    strips = 1 if scan < 256 else scan // (8 if scan >= 1024 else 16)
    for waves in (1, 2, 3, 4):
        c = max(1, (waves * sms) // (n_cand * strips))
        opts.update({c, c + 1} if c * n_cand * strips < waves * sms else {c})
    return sorted(c for c in opts if 1 <= c <= min(n_bf, _lib.QSSB_FLAG_CHUNKS_MAX))


def tune_loss(g_half, bf_geom, q_row, q_col, cal, candidates: torch.Tensor, flags: int,
              workspace: ops.Workspace, reps: int = 2, overlap: torch.Tensor | None = None) -> int:
    """Best chunks-per-candidate for this batch shape (cached); 0 keeps the
    built-in plan when it is the fastest."""
    dev = g_half.device
    n_cand = int(candidates.shape[0])
    key = _key("loss" if overlap is None else "loss_table", dev, int(cal.scan_rows), int(cal.n_bf),
               n_cand, flags & 0xFFFF)
    hit = _cache().get(key)
    if hit is not None:
        return hit
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    out = torch.empty(n_cand, dtype=torch.float32, device=dev)
    timings = {}
    opts = loss_chunk_options(int(cal.n_bf), n_cand, sms, int(cal.scan_rows))
    if int(cal.scan_rows) == 128:
        opts = [0] + opts  # the built-in wave-aware plan competes too
    for c in opts:
        f = flags | _lib.flag_chunks(c)
        timings[c] = _time_ms(lambda: ops.loss_batch(g_half, bf_geom, q_row, q_col, cal, candidates,
                                                     flags=f, workspace=workspace, out=out,
                                                     overlap=overlap), dev, reps)
    best = min(timings, key=timings.get)
    _store(key, best)
    return best


def _object_key(device, scan_rows: int, n_bf: int, flags: int, quadratic: bool) -> str:
    return _key("object", device, int(scan_rows), int(n_bf), flags & 0xFF, int(quadratic))


def cached_object(device: torch.device, scan_rows: int, n_bf: int, flags: int,
                  quadratic: bool = True) -> int:
    """The cached object tuning for this shape as flag bits (QSSB_FLAG_CHUNKS |
    QSSB_FLAG_VARIANT), or 0 (built-in plan and tile); no search."""
    return _cache().get(_object_key(device, scan_rows, n_bf, flags, quadratic), 0)


def object_options(scan_rows: int, n_bf: int, quadratic: bool) -> list[tuple[int, int]]:
    """(total BF chunks, trotter tile variant) pairs the object tuner times:
    chunk counts around the built-in plan's, each with 2, 4 and 8 frequencies
    per thread on the quadratic-chi path (variants 1, 0, 3; 0 is the built-in
    4) and the built-in tile elsewhere."""
    base = 32 if int(scan_rows) >= 256 else 128
    chunks = sorted({min(max(1, c), int(n_bf)) for c in (base // 2, base, 3 * base // 2, 2 * base)})
    variants = (0, 1, 3) if quadratic else (0,)
    return [(c, v) for c in chunks for v in variants]


def tune_object(g_half, bf_geom, q_row, q_col, cal, ab, flags: int, workspace: ops.Workspace,
                reps: int = 3) -> int:
    """Best (BF chunk count, trotter tile) for the object kernels, as flag bits
    to OR into ``flags`` (cached). ``ab`` decides the path: C30 == 0 is the
    quadratic-chi path that has tile variants."""
    dev = g_half.device
    quadratic = float(ab.C30) == 0.0
    key = _object_key(dev, int(cal.scan_rows), int(cal.n_bf), flags, quadratic)
    hit = _cache().get(key)
    if hit is not None:
        return hit
    timings = {}
    for c, v in object_options(int(cal.scan_rows), int(cal.n_bf), quadratic):
        bits = _lib.flag_chunks(c) | _lib.flag_variant(v)
        f = flags | bits
        timings[bits] = _time_ms(lambda: ops.object_wave(g_half, bf_geom, q_row, q_col, cal, ab,
                                                         flags=f, workspace=workspace), dev, reps)
    best = min(timings, key=timings.get)
    _store(key, best)
    return best


def tune_gather(counts: torch.Tensor, bf_linear: torch.Tensor, reps: int = 3) -> int:
    """Best tile shape of the BF gather for this detector, frame count and BF
    count (``qssb_gather_bf_columns_2d_ex`` variant, cached; 0 = built-in)."""
    dev = counts.device
    k0, k1 = int(counts.shape[-2]), int(counts.shape[-1])
    n_frames = counts.numel() // (k0 * k1)
    key = _key("gather", dev, k0, k1, n_frames, int(bf_linear.numel()))
    hit = _cache().get(key)
    if hit is not None:
        return hit
    timings = {}
    for v in range(_lib.GATHER_VARIANTS + 1):
        timings[v] = _time_ms(lambda: ops.gather_bf_columns(counts, bf_linear, validate=False,
                                                            variant=v), dev, reps)
    best = min(timings, key=timings.get)
    _store(key, best)
    return best


def tune_scan_fft(columns: torch.Tensor, scan_shape: tuple[int, int], reps: int = 3) -> int:
    """Best launch shape of the scan FFT for this scan size and BF count
    (``qssb_scan_fft_half_ex`` variant, cached; 0 = built-in)."""
    dev = columns.device
    r0 = int(scan_shape[0])
    key = _key("scan_fft", dev, r0, int(scan_shape[1]), int(columns.shape[0]))
    hit = _cache().get(key)
    if hit is not None:
        return hit
    timings = {}
    for v in range(ops.scan_fft_variants(r0) + 1):
        timings[v] = _time_ms(lambda: ops.scan_fft_half(columns, scan_shape, variant=v), dev, reps)
    best = min(timings, key=timings.get)
    _store(key, best)
    return best
