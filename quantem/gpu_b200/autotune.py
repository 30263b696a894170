"""Autotuner for the work partition of the SSB kernels.

The loss kernel's CTAs each own one (candidate, BF chunk); with one CTA per
SM resident, the number of chunks per candidate decides how many waves the
batch takes and how full the last one is. The trotter kernel's BF chunk count
trades grid size against the cost of folding the partial sums. Both are set
through ``QSSB_FLAG_CHUNKS`` (bits 16..30 of the flags). The tuner times a
small set of candidate partitions with CUDA events on the real inputs, keeps
the fastest and caches it per (device, kind, scan size, BF count, batch size,
chi path) in memory and in a JSON file (``$QSSB_TUNING_CACHE``, default
``~/.cache/quantem_gpu_b200/tuning.json``) so later processes skip the search.
A cached partition gives identical bits on every call; different partitions
differ only in float32 summation order.
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


def cached_object(device: torch.device, scan_rows: int, n_bf: int, flags: int) -> int:
    """The cached object partition for this shape, or 0 (built-in plan); no search."""
    return _cache().get(_key("object", device, int(scan_rows), int(n_bf), flags & 0xFFFF), 0)


def tune_object(g_half, bf_geom, q_row, q_col, cal, ab, flags: int, workspace: ops.Workspace,
                reps: int = 3) -> int:
    """Best total BF chunk count for the object (trotter) kernel (cached)."""
    dev = g_half.device
    key = _key("object", dev, int(cal.scan_rows), int(cal.n_bf), flags & 0xFFFF)
    hit = _cache().get(key)
    if hit is not None:
        return hit
    base = 32 if int(cal.scan_rows) >= 256 else 128
    timings = {}
    for c in sorted({max(1, base // 2), base, 3 * base // 2, 2 * base}):
        f = flags | _lib.flag_chunks(min(c, int(cal.n_bf)))
        timings[c] = _time_ms(lambda: ops.object_wave(g_half, bf_geom, q_row, q_col, cal, ab,
                                                      flags=f, workspace=workspace), dev, reps)
    best = min(timings, key=timings.get)
    _store(key, best)
    return best
