"""The N > 1 plumbing of bench.py on CPU with world_size-2 gloo process
groups: the barrier and max-over-ranks timing, and the reference arm launched
the way the driver launches it (torch.distributed.run, two ranks: rank 0
times and prints one JSON line, rank 1 exits 0 without work). The B200 arm's
data path has no collective (replicas only)."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2",
                      RANK=str(rank), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(REPO))
    import bench
    import torch.distributed as dist

    world, r, _ = bench._dist()
    try:
        bench._barrier(world)
        out.put((r, world, bench._max_over_ranks(0.25 + r, world)))
        bench._barrier(world)
    finally:
        dist.destroy_process_group()


def test_barrier_and_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 2, 1.25), (1, 2, 1.25)]


def test_reference_arm_on_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--gpus", "2", "--steps", "1", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="4")
    proc = subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, timeout=600, env=env)
    assert proc.returncode == 0, proc.stderr[-2000:]
    lines = [ln for ln in proc.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, proc.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
