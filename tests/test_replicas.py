"""The N > 1 path of bench.py on the host: world-size-2 gloo process groups
(the replica path has no data exchange; its only collectives are the
max-over-ranks of the timings).  Rendezvous on 127.0.0.1."""

from __future__ import annotations

import datetime
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank: int, world: int, port: int, queue) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        w, r, local = bench._dist()
        slowest = bench._max_over_ranks(1.5 + r, w, local)   # each rank's own "time"
        queue.put((r, w, slowest))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gives_every_rank_the_slowest_time():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0], codes
    got = sorted(queue.get(timeout=5) for _ in range(2))
    assert got == [(0, 2, 2.5), (1, 2, 2.5)]


@pytest.mark.timeout(300)
def test_two_rank_launch_prints_one_line_from_rank_zero():
    """The launch the benchmark driver uses, with gloo instead of NCCL: the
    reference arm runs on rank 0 alone, the other rank exits 0 without
    work, one JSON line comes out with n_gpus = 2."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"), "--gpus", "2",
           "--impl", "reference", "--dist-backend", "gloo", "--size", "24", "--steps", "3", "--warmup", "3",
           "--cpu-budget", "0.2"]
    res = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=280)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, res.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0
