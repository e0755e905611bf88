"""Host plumbing of `bench.py --gpus N` (independent replicas, one per rank) with world_size 2 on
the gloo backend: barrier, max-over-ranks time and sum-over-ranks work, and the reference arm's
rank-0-only rule.  CPU only."""

import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        ms = bench.reduce_max(10.0 + rank, world)        # the slowest rank sets the time
        work = bench.reduce_sum(1000.0 * (rank + 1), world)  # every rank's owners count
        bench.barrier(world)
        out.put((rank, ms, work))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_like_the_bench():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 11.0, 3000.0), (1, 11.0, 3000.0)]


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    args = bench.parse()
    assert bench.run_reference(args) is None
    assert capsys.readouterr().out == ""
