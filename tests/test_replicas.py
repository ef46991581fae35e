"""The multi-GPU form is replicas: each rank runs its own products and the bench reports every
rank's products over the slowest rank's time. Its cross-rank steps (the barrier and the
max-over-ranks reduction of the timings) run here on two CPU ranks over gloo."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r pretends its timed steps took 10 + r ms and its back-to-back products 3 + 2 r ms
        dist.barrier()
        total_ms, batch_ms = bench.max_over_ranks(dist, [10.0 + rank, 3.0 + 2 * rank], "cpu")
        out.put((rank, total_ms, batch_ms, bench.whole_job_rate(world, 20, total_ms)))
    finally:
        dist.destroy_process_group()


def test_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, total_ms, batch_ms, rate in got:
        assert total_ms == 11.0 and batch_ms == 5.0  # the slowest rank's time, on every rank
        assert rate == pytest.approx(2 * 20 / 11e-3)


def test_single_process_is_its_own_maximum():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(None, [4.0, 2.5], "cpu") == [4.0, 2.5]
    assert bench.whole_job_rate(1, 10, 2.0) == pytest.approx(5000.0)
