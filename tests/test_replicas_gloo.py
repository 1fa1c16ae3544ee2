"""The multi-GPU form of the benchmark is replicas: every rank solves its own
boards and the whole-job rate is all ranks' units over the slowest rank's
time.  Two gloo ranks on the CPU exercise that reduction."""

from __future__ import annotations

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        value, slowest = bench.whole_job_rate([100.0, 150.0][rank], 4, world, dist, "cpu")
        out.put((rank, value, slowest))
    finally:
        dist.destroy_process_group()


def test_whole_job_rate_is_all_units_over_the_slowest_rank() -> None:
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(out.get(timeout=5) for _ in range(2))
    for _, value, slowest in got:
        assert slowest == 150.0
        assert value == pytest.approx(2 * 4 / 0.150)


def test_one_rank_needs_no_process_group() -> None:
    import bench

    assert bench.whole_job_rate(250.0, 5, 1) == (pytest.approx(20.0), 250.0)
