"""The replica dispatcher (pcb_analysis_b200/replicas.py) on fake engines.

A fake engine has a byte budget and a slot count like the batch engine: it
admits a board when both have room and finishes it after a fixed number of
steps.  Checked: assignment to the engine with the most free bytes, a head
request that waits for memory and is admitted after a collection, refusal of
a request that fits no idle engine, results in request order; and, on two
gloo ranks, the footprint-balanced partition and the gather on rank 0.
"""

from __future__ import annotations

import os
import socket
from dataclasses import dataclass

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from pcb_analysis_b200.replicas import Dispatcher, partition, serve_on_ranks


@dataclass
class Request:
    arrays: dict
    rhs: np.ndarray
    initial_guess: None = None


def request(size: int, steps: int, value: float) -> Request:
    return Request({"bytes": size, "steps": steps}, np.full(3, value))


class FakeEngine:
    def __init__(self, budget: int, slots: int = 4) -> None:
        self.budget, self.slots = budget, slots
        self.used = 0
        self.live: dict[int, list] = {}
        self.ready: list[int] = []
        self.next = 0
        self.admitted: list[float] = []

    def info(self) -> dict:
        return {"budget_bytes": self.budget, "bytes_in_use": self.used}

    def submit(self, arrays, rhs, config, initial_guess=None):
        if len(self.live) >= self.slots or self.used + arrays["bytes"] > self.budget:
            return None
        ticket = self.next
        self.next += 1
        self.used += arrays["bytes"]
        self.live[ticket] = [arrays["steps"], arrays["bytes"], rhs]
        self.admitted.append(float(rhs[0]))
        return ticket

    def step(self) -> int:
        for ticket, entry in list(self.live.items()):
            entry[0] -= 1
            if entry[0] <= 0 and ticket not in self.ready:
                self.ready.append(ticket)
        return len(self.live)

    def finished(self) -> list[int]:
        return list(self.ready)

    def collect(self, ticket: int) -> dict:
        steps, size, rhs = self.live.pop(ticket)
        self.ready.remove(ticket)
        self.used -= size
        return {"solution": 2.0 * rhs, "converged": True}


def test_requests_go_to_the_freest_engine_wait_for_memory_and_return_in_order() -> None:
    small, large = FakeEngine(budget=100), FakeEngine(budget=250)
    reqs = [request(120, 3, 0.0), request(90, 1, 1.0), request(90, 2, 2.0), request(200, 1, 3.0),
            request(10, 1, 4.0)]
    placed = Dispatcher([small, large]).run(reqs)
    assert [p.index for p in placed] == list(range(5))
    for p, q in zip(placed, reqs):
        np.testing.assert_array_equal(p.result["solution"], 2.0 * q.rhs)
    # 0 -> large (most free); 1 -> large (130 free > 100); 2 -> small; 3 (200 B) waits for the
    # large engine to drain and nothing overtakes it; then 4.
    assert [p.engine for p in placed] == [1, 1, 0, 1, 0]
    assert large.admitted == [0.0, 1.0, 3.0] and small.admitted == [2.0, 4.0]


def test_a_request_no_idle_engine_can_hold_is_refused() -> None:
    with pytest.raises(MemoryError, match="request 1"):
        Dispatcher([FakeEngine(budget=100)]).run([request(50, 1, 0.0), request(150, 1, 1.0)])


def test_partition_balances_bytes_and_is_deterministic() -> None:
    sizes = [500, 100, 300, 300, 200, 100]
    plan = partition(sizes, 2)
    assert plan == partition(sizes, 2)
    assert sorted(plan[0] + plan[1]) == list(range(6))
    loads = [sum(sizes[i] for i in share) for share in plan]
    assert abs(loads[0] - loads[1]) <= 100


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        reqs = [request(s, 1 + i % 3, float(i)) for i, s in enumerate([300, 120, 80, 250, 60, 60, 140])]
        engine = FakeEngine(budget=400, slots=2)
        placed = serve_on_ranks(reqs, engine, lambda q: q.arrays["bytes"])
        out.put((rank, None if placed is None else [(p.index, p.engine, float(p.result["solution"][0]))
                                                    for p in placed], sorted(engine.admitted)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_by_footprint_and_gather_in_request_order() -> None:
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = dict((r, (placed, admitted)) for r, placed, admitted in (out.get(timeout=5) for _ in range(2)))
    placed = got[0][0]
    assert got[1][0] is None
    assert [i for i, _, _ in placed] == list(range(7))
    assert [v for _, _, v in placed] == [2.0 * i for i in range(7)]
    plan = partition([300, 120, 80, 250, 60, 60, 140], 2)
    for index, rank, _ in placed:
        assert index in plan[rank]
    assert sorted(got[0][1] + got[1][1]) == [float(i) for i in range(7)]
