"""Request-level data parallelism over per-GPU batch engines (replicas).

Boards are independent, so several GPUs serve one stream of requests as
replicas: every GPU owns a :class:`~pcb_analysis_b200._native.BatchEngine`,
and a host dispatcher decides where each request runs.  There is no device
collective: a board's solve never leaves its GPU, so its bits are those of
the same board on one GPU.

* :class:`Dispatcher` -- one host process drives several engines (one per
  visible device, or any object with the engine's submit / step / finished /
  collect / info calls).  Requests are taken first come first served; the
  head request goes to the engine with the most free bytes of its budget that
  admits it (the engine checks the board's resident + transient footprint,
  tb_engine_footprint, against its budget and slots); a head that no engine
  can take now waits until one frees memory -- nothing overtakes it -- and a
  head that no idle engine can ever take is refused with MemoryError.
  Results come back in request order, with the engine each ran on.
* :func:`serve_on_ranks` -- one process per GPU under torch.distributed.
  Every rank computes the same partition of the request list from the
  footprints alone (largest first, each to the rank with the fewest bytes
  assigned so far), so the assignment needs no messages; each rank serves
  its share on its own engine and rank 0 gathers the results in request
  order (``gather_object``: the results are host arrays).
"""

from __future__ import annotations

from collections import deque
from dataclasses import dataclass
from typing import Any, Callable, Protocol, Sequence

from .mpir import MPIRConfig


class Engine(Protocol):
    def submit(self, arrays: dict, rhs: Any, config: Any, initial_guess: Any | None = None) -> int | None: ...

    def step(self) -> int: ...

    def finished(self) -> list[int]: ...

    def collect(self, ticket: int) -> dict: ...

    def info(self) -> dict[str, int]: ...


@dataclass
class Placed:
    """A request's result and the engine that solved it."""

    index: int
    engine: int
    result: dict


def _free_bytes(engine: Engine) -> int:
    info = engine.info()
    return int(info["budget_bytes"]) - int(info["bytes_in_use"])


class Dispatcher:
    """First-come-first-served dispatch of board requests over engines."""

    def __init__(self, engines: Sequence[Engine], config: MPIRConfig | None = None) -> None:
        if not engines:
            raise ValueError("a dispatcher needs at least one engine")
        self.engines = list(engines)
        self.config = config or MPIRConfig()

    def _admit(self, request) -> tuple[int, int] | None:
        """Submit `request` to the engine with the most free bytes that takes
        it; (engine, ticket), or None when none can now."""

        order = sorted(range(len(self.engines)), key=lambda e: (-_free_bytes(self.engines[e]), e))
        for e in order:
            ticket = self.engines[e].submit(request.arrays, request.rhs, self.config, request.initial_guess)
            if ticket is not None:
                return e, ticket
        return None

    def run(self, requests: Sequence[Any], max_rounds: int = 1 << 40) -> list[Placed]:
        """Solve every request; the results in request order."""

        waiting = deque(enumerate(requests))
        flying: dict[tuple[int, int], int] = {}  # (engine, ticket) -> request index
        done: dict[int, Placed] = {}
        for _ in range(max_rounds):
            while waiting:
                placed = self._admit(waiting[0][1])
                if placed is None:
                    if not flying:
                        raise MemoryError(f"request {waiting[0][0]} does not fit any idle engine")
                    break
                flying[placed] = waiting.popleft()[0]
            if not flying:
                break
            busy = {e for e, _ in flying}
            for e in sorted(busy):
                engine = self.engines[e]
                engine.step()
                for ticket in engine.finished():
                    index = flying.pop((e, ticket), None)
                    if index is not None:
                        done[index] = Placed(index, e, engine.collect(ticket))
        if waiting or flying:
            raise RuntimeError("the dispatcher stopped before every request finished")
        return [done[i] for i in range(len(requests))]


def partition(footprints: Sequence[int], ranks: int) -> list[list[int]]:
    """Request indices per rank: largest footprint first, each to the rank
    with the fewest bytes so far (ties: the lower rank); every list in
    request order.  Deterministic, so every rank computes the same plan."""

    if ranks < 1:
        raise ValueError("ranks must be positive")
    load = [0] * ranks
    share: list[list[int]] = [[] for _ in range(ranks)]
    for index in sorted(range(len(footprints)), key=lambda i: (-int(footprints[i]), i)):
        rank = min(range(ranks), key=lambda r: (load[r], r))
        load[rank] += int(footprints[index])
        share[rank].append(index)
    return [sorted(s) for s in share]


def serve_on_ranks(requests: Sequence[Any], engine: Engine, footprint: Callable[[Any], int], *,
                   config: MPIRConfig | None = None, group: Any = None) -> list[Placed] | None:
    """Serve `requests` with one engine per rank of the default (or given)
    process group; rank 0 returns every result in request order (``engine``
    is the rank), the other ranks None."""

    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    plan = partition([footprint(q) for q in requests], world)
    mine = plan[rank]
    local = Dispatcher([engine], config).run([requests[i] for i in mine])
    payload = [(mine[k], p.result) for k, p in enumerate(local)]
    gathered: list[Any] | None = [None] * world if rank == 0 else None
    dist.gather_object(payload, gathered, dst=0, group=group)
    if rank != 0:
        return None
    out: dict[int, Placed] = {}
    for r, part in enumerate(gathered):
        for index, result in part:
            out[index] = Placed(index, r, result)
    return [out[i] for i in range(len(requests))]


__all__ = ["Dispatcher", "Engine", "Placed", "partition", "serve_on_ranks"]
