"""Batched and served steady solves on one device: many boards resident in HBM.

The reference solves one board per call (src/thermal/matrix_free_mpir_fem/
solve.py:39-280).  Here a :class:`~pcb_analysis_b200._native.BatchEngine`
keeps every admitted board's grid, coefficients and iterates in HBM and runs
the MPIR solves of all of them in one set of graph-captured kernels; this
module feeds it:

* :func:`board_request` turns a ``ThermalConductionProblem`` into the prepared
  arrays and right-hand side of the linear solve (the same system the single
  solve builds, reference operator.py:89-440);
* :func:`solve_batch` admits a list of boards as room allows and runs them to
  completion;
* :func:`serve` is the request loop: requests arrive over time, each is
  admitted when a slot and its HBM bytes are free, boards finish and leave
  while others run (continuous batching), and every request's latency from
  arrival to result is recorded.
"""

from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field
from typing import Any, Iterable, Sequence

import numpy as np

from ._native import BatchEngine
from .mpir import MPIRConfig, MPIRResult, result_from_native


@dataclass
class BoardRequest:
    """One linear solve: the prepared board arrays (the arguments of
    ``DeviceSystem``) and its right-hand side in the reference's node order."""

    arrays: dict[str, np.ndarray]
    rhs: np.ndarray
    initial_guess: np.ndarray | None = None
    tag: Any = None

    @property
    def nodes(self) -> int:
        return int(self.rhs.size)


@dataclass
class ServedResult:
    request: BoardRequest
    result: MPIRResult
    arrival_s: float
    admitted_s: float
    finished_s: float

    @property
    def latency_s(self) -> float:
        return self.finished_s - self.arrival_s


@dataclass
class ServeReport:
    results: list[ServedResult]
    wall_s: float
    engine: dict[str, int] = field(default_factory=dict)

    @property
    def solves_per_s(self) -> float:
        return len(self.results) / self.wall_s if self.wall_s > 0 else 0.0

    def latency_percentile(self, q: float) -> float:
        return float(np.percentile([r.latency_s for r in self.results], q))


def board_request(problem: Any, *, reference_temperature_k: float | None = None, device_id: int = 0,
                  tag: Any = None) -> BoardRequest:
    """Prepared arrays and right-hand side of ``problem``'s steady solve for
    the rise above the reference temperature (its default: the mean ambient of
    the first convection boundary, reference operator.py:389-397)."""

    from .thermal.operator import MatrixFreeThermalOperator

    op = MatrixFreeThermalOperator(problem, preconditioner="jacobi", device_id=device_id)
    try:
        reference = op.default_reference_temperature() if reference_temperature_k is None else reference_temperature_k
        rhs = op.build_rhs(float(reference))
        arrays = op.system_arrays()
    finally:
        op.close()
    return BoardRequest(arrays=arrays, rhs=rhs, tag=tag if tag is not None else float(reference))


def _result(raw: dict[str, Any]) -> MPIRResult:
    return result_from_native((raw["solution"], raw["converged"], raw["outer_iterations"], raw["inner_iterations"],
                               raw["relative_residual"], raw["high_operator_applications"],
                               raw["low_operator_applications"], raw["history"]))


def solve_batch(requests: Sequence[BoardRequest], config: MPIRConfig | None = None, *,
                engine: BatchEngine | None = None, **engine_options: Any) -> list[MPIRResult]:
    """Solve every request on one device; results in request order.

    Boards are admitted in order as slots and budget allow, so a list larger
    than the engine still runs to completion."""

    report = serve(requests, [0.0] * len(requests), config, engine=engine, **engine_options)
    by_index = {id(r.request): r.result for r in report.results}
    return [by_index[id(q)] for q in requests]


def serve(requests: Sequence[BoardRequest], arrivals_s: Iterable[float], config: MPIRConfig | None = None, *,
          engine: BatchEngine | None = None, max_steps: int = 1 << 40, **engine_options: Any) -> ServeReport:
    """Continuous-batching request loop.

    Request ``i`` arrives ``arrivals_s[i]`` seconds after the start.  Arrived
    requests are admitted first come first served whenever the engine has a
    slot and the bytes for them (a refused head waits; nothing overtakes it);
    the engine runs graph chunks over everything resident; finished boards are
    collected at once, which frees their slot and bytes for the next arrival.
    """

    config = config or MPIRConfig()
    arrivals = [float(a) for a in arrivals_s]
    if len(arrivals) != len(requests):
        raise ValueError("one arrival time per request")
    own = engine is None
    if own:
        max_slabs = max(int(np.asarray(q.arrays["slab_thickness_m"]).size) for q in requests) if requests else 1
        options = dict(capacity=min(256, max(1, len(requests))), max_slabs=max(1, max_slabs))
        options.update(engine_options)
        engine = BatchEngine(**options)
    order = sorted(range(len(requests)), key=lambda i: arrivals[i])
    pending = deque(order)
    waiting: deque[int] = deque()
    in_flight: dict[int, tuple[int, float]] = {}
    results: list[ServedResult] = []
    t0 = time.perf_counter()
    try:
        steps = 0
        while pending or waiting or in_flight:
            now = time.perf_counter() - t0
            while pending and arrivals[pending[0]] <= now:
                waiting.append(pending.popleft())
            while waiting:
                i = waiting[0]
                q = requests[i]
                ticket = engine.submit(q.arrays, q.rhs, config, q.initial_guess)
                if ticket is None:
                    if not in_flight:
                        raise MemoryError("a request does not fit the engine even when it is empty")
                    break
                waiting.popleft()
                in_flight[ticket] = (i, time.perf_counter() - t0)
            if in_flight:
                engine.step()
                steps += 1
                if steps > max_steps:
                    raise TimeoutError("the request loop exceeded its step limit")
                for ticket in engine.finished():
                    i, admitted = in_flight.pop(ticket)
                    raw = engine.collect(ticket)
                    results.append(ServedResult(requests[i], _result(raw), arrivals[i], admitted,
                                                time.perf_counter() - t0))
            elif pending:
                time.sleep(max(0.0, min(0.01, arrivals[pending[0]] - (time.perf_counter() - t0))))
        wall = time.perf_counter() - t0
        info = engine.info()
    finally:
        if own:
            engine.close()
    return ServeReport(results=results, wall_s=wall, engine=info)


def poisson_arrivals(count: int, rate_per_s: float, seed: int = 0) -> list[float]:
    """Arrival times of a Poisson stream: exponential gaps of mean 1/rate."""

    rng = np.random.default_rng(seed)
    return [float(t) for t in np.cumsum(rng.exponential(1.0 / rate_per_s, count))]
