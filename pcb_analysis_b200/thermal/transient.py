"""Transient conduction by backward Euler on one resident device system.

An implicit step of the lumped-capacity heat equation,

    (K + R + C / dt) T_{n+1} = q + R T_amb + C / dt T_n,

is the steady operator with C / dt added on the diagonal where the Robin
conductance sits (the scheme of pcb-analysis's
src/thermal/matrix_free_mpir_fem/transient.py:1-24).  The whole march runs on
one :class:`~pcb_analysis_b200.thermal.session.ResidentSolve`: a step with the
previous dt only builds its right-hand side, a new dt rewrites the lumped
totals, the diagonal and the preconditioner on the device, and the Newton
loop of a radiating board rewrites its linearised faces -- the board is
prepared once.

The call surface is the reference's (transient.py:45-258): TimeSchedule with
its uniform and geometric constructors, TransientStep,
TransientThermalSolution and solve_thermal_transient with the same keywords,
the same stopping rule and the same record per step.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Any, Iterator

import numpy as np

from ..mpir import MPIRConfig
from .mesh import Preconditioner
from .operator import B200Float32Runtime
from .problem import ThermalConductionProblem
from .session import ResidentSolve
from .solve import ThermalConductionSolution


@dataclass(frozen=True)
class TimeSchedule:
    """Time points 0 = t_0 < t_1 < ... < t_N of a transient run, in seconds."""

    times_s: tuple[float, ...]

    def __post_init__(self) -> None:
        points = np.asarray(self.times_s, dtype=np.float64).ravel()
        if points.size < 2 or points[0] != 0.0:
            raise ValueError("times_s must start at 0 and hold at least one step")
        if not (np.isfinite(points).all() and (np.diff(points) > 0.0).all()):
            raise ValueError("times_s must be finite and strictly increasing")
        object.__setattr__(self, "times_s", tuple(map(float, points)))

    @property
    def steps_s(self) -> np.ndarray:
        return np.diff(np.asarray(self.times_s))

    @property
    def end_s(self) -> float:
        return self.times_s[-1]

    @classmethod
    def uniform(cls, step_s: float, end_s: float) -> "TimeSchedule":
        """Steps of `step_s` up to the first multiple of it at or past `end_s`."""

        if not (step_s > 0.0 and end_s > 0.0):
            raise ValueError("step_s and end_s must be positive")
        steps = math.ceil(end_s / step_s - 1.0e-9)
        return cls(tuple(step_s * np.arange(steps + 1)))

    @classmethod
    def geometric(cls, first_step_s: float, end_s: float, *, growth: float = 1.5,
                  max_step_s: float | None = None) -> "TimeSchedule":
        """Steps growing by the factor `growth` from `first_step_s` (at most
        `max_step_s`), the last one shortened to end at `end_s`."""

        if not (first_step_s > 0.0 and end_s > 0.0):
            raise ValueError("first_step_s and end_s must be positive")
        if growth < 1.0:
            raise ValueError("growth must be at least one")
        cap = math.inf if max_step_s is None else float(max_step_s)
        return cls((0.0, *_growing_points(float(first_step_s), float(end_s), float(growth), cap)))


def _growing_points(first: float, end: float, growth: float, cap: float) -> Iterator[float]:
    now, step = 0.0, first
    while now < end - 1.0e-12 * end:
        now = min(now + step, end)
        yield now
        step = min(step * growth, cap)


@dataclass(frozen=True)
class TransientStep:
    index: int
    time_s: float
    step_s: float
    max_temperature_k: float
    max_change_k: float
    stored_heat_w: float
    convective_heat_w: float
    radiative_heat_w: float
    heat_balance_error_w: float
    inner_iterations: int
    radiation_iterations: int
    converged: bool


@dataclass(frozen=True)
class TransientThermalSolution:
    """Temperature history of a backward-Euler run and the last step's budget."""

    times_s: np.ndarray
    temperature_k: np.ndarray  # (len(times_s), *node_shape); only the final field with store="final"
    history: tuple[TransientStep, ...]
    final: ThermalConductionSolution
    reached_steady: bool

    @property
    def max_temperature_k(self) -> np.ndarray:
        return np.asarray([step.max_temperature_k for step in self.history])

    @property
    def final_temperature_k(self) -> np.ndarray:
        return self.temperature_k[-1]


def _start_field(problem: ThermalConductionProblem, guess: Any) -> np.ndarray:
    """T_0: the guess, else a uniform field at the first convective ambient,
    the first radiative one, or the mean fixed temperature; fixed nodes at
    their prescribed values."""

    mesh = problem.mesh
    if guess is None:
        if problem.convection:
            level = problem.convection[0].mean_ambient_k()
        elif problem.radiation:
            level = problem.radiation[0].mean_ambient_k()
        else:
            level = float(np.mean(problem.fixed_temperature_k[problem.fixed_temperature_mask]))
        field = np.full(mesh.node_shape, level)
    else:
        values = np.asarray(guess, dtype=np.float64)
        field = np.full(mesh.node_shape, float(values)) if values.ndim == 0 else values.reshape(mesh.node_shape).copy()
        if not np.isfinite(field[mesh.active_nodes]).all():
            raise ValueError("initial_temperature_k must be finite on active nodes")
    return np.where(problem.fixed_temperature_mask, problem.fixed_temperature_k, field)


class _Record:
    """Fields kept by a march: every step's, or the latest only."""

    def __init__(self, keep_all: bool, active: np.ndarray, start: np.ndarray) -> None:
        self.keep_all = keep_all
        self.active = active
        self.times = [0.0]
        self.fields = [self._shown(start)]

    def _shown(self, field: np.ndarray) -> np.ndarray:
        return np.where(self.active, field, np.nan)

    def add(self, time_s: float, field: np.ndarray) -> np.ndarray:
        shown = self._shown(field)
        if self.keep_all:
            self.times.append(time_s)
            self.fields.append(shown)
        else:
            self.times, self.fields = [time_s], [shown]
        return shown

    def arrays(self) -> tuple[np.ndarray, np.ndarray]:
        return np.asarray(self.times), np.stack(self.fields)


def solve_thermal_transient(
    problem: ThermalConductionProblem,
    schedule: TimeSchedule,
    *,
    initial_temperature_k: np.ndarray | float | None = None,
    store: str = "all",
    until_steady: bool = False,
    steady_tolerance_k_per_s: float = 1.0e-3,
    config: MPIRConfig | None = None,
    runtime: B200Float32Runtime | None = None,
    backend: str | None = None,
    device_id: int = 0,
    preconditioner: Preconditioner = "two-level",
    coarse_block_nodes: int | None = None,
    native: bool | None = None,
    radiation_max_iterations: int = 25,
    radiation_tolerance_k: float = 1.0e-4,
) -> TransientThermalSolution:
    """March `problem` from `initial_temperature_k` through `schedule` by backward Euler.

    The mesh must carry volumetric_heat_capacity_j_per_m3_k.  The initial
    field defaults to the first convective (else radiative) ambient, else the
    mean fixed temperature.  store="all" keeps every field, "final" only the
    last.  With until_steady the march stops once max |T_{n+1} - T_n| / dt
    falls below steady_tolerance_k_per_s.
    """

    if store not in ("all", "final"):
        raise ValueError("store must be 'all' or 'final'")
    if not steady_tolerance_k_per_s > 0.0:
        raise ValueError("steady_tolerance_k_per_s must be positive")
    mesh = problem.mesh
    capacity = mesh.nodal_heat_capacity_j_per_k().reshape(-1)
    field = _start_field(problem, initial_temperature_k)
    active = mesh.active_nodes
    record = _Record(store == "all", active, field)
    history: list[TransientStep] = []
    last: ThermalConductionSolution | None = None
    steady = False
    device = dict(runtime=runtime, backend=backend, device_id=device_id, preconditioner=preconditioner,
                  coarse_block_nodes=coarse_block_nodes, native=native)
    with ResidentSolve(**device) as session:
        for index, (time_s, step_s) in enumerate(zip(schedule.times_s[1:], map(float, schedule.steps_s)), start=1):
            last = session.steady(
                problem, config=config, initial_temperature_k=field, capacity_per_s=capacity / step_s,
                previous_temperature_k=field, radiation_max_iterations=radiation_max_iterations,
                radiation_tolerance_k=radiation_tolerance_k)
            solved = np.where(np.isfinite(last.temperature_k), last.temperature_k, field)
            moved = float(np.abs(solved - field)[active].max()) if active.any() else 0.0
            field = solved
            shown = record.add(float(time_s), field)
            history.append(TransientStep(
                index=index, time_s=float(time_s), step_s=step_s, max_temperature_k=float(np.nanmax(shown)),
                max_change_k=moved, stored_heat_w=last.stored_heat_w,
                convective_heat_w=float(np.sum(last.convective_heat_w)),
                radiative_heat_w=float(np.sum(last.radiative_heat_w)),
                heat_balance_error_w=last.heat_balance_error_w, inner_iterations=last.solve.inner_iterations,
                radiation_iterations=last.radiation_iterations,
                converged=last.solve.converged and last.radiation_converged))
            if until_steady and moved / step_s <= steady_tolerance_k_per_s:
                steady = True
                break
    assert last is not None
    times, fields = record.arrays()
    return TransientThermalSolution(times_s=times, temperature_k=fields, history=tuple(history), final=last,
                                    reached_steady=steady)


__all__ = ["TimeSchedule", "TransientStep", "TransientThermalSolution", "solve_thermal_transient"]
