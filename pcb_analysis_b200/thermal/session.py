"""One resident device system for every linear solve of a call.

A steady solve of a radiating board is a sequence of linear solves that
differ only in their linearised Robin faces; a transient march is a sequence
that differs in C / dt and the previous field; each of those is in turn at
most two MPIR runs (a second one when the first stalls far above its
reference temperature).  :class:`ResidentSolve` keeps the prepared system,
its preconditioner and its graphs in HBM for the whole sequence: between
solves it rewrites only the Robin totals (tb_set_convection) or the capacity
(tb_set_capacity) on the device, where the reference prepares a new system
for each one (src/thermal/matrix_free_mpir_fem/solve.py:126-280,
transient.py:129-258).

What a caller of the reference sees is unchanged: the temperatures, the heat
budget, the MPIR counts and history, the Newton iteration count, and the
error messages.
"""

from __future__ import annotations

import dataclasses
import math
from typing import Any, Iterator

import numpy as np

from ..mpir import MPIRConfig, MPIRResult, result_from_native
from .operator import MatrixFreeThermalOperator
from .problem import ThermalConductionProblem

# MPIR counts that add up when a stalled run is resumed.
_COUNTS = ("outer_iterations", "inner_iterations", "high_operator_applications", "low_operator_applications")


def default_config() -> MPIRConfig:
    """The refinement limits a solve uses when the caller gives none."""

    return MPIRConfig(max_outer_iterations=16)


def finite_or_zero(field: Any) -> np.ndarray | None:
    """Flat FP64 copy of an optional node field with NaN (void nodes) as 0."""

    if field is None:
        return None
    flat = np.asarray(field, dtype=np.float64).reshape(-1)
    return np.nan_to_num(flat, nan=0.0, posinf=0.0, neginf=0.0) if not np.all(np.isfinite(flat)) else flat.copy()


def _resumed(first: MPIRResult, second: MPIRResult) -> MPIRResult:
    """The record of a refinement run in two parts: counts and history of
    both, solution, residual and convergence of the second."""

    totals = {name: getattr(first, name) + getattr(second, name) for name in _COUNTS}
    return dataclasses.replace(second, history=tuple(first.history) + tuple(second.history), **totals)


class ResidentSolve:
    """Owner of the device system shared by the linear solves of one call."""

    def __init__(self, **operator_options: Any) -> None:
        self._options = operator_options
        self._operator: MatrixFreeThermalOperator | None = None
        self._capacity: np.ndarray | None = None

    # ------------------------------------------------------------ lifetime
    def close(self) -> None:
        if self._operator is not None:
            self._operator.close()
            self._operator = None

    def __enter__(self) -> "ResidentSolve":
        return self

    def __exit__(self, *exc: object) -> None:
        self.close()

    # ------------------------------------------------------------ binding
    def bind(self, problem: ThermalConductionProblem, capacity_per_s: np.ndarray | None = None
             ) -> MatrixFreeThermalOperator:
        """The resident operator, carrying `problem`'s boundaries and the
        given C / dt (made on first use)."""

        op = self._operator
        if op is None:
            op = MatrixFreeThermalOperator(problem, capacity_per_s=capacity_per_s, **self._options)
            self._operator = op
            self._capacity = None if capacity_per_s is None else np.array(capacity_per_s, dtype=np.float64)
            return op
        if problem is not op.problem and problem.convection is not op.problem.convection:
            op.replace_boundaries(problem)
        if capacity_per_s is not None and not (
                self._capacity is not None and np.array_equal(self._capacity, capacity_per_s)):
            op.set_capacity_per_s(capacity_per_s)
            self._capacity = np.array(capacity_per_s, dtype=np.float64)
        return op

    # ------------------------------------------------------------ solves
    def steady(
        self,
        problem: ThermalConductionProblem,
        *,
        config: MPIRConfig | None = None,
        initial_temperature_k: Any = None,
        reference_temperature_k: float | None = None,
        radiation_max_iterations: int = 25,
        radiation_tolerance_k: float = 1.0e-4,
        capacity_per_s: np.ndarray | None = None,
        previous_temperature_k: Any = None,
    ):
        """One steady (or backward-Euler) solve of `problem`, with the Newton
        loop of its radiating faces when it has any."""

        previous = finite_or_zero(previous_temperature_k)
        if not problem.radiation:
            op = self.bind(problem, capacity_per_s)
            return self.linear(op, problem, config, initial_temperature_k, reference_temperature_k, previous)
        if radiation_max_iterations < 1:
            raise ValueError("radiation_max_iterations must be positive")
        if not radiation_tolerance_k > 0.0:
            raise ValueError("radiation_tolerance_k must be positive")
        plain = len(problem.convection)
        last = None
        steps = 0
        change = math.inf
        for steps, (solution, change) in enumerate(
                self._newton(problem, config, initial_temperature_k, reference_temperature_k, capacity_per_s,
                             previous, radiation_max_iterations), start=1):
            last = solution
            if change <= radiation_tolerance_k:
                break
        assert last is not None
        removed = last.convective_heat_w
        return dataclasses.replace(
            last,
            convective_heat_w=removed[:plain],
            radiative_heat_w=removed[plain:],
            radiation_iterations=steps,
            radiation_converged=bool(change <= radiation_tolerance_k and last.solve.converged),
            radiation_change_k=change,
        )

    def _newton(self, problem, config, guess, reference, capacity_per_s, previous, limit
                ) -> Iterator[tuple[Any, float]]:
        """Newton iterates of the radiating faces: each linearises them at the
        current field (h = 4 e sigma T^3 about T), solves, and yields the
        solution with the largest change of the field."""

        mesh = problem.mesh
        field = _newton_start(problem, guess)
        for _ in range(limit):
            faces = tuple(boundary.linearize(mesh, field) for boundary in problem.radiation)
            linear = dataclasses.replace(problem, convection=tuple(problem.convection) + faces, radiation=())
            op = self.bind(linear, capacity_per_s)
            solution = self.linear(op, linear, config, field, reference, previous)
            moved = np.where(np.isfinite(solution.temperature_k), solution.temperature_k, field)
            delta = float(np.max(np.abs(moved - field)))
            field = moved
            yield solution, delta

    def linear(self, op: MatrixFreeThermalOperator, problem: ThermalConductionProblem, config: MPIRConfig | None,
               guess: Any, reference_k: float | None, previous: np.ndarray | None):
        """MPIR solve of the linear problem on the bound operator, then the
        heat budget on the device."""

        from .solve import ThermalConductionSolution

        reference = op.default_reference_temperature() if reference_k is None else float(reference_k)
        if not math.isfinite(reference):
            raise ValueError("reference_temperature_k must be finite")
        settings = config if config is not None else default_config()
        start = None if guess is None else _rise_guess(op, guess, reference)
        record, rise = _solve_in_hbm(op, reference, previous, settings, start)
        # the host free mask (a pass over every node) is needed only to restart
        free = None if record.converged else op.free_nodes.reshape(-1)
        if free is not None and free.any():
            # The FP64 residual of K theta cannot fall below about
            # eps ||K|| ||theta||: a board far above its reference stalls.
            # Moving the reference to the mean free rise and resuming from
            # the iterate takes that offset out of theta.
            offset = float(np.mean(record.solution[free]))
            if offset != 0.0:
                reference += offset
                again, rise = _solve_in_hbm(op, reference, previous, settings, record.solution - offset)
                record = _resumed(record, again)
        post = op.device_system.postprocess_rise_device(rise, reference, previous, temperature=True)
        temperature = post["temperature"].reshape(problem.mesh.node_shape)  # rise + reference, formed on the device
        if not problem.mesh.is_full:
            temperature = np.where(op.active_nodes, temperature, np.nan)
        removed = post["convective_heat_w"]
        balance = post["total_heat_input_w"] - float(np.sum(removed)) - post["fixed_temperature_heat_w"] \
            - post["stored_heat_w"]
        return ThermalConductionSolution(
            temperature_k=temperature,
            heat_flux_w_per_m2=post["heat_flux"],
            max_temperature_k=post["temperature_extrema"][1],
            min_temperature_k=post["temperature_extrema"][0],
            total_heat_input_w=post["total_heat_input_w"],
            convective_heat_w=removed,
            fixed_temperature_heat_w=post["fixed_temperature_heat_w"],
            heat_balance_error_w=balance,
            solve=record,
            stored_heat_w=post["stored_heat_w"],
        )


def _solve_in_hbm(op: MatrixFreeThermalOperator, reference: float, previous: np.ndarray | None,
                  settings: MPIRConfig, start: np.ndarray | None) -> tuple[MPIRResult, Any]:
    """The MPIR solve of the rise over `reference` with its right-hand side
    built, and its solution left, in HBM: the solve ``solve_mpir(op,
    op.build_rhs(reference, previous), ...)`` does, bit for bit, without the
    right-hand side's round trip through the host.  The solution is read
    back once (the record's ``solution``); the device copy is returned for
    the post-processing."""

    import torch

    dev = op.device_system
    device = torch.device("cuda", dev.device)
    n = op.size
    prev = None
    if previous is not None:
        prev = torch.from_numpy(np.ascontiguousarray(np.asarray(previous, dtype=np.float64).reshape(-1))).to(device)
    rhs = torch.empty(n, dtype=torch.float64, device=device)
    dev.build_rhs_device(reference, rhs, prev)
    if not bool(torch.isfinite(rhs).all()):
        raise ValueError("rhs must contain only finite values")
    if start is None:
        rise = torch.zeros(n, dtype=torch.float64, device=device)
    else:
        guess = np.ascontiguousarray(np.asarray(start, dtype=np.float64).reshape(-1))
        if guess.size != n:
            raise ValueError(f"initial_guess has size {guess.size}, expected {n}")
        rise = torch.from_numpy(guess).to(device)
    out = dev.solve_mpir_device(rhs, rise, settings)
    solution = dev.download(rise)
    record = result_from_native((solution, out["converged"], out["outer_iterations"], out["inner_iterations"],
                                 out["relative_residual"], out["high_operator_applications"],
                                 out["low_operator_applications"], out["history"]), op.runtime.name)
    return record, rise


def _rise_guess(op: MatrixFreeThermalOperator, guess: Any, reference: float) -> np.ndarray:
    """Warm start of the refinement as a rise over `reference`: the guess,
    with fixed nodes at their prescribed value (void nodes at the reference)."""

    values = np.asarray(guess, dtype=np.float64)
    flat = np.full(op.size, float(values)) if values.ndim == 0 else values.reshape(-1)
    if flat.size != op.size:
        raise ValueError("initial_temperature_k must hold one value per node")
    pinned = op.fixed_nodes.reshape(-1)
    held = op.fixed_temperature_k.reshape(-1) + reference * ~op.active_nodes.reshape(-1)
    return np.where(pinned, held, flat) - reference


def _newton_start(problem: ThermalConductionProblem, guess: Any) -> np.ndarray:
    """Field the first linearisation is taken at: the guess (void nodes at the
    first radiative ambient), else the first convective ambient, else the
    first radiative one."""

    shape = problem.mesh.node_shape
    radiant = problem.radiation[0].mean_ambient_k()
    if guess is None:
        level = problem.convection[0].mean_ambient_k() if problem.convection else float(radiant)
        return np.full(shape, level)
    values = np.asarray(guess, dtype=np.float64)
    field = np.full(shape, float(values)) if values.ndim == 0 else values.reshape(shape).copy()
    field[~np.isfinite(field)] = radiant
    return field
