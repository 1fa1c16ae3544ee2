"""Steady conduction solve on the device.

The public entry keeps the call surface of pcb-analysis's
``solve_thermal_conduction`` (src/thermal/matrix_free_mpir_fem/solve.py:19-79):
its keywords with their defaults and its solution record.  The work happens
in :class:`~pcb_analysis_b200.thermal.session.ResidentSolve`, which holds one
prepared device system for all the linear solves of the call.
"""

from __future__ import annotations

import dataclasses
from dataclasses import dataclass
from typing import Any

import numpy as np

from ..mpir import MPIRConfig, MPIRResult
from .mesh import Preconditioner
from .operator import B200Float32Runtime
from .problem import ThermalConductionProblem
from .session import ResidentSolve


@dataclass(frozen=True)
class ThermalConductionSolution:
    """Nodal temperatures and the heat budget of one steady solve.

    The fields are the reference's (solve.py:19-36): temperatures on the node
    grid (NaN on void nodes), -k grad T per element, the extremes, the heat
    put in, removed per convection boundary and through fixed nodes, the
    budget's error and the refinement record; with radiation also the heat
    radiated per boundary and the Newton loop's outcome; for a backward-Euler
    step the heat stored."""

    temperature_k: np.ndarray
    heat_flux_w_per_m2: np.ndarray
    max_temperature_k: float
    min_temperature_k: float
    total_heat_input_w: float
    convective_heat_w: np.ndarray
    fixed_temperature_heat_w: float
    heat_balance_error_w: float
    solve: MPIRResult
    radiative_heat_w: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))
    radiation_iterations: int = 0
    radiation_converged: bool = True
    radiation_change_k: float = 0.0
    stored_heat_w: float = 0.0


def solve_thermal_conduction(
    problem: ThermalConductionProblem,
    *,
    config: MPIRConfig | None = None,
    runtime: B200Float32Runtime | None = None,
    backend: str | None = None,
    device_id: int = 0,
    initial_temperature_k: np.ndarray | float | None = None,
    preconditioner: Preconditioner = "two-level",
    coarse_block_nodes: int | None = None,
    reference_temperature_k: float | None = None,
    native: bool | None = None,
    radiation_max_iterations: int = 25,
    radiation_tolerance_k: float = 1.0e-4,
) -> ThermalConductionSolution:
    """Solve steady heat conduction in a layered PCB with device MPIR.

    The unknown is the rise above ``reference_temperature_k`` (default: the
    first convective ambient, else the mean fixed temperature).
    ``initial_temperature_k`` warm-starts the refinement.  With
    ``problem.radiation`` the radiating faces are Newton-linearised and the
    linear solve repeats until the temperatures move by less than
    ``radiation_tolerance_k``.
    """

    return _solve(
        problem,
        config=config,
        initial_temperature_k=initial_temperature_k,
        reference_temperature_k=reference_temperature_k,
        radiation_max_iterations=radiation_max_iterations,
        radiation_tolerance_k=radiation_tolerance_k,
        runtime=runtime,
        backend=backend,
        device_id=device_id,
        preconditioner=preconditioner,
        coarse_block_nodes=coarse_block_nodes,
        native=native,
    )


def _solve(
    problem: ThermalConductionProblem,
    *,
    config: MPIRConfig | None = None,
    initial_temperature_k: Any = None,
    reference_temperature_k: float | None = None,
    radiation_max_iterations: int = 25,
    radiation_tolerance_k: float = 1.0e-4,
    capacity_per_s: np.ndarray | None = None,
    previous_temperature_k: Any = None,
    **device_options: Any,
) -> ThermalConductionSolution:
    """One solve on a system of its own (prepared, solved, released)."""

    with ResidentSolve(**device_options) as session:
        return session.steady(
            problem,
            config=config,
            initial_temperature_k=initial_temperature_k,
            reference_temperature_k=reference_temperature_k,
            radiation_max_iterations=radiation_max_iterations,
            radiation_tolerance_k=radiation_tolerance_k,
            capacity_per_s=capacity_per_s,
            previous_temperature_k=previous_temperature_k,
        )
