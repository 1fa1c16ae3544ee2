"""Mixed-precision iterative refinement: configuration, results and the solve entry.

Mirrors src/electrical/matrix_free_mpir_fem/solver.py of pcb-analysis
(MPIRConfig :52-79, MPIRStep :82-87, MPIRResult :90-100, solve_mpir
:580-698).  The whole refinement runs on the device through the system's
``native_solve_mpir`` hook (the hook the reference's own solve_mpir consults
first, solver.py:612-635); there is no host PCG to fall back to.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Protocol

import numpy as np

LOW_RUNTIME_NAME = "b200-fp32"


class MatrixFreeMPIRSystem(Protocol):
    """Split-precision operator contract (reference solver.py:16-38)."""

    size: int
    high_dtype: Any
    inner_solver: str

    def apply_high(self, vector: np.ndarray) -> np.ndarray: ...

    def apply_low(self, vector: Any) -> Any: ...

    def diagonal_low(self) -> Any: ...


@dataclass(frozen=True)
class MPIRConfig:
    """Accuracy and work limits of the nested solve (reference solver.py:52-79)."""

    relative_tolerance: float = 1.0e-10
    absolute_tolerance: float = 0.0
    inner_relative_tolerance: float = 2.0e-3
    max_outer_iterations: int = 8
    max_inner_iterations: int = 200
    gmres_restart: int = 24

    def __post_init__(self) -> None:
        for name in ("relative_tolerance", "absolute_tolerance", "inner_relative_tolerance"):
            value = float(getattr(self, name))
            if not np.isfinite(value) or value < 0.0:
                raise ValueError(f"{name} must be finite and non-negative")
        if self.relative_tolerance == 0.0 and self.absolute_tolerance == 0.0:
            raise ValueError("at least one outer tolerance must be positive")
        if not 0.0 < self.inner_relative_tolerance < 1.0:
            raise ValueError("inner_relative_tolerance must be between zero and one")
        if self.max_outer_iterations < 1 or self.max_inner_iterations < 1:
            raise ValueError("iteration limits must be positive")
        if self.gmres_restart < 2:
            raise ValueError("gmres_restart must be at least two")


@dataclass(frozen=True)
class MPIRStep:
    outer_iteration: int
    high_relative_residual: float
    inner_iterations: int
    inner_relative_residual: float


@dataclass(frozen=True)
class MPIRResult:
    solution: np.ndarray
    converged: bool
    outer_iterations: int
    inner_iterations: int
    relative_residual: float
    high_operator_applications: int
    low_operator_applications: int
    low_runtime: str
    history: tuple[MPIRStep, ...]


def result_from_native(result: tuple, low_runtime: str = LOW_RUNTIME_NAME) -> MPIRResult:
    solution, converged, outer, inner, rel, n_high, n_low, steps = result
    return MPIRResult(
        solution=np.asarray(solution, dtype=np.float64),
        converged=bool(converged),
        outer_iterations=int(outer),
        inner_iterations=int(inner),
        relative_residual=float(rel),
        high_operator_applications=int(n_high),
        low_operator_applications=int(n_low),
        low_runtime=low_runtime,
        history=tuple(MPIRStep(int(a), float(b), int(c), float(d)) for a, b, c, d in steps),
    )


def solve_mpir(
    system: Any,
    rhs: np.ndarray,
    *,
    config: MPIRConfig | None = None,
    initial_guess: np.ndarray | None = None,
) -> MPIRResult:
    """Solve A x = rhs with FP64 refinement around an FP32 Jacobi PCG, on the device."""

    config = config or MPIRConfig()
    rhs_high = np.asarray(rhs, dtype=np.float64).reshape(-1)
    if rhs_high.size != system.size:
        raise ValueError(f"rhs has size {rhs_high.size}, expected {system.size}")
    if not np.all(np.isfinite(rhs_high)):
        raise ValueError("rhs must contain only finite values")
    if initial_guess is not None:
        guess = np.asarray(initial_guess, dtype=np.float64).reshape(-1)
        if guess.size != system.size:
            raise ValueError(f"initial_guess has size {guess.size}, expected {system.size}")
    else:
        guess = None
    native = getattr(system, "native_solve_mpir", None)
    if native is None:
        raise TypeError("solve_mpir runs on the device: the system must provide native_solve_mpir")
    outcome = native(rhs_high, config, guess)
    if outcome is None:
        raise RuntimeError("the system declined the device solve")
    return result_from_native(outcome, getattr(getattr(system, "runtime", None), "name", LOW_RUNTIME_NAME))
