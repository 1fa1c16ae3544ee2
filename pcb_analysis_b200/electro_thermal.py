"""Staggered electro-thermal coupling on the device solves (reference
multiphysics/staggered_coupling/electro_thermal.py:1-478).

Copper resistivity grows linearly with temperature,
``sigma(T) = sigma_ref / (1 + alpha (T - T_ref))``.  The coupling alternates a
DC solve (:func:`solve_pcb_dc`) with the current conductivity and a thermal
solve (:func:`solve_thermal_conduction`) loaded with that solve's Joule loss,
then re-evaluates the conductivity at the new element temperatures.  Both
solves run the device MPIR path and are warm-started from the previous
iterate; the temperature iterate is relaxed with Aitken's delta-squared
factor.  This module is host control only: every operator action, PCG
iteration and residual runs in the CUDA library.

Voltage drive (two or more voltage terminals) gives a loss ``V^2 / R(T)``
that falls as the copper heats, so the loop contracts.  A problem whose
copper currents are all imposed (no or one voltage terminal) still runs but
warns: its loss ``I^2 R(T)`` rises with temperature and can run away.
"""

from __future__ import annotations

import dataclasses
import warnings
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from .electrical import PCBConductionProblem, PCBConductionSolution, solve_pcb_dc
from .mpir import MPIRConfig
from .thermal import (
    ConvectionBoundary,
    HeatSource,
    LayeredThermalMesh,
    ThermalConductionProblem,
    ThermalConductionSolution,
    solve_thermal_conduction,
)
from .thermal.coupling import element_joule_heat_w, via_joule_heat_sources

COPPER_TEMPERATURE_COEFFICIENT_PER_K = 3.93e-3
CURRENT_DRIVEN_DEPRECATION = (
    "current-driven electro-thermal coupling is deprecated: with fewer than two "
    "voltage terminals the current terminals fix every copper current, so the "
    "loss I^2 R(T) rises with temperature and the board can run away; hold at "
    "least two pads with VoltageTerminal (PCBConductionProblem.voltage_terminals)"
)


@dataclass(frozen=True)
class ElectroThermalScenario:
    """One board: its DC drive, thermal mesh and environment, and the
    resistivity law (reference electro_thermal.py:72-125).  ``layer_slabs[L]``
    is the thermal slab holding electrical layer ``L``."""

    electrical: PCBConductionProblem
    thermal_mesh: LayeredThermalMesh
    layer_slabs: tuple[int, ...]
    convection: tuple[ConvectionBoundary, ...] = ()
    fixed_temperature_mask: np.ndarray | None = None
    fixed_temperature_k: float | np.ndarray | None = None
    extra_heat_sources: tuple[HeatSource, ...] = ()
    extra_element_heat_w: np.ndarray | None = None
    conductivity_reference_temperature_k: float = 293.15
    temperature_coefficient_per_k: float = COPPER_TEMPERATURE_COEFFICIENT_PER_K
    radiation: tuple = ()

    def __post_init__(self) -> None:
        layers, rows, cols = self.electrical.mesh.element_active.shape
        slabs, thermal_rows, thermal_cols = self.thermal_mesh.element_grid_shape
        if (rows, cols) != (thermal_rows, thermal_cols):
            raise ValueError("electrical and thermal meshes must share (rows, cols)")
        if not (np.allclose(self.electrical.mesh.pitch_x_m, self.thermal_mesh.pitch_x_m)
                and np.allclose(self.electrical.mesh.pitch_y_m, self.thermal_mesh.pitch_y_m)):
            raise ValueError("electrical and thermal meshes must share the same grid lines")
        mapping = tuple(int(s) for s in self.layer_slabs)
        if len(mapping) != layers or any(not 0 <= s < slabs for s in mapping):
            raise ValueError("layer_slabs must name one thermal slab per electrical layer")
        alpha = self.temperature_coefficient_per_k
        if not np.isfinite(alpha) or alpha < 0.0:
            raise ValueError("temperature_coefficient_per_k must be finite and non-negative")
        object.__setattr__(self, "layer_slabs", mapping)
        for name in ("convection", "extra_heat_sources", "radiation"):
            object.__setattr__(self, name, tuple(getattr(self, name)))
        # The boundary conditions are checked once here, before any heat exists.
        ThermalConductionProblem(
            self.thermal_mesh,
            convection=self.convection,
            fixed_temperature_mask=self.fixed_temperature_mask,
            fixed_temperature_k=self.fixed_temperature_k,
            heat_sources=self.extra_heat_sources,
            element_heat_w=self.extra_element_heat_w,
            radiation=self.radiation,
        )
        # With at most one voltage terminal (a gauge that absorbs the current
        # terminals' sum) every copper current is imposed.
        if len(self.electrical.voltage_terminals) < 2:
            warnings.warn(CURRENT_DRIVEN_DEPRECATION, DeprecationWarning, stacklevel=3)


@dataclass(frozen=True)
class CouplingConfig:
    """Fixed-point limits (reference electro_thermal.py:128-149).  ``electrical``
    and ``thermal`` are the MPIR configs of the two solves (None: defaults)."""

    max_iterations: int = 20
    temperature_tolerance_k: float = 1.0e-3
    relative_loss_tolerance: float = 1.0e-6
    relaxation: float = 1.0
    aitken: bool = True
    max_relaxation: float = 4.0
    electrical: MPIRConfig | None = None
    thermal: MPIRConfig | None = None

    def __post_init__(self) -> None:
        if self.max_iterations < 1:
            raise ValueError("max_iterations must be positive")
        if self.temperature_tolerance_k <= 0.0 or self.relative_loss_tolerance <= 0.0:
            raise ValueError("tolerances must be positive")
        if not 0.0 < self.relaxation <= self.max_relaxation:
            raise ValueError("relaxation must lie in (0, max_relaxation]")
        if self.max_relaxation < 1.0:
            raise ValueError("max_relaxation must be at least one")


@dataclass(frozen=True)
class CouplingStep:
    """One pass of the loop (reference electro_thermal.py:152-161)."""

    iteration: int
    joule_loss_w: float
    max_temperature_k: float
    temperature_change_k: float
    relative_loss_change: float
    relaxation: float
    electrical_inner_iterations: int
    thermal_inner_iterations: int


@dataclass(frozen=True)
class ElectroThermalResult:
    """The last solves, the conductivity and via resistances the last DC solve
    used, the element temperature of every electrical layer and the history
    (reference electro_thermal.py:164-177)."""

    electrical: PCBConductionSolution
    thermal: ThermalConductionSolution
    conductivity_s_per_m: np.ndarray
    via_resistance_ohm: np.ndarray
    element_temperature_k: np.ndarray
    converged: bool
    iterations: int
    history: tuple[CouplingStep, ...]
    cold_joule_loss_w: float

    @property
    def loss_increase_ratio(self) -> float:
        cold = self.cold_joule_loss_w
        return self.electrical.joule_loss_w / cold if cold else float("nan")


def slab_element_temperature_k(temperature_k: np.ndarray, thermal_mesh: LayeredThermalMesh,
                               slab: int) -> np.ndarray:
    """Mean of the eight corner temperatures of every element of one slab
    (reference electro_thermal.py:180-190)."""
    grid = np.asarray(temperature_k, dtype=np.float64).reshape(thermal_mesh.node_shape)
    lo, hi = grid[slab], grid[slab + 1]
    return 0.125 * (lo[:-1, :-1] + lo[:-1, 1:] + lo[1:, :-1] + lo[1:, 1:]
                    + hi[:-1, :-1] + hi[:-1, 1:] + hi[1:, :-1] + hi[1:, 1:])


def electrical_layer_temperature_k(temperature_k: np.ndarray, thermal_mesh: LayeredThermalMesh,
                                   layer_slabs: Sequence[int]) -> np.ndarray:
    """Element temperatures ``(layers, rows, cols)`` of the electrical layers
    (reference electro_thermal.py:193-200)."""
    return np.stack([slab_element_temperature_k(temperature_k, thermal_mesh, s) for s in layer_slabs])


def via_temperature_k(temperature_k: np.ndarray, thermal_mesh: LayeredThermalMesh,
                      layer_slabs: Sequence[int], vias: Sequence) -> np.ndarray:
    """Temperature of every via: the mean of its two ends, an end being the
    mean of the node faces below and above its copper slab (reference
    electro_thermal.py:203-231)."""
    grid = np.asarray(temperature_k, dtype=np.float64).reshape(thermal_mesh.node_shape)
    out = np.empty(len(vias), dtype=np.float64)
    for index, via in enumerate(vias):
        ends = []
        for layer, row, col in (via.lower, via.upper):
            slab = layer_slabs[layer]
            ends.append(0.5 * (grid[slab, row, col] + grid[slab + 1, row, col]))
        out[index] = 0.5 * (ends[0] + ends[1])
    return out


def via_node_temperature_k(temperature_k: np.ndarray, thermal_mesh: LayeredThermalMesh,
                           layer_slabs: Sequence[int], problem: PCBConductionProblem) -> np.ndarray:
    """:func:`via_temperature_k` over the vias of ``problem``."""
    return via_temperature_k(temperature_k, thermal_mesh, layer_slabs, problem.vias)


def conductivity_at_temperature(reference_conductivity: np.ndarray, temperature_k: np.ndarray, *,
                                reference_temperature_k: float, coefficient_per_k: float) -> np.ndarray:
    """``sigma_ref / (1 + alpha (T - T_ref))``; a non-positive denominator is a
    ValueError (reference electro_thermal.py:234-244)."""
    factor = 1.0 + coefficient_per_k * (np.asarray(temperature_k) - reference_temperature_k)
    if np.any(factor <= 0.0):
        raise ValueError("the linear resistivity model left the valid range (σ ≤ 0)")
    return np.asarray(reference_conductivity) / factor


def thermal_problem_with_joule_heat(scenario: ElectroThermalScenario,
                                    electrical: PCBConductionSolution) -> ThermalConductionProblem:
    """The scenario's thermal problem loaded with a DC solution's element and
    via losses (reference electro_thermal.py:247-266)."""
    heat = element_joule_heat_w(electrical, scenario.thermal_mesh, scenario.layer_slabs)
    if scenario.extra_element_heat_w is not None:
        heat = heat + np.asarray(scenario.extra_element_heat_w, dtype=np.float64)
    sources = via_joule_heat_sources(scenario.electrical, electrical, scenario.thermal_mesh, scenario.layer_slabs)
    return ThermalConductionProblem(
        scenario.thermal_mesh,
        convection=scenario.convection,
        fixed_temperature_mask=scenario.fixed_temperature_mask,
        fixed_temperature_k=scenario.fixed_temperature_k,
        heat_sources=sources + scenario.extra_heat_sources,
        element_heat_w=heat,
        radiation=scenario.radiation,
    )


def heated_electrical_problem(scenario: ElectroThermalScenario, temperature_k: np.ndarray) -> PCBConductionProblem:
    """The DC problem with copper conductivity and via resistance evaluated at
    the given board temperature (reference electro_thermal.py:269-300).  Via
    barrels follow the copper law at the temperature of their ends."""
    sigma = conductivity_at_temperature(
        np.asarray(scenario.electrical.mesh.conductivity_s_per_m, dtype=np.float64),
        electrical_layer_temperature_k(temperature_k, scenario.thermal_mesh, scenario.layer_slabs),
        reference_temperature_k=scenario.conductivity_reference_temperature_k,
        coefficient_per_k=scenario.temperature_coefficient_per_k,
    )
    via_t = via_node_temperature_k(temperature_k, scenario.thermal_mesh, scenario.layer_slabs, scenario.electrical)
    via_factor = 1.0 + scenario.temperature_coefficient_per_k * (via_t - scenario.conductivity_reference_temperature_k)
    vias = tuple(dataclasses.replace(via, resistance_ohm=via.resistance_ohm * float(f))
                 for via, f in zip(scenario.electrical.vias, via_factor))
    return dataclasses.replace(
        scenario.electrical,
        mesh=dataclasses.replace(scenario.electrical.mesh, conductivity_s_per_m=sigma),
        vias=vias,
    )


class TemperatureFixedPoint:
    """Relaxed fixed point on the temperature field with Aitken's delta-squared
    factor (reference electro_thermal.py:303-351).

    With increments d_k = proposed_k - T_k the factor becomes
    ``w_k = -w_{k-1} (d_{k-1} . (d_k - d_{k-1})) / |d_k - d_{k-1}|^2``, clipped
    to [0.05, max_relaxation]: above one for a slowly contracting loop, below
    one for an oscillating one.  A relaxed step that would take the minimum
    temperature below the floor where ``1 + alpha (T - T_ref)`` reaches 1e-3,
    while the plain proposal stays above it, is replaced by the plain
    proposal with the factor reset to one."""

    def __init__(self, scenario: ElectroThermalScenario, config: CouplingConfig) -> None:
        self.config = config
        self.relaxation = config.relaxation
        self.temperature: np.ndarray | None = None
        self._previous: np.ndarray | None = None
        alpha = scenario.temperature_coefficient_per_k
        self._floor = (scenario.conductivity_reference_temperature_k - (1.0 - 1.0e-3) / alpha
                       if alpha > 0.0 else -np.inf)

    def update(self, proposed: np.ndarray) -> float:
        """Take a proposed field; return the largest change of the relaxed iterate
        (infinity on the first call)."""
        proposed = np.asarray(proposed, dtype=np.float64)
        if self.temperature is None:
            self.temperature = proposed.copy()
            self._previous = None
            return float("inf")
        increment = proposed - self.temperature
        if self.config.aitken and self._previous is not None:
            diff = (increment - self._previous).reshape(-1)
            denominator = float(np.dot(diff, diff))
            if denominator > 0.0:
                w = -self.relaxation * float(np.dot(self._previous.reshape(-1), diff)) / denominator
                self.relaxation = float(np.clip(w, 0.05, self.config.max_relaxation))
        candidate = self.temperature + self.relaxation * increment
        if float(np.min(candidate)) < self._floor <= float(np.min(proposed)):
            self.relaxation = 1.0
            candidate = proposed.copy()
        change = float(np.max(np.abs(candidate - self.temperature)))
        self.temperature = candidate
        self._previous = increment
        return change


def run_electro_thermal(
    scenario: ElectroThermalScenario,
    *,
    config: CouplingConfig | None = None,
    backend: str | None = None,
    device_id: int = 0,
    native: bool | None = None,
) -> ElectroThermalResult:
    """Iterate DC and thermal device solves to a self-consistent sigma(T) state
    (reference electro_thermal.py:354-478).

    Each pass: DC solve warm-started from the last potential; thermal solve
    with its Joule loss, warm-started from the relaxed temperature; relaxed
    update of the temperature.  The loop stops after one pass when the
    temperature coefficient is zero, or when the temperature change and the
    relative loss change are both within tolerance and both solves
    converged; otherwise the DC problem is re-heated and the loop continues,
    up to ``config.max_iterations`` passes (non-convergence is reported in
    the result, not raised).  ``backend`` and ``native`` are passed to the
    two solves unchanged."""
    config = config or CouplingConfig()
    problem = scenario.electrical
    fixed_point = TemperatureFixedPoint(scenario, config)
    history: list[CouplingStep] = []
    potential: np.ndarray | None = None
    cold_loss = float("nan")
    previous_loss = float("nan")
    converged = False
    dc = thermal = None
    for iteration in range(1, config.max_iterations + 1):
        dc = solve_pcb_dc(problem, config=config.electrical, backend=backend, device_id=device_id,
                          initial_potential_v=potential, native=native)
        potential = dc.potential_v
        loss = dc.joule_loss_w
        if iteration == 1:
            cold_loss = loss
        thermal = solve_thermal_conduction(
            thermal_problem_with_joule_heat(scenario, dc), config=config.thermal, backend=backend,
            device_id=device_id, initial_temperature_k=fixed_point.temperature, native=native,
        )
        # Nodes of void elements come back NaN; they hold no copper, so they
        # are held at the coldest node to keep the iterate finite.
        proposed = np.where(np.isfinite(thermal.temperature_k), thermal.temperature_k, thermal.min_temperature_k)
        change = fixed_point.update(proposed)
        temperature = fixed_point.temperature
        loss_change = (abs(loss - previous_loss) / abs(loss)
                       if np.isfinite(previous_loss) and loss else float("inf"))
        previous_loss = loss
        history.append(CouplingStep(
            iteration=iteration,
            joule_loss_w=loss,
            max_temperature_k=float(np.max(temperature)),
            temperature_change_k=change,
            relative_loss_change=loss_change,
            relaxation=fixed_point.relaxation,
            electrical_inner_iterations=dc.solve.inner_iterations,
            thermal_inner_iterations=thermal.solve.inner_iterations,
        ))
        both_converged = dc.solve.converged and thermal.solve.converged
        if scenario.temperature_coefficient_per_k == 0.0:
            converged = both_converged
            break
        if (change <= config.temperature_tolerance_k and loss_change <= config.relative_loss_tolerance
                and both_converged):
            converged = True
            break
        problem = heated_electrical_problem(scenario, temperature)
    return ElectroThermalResult(
        electrical=dc,
        thermal=thermal,
        conductivity_s_per_m=np.asarray(problem.mesh.conductivity_s_per_m, dtype=np.float64),
        via_resistance_ohm=np.asarray([via.resistance_ohm for via in problem.vias], dtype=np.float64),
        element_temperature_k=electrical_layer_temperature_k(temperature, scenario.thermal_mesh,
                                                             scenario.layer_slabs),
        converged=converged,
        iterations=len(history),
        history=tuple(history),
        cold_joule_loss_w=cold_loss,
    )
