"""Staggered electro-thermal coupling over the device DC and thermal solves.

Copper conducts less as it heats, sigma(T) = sigma_ref / (1 + alpha (T - T_ref)).
The coupling alternates a DC solve (:func:`solve_pcb_dc`) at the current
conductivity with a thermal solve (:func:`solve_thermal_conduction`) loaded by
that solve's Joule loss, then evaluates the conductivity at the new element
temperatures; both solves are warm-started from the previous pass and the
temperature iterate is relaxed by Aitken's delta-squared factor.  This module
is host control only: every operator action, PCG iteration and residual runs
in the CUDA library.

The call surface is that of pcb-analysis's
src/multiphysics/staggered_coupling/electro_thermal.py:72-478 (the scenario,
config, step and result records, the resistivity helpers, the relaxed fixed
point and run_electro_thermal), and so are the numbers a pass produces: the
same pass count, the same losses and temperatures, because the stopping
rules and the relaxation are the reference's.

Voltage drive (two or more voltage terminals) gives a loss V^2 / R(T) that
falls as the copper heats, so the loop contracts.  With fewer voltage
terminals every copper current is imposed; such a scenario still runs but
warns, since its loss I^2 R(T) rises with temperature and can run away.
"""

from __future__ import annotations

import dataclasses
import itertools
import math
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

# Lower clip of the Aitken factor.
_MIN_RELAXATION = 0.05
# A relaxed field may not cool copper to where 1 + alpha (T - T_ref) < this.
_MIN_RESISTIVITY_FACTOR = 1.0e-3


def _same_grid_lines(electrical_mesh, thermal_mesh: LayeredThermalMesh) -> bool:
    return bool(np.allclose(electrical_mesh.pitch_x_m, thermal_mesh.pitch_x_m)
                and np.allclose(electrical_mesh.pitch_y_m, thermal_mesh.pitch_y_m))


@dataclass(frozen=True)
class ElectroThermalScenario:
    """One board: its DC drive, its thermal mesh and environment, and the
    resistivity law; ``layer_slabs[L]`` is the thermal slab that holds
    electrical layer ``L``."""

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
        slabs = self.thermal_mesh.element_grid_shape[0]
        if tuple(self.thermal_mesh.element_grid_shape[1:]) != (rows, cols):
            raise ValueError("electrical and thermal meshes must share (rows, cols)")
        if not _same_grid_lines(self.electrical.mesh, self.thermal_mesh):
            raise ValueError("electrical and thermal meshes must share the same grid lines")
        slabs_of = tuple(map(int, self.layer_slabs))
        if len(slabs_of) != layers or not all(0 <= s < slabs for s in slabs_of):
            raise ValueError("layer_slabs must name one thermal slab per electrical layer")
        alpha = float(self.temperature_coefficient_per_k)
        if not (math.isfinite(alpha) and alpha >= 0.0):
            raise ValueError("temperature_coefficient_per_k must be finite and non-negative")
        object.__setattr__(self, "layer_slabs", slabs_of)
        for name in ("convection", "extra_heat_sources", "radiation"):
            object.__setattr__(self, name, tuple(getattr(self, name)))
        self.thermal_problem()  # the thermal boundary conditions are checked here, before any heat
        if len(self.electrical.voltage_terminals) < 2:  # every copper current is imposed
            warnings.warn(CURRENT_DRIVEN_DEPRECATION, DeprecationWarning, stacklevel=3)

    def thermal_problem(self, element_heat_w: np.ndarray | None = None,
                        heat_sources: tuple[HeatSource, ...] = ()) -> ThermalConductionProblem:
        """The scenario's thermal problem with the given loads added to its own."""

        heat = self.extra_element_heat_w
        if element_heat_w is not None:
            heat = element_heat_w if heat is None else element_heat_w + np.asarray(heat, dtype=np.float64)
        return ThermalConductionProblem(
            self.thermal_mesh, convection=self.convection, fixed_temperature_mask=self.fixed_temperature_mask,
            fixed_temperature_k=self.fixed_temperature_k, heat_sources=heat_sources + self.extra_heat_sources,
            element_heat_w=heat, radiation=self.radiation)

    def resistivity_factor(self, temperature_k):
        """1 + alpha (T - T_ref)."""

        return 1.0 + self.temperature_coefficient_per_k * (
            np.asarray(temperature_k) - self.conductivity_reference_temperature_k)


@dataclass(frozen=True)
class CouplingConfig:
    """Limits of the fixed point; ``electrical`` and ``thermal`` are the MPIR
    configs of the two solves (None: their defaults)."""

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
        if min(self.temperature_tolerance_k, self.relative_loss_tolerance) <= 0.0:
            raise ValueError("tolerances must be positive")
        if not 0.0 < self.relaxation <= self.max_relaxation:
            raise ValueError("relaxation must lie in (0, max_relaxation]")
        if self.max_relaxation < 1.0:
            raise ValueError("max_relaxation must be at least one")


@dataclass(frozen=True)
class CouplingStep:
    """One pass of the loop."""

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
    used, the element temperature of every electrical layer, and the passes."""

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


# ------------------------------------------------------------------ fields
def slab_element_temperature_k(temperature_k: np.ndarray, thermal_mesh: LayeredThermalMesh,
                               slab: int) -> np.ndarray:
    """Mean of the eight corner temperatures of every element of one slab,
    summed in the corner order 4 dz + 2 dy + dx."""

    grid = np.asarray(temperature_k, dtype=np.float64).reshape(thermal_mesh.node_shape)
    total = None
    for dz, dy, dx in itertools.product((0, 1), repeat=3):
        corner = grid[slab + dz, dy:grid.shape[1] - 1 + dy, dx:grid.shape[2] - 1 + dx]
        total = corner if total is None else total + corner
    return 0.125 * total


def electrical_layer_temperature_k(temperature_k: np.ndarray, thermal_mesh: LayeredThermalMesh,
                                   layer_slabs: Sequence[int]) -> np.ndarray:
    """Element temperatures ``(layers, rows, cols)`` of the electrical layers."""

    return np.stack([slab_element_temperature_k(temperature_k, thermal_mesh, slab) for slab in layer_slabs])


def via_temperature_k(temperature_k: np.ndarray, thermal_mesh: LayeredThermalMesh,
                      layer_slabs: Sequence[int], vias: Sequence) -> np.ndarray:
    """Temperature of every via: the mean of its two ends, an end being the
    mean of the node faces below and above its copper slab."""

    if not len(vias):
        return np.zeros(0)
    grid = np.asarray(temperature_k, dtype=np.float64).reshape(thermal_mesh.node_shape)
    slab_of = np.asarray(layer_slabs)

    def end(points: np.ndarray) -> np.ndarray:
        slab, row, col = slab_of[points[:, 0]], points[:, 1], points[:, 2]
        return 0.5 * (grid[slab, row, col] + grid[slab + 1, row, col])

    lower = np.array([via.lower for via in vias], dtype=np.int64)
    upper = np.array([via.upper for via in vias], dtype=np.int64)
    return 0.5 * (end(lower) + end(upper))


def via_node_temperature_k(temperature_k: np.ndarray, thermal_mesh: LayeredThermalMesh,
                           layer_slabs: Sequence[int], problem: PCBConductionProblem) -> np.ndarray:
    """:func:`via_temperature_k` over the vias of ``problem``."""

    return via_temperature_k(temperature_k, thermal_mesh, layer_slabs, problem.vias)


def conductivity_at_temperature(reference_conductivity: np.ndarray, temperature_k: np.ndarray, *,
                                reference_temperature_k: float, coefficient_per_k: float) -> np.ndarray:
    """``sigma_ref / (1 + alpha (T - T_ref))``; a non-positive denominator is a ValueError."""

    factor = 1.0 + coefficient_per_k * (np.asarray(temperature_k) - reference_temperature_k)
    if (factor <= 0.0).any():
        raise ValueError("the linear resistivity model left the valid range (σ ≤ 0)")
    return np.asarray(reference_conductivity) / factor


def thermal_problem_with_joule_heat(scenario: ElectroThermalScenario,
                                    electrical: PCBConductionSolution) -> ThermalConductionProblem:
    """The scenario's thermal problem loaded with a DC solution's element and via losses."""

    heat = element_joule_heat_w(electrical, scenario.thermal_mesh, scenario.layer_slabs)
    sources = via_joule_heat_sources(scenario.electrical, electrical, scenario.thermal_mesh, scenario.layer_slabs)
    return scenario.thermal_problem(heat, sources)


def heated_electrical_problem(scenario: ElectroThermalScenario, temperature_k: np.ndarray) -> PCBConductionProblem:
    """The DC problem with the copper conductivity and the via resistances at
    the given board temperature; via barrels follow the copper law at the
    temperature of their ends."""

    cold = scenario.electrical
    sigma = conductivity_at_temperature(
        np.asarray(cold.mesh.conductivity_s_per_m, dtype=np.float64),
        electrical_layer_temperature_k(temperature_k, scenario.thermal_mesh, scenario.layer_slabs),
        reference_temperature_k=scenario.conductivity_reference_temperature_k,
        coefficient_per_k=scenario.temperature_coefficient_per_k)
    factors = scenario.resistivity_factor(
        via_node_temperature_k(temperature_k, scenario.thermal_mesh, scenario.layer_slabs, cold))
    vias = tuple(dataclasses.replace(via, resistance_ohm=via.resistance_ohm * float(f))
                 for via, f in zip(cold.vias, factors))
    return dataclasses.replace(cold, mesh=dataclasses.replace(cold.mesh, conductivity_s_per_m=sigma), vias=vias)


# ------------------------------------------------------------------ fixed point
class TemperatureFixedPoint:
    """Relaxed fixed point on the temperature field (Aitken's delta-squared).

    With the increments d_k = proposed_k - T_k the factor is
    w_k = -w_{k-1} (d_{k-1} . (d_k - d_{k-1})) / |d_k - d_{k-1}|^2, clipped to
    [0.05, max_relaxation]: above one for a slowly contracting loop, below one
    for an oscillating one.  A relaxed step that would cool the coldest node
    below the temperature where 1 + alpha (T - T_ref) reaches 1e-3, while the
    plain proposal stays above it, gives way to the plain proposal, and the
    factor restarts at one."""

    def __init__(self, scenario: ElectroThermalScenario, config: CouplingConfig) -> None:
        self.config = config
        self.relaxation = config.relaxation
        self.temperature: np.ndarray | None = None
        self._last_step: np.ndarray | None = None
        alpha = scenario.temperature_coefficient_per_k
        self._coldest_allowed = (
            scenario.conductivity_reference_temperature_k - (1.0 - _MIN_RESISTIVITY_FACTOR) / alpha
            if alpha > 0.0 else -math.inf)

    def _aitken(self, step: np.ndarray) -> None:
        if not self.config.aitken or self._last_step is None:
            return
        bend = (step - self._last_step).ravel()
        curvature = float(bend @ bend)
        if curvature > 0.0:
            proposal = -self.relaxation * float(self._last_step.ravel() @ bend) / curvature
            self.relaxation = min(max(proposal, _MIN_RELAXATION), self.config.max_relaxation)

    def update(self, proposed: np.ndarray) -> float:
        """Take a proposed field; return the largest change of the relaxed
        iterate (infinity on the first call)."""

        target = np.asarray(proposed, dtype=np.float64)
        if self.temperature is None:
            self.temperature, self._last_step = target.copy(), None
            return math.inf
        step = target - self.temperature
        self._aitken(step)
        relaxed = self.temperature + self.relaxation * step
        if relaxed.min() < self._coldest_allowed <= target.min():
            self.relaxation, relaxed = 1.0, target.copy()
        change = float(np.abs(relaxed - self.temperature).max())
        self.temperature, self._last_step = relaxed, step
        return change


# ------------------------------------------------------------------ the loop
@dataclass
class _Coupling:
    """State the passes carry from one to the next."""

    problem: PCBConductionProblem
    potential: np.ndarray | None = None
    cold_loss: float = math.nan
    last_loss: float = math.nan
    dc: PCBConductionSolution | None = None
    thermal: ThermalConductionSolution | None = None

    def loss_change(self, loss: float) -> float:
        """|loss - last| / |loss| (infinite on the first pass or at zero loss)."""

        change = abs(loss - self.last_loss) / abs(loss) if math.isfinite(self.last_loss) and loss else math.inf
        self.last_loss = loss
        return change


def run_electro_thermal(
    scenario: ElectroThermalScenario,
    *,
    config: CouplingConfig | None = None,
    backend: str | None = None,
    device_id: int = 0,
    native: bool | None = None,
) -> ElectroThermalResult:
    """Iterate DC and thermal device solves to a self-consistent sigma(T) state.

    A pass: the DC solve warm-started from the last potential; the thermal
    solve loaded with its Joule loss, warm-started from the relaxed field; the
    relaxed update of the field.  The loop ends after one pass when the
    temperature coefficient is zero; otherwise once the field change and the
    relative loss change are both within tolerance with both solves
    converged, or after ``config.max_iterations`` passes (reported, not
    raised).  ``backend`` and ``native`` go to both solves unchanged."""

    settings = config or CouplingConfig()
    solver_options = dict(backend=backend, device_id=device_id, native=native)
    relaxed = TemperatureFixedPoint(scenario, settings)
    state = _Coupling(problem=scenario.electrical)
    passes: list[CouplingStep] = []
    converged = False
    isothermal = scenario.temperature_coefficient_per_k == 0.0
    for number in range(1, settings.max_iterations + 1):
        state.dc = solve_pcb_dc(state.problem, config=settings.electrical, initial_potential_v=state.potential,
                                **solver_options)
        state.potential = state.dc.potential_v
        loss = state.dc.joule_loss_w
        if number == 1:
            state.cold_loss = loss
        state.thermal = solve_thermal_conduction(
            thermal_problem_with_joule_heat(scenario, state.dc), config=settings.thermal,
            initial_temperature_k=relaxed.temperature, **solver_options)
        # Void elements' nodes come back NaN; they hold no copper and are
        # held at the coldest node so that the iterate stays finite.
        field = state.thermal.temperature_k
        change = relaxed.update(np.where(np.isfinite(field), field, state.thermal.min_temperature_k))
        loss_change = state.loss_change(loss)
        passes.append(CouplingStep(
            iteration=number, joule_loss_w=loss, max_temperature_k=float(relaxed.temperature.max()),
            temperature_change_k=change, relative_loss_change=loss_change, relaxation=relaxed.relaxation,
            electrical_inner_iterations=state.dc.solve.inner_iterations,
            thermal_inner_iterations=state.thermal.solve.inner_iterations))
        solved = state.dc.solve.converged and state.thermal.solve.converged
        settled = change <= settings.temperature_tolerance_k and loss_change <= settings.relative_loss_tolerance
        if isothermal or (settled and solved):
            converged = solved
            break
        state.problem = heated_electrical_problem(scenario, relaxed.temperature)
    return ElectroThermalResult(
        electrical=state.dc,
        thermal=state.thermal,
        conductivity_s_per_m=np.asarray(state.problem.mesh.conductivity_s_per_m, dtype=np.float64),
        via_resistance_ohm=np.asarray([via.resistance_ohm for via in state.problem.vias], dtype=np.float64),
        element_temperature_k=electrical_layer_temperature_k(relaxed.temperature, scenario.thermal_mesh,
                                                             scenario.layer_slabs),
        converged=converged,
        iterations=len(passes),
        history=tuple(passes),
        cold_joule_loss_w=state.cold_loss,
    )
