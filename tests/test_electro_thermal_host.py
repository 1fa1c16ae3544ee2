"""Host side of the electro-thermal coupling, without a GPU.

* the host steps (resistivity law, layer and via temperatures, loss placement,
  Aitken fixed point) equal the reference's on seeded inputs
  (tests/golden/coupling/electro_thermal.npz, made by make_golden_electro_thermal.py);
* scenario and config validation and the current-drive warning follow
  pcb-analysis tests/test_staggered_coupling.py:240-271;
* the loop's control (warm starts, stopping rules, iteration limit, the
  conductivity it reports) is checked with the two device solves replaced
  by closed-form fakes.
"""

from __future__ import annotations

import types
import warnings
from pathlib import Path

import numpy as np
import pytest

import pcb_analysis_b200.electrical as ed
import pcb_analysis_b200.electro_thermal as et
import pcb_analysis_b200.thermal as td
from pcb_analysis_b200.thermal.coupling import element_heat_from_losses, via_heat_sources
from tests import electro_thermal_cases as cases
from tests.golden.make_golden_electro_thermal import fixed_point_proposals

GOLDEN = Path(__file__).resolve().parent / "golden" / "coupling" / "electro_thermal.npz"


@pytest.fixture(scope="module")
def golden() -> dict:
    with np.load(GOLDEN) as data:
        return {k: data[k] for k in data.files}


def _scenario(**overrides):
    return cases.scenario(ed, td, et, cases.voltage_loop(ed, cases.GOLDEN_VOLTAGE_V), **overrides)


def test_heated_problem_matches_the_reference(golden) -> None:
    scenario = _scenario()
    temperature = golden["seeded_temperature"]
    heated = et.heated_electrical_problem(scenario, temperature)
    np.testing.assert_array_equal(np.asarray(heated.mesh.conductivity_s_per_m), golden["heated_conductivity"])
    np.testing.assert_array_equal([v.resistance_ohm for v in heated.vias], golden["heated_via_resistance"])
    np.testing.assert_array_equal(
        et.electrical_layer_temperature_k(temperature, scenario.thermal_mesh, scenario.layer_slabs),
        golden["seeded_layer_temperature"])


def test_loss_placement_matches_the_reference(golden) -> None:
    scenario = _scenario()
    heat = element_heat_from_losses(golden["seeded_element_loss"], scenario.thermal_mesh, (0, 2))
    np.testing.assert_array_equal(heat, golden["seeded_element_heat"])
    sources = via_heat_sources(scenario.electrical.vias, golden["seeded_via_loss"], 2, scenario.thermal_mesh, (0, 2))
    np.testing.assert_array_equal(np.array([s.nodes for s in sources]), golden["via_source_nodes"])
    np.testing.assert_array_equal([s.power_w for s in sources], golden["via_source_power"])
    with pytest.raises(ValueError, match="layer_slabs"):
        element_heat_from_losses(golden["seeded_element_loss"], scenario.thermal_mesh, (0,))
    with pytest.raises(ValueError, match="one value per via"):
        via_heat_sources(scenario.electrical.vias, golden["seeded_via_loss"][:-1], 2, scenario.thermal_mesh, (0, 2))


def test_fixed_point_matches_the_reference(golden) -> None:
    scenario = _scenario()
    fixed_point = et.TemperatureFixedPoint(scenario, et.CouplingConfig())
    changes, relaxations = [], []
    for proposal in fixed_point_proposals(scenario.thermal_mesh.node_shape):
        changes.append(fixed_point.update(proposal))
        relaxations.append(fixed_point.relaxation)
    np.testing.assert_allclose(changes, golden["fixed_point_change"], rtol=1e-13)
    np.testing.assert_allclose(relaxations, golden["fixed_point_relaxation"], rtol=1e-13)
    np.testing.assert_allclose(fixed_point.temperature, golden["fixed_point_temperature"], rtol=1e-14)
    assert any(r != 1.0 for r in relaxations[2:])  # Aitken moved the factor


def test_resistivity_law_and_its_range() -> None:
    sigma = et.conductivity_at_temperature(np.array([5.8e7]), np.array([353.15]), reference_temperature_k=293.15,
                                           coefficient_per_k=3.93e-3)
    assert sigma[0] == pytest.approx(5.8e7 / (1.0 + 3.93e-3 * 60.0), rel=1e-15)
    with pytest.raises(ValueError, match="valid range"):
        et.conductivity_at_temperature(np.array([5.8e7]), np.array([0.0]), reference_temperature_k=293.15,
                                       coefficient_per_k=3.93e-3)


def test_scenario_and_config_validation() -> None:
    problem = cases.voltage_loop(ed, 1e-3)
    thermal = cases.loop_thermal_mesh(td, problem)
    top = (td.ConvectionBoundary("top", 5.0, cases.AMBIENT),)
    with pytest.raises(ValueError, match="one thermal slab per electrical layer"):
        et.ElectroThermalScenario(problem, thermal, (0,), convection=top)
    with pytest.raises(ValueError, match="positive film coefficient, a radiating face or a fixed node"):
        et.ElectroThermalScenario(problem, thermal, (0, 2))
    with pytest.raises(ValueError, match="non-negative"):
        et.ElectroThermalScenario(problem, thermal, (0, 2), convection=top, temperature_coefficient_per_k=-1.0)
    with pytest.raises(ValueError, match="relaxation"):
        et.CouplingConfig(relaxation=0.0)
    with pytest.raises(ValueError, match="max_iterations"):
        et.CouplingConfig(max_iterations=0)


def test_only_current_driven_scenarios_warn() -> None:
    with warnings.catch_warnings():
        warnings.simplefilter("error", DeprecationWarning)
        _scenario()
    with pytest.warns(DeprecationWarning, match="current-driven"):
        cases.scenario(ed, td, et, cases.current_loop(ed))
    board = cases.voltage_loop(ed, 1e-3)
    source, sink = board.voltage_terminals
    pinned = ed.PCBConductionProblem(board.mesh, terminals=(ed.CurrentTerminal(sink.nodes, -2.0, "load"),),
                                     voltage_terminals=(source,), vias=board.vias)
    with pytest.warns(DeprecationWarning, match="fewer than two voltage terminals"):
        cases.scenario(ed, td, et, pinned)


class _FakeSolves:
    """Closed-form stand-ins for the two device solves: the loss is V^2 over a
    resistance proportional to the mean copper resistivity, and the board is
    isothermal at ambient + theta * loss."""

    def __init__(self, scenario, theta: float = 400.0) -> None:
        self.scenario = scenario
        self.theta = theta
        self.dc_starts: list = []
        self.thermal_starts: list = []

    def solve_pcb_dc(self, problem, *, config, backend, device_id, initial_potential_v, native):
        self.dc_starts.append(initial_potential_v)
        sigma0 = np.asarray(self.scenario.electrical.mesh.conductivity_s_per_m, dtype=np.float64)
        ratio = float(np.mean(np.asarray(problem.mesh.conductivity_s_per_m) / sigma0))
        loss = 0.05 * ratio
        shape = problem.mesh.element_active.shape
        return types.SimpleNamespace(
            potential_v=np.full(problem.mesh.node_shape, ratio), joule_loss_w=loss,
            element_joule_loss_w=np.full(shape, loss / np.prod(shape)), via_joule_loss_w=np.zeros(len(problem.vias)),
            solve=types.SimpleNamespace(inner_iterations=7, converged=True))

    def solve_thermal_conduction(self, problem, *, config, backend, device_id, initial_temperature_k, native):
        self.thermal_starts.append(None if initial_temperature_k is None else np.array(initial_temperature_k))
        heat = float(np.sum(problem.element_heat_w))
        t = np.full(problem.mesh.node_shape, cases.AMBIENT + self.theta * heat)
        return types.SimpleNamespace(temperature_k=t, min_temperature_k=float(t.min()),
                                     solve=types.SimpleNamespace(inner_iterations=3, converged=True))


def _run_with_fakes(monkeypatch, scenario, config=None, theta=400.0):
    fakes = _FakeSolves(scenario, theta)
    monkeypatch.setattr(et, "solve_pcb_dc", fakes.solve_pcb_dc)
    monkeypatch.setattr(et, "solve_thermal_conduction", fakes.solve_thermal_conduction)
    return et.run_electro_thermal(scenario, config=config), fakes


def test_loop_control_with_closed_form_solves(monkeypatch) -> None:
    scenario = _scenario()
    result, fakes = _run_with_fakes(monkeypatch, scenario)
    assert result.converged and 2 < result.iterations < 20
    # Warm starts: nothing on the first pass, the previous iterate after it.
    assert fakes.dc_starts[0] is None and all(s is not None for s in fakes.dc_starts[1:])
    assert fakes.thermal_starts[0] is None and all(s is not None for s in fakes.thermal_starts[1:])
    # The fixed point of T = T_amb + theta * 0.05 / (1 + alpha (T - T_ref)).
    alpha, t_ref = 3.93e-3, 293.15
    t = result.thermal.temperature_k.max()
    assert t == pytest.approx(cases.AMBIENT + 400.0 * 0.05 / (1.0 + alpha * (t - t_ref)), abs=2e-3)
    assert result.loss_increase_ratio < 1.0
    assert result.history[-1].temperature_change_k <= 1e-3
    assert [s.iteration for s in result.history] == list(range(1, result.iterations + 1))
    # The conductivity reported is the one the last DC solve used.
    sigma0 = np.asarray(scenario.electrical.mesh.conductivity_s_per_m, dtype=np.float64)
    np.testing.assert_allclose(np.mean(result.conductivity_s_per_m / sigma0), result.electrical.potential_v.flat[0],
                               rtol=1e-12)


def test_zero_coefficient_and_iteration_limit(monkeypatch) -> None:
    one_pass, _ = _run_with_fakes(monkeypatch, _scenario(temperature_coefficient_per_k=0.0))
    assert one_pass.converged and one_pass.iterations == 1 and one_pass.loss_increase_ratio == 1.0
    capped, _ = _run_with_fakes(monkeypatch, _scenario(), config=et.CouplingConfig(max_iterations=2))
    assert not capped.converged and capped.iterations == 2
