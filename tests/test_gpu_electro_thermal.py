"""The electro-thermal coupling on the device solves.

* the voltage-driven loop reaches the reference's coupled state
  (tests/golden/coupling/electro_thermal.npz): the same number of passes with and
  without Aitken relaxation, the same loss per pass, and the final
  temperature, potential, conductivity and terminal currents within the
  solve tolerance;
* the closed-form cases of pcb-analysis tests/test_staggered_coupling.py:120-238
  hold: an isothermal board reproduces the resistivity law (I^2 R(T) under
  current drive, V^2 / R(T) under voltage drive), a zero coefficient needs one
  pass, the coupled state is self-consistent, and an iteration limit is
  reported instead of raised.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import pcb_analysis_b200.electrical as ed
import pcb_analysis_b200.electro_thermal as et
import pcb_analysis_b200.thermal as td
from tests import electro_thermal_cases as cases

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "coupling" / "electro_thermal.npz"
ALPHA, T_REF, HOT = 3.93e-3, 293.15, 353.15


@pytest.fixture(scope="module")
def golden() -> dict:
    with np.load(GOLDEN) as data:
        return {k: data[k] for k in data.files}


def _voltage_scenario(voltage_v: float = cases.GOLDEN_VOLTAGE_V, **overrides):
    return cases.scenario(ed, td, et, cases.voltage_loop(ed, voltage_v), **overrides)


def _current_scenario(current_a: float, **overrides):
    with pytest.warns(DeprecationWarning, match="current-driven"):
        return cases.scenario(ed, td, et, cases.current_loop(ed, current_a), **overrides)


def _voltage_for_cold_current(current_a: float) -> float:
    probe = ed.solve_pcb_dc(cases.voltage_loop(ed, 1.0))
    return current_a / float(probe.voltage_terminal_current_a[0])


@pytest.mark.parametrize("tag", ["aitken", "plain"])
def test_coupled_loop_matches_the_reference(golden, tag: str) -> None:
    config = et.CouplingConfig(aitken=(tag == "aitken"))
    result = et.run_electro_thermal(_voltage_scenario(), config=config)
    assert result.converged
    assert result.iterations == int(golden[f"{tag}_passes"][0])
    np.testing.assert_allclose([s.joule_loss_w for s in result.history], golden[f"{tag}_loss"], rtol=1e-8)
    np.testing.assert_allclose([s.relaxation for s in result.history], golden[f"{tag}_relaxation"], rtol=1e-5)
    t, t_ref = result.thermal.temperature_k.reshape(-1), golden[f"{tag}_temperature"]
    rise = float(np.max(t_ref) - cases.AMBIENT)
    assert float(np.max(np.abs(t - t_ref))) <= 1e-6 * rise
    v_ref = golden[f"{tag}_potential"]
    finite = np.isfinite(v_ref)
    np.testing.assert_array_equal(np.isfinite(result.electrical.potential_v.reshape(-1)), finite)
    np.testing.assert_allclose(result.electrical.potential_v.reshape(-1)[finite], v_ref[finite],
                               atol=1e-8 * cases.GOLDEN_VOLTAGE_V)
    np.testing.assert_allclose(result.conductivity_s_per_m, golden[f"{tag}_conductivity"], rtol=1e-8)
    np.testing.assert_allclose(result.via_resistance_ohm, golden[f"{tag}_via_resistance"], rtol=1e-8)
    np.testing.assert_allclose(result.element_temperature_k, golden[f"{tag}_layer_temperature"], rtol=1e-8)
    np.testing.assert_allclose(result.electrical.voltage_terminal_current_a, golden[f"{tag}_terminal_current"],
                               rtol=1e-7)
    assert result.cold_joule_loss_w == pytest.approx(float(golden[f"{tag}_cold_loss"][0]), rel=1e-9)
    assert result.thermal.total_heat_input_w == pytest.approx(result.electrical.joule_loss_w, rel=1e-12)


def test_isothermal_current_drive_reproduces_the_resistivity_law() -> None:
    problem = cases.current_loop(ed)
    thermal = cases.loop_thermal_mesh(td, problem)
    with pytest.warns(DeprecationWarning, match="current-driven"):
        scenario = et.ElectroThermalScenario(
            problem, thermal, (0, 2), fixed_temperature_mask=np.ones(thermal.node_shape, dtype=bool),
            fixed_temperature_k=HOT, conductivity_reference_temperature_k=T_REF)
    result = et.run_electro_thermal(scenario)
    cold = ed.solve_pcb_dc(problem)
    factor = 1.0 + ALPHA * (HOT - T_REF)
    assert result.converged and result.iterations == 3  # the hot solve, then a confirming pass
    assert result.electrical.joule_loss_w == pytest.approx(cold.joule_loss_w * factor, rel=1e-9)
    assert result.loss_increase_ratio == pytest.approx(factor, rel=1e-9)
    np.testing.assert_allclose(result.element_temperature_k, HOT)
    np.testing.assert_allclose(result.thermal.temperature_k, HOT)


def test_isothermal_voltage_drive_loses_in_inverse_proportion_to_resistance() -> None:
    problem = cases.voltage_loop(ed, 20e-3)
    thermal = cases.loop_thermal_mesh(td, problem)
    scenario = et.ElectroThermalScenario(
        problem, thermal, (0, 2), fixed_temperature_mask=np.ones(thermal.node_shape, dtype=bool),
        fixed_temperature_k=HOT, conductivity_reference_temperature_k=T_REF)
    result = et.run_electro_thermal(scenario)
    cold = ed.solve_pcb_dc(problem)
    factor = 1.0 + ALPHA * (HOT - T_REF)
    assert result.converged
    assert result.electrical.joule_loss_w == pytest.approx(cold.joule_loss_w / factor, rel=1e-9)
    np.testing.assert_allclose(result.electrical.voltage_terminal_current_a,
                               cold.voltage_terminal_current_a / factor, rtol=1e-9)


def test_zero_coefficient_needs_one_pass() -> None:
    result = et.run_electro_thermal(_voltage_scenario(temperature_coefficient_per_k=0.0))
    assert result.converged and result.iterations == 1
    assert result.loss_increase_ratio == 1.0
    np.testing.assert_allclose(result.conductivity_s_per_m, cases.loop_mesh(ed).conductivity_s_per_m)


def test_coupled_state_is_self_consistent_and_aitken_saves_passes() -> None:
    scenario = _voltage_scenario(_voltage_for_cold_current(3.0))
    accelerated = et.run_electro_thermal(scenario)
    plain = et.run_electro_thermal(scenario, config=et.CouplingConfig(aitken=False))
    assert accelerated.converged and plain.converged
    assert accelerated.iterations < plain.iterations
    assert accelerated.loss_increase_ratio < 0.9
    assert accelerated.thermal.max_temperature_k > cases.AMBIENT + 10.0
    np.testing.assert_allclose(accelerated.electrical.joule_loss_w, plain.electrical.joule_loss_w, rtol=1e-6)
    layer_t = et.electrical_layer_temperature_k(accelerated.thermal.temperature_k, scenario.thermal_mesh,
                                                scenario.layer_slabs)
    expected = et.conductivity_at_temperature(scenario.electrical.mesh.conductivity_s_per_m, layer_t,
                                              reference_temperature_k=T_REF, coefficient_per_k=ALPHA)
    np.testing.assert_allclose(accelerated.conductivity_s_per_m, expected, rtol=1e-6)
    assert accelerated.thermal.total_heat_input_w == pytest.approx(accelerated.electrical.joule_loss_w, rel=1e-12)
    assert accelerated.history[-1].temperature_change_k <= 1e-3
    assert all(step.relaxation > 0.0 for step in accelerated.history)


def test_iteration_limit_is_reported_and_voltage_drive_settles() -> None:
    capped = et.run_electro_thermal(_current_scenario(6.0), config=et.CouplingConfig(max_iterations=3))
    assert not capped.converged and capped.iterations == 3
    assert capped.electrical.joule_loss_w > capped.cold_joule_loss_w
    settled = et.run_electro_thermal(_voltage_scenario(_voltage_for_cold_current(6.0)))
    assert settled.converged and settled.iterations <= 10
    assert settled.loss_increase_ratio < 1.0
    assert float(settled.electrical.voltage_terminal_current_a[0]) < 6.0
