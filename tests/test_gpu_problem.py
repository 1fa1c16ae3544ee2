"""Problem preparation and post-processing on the device, against the
reference's own arrays.

Mirrors tests/test_native_thermal_system.py:85-121 of pcb-analysis (the
prepared system bit-identical to the NumPy operator's) for the device path:

* node masks, lumped Robin conductance and R T_amb (per boundary and in
  total) and the nodal load equal the reference's golden arrays bit for bit;
* the right-hand side and the unconstrained residual equal the reference's
  formulas (operator.py:411-482) evaluated in NumPy on those arrays with the
  device's own stiffness action, bit for bit, and the golden right-hand side
  within the stiffness action's rounding;
* -k grad T of the reference's solution equals the reference's flux bit for
  bit; the per-boundary heat and the budget (compensated sums on the device,
  pairwise NumPy sums in the reference) agree within rounding;
* new boundaries or a new C / dt on a resident problem system give the arrays
  and diagonal of a system made fresh with them.
"""

from __future__ import annotations

import dataclasses

import numpy as np
import pytest

import pcb_analysis_b200.thermal as ns
from pcb_analysis_b200.thermal.system import prepare, problem_inputs
from tests.conftest import golden_cases, load_golden
from tests.problems import CASES

pytestmark = pytest.mark.gpu


def _system(problem, capacity=None):
    from pcb_analysis_b200._native import DeviceSystem

    return DeviceSystem.from_problem(**problem_inputs(problem, capacity))


def _rhs_in_numpy(prepared, robin_total, stiffness, reference, capacity=None, previous=None):
    """operator.py:411-440 on host arrays, with the given stiffness action."""

    mask = prepared.fixed_nodes.reshape(-1)
    active = prepared.active_nodes.reshape(-1)
    shifted = np.where(mask & active, prepared.fixed_temperature_k.reshape(-1) - reference, 0.0)
    cap_load = np.zeros(mask.size) if previous is None else capacity * np.where(np.isfinite(previous), previous, 0.0)
    rhs = prepared.load + (prepared.robin_rhs - robin_total * reference) + cap_load - stiffness(shifted)
    rhs[mask] = shifted[mask]
    return rhs


@pytest.mark.parametrize("name", golden_cases())
def test_prepared_arrays_equal_the_reference_bit_for_bit(name: str) -> None:
    g = load_golden(name)
    problem = CASES[name](ns)
    with _system(problem) as dev:
        p = dev.prepared()
        np.testing.assert_array_equal(p["robin_total"], g["robin_total"])
        np.testing.assert_array_equal(p["robin_rhs"], g["robin_rhs"])
        np.testing.assert_array_equal(p["load"], g["load"])
        np.testing.assert_array_equal(p["free_nodes"], g["free"])
        np.testing.assert_array_equal(p["active_nodes"], g["active_nodes"])
        for b in range(g["robin_weights"].shape[0]):
            w, rw = dev.boundary_weights(b)
            np.testing.assert_array_equal(w, g["robin_weights"][b])
            np.testing.assert_array_equal(rw, g["robin_rhs_weights"][b])
        np.testing.assert_array_equal(dev.diagonal(), g["diagonal"])


@pytest.mark.parametrize("name", golden_cases())
def test_right_hand_side_and_residual_follow_the_reference_formulas(name: str) -> None:
    g = load_golden(name)
    problem = CASES[name](ns)
    host = prepare(problem)
    reference = float(g["reference_temperature"])
    with _system(problem) as dev:
        rhs = dev.build_rhs(reference)
        np.testing.assert_array_equal(rhs, _rhs_in_numpy(host, host.robin_total, dev.stiffness_f64, reference))
        scale = np.abs(g["rhs"]).max()
        np.testing.assert_allclose(rhs, g["rhs"], rtol=0, atol=1e-12 * scale)
        temperature = np.where(np.isfinite(g["two_level_temperature"]), g["two_level_temperature"], reference)
        out = dev.postprocess(temperature, residual=True)
        expected = dev.stiffness_f64(temperature) + host.robin_only * temperature - host.robin_rhs + 0.0 - host.load
        np.testing.assert_array_equal(out["residual"], expected)


@pytest.mark.parametrize("name", golden_cases())
def test_flux_and_heat_budget_of_the_reference_solution(name: str) -> None:
    g = load_golden(name)
    problem = CASES[name](ns)
    reference = float(g["reference_temperature"])
    temperature = g["two_level_temperature"]
    with _system(problem) as dev:
        out = dev.postprocess(np.where(np.isfinite(temperature), temperature, reference), residual=True)
        fixed = dev.prepared()["free_nodes"] == 0
    np.testing.assert_array_equal(out["heat_flux"], g["two_level_flux"])
    budget = g["two_level_budget"]
    # heat that crosses the board: input, removed by convection, through fixed nodes
    scale = abs(budget[0]) + np.abs(g["two_level_convective"]).sum() + np.abs(out["residual"][fixed]).sum()
    assert out["total_heat_input_w"] == pytest.approx(budget[0], rel=1e-13, abs=1e-15)
    np.testing.assert_allclose(out["convective_heat_w"], g["two_level_convective"], rtol=0, atol=1e-11 * scale)
    assert out["fixed_temperature_heat_w"] == pytest.approx(budget[1], rel=0, abs=1e-9 * scale)


def test_transient_terms_match_numpy_with_the_same_stiffness() -> None:
    problem = CASES["voxel_body"](ns)
    host = prepare(problem)
    rng = np.random.default_rng(3)
    capacity = rng.uniform(0.0, 2e-3, problem.mesh.size) * host.active_nodes.reshape(-1)
    previous = 300.0 + rng.standard_normal(problem.mesh.size)
    previous[5] = np.nan  # non-finite history counts as zero
    with _system(problem, capacity) as dev:
        robin_total = host.robin_only + capacity
        np.testing.assert_array_equal(dev.prepared()["robin_total"], robin_total)
        rhs = dev.build_rhs(297.0, previous)
        expected = _rhs_in_numpy(host, robin_total, dev.stiffness_f64, 297.0, capacity, previous)
        np.testing.assert_array_equal(rhs, expected)
        with pytest.raises(ValueError, match="previous_temperature_k"):
            dev.build_rhs(297.0)
        temperature = 301.0 + rng.standard_normal(problem.mesh.size)
        out = dev.postprocess(temperature, previous, residual=True)
        stored = np.where(np.isfinite(temperature) & np.isfinite(previous), capacity * (temperature - previous), 0.0)
        expected = dev.stiffness_f64(temperature) + host.robin_only * temperature - host.robin_rhs + stored - host.load
        np.testing.assert_array_equal(out["residual"], expected)
        assert out["stored_heat_w"] == pytest.approx(float(np.sum(stored)), rel=1e-13, abs=1e-15)


def test_new_boundaries_and_capacity_on_a_resident_system_equal_a_fresh_one() -> None:
    problem = CASES["voxel_body"](ns)
    rows, cols = problem.mesh.element_shape
    other = dataclasses.replace(problem, convection=(
        ns.ConvectionBoundary("bottom", np.linspace(1.0, 9.0, rows * cols).reshape(rows, cols), 290.0),
        ns.ExposedFaceConvection(3.0, np.full(problem.mesh.element_grid_shape, 310.0), directions=("+z", "-x")),
        ns.ConvectionBoundary("top", 4.0, 305.0),
    ))
    capacity = np.full(problem.mesh.size, 1e-3)
    with _system(problem) as dev, _system(other, capacity) as fresh:
        from pcb_analysis_b200.thermal.system import convection_specs

        dev.set_convection(convection_specs(other.convection))
        dev.set_capacity(capacity)
        a, b = dev.prepared(), fresh.prepared()
        for key in a:
            np.testing.assert_array_equal(a[key], b[key])
        np.testing.assert_array_equal(dev.diagonal(), fresh.diagonal())
        for i in range(3):
            np.testing.assert_array_equal(dev.boundary_weights(i)[0], fresh.boundary_weights(i)[0])
        host = prepare(other, capacity)
        np.testing.assert_array_equal(a["robin_total"], host.robin_total)
        np.testing.assert_array_equal(a["robin_rhs"], host.robin_rhs)


def test_invalid_problems_and_misuse_are_refused() -> None:
    from pcb_analysis_b200._native import DeviceSystem

    problem = CASES["voxel_body"](ns)
    inputs = problem_inputs(problem)
    bad = dict(inputs, convection=[dict(inputs["convection"][0], coefficient=-np.ones((7, 9)))])
    with pytest.raises(ValueError, match="film coefficient"):
        DeviceSystem.from_problem(**bad)
    bad = dict(inputs, sources=[(np.array([problem.mesh.size]), 1.0)])
    with pytest.raises(ValueError, match="outside the grid"):
        DeviceSystem.from_problem(**bad)
    bad = dict(inputs, k_in=np.full(problem.mesh.element_grid_shape, np.nan))
    with pytest.raises(ValueError, match="conductivities"):
        DeviceSystem.from_problem(**bad)
    with DeviceSystem.from_problem(**inputs) as dev:
        with pytest.raises(ValueError, match="tb_set_convection"):
            dev.set_robin(np.zeros(problem.mesh.size))
        with pytest.raises(ValueError, match="capacity_per_s"):
            dev.set_capacity(np.full(problem.mesh.size, -1.0))
