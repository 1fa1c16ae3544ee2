"""Backward-Euler transients on the resident device system, held to the
known answers of the reference's tests/test_thermal_transient.py (discrete
cooling law of a lumped block, march to the steady state, a radiating body)
and to a march that prepares a fresh system for every step."""

from __future__ import annotations

import numpy as np
import pytest

import pcb_analysis_b200.thermal as ns
from pcb_analysis_b200.thermal.solve import _solve

pytestmark = pytest.mark.gpu

AMBIENT = 300.0
COPPER_RHO_C = 3.45e6  # J/m3K


def test_lumped_block_follows_the_discrete_backward_euler_law() -> None:
    """T_{n+1} = T_a + (T_n - T_a) / (1 + dt / tau), tau = rho c t / h, for a
    nearly isothermal copper block cooled on top."""

    thickness, h, start = 2.0e-3, 20.0, 350.0
    mesh = ns.LayeredThermalMesh((thickness,), 1e-3, 1e-3, 4000.0, element_shape=(4, 5),
                                 volumetric_heat_capacity_j_per_m3_k=COPPER_RHO_C)
    problem = ns.ThermalConductionProblem(mesh, convection=(ns.ConvectionBoundary("top", h, AMBIENT),))
    schedule = ns.TimeSchedule.uniform(20.0, 400.0)
    solution = ns.solve_thermal_transient(problem, schedule, initial_temperature_k=start)
    assert solution.temperature_k.shape == (21, *mesh.node_shape)
    np.testing.assert_allclose(solution.temperature_k[0], start)
    tau = COPPER_RHO_C * thickness / h
    expected = start
    for step in solution.history:
        expected = AMBIENT + (expected - AMBIENT) / (1.0 + step.step_s / tau)
        assert step.max_temperature_k == pytest.approx(expected, abs=2.0e-4)
        assert step.converged
        assert step.stored_heat_w == pytest.approx(-step.convective_heat_w, rel=1e-9)
        assert abs(step.heat_balance_error_w) < 1e-9
    analytic = AMBIENT + (start - AMBIENT) * np.exp(-schedule.end_s / tau)
    assert abs(solution.history[-1].max_temperature_k - analytic) < 0.6
    finer = ns.solve_thermal_transient(problem, ns.TimeSchedule.uniform(5.0, 400.0), initial_temperature_k=start,
                                       store="final")
    assert finer.temperature_k.shape == (1, *mesh.node_shape)
    assert abs(finer.history[-1].max_temperature_k - analytic) < 0.16


def _heated_plate():
    mesh = ns.LayeredThermalMesh(
        (35e-6, 1.5e-3, 35e-6), 0.5e-3, 0.5e-3, (385.0, 0.8, 385.0), element_shape=(8, 12),
        through_plane_conductivity_w_per_m_k=(385.0, 0.3, 385.0),
        volumetric_heat_capacity_j_per_m3_k=(COPPER_RHO_C, 1.8e6, COPPER_RHO_C),
    )
    heat = np.zeros((3, 8, 12))
    heat[2, 3:5, 5:7] = 0.1
    return ns.ThermalConductionProblem(
        mesh, convection=(ns.ConvectionBoundary("top", 10.0, AMBIENT), ns.ConvectionBoundary("bottom", 10.0, AMBIENT)),
        element_heat_w=heat,
    )


def test_heated_plate_marches_to_the_steady_solution_and_stops() -> None:
    problem = _heated_plate()
    steady = ns.solve_thermal_conduction(problem)
    schedule = ns.TimeSchedule.geometric(0.01, 20000.0, growth=1.6)
    transient = ns.solve_thermal_transient(problem, schedule, until_steady=True, steady_tolerance_k_per_s=2e-5)
    assert transient.reached_steady and len(transient.history) < len(schedule.steps_s)
    rise = steady.max_temperature_k - AMBIENT
    assert rise > 5.0
    assert np.nanmax(np.abs(transient.final_temperature_k - steady.temperature_k)) < 2e-3 * rise
    peaks = transient.max_temperature_k
    assert peaks[0] > AMBIENT and np.all(np.diff(peaks) >= -1e-9)
    for step in transient.history:
        assert abs(step.heat_balance_error_w) < 1e-9
        assert step.stored_heat_w + step.convective_heat_w == pytest.approx(0.4, rel=1e-9)


@pytest.mark.parametrize("preconditioner", ["two-level", "jacobi"])
def test_resident_march_equals_a_fresh_system_per_step(preconditioner) -> None:
    """Rewriting C / dt on the resident system gives the bits of preparing
    the step's system from scratch."""

    problem = _heated_plate()
    schedule = ns.TimeSchedule((0.0, 0.5, 1.5, 2.5, 4.5))  # dt 0.5, 1, 1, 2: rewrites and one reuse
    march = ns.solve_thermal_transient(problem, schedule, preconditioner=preconditioner)
    capacity = problem.mesh.nodal_heat_capacity_j_per_k().reshape(-1)
    current = np.full(problem.mesh.node_shape, AMBIENT)
    for k, step_s in enumerate(schedule.steps_s, start=1):
        fresh = _solve(problem, initial_temperature_k=current, capacity_per_s=capacity / step_s,
                       previous_temperature_k=current, preconditioner=preconditioner)
        current = np.where(np.isfinite(fresh.temperature_k), fresh.temperature_k, current)
        np.testing.assert_array_equal(march.temperature_k[k], current)


def test_radiating_masked_body_relaxes_to_its_steady_state() -> None:
    active = np.zeros((3, 5, 5), dtype=bool)
    active[:, 1:4, 1:4] = True
    mesh = ns.LayeredThermalMesh((1e-3,) * 3, 1e-3, 1e-3, np.where(active, 200.0, 1.0), active=active,
                                 volumetric_heat_capacity_j_per_m3_k=np.where(active, 2.4e6, 1.0))
    problem = ns.ThermalConductionProblem(
        mesh, convection=(ns.ExposedFaceConvection(5.0, AMBIENT),),
        radiation=(ns.RadiationBoundary("top", 0.9, AMBIENT),), element_heat_w=np.where(active, 0.3 / 27, 0.0),
    )
    steady = ns.solve_thermal_conduction(problem)
    transient = ns.solve_thermal_transient(problem, ns.TimeSchedule.geometric(0.1, 20000.0, growth=1.7),
                                           until_steady=True, steady_tolerance_k_per_s=1e-5)
    assert transient.reached_steady
    assert np.all(np.isnan(transient.final_temperature_k[:, 0]))
    assert np.nanmax(np.abs(transient.final_temperature_k - steady.temperature_k)) < 1e-2
    last = transient.history[-1]
    assert last.radiation_iterations >= 1 and last.radiative_heat_w > 0.0
    assert last.stored_heat_w + last.convective_heat_w + last.radiative_heat_w == pytest.approx(0.3, rel=1e-9)
