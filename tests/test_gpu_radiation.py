"""Radiation as a Newton-linearised Robin boundary, on one resident device
system per solve, held to the known answers of the reference's
tests/test_thermal_radiation.py (analytic surface temperatures of a
radiating plate, the shared convection/radiation budget, a radiating cube in
a void)."""

from __future__ import annotations

import numpy as np
import pytest

import pcb_analysis_b200.thermal as ns

pytestmark = pytest.mark.gpu

SIGMA = ns.STEFAN_BOLTZMANN_W_PER_M2_K4
ROWS, COLS, PITCH, THICKNESS, K = 8, 10, 1.0e-3, 1.0e-3, 200.0
AREA = ROWS * COLS * PITCH * PITCH
AMBIENT = 300.0


def _plate(power_w):
    mesh = ns.LayeredThermalMesh((THICKNESS,), PITCH, PITCH, K, element_shape=(ROWS, COLS))
    return mesh, np.full((1, ROWS, COLS), power_w / (ROWS * COLS))


@pytest.mark.parametrize("power_w, emissivity", [(0.05, 0.9), (0.6, 0.8), (3.0, 0.8)])
@pytest.mark.parametrize("kind", ["top", "exposed"])
def test_radiating_plate_reaches_the_analytic_surface_temperature(kind, power_w, emissivity) -> None:
    mesh, heat = _plate(power_w)
    radiation = (ns.RadiationBoundary("top", emissivity, AMBIENT) if kind == "top"
                 else ns.ExposedFaceRadiation(emissivity, AMBIENT, directions=("+z",)))
    solution = ns.solve_thermal_conduction(ns.ThermalConductionProblem(mesh, radiation=(radiation,),
                                                                       element_heat_w=heat))
    surface = (AMBIENT**4 + power_w / (emissivity * SIGMA * AREA)) ** 0.25
    drop = power_w / AREA * THICKNESS / (2.0 * K)  # uniform heat conducted to the top face
    assert solution.radiation_converged and solution.solve.converged
    assert solution.radiation_iterations <= 15
    np.testing.assert_allclose(solution.temperature_k[1], surface, rtol=1.0e-7)
    np.testing.assert_allclose(solution.temperature_k[0], surface + drop, rtol=1.0e-7)
    assert solution.radiative_heat_w.shape == (1,) and solution.convective_heat_w.shape == (0,)
    assert solution.radiative_heat_w[0] == pytest.approx(power_w, rel=1.0e-9)
    assert abs(solution.heat_balance_error_w) < 1.0e-9 * max(power_w, 1.0)


def test_newton_loop_is_short_and_confirms_a_warm_start_in_one_step() -> None:
    mesh, heat = _plate(0.05)
    problem = ns.ThermalConductionProblem(mesh, radiation=(ns.RadiationBoundary("top", 0.8, AMBIENT),),
                                          element_heat_w=heat)
    solution = ns.solve_thermal_conduction(problem)
    assert 40.0 < solution.max_temperature_k - AMBIENT < 120.0
    assert solution.radiation_iterations <= 6
    again = ns.solve_thermal_conduction(problem, initial_temperature_k=solution.temperature_k)
    assert again.radiation_iterations == 1


def test_convection_and_radiation_share_the_budget() -> None:
    mesh, heat = _plate(0.6)
    h, emissivity = 8.0, 0.85
    solution = ns.solve_thermal_conduction(ns.ThermalConductionProblem(
        mesh, convection=(ns.ConvectionBoundary("top", h, AMBIENT),),
        radiation=(ns.RadiationBoundary("top", emissivity, AMBIENT),), element_heat_w=heat))
    surface = float(np.mean(solution.temperature_k[1]))
    convective = h * AREA * (surface - AMBIENT)
    radiative = emissivity * SIGMA * AREA * (surface**4 - AMBIENT**4)
    assert solution.convective_heat_w[0] == pytest.approx(convective, rel=1.0e-6)
    assert solution.radiative_heat_w[0] == pytest.approx(radiative, rel=1.0e-6)
    assert convective + radiative == pytest.approx(0.6, rel=1.0e-6)
    only_convection = ns.solve_thermal_conduction(ns.ThermalConductionProblem(
        mesh, convection=(ns.ConvectionBoundary("top", h, AMBIENT),), element_heat_w=heat))
    assert AMBIENT < solution.max_temperature_k < only_convection.max_temperature_k


def test_cube_in_a_void_radiates_from_its_exposed_faces() -> None:
    active = np.zeros((4, 6, 6), dtype=bool)
    active[1:3, 2:4, 2:4] = True
    mesh = ns.LayeredThermalMesh((1e-3,) * 4, 1e-3, 1e-3, np.where(active, 200.0, 1.0), active=active)
    solution = ns.solve_thermal_conduction(ns.ThermalConductionProblem(
        mesh, radiation=(ns.ExposedFaceRadiation(0.9, AMBIENT),), element_heat_w=np.where(active, 0.5 / 8, 0.0)))
    surface = (AMBIENT**4 + 0.5 / (0.9 * SIGMA * 6 * (2e-3) ** 2)) ** 0.25
    assert solution.radiation_converged
    assert solution.radiative_heat_w[0] == pytest.approx(0.5, rel=1.0e-9)
    assert surface - 0.5 < np.nanmin(solution.temperature_k) and np.nanmax(solution.temperature_k) < surface + 0.5
    assert np.all(np.isnan(solution.temperature_k[0])) and np.all(np.isnan(solution.temperature_k[:, 0]))
