"""Time schedules and the argument checks of the transient march (no device
needed; reference tests/test_thermal_transient.py:24-36,124-150)."""

from __future__ import annotations

import numpy as np
import pytest

import pcb_analysis_b200.thermal as ns


def test_time_schedules() -> None:
    assert ns.TimeSchedule.uniform(0.5, 2.0).times_s == (0.0, 0.5, 1.0, 1.5, 2.0)
    geometric = ns.TimeSchedule.geometric(1.0, 100.0, growth=2.0)
    assert geometric.times_s[:4] == (0.0, 1.0, 3.0, 7.0) and geometric.end_s == 100.0
    assert np.all(np.diff(geometric.times_s) > 0.0)
    assert max(ns.TimeSchedule.geometric(1.0, 20.0, growth=2.0, max_step_s=4.0).steps_s) == 4.0
    with pytest.raises(ValueError, match="start at 0"):
        ns.TimeSchedule((1.0, 2.0))
    with pytest.raises(ValueError, match="increasing"):
        ns.TimeSchedule((0.0, 2.0, 1.0))


def test_transient_arguments_are_checked_before_any_device_work() -> None:
    plain = ns.LayeredThermalMesh((1e-3,), 1e-3, 1e-3, 200.0, element_shape=(2, 2))
    problem = ns.ThermalConductionProblem(plain, convection=(ns.ConvectionBoundary("top", 5.0, 300.0),))
    with pytest.raises(ValueError, match="volumetric_heat_capacity"):
        ns.solve_thermal_transient(problem, ns.TimeSchedule.uniform(1.0, 2.0))
    with pytest.raises(ValueError, match="positive on active"):
        ns.LayeredThermalMesh((1e-3,), 1e-3, 1e-3, 200.0, element_shape=(2, 2),
                              volumetric_heat_capacity_j_per_m3_k=0.0)
    with_capacity = ns.LayeredThermalMesh((1e-3,), 1e-3, 1e-3, 200.0, element_shape=(2, 2),
                                          volumetric_heat_capacity_j_per_m3_k=1e6)
    np.testing.assert_allclose(with_capacity.nodal_heat_capacity_j_per_k().sum(), 1e6 * 4e-9)
    heated = ns.ThermalConductionProblem(with_capacity, convection=(ns.ConvectionBoundary("top", 5.0, 300.0),))
    with pytest.raises(ValueError, match="store"):
        ns.solve_thermal_transient(heated, ns.TimeSchedule.uniform(1.0, 2.0), store="none")
