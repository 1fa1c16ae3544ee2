"""The public steady solve keeps its right-hand side and solution in HBM.

solve_thermal_conduction builds the right-hand side on the device
(tb_build_rhs_device), solves from it (tb_solve_mpir_device), reads the
solution back once and post-processes T = rise + reference on the device
(tb_postprocess_rise_device).  The host-array route it replaces (reference
solve.py: operator.build_rhs, solve_mpir, the post-processing of the host
temperature) must give the same bits: temperature, flux, removed heat,
budget, the temperature extrema and the MPIR record, on boards with fixed
nodes, void elements, every preconditioner, and a transient step (previous
temperature on the device).
"""

from __future__ import annotations

import numpy as np
import pytest

import pcb_analysis_b200.thermal as ns
from pcb_analysis_b200.mpir import MPIRConfig, solve_mpir
from pcb_analysis_b200.thermal.operator import MatrixFreeThermalOperator
from pcb_analysis_b200.thermal.session import ResidentSolve
from tests.problems import CASES

pytestmark = pytest.mark.gpu

CONFIG = MPIRConfig(inner_relative_tolerance=1e-4, max_outer_iterations=40, max_inner_iterations=200000)


def _host_route(problem, preconditioner, reference, capacity=None, previous=None):
    op = MatrixFreeThermalOperator(problem, preconditioner=preconditioner, capacity_per_s=capacity)
    try:
        record = solve_mpir(op, op.build_rhs(reference, previous), config=CONFIG)
        temperature = record.solution.reshape(problem.mesh.node_shape) + reference
        post = op.postprocess(temperature, previous)
    finally:
        op.close()
    return record, temperature, post


@pytest.mark.parametrize("name", ["stack_12x20_fixed", "mixed_board", "voxel_body", "seeded_board_24x30"])
@pytest.mark.parametrize("preconditioner", ["jacobi", "two-level", "multilevel"])
def test_public_solve_equals_the_host_array_route_bit_for_bit(name: str, preconditioner: str) -> None:
    problem = CASES[name](ns)
    reference = 291.5
    solution = ns.solve_thermal_conduction(problem, preconditioner=preconditioner, config=CONFIG,
                                           reference_temperature_k=reference)
    record, temperature, post = _host_route(problem, preconditioner, reference)
    assert solution.solve.converged and record.converged
    np.testing.assert_array_equal(solution.solve.solution, record.solution)
    assert solution.solve.history == record.history
    assert solution.solve.inner_iterations == record.inner_iterations
    active = np.isfinite(solution.temperature_k)
    np.testing.assert_array_equal(solution.temperature_k[active], temperature[active])
    np.testing.assert_array_equal(solution.heat_flux_w_per_m2, post["heat_flux"])
    np.testing.assert_array_equal(solution.convective_heat_w, post["convective_heat_w"])
    assert solution.total_heat_input_w == post["total_heat_input_w"]
    assert solution.fixed_temperature_heat_w == post["fixed_temperature_heat_w"]
    # extrema reduced on the device over the active nodes, as nanmax / nanmin of the field with NaN on void nodes
    assert solution.max_temperature_k == float(np.max(temperature[active]))
    assert solution.min_temperature_k == float(np.min(temperature[active]))


def test_transient_step_with_the_previous_field_on_the_device() -> None:
    problem = CASES["stack_12x20_fixed"](ns)
    n = problem.mesh.size
    rng = np.random.default_rng(4)
    capacity = rng.uniform(1e-4, 1e-3, n)
    previous = 300.0 + rng.uniform(-2.0, 2.0, n)
    reference = 300.0
    with ResidentSolve(preconditioner="two-level") as session:
        solution = session.steady(problem, config=CONFIG, reference_temperature_k=reference,
                                  capacity_per_s=capacity, previous_temperature_k=previous)
    record, temperature, post = _host_route(problem, "two-level", reference, capacity, previous)
    np.testing.assert_array_equal(solution.solve.solution, record.solution)
    np.testing.assert_array_equal(solution.temperature_k.reshape(-1), temperature.reshape(-1))
    assert solution.stored_heat_w == post["stored_heat_w"]
    np.testing.assert_array_equal(solution.heat_flux_w_per_m2, post["heat_flux"])


def test_device_entry_points_refuse_wrong_tensors() -> None:
    import torch

    problem = CASES["stack_1x4"](ns)
    op = MatrixFreeThermalOperator(problem, preconditioner="jacobi")
    try:
        dev = op.device_system
        short = torch.zeros(op.size - 1, dtype=torch.float64, device="cuda:0")
        with pytest.raises(ValueError):
            dev.build_rhs_device(290.0, short)
        wrong = torch.zeros(op.size, dtype=torch.float32, device="cuda:0")
        with pytest.raises(ValueError):
            dev.postprocess_rise_device(wrong, 290.0)
        host = torch.zeros(op.size, dtype=torch.float64)
        with pytest.raises(ValueError):
            dev.build_rhs_device(290.0, host)
    finally:
        op.close()
