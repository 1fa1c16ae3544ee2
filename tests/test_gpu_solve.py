"""Device MPIR and FP64 PCG solves against the reference's converged temperatures.

The reference's solutions (tests/golden) were converged to relative residual
1e-10; so are these.  Temperatures are compared with the reference's own
cross-implementation tolerance (tests/test_cuda_thermal_conduction.py:101:
rtol 1e-8, atol 1e-7 K), the analytic cases with the bounds of
tests/test_thermal_conduction.py.
"""

from __future__ import annotations

import numpy as np
import pytest

import pcb_analysis_b200.thermal as ns
from oracle.oracle import OracleSystem
from pcb_analysis_b200.mpir import MPIRConfig, solve_mpir
from tests.conftest import golden_cases, load_golden
from tests.problems import CASES, fixed_faces, parabola

pytestmark = pytest.mark.gpu

CONFIG = MPIRConfig(inner_relative_tolerance=1e-4, max_outer_iterations=30, max_inner_iterations=100000)


@pytest.mark.parametrize("name", golden_cases())
def test_device_mpir_reaches_the_reference_temperatures(name: str) -> None:
    g = load_golden(name)
    problem = CASES[name](ns)
    solution = ns.solve_thermal_conduction(problem, preconditioner="jacobi", config=CONFIG)
    assert solution.solve.converged
    assert solution.solve.relative_residual <= 1e-10
    assert solution.solve.low_runtime == "b200-fp32"
    t = solution.temperature_k.reshape(-1)
    for tag in ("fp64_pcg", "two_level"):
        ref = g[f"{tag}_temperature"]
        finite = np.isfinite(ref)
        np.testing.assert_array_equal(finite, np.isfinite(t))
        np.testing.assert_allclose(t[finite], ref[finite], rtol=1e-8, atol=1e-7)
    budget = g["fp64_pcg_budget"]
    assert solution.total_heat_input_w == pytest.approx(budget[0], rel=1e-12, abs=1e-15)
    np.testing.assert_allclose(solution.convective_heat_w, g["fp64_pcg_convective"], rtol=1e-6, atol=1e-9)
    assert solution.heat_balance_error_w == pytest.approx(0.0, abs=1e-8)
    np.testing.assert_allclose(solution.heat_flux_w_per_m2, g["fp64_pcg_flux"], rtol=1e-6,
                               atol=1e-6 * np.abs(g["fp64_pcg_flux"]).max())


def test_fixed_faces_give_a_linear_profile_and_the_exact_flux() -> None:
    solution = ns.solve_thermal_conduction(fixed_faces(ns), preconditioner="jacobi", config=CONFIG)
    assert solution.solve.converged
    for face, temperature in zip(300.0 + 12.5 * np.arange(5), solution.temperature_k):
        np.testing.assert_allclose(temperature, face, rtol=1e-8)
    flux_error = 2.0 * 1e-8 * 350.0 / 0.5e-3
    np.testing.assert_allclose(solution.heat_flux_w_per_m2[..., 2], -50.0 / 2.0e-3, rtol=0, atol=flux_error)
    assert solution.fixed_temperature_heat_w == pytest.approx(0.0, abs=1e-9)
    assert solution.heat_balance_error_w == pytest.approx(0.0, abs=1e-9)


def test_uniform_heating_with_one_cooled_face_matches_the_parabola() -> None:
    solution = ns.solve_thermal_conduction(parabola(ns), preconditioner="jacobi", config=CONFIG,
                                           initial_temperature_k=300.0)
    area, thickness, flux = 4.0e-3 * 5.0e-3, 2.0e-3, 1.0 / (4.0e-3 * 5.0e-3)
    top = 300.0 + flux / 100.0
    bottom = top + flux * thickness / (2.0 * 0.3)
    assert solution.solve.converged
    assert solution.temperature_k[-1, 2, 2] == pytest.approx(top, rel=1e-9)
    assert solution.temperature_k[0, 2, 2] == pytest.approx(bottom, rel=1e-9)
    assert solution.convective_heat_w[0] == pytest.approx(1.0, rel=1e-9)
    assert solution.heat_balance_error_w == pytest.approx(0.0, abs=1e-9)


def test_mpir_history_and_counts_follow_the_reference_contract() -> None:
    problem = CASES["stack_12x20_fixed"](ns)
    op = ns.MatrixFreeThermalOperator(problem, preconditioner="jacobi")
    try:
        rhs = op.build_rhs(op.default_reference_temperature())
        result = solve_mpir(op, rhs, config=CONFIG)
        assert result.converged
        assert result.low_operator_applications > 5 * result.high_operator_applications
        assert result.high_operator_applications == result.outer_iterations + 1
        assert len(result.history) == result.outer_iterations
        assert sum(s.inner_iterations for s in result.history) == result.inner_iterations
        assert result.history[0].high_relative_residual == pytest.approx(1.0)
        residual = rhs - op.apply_high(result.solution)
        assert np.linalg.norm(residual) <= 1.0000001e-10 * np.linalg.norm(rhs)
        again = solve_mpir(op, rhs, config=CONFIG)
        np.testing.assert_array_equal(again.solution, result.solution)  # bit-repeatable
        assert again.history == result.history
    finally:
        op.close()


def test_power_of_two_scaling_keeps_a_tiny_correction_to_the_bit() -> None:
    """A 2^-70 right-hand side gives the unit answer times 2^-70 exactly
    (tests/test_matrix_free_mpir_fem.py:268 of pcb-analysis)."""

    problem = CASES["mixed_board"](ns)
    op = ns.MatrixFreeThermalOperator(problem, preconditioner="jacobi")
    try:
        rhs = op.build_rhs(op.default_reference_temperature())
        config = MPIRConfig(inner_relative_tolerance=1e-4, max_outer_iterations=3, max_inner_iterations=5000)
        big = solve_mpir(op, rhs, config=config)
        small = solve_mpir(op, rhs * 2.0**-70, config=config)
        np.testing.assert_array_equal(small.solution * 2.0**70, big.solution)
        assert [s.inner_iterations for s in small.history] == [s.inner_iterations for s in big.history]
    finally:
        op.close()


def test_device_fp64_pcg_matches_the_oracle() -> None:
    g = load_golden("seeded_board_24x30")
    problem = CASES["seeded_board_24x30"](ns)
    op = ns.MatrixFreeThermalOperator(problem, preconditioner="jacobi")
    try:
        out = op.device_system.solve_pcg_f64(g["rhs"], relative_tolerance=1e-10, max_iterations=200000)
        assert out["converged"] and out["relative_residual"] <= 1e-10
        oracle = OracleSystem(g["coef"], g["robin_total"], g["free"])
        x, _, _ = oracle.pcg_f64(g["rhs"], rtol=1e-10)
        np.testing.assert_allclose(out["solution"], x, rtol=1e-7, atol=1e-9 * np.abs(x).max())
    finally:
        op.close()


def test_zero_rhs_returns_zero_without_iterating() -> None:
    problem = CASES["stack_12x20"](ns)
    op = ns.MatrixFreeThermalOperator(problem, preconditioner="jacobi")
    try:
        result = solve_mpir(op, np.zeros(op.size), config=CONFIG)
        assert result.converged and result.inner_iterations == 0
        assert not np.any(result.solution)
    finally:
        op.close()


def test_both_operator_kernels_reach_the_same_solution() -> None:
    """The z-marching tile kernel (one block per tile, or one balanced wave)
    and the warp-marching kernel solve to the same temperatures."""

    problem = CASES["seeded_board_24x30"](ns)
    op = ns.MatrixFreeThermalOperator(problem, preconditioner="jacobi")
    try:
        rhs = op.build_rhs(op.default_reference_temperature())
        op.device_system.apply_plan = (0, 16, 0, 0, 0)
        tiles = solve_mpir(op, rhs, config=CONFIG)
        op.device_system.apply_plan = (1, 16, 2, 2, 8)
        warps = solve_mpir(op, rhs, config=CONFIG)
        op.device_system.apply_plan = (2, 8, 0, 0, 0)
        balanced = solve_mpir(op, rhs, config=CONFIG)
        assert tiles.converged and warps.converged and balanced.converged
        scale = np.abs(tiles.solution).max()
        np.testing.assert_allclose(warps.solution, tiles.solution, rtol=0, atol=1e-8 * scale)
        np.testing.assert_allclose(balanced.solution, tiles.solution, rtol=0, atol=1e-8 * scale)
    finally:
        op.close()


def test_tensor_copy_staging_gives_the_same_two_level_solve() -> None:
    """The two-level MPIR solve with the operator fed by tensor copies
    reproduces the cp.async-fed solve bit for bit: same inner products, same
    iteration counts, same temperatures."""

    problem = CASES["seeded_board_24x30"](ns)
    op = ns.MatrixFreeThermalOperator(problem)
    try:
        rhs = op.build_rhs(op.default_reference_temperature())
        for kind, rows in ((0, 8), (2, 16)):
            op.device_system.apply_plan = (kind, rows, 0, 0, 0)
            plain = solve_mpir(op, rhs, config=CONFIG)
            op.device_system.apply_plan = (kind, rows, 1, 0, 0)
            staged = solve_mpir(op, rhs, config=CONFIG)
            assert plain.converged and staged.converged
            assert staged.inner_iterations == plain.inner_iterations
            np.testing.assert_array_equal(staged.solution, plain.solution)
    finally:
        op.close()
