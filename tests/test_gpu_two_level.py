"""The device two-level preconditioner against the reference's coarse space
(tests/golden/coarse) and the oracle's restatement, and two-level MPIR solves
against the reference's converged temperatures.

Tolerances:
* Z^T A Z: every entry within 1e-11 of the largest (sums of FP64 actions
  that agree with the reference's to 64 eps);
* the inverse: within 1e-8 of the largest entry (Gauss-Jordan here, Cholesky
  in the reference; both FP64);
* the FP32 preconditioner action: ||y - y_ref|| <= 1e-5 ||y_ref||;
* temperatures: the reference's cross-implementation bound rtol 1e-8,
  atol 1e-7 K, both solves converged to relative residual 1e-10.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import pcb_analysis_b200.thermal as ns
from oracle.oracle import CoarseSpaceOracle, OracleSystem
from pcb_analysis_b200.mpir import MPIRConfig, solve_mpir
from tests.conftest import golden_cases, load_golden
from tests.problems import CASES

pytestmark = pytest.mark.gpu

COARSE = Path(__file__).resolve().parent / "golden" / "coarse"
CONFIG = MPIRConfig(inner_relative_tolerance=1e-4, max_outer_iterations=30, max_inner_iterations=100000)


def _split(tag: str):
    name, _, block = tag.rpartition("_b")
    if not name or not block.isdigit():
        return tag, None
    return name, int(block)


@pytest.mark.parametrize("tag", sorted(p.stem for p in COARSE.glob("*.npz")))
def test_coarse_space_matches_the_reference(tag: str) -> None:
    name, block = _split(tag)
    ref = np.load(COARSE / f"{tag}.npz")
    g = load_golden(name)
    op = ns.MatrixFreeThermalOperator(CASES[name](ns), coarse_block_nodes=block)
    try:
        info = op.device_system.preconditioner()
        assert info["kind"] == "two-level"
        assert info["block"] == int(ref["block"])
        assert info["coarse_shape"] == tuple(int(v) for v in ref["coarse_shape"])
        matrix, inverse = op.device_system.coarse()
        np.testing.assert_allclose(matrix, ref["coarse_matrix"], rtol=0,
                                   atol=1e-11 * np.abs(ref["coarse_matrix"]).max())
        np.testing.assert_allclose(inverse, ref["coarse_inverse"], rtol=0,
                                   atol=1e-8 * np.abs(ref["coarse_inverse"]).max())
        x32 = g["v64"].astype(np.float32)
        y = op.precondition_low(x32)
        oracle = OracleSystem(g["coef"], g["robin_total"], g["free"])
        expect = CoarseSpaceOracle(oracle, block=block).precondition_f64(x32.astype(np.float64))
        assert np.linalg.norm(y - expect) <= 1e-5 * np.linalg.norm(expect)
    finally:
        op.close()


def _board(slabs, rows, cols, seed, fixed=0.0):
    rng = np.random.default_rng(seed)
    k_in = np.where(rng.random((slabs, rows, cols)) < 0.5, 385.0, 0.3)
    node_shape = (slabs + 1, rows + 1, cols + 1)
    robin = np.zeros(node_shape)
    robin[-1] = rng.uniform(1e-7, 1e-6, robin[-1].shape)
    free = np.ones(node_shape, dtype=np.uint8)
    if fixed:
        free[0][rng.random(free[0].shape) < fixed] = 0
    return dict(slab_thickness_m=rng.uniform(0.035e-3, 0.4e-3, slabs), pitch_x_m=np.full(cols, 0.25e-3),
                pitch_y_m=np.full(rows, 0.25e-3), k_in=k_in, k_z=0.8 * k_in, robin_total=robin.reshape(-1),
                free_nodes=free.reshape(-1))


@pytest.mark.parametrize("shape,block", [((4, 80, 80), None), ((3, 30, 41), 3), ((2, 45, 37), 7), ((6, 9, 11), 1)])
def test_coarse_space_matches_the_oracle_on_other_patch_widths(shape, block) -> None:
    from pcb_analysis_b200._native import DeviceSystem

    arrays = _board(*shape, seed=sum(shape), fixed=0.1)
    free = arrays.pop("free_nodes")
    oracle = OracleSystem.from_arrays(free=free, **arrays)
    expect = CoarseSpaceOracle(oracle, block=block)
    with DeviceSystem(free_nodes=free, **arrays) as dev:
        dev.set_preconditioner("two-level", block)
        info = dev.preconditioner()
        assert info["block"] == expect.block and info["coarse_shape"] == tuple(expect.coarse_shape)
        matrix, inverse = dev.coarse()
        np.testing.assert_allclose(matrix, expect.coarse_matrix, rtol=0,
                                   atol=1e-11 * np.abs(expect.coarse_matrix).max())
        np.testing.assert_allclose(inverse, expect.coarse_inverse, rtol=0,
                                   atol=1e-8 * np.abs(expect.coarse_inverse).max())
        x = np.random.default_rng(3).standard_normal(oracle.size).astype(np.float32)
        y = dev.precondition_f32(x)
        ref = expect.precondition_f64(x.astype(np.float64))
        assert np.linalg.norm(y - ref) <= 1e-5 * np.linalg.norm(ref)


@pytest.mark.parametrize("name", golden_cases())
def test_two_level_mpir_reaches_the_reference_temperatures(name: str) -> None:
    g = load_golden(name)
    solution = ns.solve_thermal_conduction(CASES[name](ns), config=CONFIG)
    assert solution.solve.converged
    assert solution.solve.relative_residual <= 1e-10
    t = solution.temperature_k.reshape(-1)
    for tag in ("two_level", "fp64_pcg"):
        ref = g[f"{tag}_temperature"]
        finite = np.isfinite(ref)
        np.testing.assert_array_equal(finite, np.isfinite(t))
        np.testing.assert_allclose(t[finite], ref[finite], rtol=1e-8, atol=1e-7)
    assert solution.heat_balance_error_w == pytest.approx(0.0, abs=1e-8)


def test_two_level_cuts_iterations_and_is_bit_repeatable() -> None:
    problem = CASES["seeded_board_24x30"](ns)
    two = ns.MatrixFreeThermalOperator(problem)
    jac = ns.MatrixFreeThermalOperator(problem, preconditioner="jacobi")
    try:
        rhs = two.build_rhs(two.default_reference_temperature())
        a = solve_mpir(two, rhs, config=CONFIG)
        b = solve_mpir(two, rhs, config=CONFIG)
        j = solve_mpir(jac, rhs, config=CONFIG)
        assert a.converged and j.converged
        assert a.inner_iterations < j.inner_iterations
        np.testing.assert_array_equal(a.solution, b.solution)
        assert a.history == b.history
        residual = rhs - two.apply_high(a.solution)
        assert np.linalg.norm(residual) <= 1.0000001e-10 * np.linalg.norm(rhs)
        scale = np.abs(j.solution).max()
        np.testing.assert_allclose(a.solution, j.solution, rtol=0, atol=1e-8 * scale)
    finally:
        two.close()
        jac.close()


def test_switching_back_to_jacobi_restores_its_solve() -> None:
    problem = CASES["mixed_board"](ns)
    op = ns.MatrixFreeThermalOperator(problem, preconditioner="jacobi")
    try:
        rhs = op.build_rhs(op.default_reference_temperature())
        before = solve_mpir(op, rhs, config=CONFIG)
        op.device_system.set_preconditioner("two-level")
        middle = solve_mpir(op, rhs, config=CONFIG)
        op.device_system.set_preconditioner("jacobi")
        after = solve_mpir(op, rhs, config=CONFIG)
        np.testing.assert_array_equal(after.solution, before.solution)
        assert middle.converged and middle.inner_iterations <= before.inner_iterations
    finally:
        op.close()
