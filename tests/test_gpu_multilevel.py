"""The device multilevel preconditioner against its CPU restatement
(oracle/multilevel.py), and multilevel MPIR solves against the reference's
converged temperatures and the FP64 oracle.

Tolerances:
* grid shapes: equal;
* coarse stencils (FP32 copies of FP64 Galerkin sums): within 1e-6 of the
  level's largest coefficient;
* the coarsest dense matrix (FP64): within 1e-11 of its largest entry;
* the FP32 preconditioner action: ||y - y_ref|| <= 1e-4 ||y_ref|| (an FP32
  V-cycle against the FP64 restatement);
* temperatures: rtol 1e-8, atol 1e-7 K against the reference's fixtures
  (as the two-level solves), and 1e-8 of the peak rise against the FP64
  oracle PCG on seeded boards, every solve converged to 1e-10.
"""

from __future__ import annotations

import numpy as np
import pytest

import pcb_analysis_b200.thermal as ns
from oracle.multilevel import MultilevelOracle
from oracle.oracle import OracleSystem
from pcb_analysis_b200.mpir import MPIRConfig, solve_mpir
from pcb_analysis_b200.workloads import board_c3
from tests.conftest import golden_cases, load_golden
from tests.problems import CASES

pytestmark = pytest.mark.gpu

CONFIG = MPIRConfig(inner_relative_tolerance=1e-4, max_outer_iterations=30, max_inner_iterations=100000)


def _board(slabs, rows, cols, seed, fixed=0.0):
    rng = np.random.default_rng(seed)
    k_in = np.where(rng.random((slabs, rows, cols)) < 0.6, 385.0, 0.3)
    k_in[1::2] = 0.3
    node_shape = (slabs + 1, rows + 1, cols + 1)
    robin = np.zeros(node_shape)
    robin[-1] = 25.0 * 0.0625e-6
    robin[0] = 5.0 * 0.0625e-6
    free = np.ones(node_shape, dtype=np.uint8)
    if fixed:
        free[0, :, : max(1, int(fixed * (cols + 1)))] = 0
    thick = np.where(np.arange(slabs) % 2 == 0, 35e-6, 0.16e-3)
    return dict(slab_thickness_m=thick, pitch_x_m=np.full(cols, 0.25e-3), pitch_y_m=np.full(rows, 0.25e-3),
                k_in=k_in, k_z=k_in.copy(), robin_total=robin.reshape(-1), free_nodes=free.reshape(-1))


# (slabs, rows, cols): one coarse grid only; two and three V-cycle levels; a
# ragged 9-plane stack (the smallest plane bucket); 17 and 25 planes; first
# coarse grids more than 200 columns across along x and along y, which form
# the next grid from 2 x 2 aggregates (then 4 x 4).
SHAPES = [(3, 30, 41), (7, 72, 84), (8, 150, 131), (8, 61, 203), (16, 90, 70), (24, 40, 36), (3, 40, 830),
          (5, 850, 45)]


@pytest.mark.parametrize("shape", SHAPES)
def test_hierarchy_matches_the_oracle(shape) -> None:
    from pcb_analysis_b200._native import DeviceSystem

    arrays = _board(*shape, seed=sum(shape), fixed=0.08)
    free = arrays.pop("free_nodes")
    oracle = OracleSystem.from_arrays(free=free, **arrays)
    expect = MultilevelOracle(oracle.coef, oracle.robin_total, oracle.free)
    with DeviceSystem(free_nodes=free, **arrays) as dev:
        dev.set_preconditioner("multilevel")
        info = dev.preconditioner()
        assert info["kind"] == "multilevel"
        assert info["levels"] == expect.grids
        for level in range(1, len(expect.grids)):
            st = dev.multilevel_stencil(level)
            ref = expect.stencil(level)
            np.testing.assert_allclose(st, ref, rtol=0, atol=1e-6 * np.abs(ref).max())
        matrix, _ = dev.coarse()
        dense = expect.A[-1].toarray()
        np.testing.assert_allclose(matrix, dense, rtol=0, atol=1e-11 * np.abs(dense).max())
        for seed in (3, 4):
            x = np.random.default_rng(seed).standard_normal(oracle.size).astype(np.float32)
            y = dev.precondition_f32(x)
            ref = expect.precondition(x.astype(np.float64))
            assert np.linalg.norm(y - ref) <= 1e-4 * np.linalg.norm(ref)


@pytest.mark.parametrize("name", golden_cases())
def test_multilevel_mpir_reaches_the_reference_temperatures(name: str) -> None:
    g = load_golden(name)
    solution = ns.solve_thermal_conduction(CASES[name](ns), config=CONFIG, preconditioner="multilevel")
    assert solution.solve.converged
    assert solution.solve.relative_residual <= 1e-10
    t = solution.temperature_k.reshape(-1)
    for tag in ("two_level", "fp64_pcg"):
        ref = g[f"{tag}_temperature"]
        finite = np.isfinite(ref)
        np.testing.assert_array_equal(finite, np.isfinite(t))
        np.testing.assert_allclose(t[finite], ref[finite], rtol=1e-8, atol=1e-7)
    assert solution.heat_balance_error_w == pytest.approx(0.0, abs=1e-8)


def test_multilevel_solve_of_a_c3_cut_matches_the_fp64_oracle_and_cuts_iterations() -> None:
    problem = board_c3(seed=0, rows=192, cols=224)
    ml = ns.MatrixFreeThermalOperator(problem, preconditioner="multilevel")
    two = ns.MatrixFreeThermalOperator(problem)
    try:
        assert len(ml.device_system.preconditioner()["levels"]) >= 2
        rhs = ml.build_rhs(ml.default_reference_temperature())
        a = solve_mpir(ml, rhs, config=CONFIG)
        b = solve_mpir(ml, rhs, config=CONFIG)
        t = solve_mpir(two, rhs, config=CONFIG)
        assert a.converged and a.relative_residual <= 1e-10
        np.testing.assert_array_equal(a.solution, b.solution)  # bit-repeatable
        assert a.history == b.history
        assert 4 * a.inner_iterations < t.inner_iterations, (a.inner_iterations, t.inner_iterations)
        from pcb_analysis_b200.thermal.system import prepare

        host = prepare(problem)
        oracle = OracleSystem(np.stack(problem.mesh.element_coefficients()), host.robin_total,
                              host.free_nodes.reshape(-1).astype(np.uint8))
        theta, _, rel = oracle.pcg_f64(rhs, rtol=1e-11)
        assert rel <= 1e-11
        np.testing.assert_allclose(a.solution, theta, rtol=0, atol=1e-8 * np.abs(theta).max())
    finally:
        ml.close()
        two.close()


def test_resident_boundary_change_rebuilds_the_hierarchy() -> None:
    problem = CASES["seeded_board_24x30"](ns)
    op = ns.MatrixFreeThermalOperator(problem, preconditioner="multilevel")
    try:
        capacity = np.full(op.size, 1e-4)
        op.set_capacity_per_s(capacity)
        fresh = ns.MatrixFreeThermalOperator(problem, preconditioner="multilevel", capacity_per_s=capacity)
        try:
            x = np.random.default_rng(9).standard_normal(op.size).astype(np.float32)
            np.testing.assert_array_equal(op.precondition_low(x), fresh.precondition_low(x))
        finally:
            fresh.close()
    finally:
        op.close()


# (slabs, rows, cols): the plane buckets 9, 17 and 33 (2 to 4 stages), a
# ragged board whose last column and row tiles reach past the field, and a
# board with fewer column tiles than the device has SMs.
STAGED_SHAPES = [(8, 150, 131), (16, 192, 224), (24, 61, 203), (5, 20, 30)]


@pytest.mark.parametrize("shape", STAGED_SHAPES)
def test_staged_fine_pass_matches_the_loading_kernel(shape) -> None:
    """The fine pass fed by tensor copies against the kernel that loads its own
    columns (the default): the same arithmetic per column, only the merge order
    of r.r and r.T^-1 r differs, so both solves converge to the same
    temperatures (1e-8 of the peak rise) in nearly the same iteration count,
    and the staged solve is bit-repeatable."""

    from pcb_analysis_b200._native import DeviceSystem

    arrays = _board(*shape, seed=sum(shape) + 5, fixed=0.05)
    rhs = np.zeros((shape[0] + 1, shape[1] + 1, shape[2] + 1))
    rhs[-1, shape[1] // 2, shape[2] // 3] = 1.0
    rhs[0, shape[1] // 3, shape[2] // 2] = 0.5
    rhs = rhs.reshape(-1) * arrays["free_nodes"]
    with DeviceSystem(**arrays) as dev:
        dev.set_preconditioner("multilevel")
        assert not dev.ml_staging
        dev.ml_staging = True
        assert dev.ml_staging
        a = dev.solve_mpir(rhs, CONFIG)
        b = dev.solve_mpir(rhs, CONFIG)
        dev.ml_staging = False
        assert not dev.ml_staging
        c = dev.solve_mpir(rhs, CONFIG)
        dev.ml_staging = True
        d = dev.solve_mpir(rhs, CONFIG)
    for out in (a, c):
        assert out["converged"] and out["relative_residual"] <= 1e-10
    np.testing.assert_array_equal(a["solution"], b["solution"])
    np.testing.assert_array_equal(a["solution"], d["solution"])
    assert a["history"] == b["history"] == d["history"]
    peak = np.abs(c["solution"]).max()
    np.testing.assert_allclose(a["solution"], c["solution"], rtol=0, atol=1e-8 * peak)
    assert abs(a["inner_iterations"] - c["inner_iterations"]) <= max(3, c["inner_iterations"] // 20)


def test_staged_fine_pass_wait_that_runs_out_is_reported_and_the_system_stays_usable() -> None:
    """With the operator on its cp.async staging, the stage test switch leaves
    only the staged fine pass waiting for copies that are never issued: every
    wait gives up after 64 polls, the solve fails with TimeoutError, and with
    the switch off the system gives the bits it gave before."""

    from pcb_analysis_b200._native import DeviceSystem

    arrays = _board(8, 72, 84, seed=21)
    rhs = np.zeros((9, 73, 85))
    rhs[-1, 36, 42] = 1.0
    rhs = rhs.reshape(-1)
    with DeviceSystem(**arrays) as dev:
        dev.set_preconditioner("multilevel")
        dev.apply_plan = (0, 16, 0, 0, 0)
        dev.ml_staging = True
        before = dev.solve_mpir(rhs, CONFIG)
        assert before["converged"]
        dev.set_stage_test(64)
        with pytest.raises(TimeoutError, match="staged tiles"):
            dev.solve_mpir(rhs, CONFIG)
        dev.set_stage_test(0)
        again = dev.solve_mpir(rhs, CONFIG)
        np.testing.assert_array_equal(again["solution"], before["solution"])
        assert again["history"] == before["history"]
