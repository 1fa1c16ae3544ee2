"""Parity at the benchmark configurations, and the re-reference restart.

* c1 (128 x 128 x 8, 149,769 nodes) solved by solve_thermal_conduction with
  each preconditioner: the temperature rise within 1e-6 of the peak rise of
  the FP64 oracle's Jacobi PCG converged to 1e-11 (the accuracy bar of the
  solve: <= 1e-6 relative in temperature, both at rtol <= 1e-10; reference
  tests/test_cuda_thermal_conduction.py:89-101 holds its GPU solve to the CPU
  one at rtol 1e-8).
* Boards drawn by the c4 (batched) and c5 (served) rules, solved together in
  the batch engine: each rise within 1e-6 of its peak rise of the FP64
  restatement (oracle/multilevel.py PCG, converged to 1e-11), residual 1e-10.
* A solve that does not converge in its first refinement run re-references
  to the mean free rise and resumes from the iterate (reference
  src/thermal/matrix_free_mpir_fem/solve.py:228-254): both runs' histories,
  and their counts summed, make the record.
"""

from __future__ import annotations

import numpy as np
import pytest

import pcb_analysis_b200.thermal as ns
from oracle.multilevel import MultilevelOracle
from oracle.oracle import OracleSystem
from pcb_analysis_b200.mpir import MPIRConfig
from pcb_analysis_b200.thermal.system import prepare
from pcb_analysis_b200.workloads import board_c1, board_random, request_c5
from tests.problems import CASES

pytestmark = pytest.mark.gpu

CONFIG = MPIRConfig(inner_relative_tolerance=1e-4, max_outer_iterations=40, max_inner_iterations=400000)


def _oracle(problem) -> OracleSystem:
    host = prepare(problem)
    return OracleSystem(np.stack(problem.mesh.element_coefficients()), host.robin_total,
                        host.free_nodes.reshape(-1).astype(np.uint8))


@pytest.fixture(scope="module")
def c1_reference():
    problem = board_c1(0)
    op = ns.MatrixFreeThermalOperator(problem, preconditioner="jacobi")
    try:
        reference = op.default_reference_temperature()
        rhs = op.build_rhs(reference)
    finally:
        op.close()
    theta, _, rel = _oracle(problem).pcg_f64(rhs, rtol=1e-11)
    assert rel <= 1e-10
    return problem, reference, theta


@pytest.mark.parametrize("preconditioner", ["jacobi", "two-level", "multilevel"])
def test_c1_board_matches_the_fp64_oracle(c1_reference, preconditioner: str) -> None:
    problem, reference, theta = c1_reference
    solution = ns.solve_thermal_conduction(problem, preconditioner=preconditioner, config=CONFIG)
    assert solution.solve.converged and solution.solve.relative_residual <= 1e-10
    rise = solution.temperature_k.reshape(-1) - reference
    peak = np.abs(theta).max()
    assert peak > 1.0
    assert np.abs(rise - theta).max() <= 1e-6 * peak
    assert abs(solution.heat_balance_error_w) <= 1e-8 * solution.total_heat_input_w


def _small_boards(count: int) -> list:
    """The first seeded boards of the c4 and c5 rules small enough for the
    scipy restatement (at most 400,000 nodes)."""

    boards = []
    for seed in range(400):
        for problem in (board_random(seed), request_c5(seed)):
            if problem.mesh.size <= 400_000 and len(boards) < count:
                boards.append(problem)
        if len(boards) >= count:
            break
    return boards


def test_engine_boards_of_the_c4_and_c5_rules_match_the_fp64_restatement() -> None:
    from pcb_analysis_b200._native import BatchEngine
    from pcb_analysis_b200.serve import board_request

    problems = _small_boards(3)
    requests = [board_request(p, tag=i) for i, p in enumerate(problems)]
    with BatchEngine(capacity=4, max_slabs=max(len(q.arrays["slab_thickness_m"]) for q in requests),
                     preconditioner="two-level") as engine:
        tickets = [engine.submit(q.arrays, q.rhs, CONFIG) for q in requests]
        assert all(t is not None for t in tickets)
        done: dict[int, dict] = {}
        for _ in range(1_000_000):
            if len(done) == len(tickets):
                break
            engine.step()
            for t in engine.finished():
                done[t] = engine.collect(t)
    for q, t in zip(requests, tickets):
        result = done[t]
        assert result["converged"] and result["relative_residual"] <= 1e-10
        a = q.arrays
        oracle = OracleSystem.from_arrays(free=a["free_nodes"], **{k: v for k, v in a.items() if k != "free_nodes"})
        theta, _, rel = MultilevelOracle(oracle.coef, oracle.robin_total, oracle.free).pcg(q.rhs, rtol=1e-11)
        assert rel <= 1e-10
        free = a["free_nodes"].astype(bool)
        peak = np.abs(theta[free]).max()
        assert np.abs(result["solution"][free] - theta[free]).max() <= 1e-6 * peak


def test_unconverged_first_run_re_references_and_resumes() -> None:
    problem = CASES["stack_12x20"](ns)
    # One outer step per refinement run cannot reach 1e-10, so the first run
    # ends unconverged and the solve moves its reference temperature.
    short = MPIRConfig(inner_relative_tolerance=1e-4, max_outer_iterations=1, max_inner_iterations=100000)
    restarted = ns.solve_thermal_conduction(problem, config=short, reference_temperature_k=250.0)
    record = restarted.solve
    assert [step.outer_iteration for step in record.history] == [1, 1]
    assert record.outer_iterations == 2
    assert record.inner_iterations == sum(step.inner_iterations for step in record.history)
    # the resumed run starts from the iterate (shifted), not from zero: its
    # first residual, relative to its own right-hand side, is below one
    assert record.history[1].high_relative_residual < 0.5
    full = ns.solve_thermal_conduction(problem, config=CONFIG, reference_temperature_k=250.0)
    assert full.solve.converged
    rise = full.temperature_k - 250.0
    err = np.nanmax(np.abs(restarted.temperature_k - full.temperature_k))
    assert err <= 1e-2 * np.nanmax(np.abs(rise))
