"""The layered DC path on the device against the reference and its known answers.

* masks and the FP64 diagonal equal the reference's golden arrays bit for bit;
  the FP64 actions (constrained and unconstrained) agree with the reference's
  within FP64 rounding, the FP32 action with the oracle's exact action within
  16 FP32 ulps of its norm;
* solve_pcb_dc, with the two-level preconditioner (the reference default) and
  with Jacobi, reaches the reference's potential, current density, via
  currents, Joule losses and terminal currents;
* the closed-form cases of pcb-analysis tests/test_matrix_free_mpir_fem.py:84-219
  (strip resistance and current density, the only via current, the
  voltage-driven strip, the dense lifted system, warm starts) hold.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import pcb_analysis_b200.electrical as ed
from oracle.dc_oracle import from_problem
from tests.dc_cases import DC_CASES

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "dc"
EPS64 = np.finfo(np.float64).eps
EPS32 = np.finfo(np.float32).eps
CONFIG = ed.MPIRConfig(relative_tolerance=1e-12, max_outer_iterations=40)


def _golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as data:
        return {k: data[k] for k in data.files}


def _operator(problem, preconditioner="jacobi"):
    return ed.MatrixFreePCBOperator(
        problem.mesh,
        reference_node=problem.reference_node,
        dirichlet_nodes=tuple(node for t in problem.voltage_terminals for node in t.nodes),
        vias=problem.vias,
        preconditioner=preconditioner,
    )


@pytest.mark.parametrize("name", sorted(DC_CASES))
def test_device_operator_matches_the_reference(name: str) -> None:
    g = _golden(name)
    problem = DC_CASES[name](ed)
    op = _operator(problem)
    try:
        np.testing.assert_array_equal(op.active_nodes.reshape(-1).astype(np.uint8), g["active_nodes"])
        np.testing.assert_array_equal(op.free_nodes.reshape(-1).astype(np.uint8), g["free"])
        np.testing.assert_array_equal(op.diagonal_high(), g["diagonal"])
        for got, want in ((op.apply_high(g["v"]), g["apply_high"]), (op.apply_full_high(g["v"]), g["apply_full"])):
            assert np.linalg.norm(got - want) <= 64 * EPS64 * np.linalg.norm(want)
        v32 = g["v"].astype(np.float32)
        exact = from_problem(problem).apply_f64(v32.astype(np.float64))
        assert np.linalg.norm(op.apply_low(v32) - exact) <= 16 * EPS32 * np.linalg.norm(exact)
        rhs = op.build_rhs(problem.terminals, problem.voltage_terminals)
        assert np.linalg.norm(rhs - g["rhs"]) <= 64 * EPS64 * np.linalg.norm(g["rhs"])
    finally:
        op.close()


@pytest.mark.parametrize("preconditioner", ["two-level", "jacobi"])
@pytest.mark.parametrize("name", sorted(DC_CASES))
def test_solve_reaches_the_reference_solution(name: str, preconditioner: str) -> None:
    g = _golden(name)
    problem = DC_CASES[name](ed)
    solution = ed.solve_pcb_dc(problem, config=CONFIG, preconditioner=preconditioner)
    assert solution.solve.converged and solution.solve.relative_residual <= 1e-12
    assert solution.solve.low_runtime == "b200-fp32"
    got, want = solution.potential_v.reshape(-1), g["potential"]
    np.testing.assert_array_equal(np.isfinite(got), np.isfinite(want))
    finite = np.isfinite(want)
    scale = np.abs(want[finite]).max()
    np.testing.assert_allclose(got[finite], want[finite], rtol=1e-8, atol=1e-9 * scale)
    jscale = np.abs(g["current_density"]).max()
    np.testing.assert_allclose(solution.current_density_a_per_m2, g["current_density"], rtol=0, atol=1e-7 * jscale)
    np.testing.assert_allclose(solution.via_current_a, g["via_current"], rtol=1e-7, atol=1e-9)
    assert solution.joule_loss_w == pytest.approx(g["joule"][0], rel=1e-7)
    assert solution.max_current_density_a_per_m2 == pytest.approx(g["joule"][1], rel=1e-7)
    np.testing.assert_allclose(solution.element_joule_loss_w, g["element_joule"], rtol=0,
                               atol=1e-7 * max(np.abs(g["element_joule"]).max(), 1e-300))
    np.testing.assert_allclose(solution.voltage_terminal_current_a, g["terminal_current"], rtol=1e-7, atol=1e-9)


def test_uniform_strip_matches_closed_form_resistance_and_current_density() -> None:
    problem = DC_CASES["strip"](ed, columns=4)
    solution = ed.solve_pcb_dc(problem)
    conductivity = float(problem.mesh.conductivity_s_per_m[0, 0, 0])
    width, thickness = 1.0e-3, problem.mesh.layer_thickness_m[0]
    expected = 4.0e-3 / (conductivity * width * thickness)
    assert solution.solve.converged
    assert solution.joule_loss_w == pytest.approx(expected, rel=2.0e-10)
    assert solution.max_current_density_a_per_m2 == pytest.approx(1.0 / (width * thickness), rel=2.0e-10)
    np.testing.assert_allclose(solution.current_density_a_per_m2[..., 1], 0.0, atol=1.0e-9 / (width * thickness))


def test_layered_problem_reports_the_only_via_current() -> None:
    solution = ed.solve_pcb_dc(DC_CASES["two_layer_via"](ed))
    assert solution.solve.converged
    assert abs(solution.via_current_a[0]) == pytest.approx(1.0, rel=2.0e-9)


def test_voltage_driven_strip_and_the_dense_lifted_system() -> None:
    voltage = 1.0e-3
    mesh = DC_CASES["strip"](ed).mesh
    problem = ed.PCBConductionProblem(mesh=mesh, voltage_terminals=(
        ed.VoltageTerminal(((0, 0, 0), (0, 1, 0)), voltage, "source"),
        ed.VoltageTerminal(((0, 0, 4), (0, 1, 4)), 0.0, "sink")))
    solution = ed.solve_pcb_dc(problem)
    conductivity = float(mesh.conductivity_s_per_m[0, 0, 0])
    current = voltage / (4.0e-3 / (conductivity * 1.0e-3 * mesh.layer_thickness_m[0]))
    assert solution.solve.converged
    np.testing.assert_allclose(solution.voltage_terminal_current_a, (current, -current), rtol=2.0e-10)
    assert solution.joule_loss_w == pytest.approx(voltage * current, rel=2.0e-10)
    np.testing.assert_allclose(solution.potential_v[0, 0], voltage * np.linspace(1.0, 0.0, 5), atol=1.0e-12)

    lifted = DC_CASES["lifted"](ed)
    solution = ed.solve_pcb_dc(lifted, config=ed.MPIRConfig(relative_tolerance=1.0e-12))
    oracle = from_problem(lifted)
    full = np.column_stack([oracle.apply_full(column) for column in np.eye(oracle.size).T])
    known = ~oracle.free.reshape(-1)
    free = ~known
    fixed = np.zeros(oracle.size)
    for t in lifted.voltage_terminals:
        for node in t.nodes:
            fixed[np.ravel_multi_index(node, lifted.mesh.node_shape)] = t.voltage_v
    injection = np.zeros(oracle.size)
    injection[np.ravel_multi_index((0, 3, 2), lifted.mesh.node_shape)] = -0.25
    expected = fixed.copy()
    expected[free] = np.linalg.solve(full[np.ix_(free, free)], injection[free] - full[np.ix_(free, known)] @ fixed[known])
    assert solution.solve.converged
    np.testing.assert_allclose(solution.potential_v.reshape(-1), expected, rtol=1.0e-10, atol=1.0e-13)
    assert float(np.sum(solution.voltage_terminal_current_a)) == pytest.approx(0.25, rel=1.0e-9)
    supplied = float(np.dot(solution.voltage_terminal_current_a, (1.2, 0.0)))
    assert solution.joule_loss_w == pytest.approx(supplied - 0.25 * float(solution.potential_v[0, 3, 2]), rel=1.0e-9)


def test_warm_start_and_bitwise_repeatable_solves() -> None:
    problem = DC_CASES["power_net"](ed)
    cold = ed.solve_pcb_dc(problem)
    again = ed.solve_pcb_dc(problem)
    warm = ed.solve_pcb_dc(problem, initial_potential_v=cold.potential_v)
    assert cold.solve.converged and warm.solve.converged
    assert warm.solve.inner_iterations < cold.solve.inner_iterations
    np.testing.assert_array_equal(again.potential_v, cold.potential_v)
    np.testing.assert_allclose(warm.potential_v, cold.potential_v, rtol=1.0e-9, atol=1.0e-15)


def test_operator_refuses_nodes_off_the_copper() -> None:
    mesh = ed.LayeredPCBMesh(np.array([[[True, False]]]), (35e-6,), 1e-3, 1e-3)
    with pytest.raises(ValueError, match="reference_node must lie on active copper"):
        ed.MatrixFreePCBOperator(mesh, reference_node=(0, 0, 2))
    with pytest.raises(ValueError, match="dirichlet_nodes must lie on active copper"):
        ed.MatrixFreePCBOperator(mesh, dirichlet_nodes=[(0, 1, 2)])
    with pytest.raises(ValueError, match="reference_node or dirichlet_nodes"):
        ed.MatrixFreePCBOperator(mesh)


@pytest.mark.parametrize("name", sorted(DC_CASES))
def test_device_post_processing_matches_the_host_formulas(name: str) -> None:
    """tb_dc_post against the reference's NumPy formulas (pcb.py:810-848) on a
    seeded potential: the field bit for bit, the element loss to FP64 rounding."""
    problem = DC_CASES[name](ed)
    op = _operator(problem)
    try:
        v = _golden(name)["v"]
        field, loss = op.element_post(v)
        grid = v.reshape(problem.mesh.node_shape)
        v00, v01, v10, v11 = grid[:, :-1, :-1], grid[:, :-1, 1:], grid[:, 1:, :-1], grid[:, 1:, 1:]
        hx = np.asarray(problem.mesh.pitch_x_m, dtype=np.float64) * np.ones(problem.mesh.element_active.shape[2])
        hy = np.asarray(problem.mesh.pitch_y_m, dtype=np.float64) * np.ones(problem.mesh.element_active.shape[1])
        fx = -((v01 + v11) - (v00 + v10)) / (2.0 * hx[None, None, :])
        fy = -((v10 + v11) - (v00 + v01)) / (2.0 * hy[None, :, None])
        want = np.where(problem.mesh.element_active[..., None], np.stack((fx, fy), axis=-1), 0.0)
        np.testing.assert_array_equal(field, want)
        values = np.stack((v00, v01, v10, v11), axis=-1)
        ux, uy = ed.unit_sheet_matrices()
        cx, cy = problem.mesh.element_coefficients()
        quad = lambda u: np.einsum("...i,ij,...j->...", values, u, values)  # noqa: E731
        want_loss = cx * quad(ux) + cy * quad(uy)
        scale = max(float(np.abs(want_loss).max()), 1e-300)
        np.testing.assert_allclose(loss, want_loss, rtol=0, atol=64 * EPS64 * scale)
        assert op.joule_loss(v) == pytest.approx(float(np.sum(want_loss) + np.sum(op.via_joule_loss(v))), rel=1e-12)
    finally:
        op.close()
