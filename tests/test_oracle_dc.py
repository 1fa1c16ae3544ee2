"""The layered DC oracle against the reference's golden vectors, and the DC
problem records' validation (CPU only).

Pins oracle/dc_oracle.py to arrays recorded from the reference's NumPy
operator (tests/golden/make_golden_dc.py): element coefficients, masks and
diagonal bit for bit; actions within a few FP64 ulps of the reference's (the
same formula, evaluated in the same order); the reference's solution solves
the oracle's system.  Mirrors the validation cases of
tests/test_matrix_free_mpir_fem.py:126-266 of pcb-analysis.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import pcb_analysis_b200.electrical as ed
from oracle.dc_oracle import from_problem
from tests.dc_cases import DC_CASES

GOLDEN = Path(__file__).resolve().parent / "golden" / "dc"


def _golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as data:
        return {k: data[k] for k in data.files}


@pytest.mark.parametrize("name", sorted(DC_CASES))
def test_oracle_matches_the_reference_arrays(name: str) -> None:
    g = _golden(name)
    problem = DC_CASES[name](ed)
    oracle = from_problem(problem)
    np.testing.assert_array_equal(np.stack(problem.mesh.element_coefficients()), g["coef"])
    np.testing.assert_array_equal(oracle.coef, g["coef"])
    np.testing.assert_array_equal(oracle.active_nodes.reshape(-1).astype(np.uint8), g["active_nodes"])
    np.testing.assert_array_equal(oracle.free.reshape(-1).astype(np.uint8), g["free"])
    np.testing.assert_array_equal(oracle.diagonal(), g["diagonal"])
    np.testing.assert_array_equal(oracle.apply_f64(g["v"]), g["apply_high"])
    np.testing.assert_array_equal(oracle.apply_full(g["v"]), g["apply_full"])


@pytest.mark.parametrize("name", sorted(DC_CASES))
def test_reference_solution_solves_the_oracle_system(name: str) -> None:
    g = _golden(name)
    oracle = from_problem(DC_CASES[name](ed))
    potential = np.where(np.isfinite(g["potential"]), g["potential"], 0.0)
    residual = g["rhs"] - oracle.apply_f64(potential)
    assert np.linalg.norm(residual) <= 1e-11 * np.linalg.norm(g["rhs"])


def test_invalid_records_are_rejected_with_the_reference_messages() -> None:
    strip = DC_CASES["strip"](ed)
    mesh = strip.mesh
    with pytest.raises(ValueError, match="sum to zero"):
        ed.PCBConductionProblem(mesh=mesh, terminals=(ed.CurrentTerminal(((0, 0, 0),), 1.0),),
                                reference_node=(0, 0, 0))
    source = ed.VoltageTerminal(((0, 0, 0),), 1.0, "source")
    with pytest.raises(ValueError, match="reference_node must be None"):
        ed.PCBConductionProblem(mesh=mesh, voltage_terminals=(source,), reference_node=(0, 0, 1))
    with pytest.raises(ValueError, match="belongs to terminals"):
        ed.PCBConductionProblem(mesh=mesh, terminals=(ed.CurrentTerminal(((0, 0, 0),), 1.0, "load"),),
                                voltage_terminals=(source,))
    with pytest.raises(ValueError, match="needs a reference_node"):
        ed.PCBConductionProblem(mesh=mesh, terminals=(ed.CurrentTerminal(((0, 0, 0),), 1.0),
                                                      ed.CurrentTerminal(((0, 0, 1),), -1.0)))
    with pytest.raises(ValueError, match="current or voltage terminals"):
        ed.PCBConductionProblem(mesh=mesh, reference_node=(0, 0, 0))
    with pytest.raises(ValueError, match="different layers"):
        ed.ViaConnection((0, 0, 0), (0, 1, 1), 1.0)
    with pytest.raises(ValueError, match="finite and positive"):
        ed.ViaConnection((0, 0, 0), (1, 0, 0), 0.0)
    with pytest.raises(ValueError, match="conductivity must be finite and positive"):
        ed.LayeredPCBMesh(np.ones((1, 1, 1), dtype=bool), (35e-6,), 1e-3, 1e-3, conductivity_s_per_m=-1.0)
    with pytest.raises(ValueError, match="one value per layer"):
        ed.LayeredPCBMesh(np.ones((2, 1, 1), dtype=bool), (35e-6,), 1e-3, 1e-3)
