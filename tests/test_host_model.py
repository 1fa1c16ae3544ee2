"""The host problem model against the reference's prepared arrays, bit for bit.

Mirrors tests/test_native_thermal_system.py:85-121 of pcb-analysis (prepared
system bit-identical to NumPy) and the validation cases of
tests/test_thermal_conduction.py:212-237.
"""

from __future__ import annotations

import numpy as np
import pytest

import pcb_analysis_b200.thermal as ns
from pcb_analysis_b200.mpir import MPIRConfig
from pcb_analysis_b200.thermal.mesh import unit_hexahedron_matrices
from pcb_analysis_b200.thermal.system import prepare
from tests.conftest import golden_cases, load_golden
from tests.problems import CASES


@pytest.mark.parametrize("name", golden_cases())
def test_prepared_arrays_are_bit_identical_to_the_reference(name: str) -> None:
    g = load_golden(name)
    problem = CASES[name](ns)
    p = prepare(problem)
    np.testing.assert_array_equal(np.stack(problem.mesh.element_coefficients()), g["coef"])
    np.testing.assert_array_equal(np.stack(unit_hexahedron_matrices()), g["unit"])
    np.testing.assert_array_equal(p.robin_total, g["robin_total"])
    np.testing.assert_array_equal(p.robin_rhs, g["robin_rhs"])
    np.testing.assert_array_equal(p.load, g["load"])
    np.testing.assert_array_equal(p.free_nodes.reshape(-1).astype(np.uint8), g["free"])
    np.testing.assert_array_equal(p.active_nodes.reshape(-1).astype(np.uint8), g["active_nodes"])
    if g["robin_weights"].shape[0]:
        np.testing.assert_array_equal(np.stack(p.robin_weights), g["robin_weights"])
        np.testing.assert_array_equal(np.stack(p.robin_rhs_weights), g["robin_rhs_weights"])


def _uniform(slabs, thickness, shape, k):
    return ns.LayeredThermalMesh((thickness,) * slabs, 1.0e-3, 1.0e-3, k, element_shape=shape)


def test_floating_problem_and_bad_inputs_are_rejected() -> None:
    mesh = _uniform(1, 1.0e-3, (1, 1), 1.0)
    with pytest.raises(ValueError, match="positive film coefficient, a radiating face or a fixed node"):
        ns.ThermalConductionProblem(mesh)
    with pytest.raises(ValueError, match="positive film coefficient, a radiating face or a fixed node"):
        ns.ThermalConductionProblem(mesh, convection=(ns.ConvectionBoundary("top", 0.0, 300.0),))
    with pytest.raises(ValueError, match="element_shape is required"):
        ns.LayeredThermalMesh((1.0e-3,), 1.0e-3, 1.0e-3, 1.0)
    with pytest.raises(ValueError, match="finite and positive"):
        ns.LayeredThermalMesh((1.0e-3,), 1.0e-3, 1.0e-3, 0.0, element_shape=(1, 1))
    with pytest.raises(ValueError, match="side"):
        ns.ConvectionBoundary("left", 1.0, 300.0)  # type: ignore[arg-type]
    with pytest.raises(ValueError, match="outside mesh shape"):
        ns.ThermalConductionProblem(
            mesh,
            convection=(ns.ConvectionBoundary("top", 1.0, 300.0),),
            heat_sources=(ns.HeatSource(((5, 0, 0),), 1.0),),
        )
    with pytest.raises(ValueError, match="element_heat_w"):
        ns.ThermalConductionProblem(
            mesh, convection=(ns.ConvectionBoundary("top", 1.0, 300.0),), element_heat_w=np.zeros((2, 1, 1))
        )
    with pytest.raises(ValueError, match="unique"):
        ns.HeatSource(((0, 0, 0), (0, 0, 0)), 1.0)
    with pytest.raises(ValueError, match="emissivity"):
        ns.RadiationBoundary("top", 1.5, 300.0)
    with pytest.raises(ValueError, match="directions"):
        ns.ExposedFaceConvection(1.0, 300.0, directions=("+w",))  # type: ignore[arg-type]


def test_mesh_broadcasts_per_slab_conductivity_and_reports_volumes() -> None:
    mesh = ns.LayeredThermalMesh(
        slab_thickness_m=(35.0e-6, 1.5e-3),
        pitch_x_m=0.2e-3,
        pitch_y_m=0.1e-3,
        conductivity_w_per_m_k=(385.0, 0.8),
        element_shape=(2, 3),
        through_plane_conductivity_w_per_m_k=(385.0, 0.3),
    )
    assert mesh.element_grid_shape == (2, 2, 3)
    assert mesh.node_shape == (3, 3, 4)
    np.testing.assert_allclose(mesh.conductivity_w_per_m_k[1], 0.8)
    np.testing.assert_allclose(mesh.through_plane_conductivity_w_per_m_k[1], 0.3)
    np.testing.assert_allclose(mesh.element_volume_m3[0], 35.0e-6 * 0.2e-3 * 0.1e-3)


def test_lumped_robin_weights_are_the_exact_face_shares() -> None:
    """hA/4, hA/2, hA at corner, edge and interior top nodes (test_thermal_conduction.py:70-76)."""

    mesh = ns.LayeredThermalMesh(
        slab_thickness_m=(35.0e-6, 0.4e-3), pitch_x_m=0.2e-3, pitch_y_m=0.3e-3,
        conductivity_w_per_m_k=1.0, element_shape=(2, 2),
    )
    p = prepare(ns.ThermalConductionProblem(mesh, convection=(ns.ConvectionBoundary("top", 12.0, 300.0),)))
    top = p.robin_total.reshape(mesh.node_shape)[-1]
    area = 0.2e-3 * 0.3e-3
    assert top[1, 1] == pytest.approx(12.0 * area)
    assert top[0, 0] == pytest.approx(12.0 * area / 4.0)
    assert top[0, 1] == pytest.approx(12.0 * area / 2.0)
    assert float(np.sum(top)) == pytest.approx(12.0 * area * 4)
    assert not np.any(p.robin_total.reshape(mesh.node_shape)[:-1])


def test_exposed_faces_of_a_full_block_are_its_outer_surfaces() -> None:
    faces = ns.exposed_element_faces(np.ones((2, 3, 4), dtype=bool))
    assert faces["+z"][1].all() and not faces["+z"][0].any()
    assert faces["-x"][:, :, 0].all() and not faces["-x"][:, :, 1:].any()
    pocket = np.ones((3, 3, 3), dtype=bool)
    pocket[1, 1, 1] = False
    inner = ns.exposed_element_faces(pocket)
    assert inner["+x"][1, 1, 0] and inner["-x"][1, 1, 2] and inner["+z"][0, 1, 1]


def test_mpir_config_validation() -> None:
    with pytest.raises(ValueError, match="at least one outer tolerance"):
        MPIRConfig(relative_tolerance=0.0)
    with pytest.raises(ValueError, match="between zero and one"):
        MPIRConfig(inner_relative_tolerance=1.0)
    with pytest.raises(ValueError, match="iteration limits"):
        MPIRConfig(max_inner_iterations=0)


def test_radiation_linearisation_is_newtons_step() -> None:
    from pcb_analysis_b200.thermal.radiation import STEFAN_BOLTZMANN_W_PER_M2_K4 as SIGMA

    h, t_eff = ns.newton_linearisation(0.8, np.array([350.0]), 300.0)
    assert h[0] == pytest.approx(4 * 0.8 * SIGMA * 350.0**3)
    # q = h (T - T_eff) equals the radiated flux at the linearisation point
    assert h[0] * (350.0 - t_eff[0]) == pytest.approx(0.8 * SIGMA * (350.0**4 - 300.0**4))


def test_optional_input_scan_finds_any_nonzero_bit_across_chunks() -> None:
    """The threaded scan for absent optional inputs: +0.0 everywhere is absent;
    one nonzero word anywhere (first, last, chunk edges), including -0.0 and
    the smallest subnormal, makes the input present."""

    from pcb_analysis_b200.thermal import system

    n = 3 * system._SCAN_CHUNK + 5
    values = np.zeros(n)
    assert system._optional(values) is None
    for at in (0, system._SCAN_CHUNK - 1, system._SCAN_CHUNK, 2 * system._SCAN_CHUNK + 1, n - 1):
        for bits in (-0.0, 5e-324, 1.0):
            values[at] = bits
            assert system._optional(values) is values, (at, bits)
            values[at] = 0.0
    assert system._optional(np.zeros(7)) is None
    assert system._optional(np.array([0.0, -0.0])) is not None
