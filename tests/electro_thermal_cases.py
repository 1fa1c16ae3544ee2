"""Electro-thermal boards shared by the golden-vector generator and the tests.

The builders take namespaces, so the same board is made from the reference's
modules (``electrical.matrix_free_mpir_fem``, ``thermal.matrix_free_mpir_fem``,
``multiphysics.staggered_coupling``) and from this package's
(``pcb_analysis_b200.electrical``, ``pcb_analysis_b200.thermal``,
``pcb_analysis_b200.electro_thermal``).  The board is the two-layer current
loop of pcb-analysis tests/test_staggered_coupling.py:50-108: a 2 mm wide,
12 mm long copper track on each side of a 1.5 mm core, joined at the far end
by six 1.5 mOhm vias, over a three-slab stack (Cu, FR4, Cu).
"""

from __future__ import annotations

import numpy as np

AMBIENT = 298.15
PITCH = 0.5e-3
ROWS, COLS = 6, 24


def loop_mesh(ed):
    active = np.zeros((2, ROWS, COLS), dtype=bool)
    active[:, 1:5, :] = True
    return ed.LayeredPCBMesh(active, (35e-6, 35e-6), PITCH, PITCH)


def loop_vias(ed):
    return tuple(ed.ViaConnection((0, r, c), (1, r, c), 1.5e-3) for r in (2, 3, 4) for c in (COLS - 1, COLS))


def current_loop(ed, current_a: float = 2.0):
    """Current-driven loop: the deprecated drive, kept for its runaway checks."""
    rows = tuple(range(1, 6))
    return ed.PCBConductionProblem(
        loop_mesh(ed),
        (ed.CurrentTerminal(tuple((1, r, 0) for r in rows), current_a, "source"),
         ed.CurrentTerminal(tuple((0, r, 0) for r in rows), -current_a, "return")),
        reference_node=(0, 1, 0),
        vias=loop_vias(ed),
    )


def voltage_loop(ed, voltage_v: float):
    rows = tuple(range(1, 6))
    return ed.PCBConductionProblem(
        loop_mesh(ed),
        voltage_terminals=(ed.VoltageTerminal(tuple((1, r, 0) for r in rows), voltage_v, "source"),
                           ed.VoltageTerminal(tuple((0, r, 0) for r in rows), 0.0, "return")),
        vias=loop_vias(ed),
    )


def loop_thermal_mesh(td, problem):
    active = problem.mesh.element_active
    _, rows, cols = active.shape
    k = np.full((3, rows, cols), 0.8)
    k[0] = np.where(active[0], 385.0, 0.8)
    k[2] = np.where(active[1], 385.0, 0.8)
    kz = k.copy()
    kz[1] = 0.3
    return td.LayeredThermalMesh((35e-6, 1.5e-3, 35e-6), PITCH, PITCH, k, through_plane_conductivity_w_per_m_k=kz)


def scenario(ed, td, et, problem, **overrides):
    options = dict(
        convection=(td.ConvectionBoundary("top", 10.0, AMBIENT), td.ConvectionBoundary("bottom", 10.0, AMBIENT)),
        conductivity_reference_temperature_k=293.15,
    )
    options.update(overrides)
    return et.ElectroThermalScenario(problem, loop_thermal_mesh(td, problem), (0, 2), **options)


# The source voltage of the golden coupled solve: about 3 A through the cold loop.
GOLDEN_VOLTAGE_V = 18.5e-3
