"""Layered DC problems shared by the golden-vector generator and the tests.

Each case builds a problem from the module ``ns`` it is given (the reference's
``electrical.matrix_free_mpir_fem`` or ``pcb_analysis_b200.electrical``), so the
same board is solved by both.  They cover current and voltage drives, vias
between adjacent and distant layers, graded pitches, per-element
conductivity and void copper.
"""

from __future__ import annotations

import numpy as np


def strip(ns, columns: int = 4):
    """A uniform 1 mm strip driven end to end (test_matrix_free_mpir_fem.py:19-35)."""

    mesh = ns.LayeredPCBMesh(element_active=np.ones((1, 1, columns), dtype=bool), layer_thickness_m=(35.0e-6,),
                             pitch_x_m=1.0e-3, pitch_y_m=1.0e-3)
    return ns.PCBConductionProblem(
        mesh=mesh,
        terminals=(ns.CurrentTerminal(((0, 0, 0), (0, 1, 0)), 1.0, "source"),
                   ns.CurrentTerminal(((0, 0, columns), (0, 1, columns)), -1.0, "sink")),
        reference_node=(0, 0, columns),
    )


def two_layer_via(ns):
    """Two 1x1 sheets joined by one via (test_matrix_free_mpir_fem.py:104-123)."""

    mesh = ns.LayeredPCBMesh(element_active=np.ones((2, 1, 1), dtype=bool), layer_thickness_m=(35.0e-6, 35.0e-6),
                             pitch_x_m=1.0e-3, pitch_y_m=1.0e-3)
    return ns.PCBConductionProblem(
        mesh=mesh,
        terminals=(ns.CurrentTerminal(((0, 0, 0),), 1.0, "source"), ns.CurrentTerminal(((1, 0, 0),), -1.0, "sink")),
        reference_node=(1, 0, 0),
        vias=(ns.ViaConnection((0, 0, 1), (1, 0, 1), 2.0e-3),),
    )


def lifted(ns):
    """Voltage and current drives with graded pitches and a via (test_matrix_free_mpir_fem.py:169-186)."""

    mesh = ns.LayeredPCBMesh(element_active=np.ones((2, 3, 4), dtype=bool), layer_thickness_m=(35.0e-6, 18.0e-6),
                             pitch_x_m=(0.4e-3, 0.5e-3, 0.6e-3, 0.4e-3), pitch_y_m=0.5e-3)
    return ns.PCBConductionProblem(
        mesh=mesh,
        terminals=(ns.CurrentTerminal(((0, 3, 2),), -0.25, "load"),),
        voltage_terminals=(ns.VoltageTerminal(((0, 0, 0), (0, 1, 0)), 1.2, "vrm"),
                           ns.VoltageTerminal(((1, 3, 4), (1, 2, 4)), 0.0, "return")),
        vias=(ns.ViaConnection((0, 1, 2), (1, 1, 2), 1.0e-3),),
    )


def power_net(ns, seed: int = 0, layers: int = 4, rows: int = 23, cols: int = 37):
    """A seeded four-layer power net: planes with voids, a trace layer, stitching
    vias between adjacent and distant layers, a regulator and two loads."""

    rng = np.random.default_rng(seed)
    active = np.ones((layers, rows, cols), dtype=bool)
    active[1] = rng.random((rows, cols)) > 0.12
    active[2] = False
    active[2, rows // 2 - 2 : rows // 2 + 2, :] = True  # a wide trace across the board
    active[2, :, 3:6] = True
    conductivity = ns.COPPER_CONDUCTIVITY_S_PER_M * rng.uniform(0.7, 1.0, (layers, rows, cols))
    mesh = ns.LayeredPCBMesh(element_active=active, layer_thickness_m=(35e-6, 17.5e-6, 35e-6, 70e-6),
                             pitch_x_m=np.linspace(0.2e-3, 0.35e-3, cols), pitch_y_m=np.linspace(0.3e-3, 0.25e-3, rows),
                             conductivity_s_per_m=conductivity)
    vias = []
    for k in range(14):
        y, x = int(rng.integers(1, rows)), int(rng.integers(1, cols))
        lower, upper = sorted(rng.choice(layers, size=2, replace=False).tolist())
        vias.append(ns.ViaConnection((lower, y, x), (upper, y, x), float(rng.uniform(0.5e-3, 3e-3))))
    vias.append(ns.ViaConnection((0, rows // 2, 4), (3, rows // 2, 4), 1e-3))  # layers 0 and 3 (same colour)
    vias.append(ns.ViaConnection((2, rows // 2, 20), (3, rows // 2 + 1, 21), 2e-3))
    regulator = tuple((0, y, 0) for y in range(rows // 2 - 2, rows // 2 + 3))
    ground = tuple((3, y, cols) for y in range(0, rows + 1, 2))
    load_a = tuple((0, y, x) for y in (rows // 2, rows // 2 + 1) for x in (cols - 3, cols - 2))
    load_b = tuple((2, rows // 2 - 1, x) for x in (10, 11, 12))
    return ns.PCBConductionProblem(
        mesh=mesh,
        terminals=(ns.CurrentTerminal(load_a, -0.8, "load_a"), ns.CurrentTerminal(load_b, -0.3, "load_b")),
        voltage_terminals=(ns.VoltageTerminal(regulator, 1.0, "vrm"), ns.VoltageTerminal(ground, 0.0, "gnd")),
        vias=tuple(vias),
    )


def current_net(ns, seed: int = 1):
    """The power net driven by currents only, with a reference node."""

    base = power_net(ns, seed=seed)
    rows = base.mesh.element_active.shape[1]
    return ns.PCBConductionProblem(
        mesh=base.mesh,
        terminals=(ns.CurrentTerminal(((0, rows // 2, 0), (0, rows // 2 + 1, 0)), 1.5, "in"),
                   ns.CurrentTerminal(((3, 0, 10), (3, 1, 10)), -1.5, "out")),
        reference_node=(3, 0, 10),
        vias=base.vias,
    )


DC_CASES = {
    "strip": strip,
    "two_layer_via": two_layer_via,
    "lifted": lifted,
    "power_net": power_net,
    "current_net": current_net,
}
