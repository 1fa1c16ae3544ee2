"""Conduction problems shared by the golden-fixture script and the tests.

Each builder takes ``ns``, a namespace holding LayeredThermalMesh,
ConvectionBoundary, ExposedFaceConvection, HeatSource and
ThermalConductionProblem, so the same problem is built once with the
reference package (to record golden vectors) and once with this package (to
check against them).  The stacks follow the shapes the reference's own tests
use (tests/test_native_thermal.py:26-52, tests/test_cuda_thermal_conduction.py:25-50,
tests/test_thermal_conduction.py:240-256), plus a void pocket, graded pitches
and every boundary kind.
"""

from __future__ import annotations

import numpy as np


def stack(ns, rows: int, cols: int, fixed: bool = False):
    """Cu / FR-4 / Cu stack with a heated trace and one nodal source."""

    mesh = ns.LayeredThermalMesh(
        slab_thickness_m=(35.0e-6, 1.5e-3, 35.0e-6),
        pitch_x_m=0.2e-3,
        pitch_y_m=0.2e-3,
        conductivity_w_per_m_k=(385.0, 0.8, 385.0),
        through_plane_conductivity_w_per_m_k=(385.0, 0.3, 385.0),
        element_shape=(rows, cols),
    )
    heat = np.zeros(mesh.element_grid_shape)
    heat[2, rows // 2, cols // 4 : 3 * cols // 4] = 0.5 / max(1, cols // 2)
    fixed_mask = np.zeros(mesh.node_shape, dtype=bool)
    fixed_k = np.full(mesh.node_shape, 298.15)
    if fixed:
        fixed_mask[0, ::3, 1::2] = True
        fixed_k[0] = 310.0
    return ns.ThermalConductionProblem(
        mesh,
        convection=(
            ns.ConvectionBoundary("top", 10.0, 298.15),
            ns.ConvectionBoundary("bottom", 10.0, 298.15),
        ),
        element_heat_w=heat,
        fixed_temperature_mask=fixed_mask if fixed else None,
        fixed_temperature_k=fixed_k if fixed else None,
        heat_sources=(ns.HeatSource(((1, rows // 3, cols // 3),), 0.05),),
    )


def mixed_board(ns):
    """12 x 12 x 3 board with per-element conductivity, a fixed edge and both load kinds."""

    rows = cols = 12
    conductivity = np.full((3, rows, cols), 0.8)
    conductivity[0] = conductivity[2] = 385.0
    conductivity[1, 4:8, 4:8] = 385.0
    through = conductivity.copy()
    through[1, :4] = 0.3
    mesh = ns.LayeredThermalMesh(
        slab_thickness_m=(35.0e-6, 0.4e-3, 35.0e-6),
        pitch_x_m=0.25e-3,
        pitch_y_m=0.25e-3,
        conductivity_w_per_m_k=conductivity,
        through_plane_conductivity_w_per_m_k=through,
    )
    heat = np.zeros(mesh.element_grid_shape)
    heat[2, 5:7, 2:10] = 0.02
    mask = np.zeros(mesh.node_shape, dtype=bool)
    mask[0, :, 0] = True
    return ns.ThermalConductionProblem(
        mesh,
        convection=(ns.ConvectionBoundary("top", 10.0, 300.0),),
        fixed_temperature_mask=mask,
        fixed_temperature_k=300.0,
        heat_sources=(ns.HeatSource(((3, 6, 6),), 0.05),),
        element_heat_w=heat,
    )


def voxel_body(ns):
    """Graded pitches, a void pocket, exposed-face cooling and a top face with per-face h."""

    slabs, rows, cols = 4, 7, 9
    active = np.ones((slabs, rows, cols), dtype=bool)
    active[2:, 2:5, 3:6] = False  # pocket open to the top
    k = np.full((slabs, rows, cols), 2.0)
    k[0] = 200.0
    mesh = ns.LayeredThermalMesh(
        slab_thickness_m=(0.5e-3, 0.4e-3, 0.4e-3, 0.3e-3),
        pitch_x_m=np.linspace(0.2e-3, 0.5e-3, cols),
        pitch_y_m=np.linspace(0.3e-3, 0.25e-3, rows),
        conductivity_w_per_m_k=k,
        through_plane_conductivity_w_per_m_k=0.5 * k,
        active=active,
    )
    h_top = np.linspace(5.0, 25.0, rows * cols).reshape(rows, cols)
    heat = np.zeros(mesh.element_grid_shape)
    heat[0, 3, 4] = 0.2
    heat[1, 1, 1] = 0.05
    return ns.ThermalConductionProblem(
        mesh,
        convection=(
            ns.ConvectionBoundary("top", h_top, 295.0),
            ns.ExposedFaceConvection(8.0, 300.0, directions=("-x", "+x", "-y", "+y")),
        ),
        element_heat_w=heat,
    )


def fixed_faces(ns):
    """Two fixed faces, no convection: the linear-profile case (test_thermal_conduction.py:110)."""

    mesh = ns.LayeredThermalMesh(
        slab_thickness_m=(0.5e-3,) * 4,
        pitch_x_m=1.0e-3,
        pitch_y_m=1.0e-3,
        conductivity_w_per_m_k=1.0,
        element_shape=(2, 3),
    )
    mask = np.zeros(mesh.node_shape, dtype=bool)
    mask[0] = mask[-1] = True
    values = np.zeros(mesh.node_shape)
    values[0] = 300.0
    values[-1] = 350.0
    return ns.ThermalConductionProblem(mesh, fixed_temperature_mask=mask, fixed_temperature_k=values)


def parabola(ns):
    """Uniform heating, one cooled face (test_thermal_conduction.py:141)."""

    mesh = ns.LayeredThermalMesh(
        slab_thickness_m=(0.25e-3,) * 8,
        pitch_x_m=1.0e-3,
        pitch_y_m=1.0e-3,
        conductivity_w_per_m_k=0.3,
        element_shape=(4, 5),
    )
    count = int(np.prod(mesh.element_grid_shape))
    return ns.ThermalConductionProblem(
        mesh,
        convection=(ns.ConvectionBoundary("top", 100.0, 300.0),),
        element_heat_w=np.full(mesh.element_grid_shape, 1.0 / count),
    )


def seeded_board(ns, rows: int, cols: int, seed: int = 0):
    """A small copper/FR-4 board in the shape of the benchmark boards: 4 slabs,
    random copper fill on the outer layers, a few pads, h = 10 both faces."""

    rng = np.random.default_rng(seed)
    slabs = 4
    k_in = np.full((slabs, rows, cols), 0.3)
    for layer in (0, slabs - 1):
        fill = rng.random((rows, cols)) < 0.6
        k_in[layer] = np.where(fill, 385.0, 0.3)
    mesh = ns.LayeredThermalMesh(
        slab_thickness_m=(35e-6, 0.8e-3, 0.8e-3, 35e-6),
        pitch_x_m=0.25e-3,
        pitch_y_m=0.25e-3,
        conductivity_w_per_m_k=k_in,
    )
    sources = []
    for i in range(3):
        r = int(rng.integers(1, rows))
        c = int(rng.integers(1, cols))
        sources.append(ns.HeatSource(((slabs, r, c),), float(rng.uniform(0.1, 1.0)), f"pad{i}"))
    return ns.ThermalConductionProblem(
        mesh,
        convection=(ns.ConvectionBoundary("top", 10.0, 298.15), ns.ConvectionBoundary("bottom", 10.0, 298.15)),
        heat_sources=tuple(sources),
    )


# name -> builder(ns); the golden fixtures are keyed by these names.
CASES = {
    "stack_1x1": lambda ns: stack(ns, 1, 1),
    "stack_1x4": lambda ns: stack(ns, 1, 4),
    "stack_3x2_fixed": lambda ns: stack(ns, 3, 2, fixed=True),
    "stack_12x20": lambda ns: stack(ns, 12, 20),
    "stack_12x20_fixed": lambda ns: stack(ns, 12, 20, fixed=True),
    "mixed_board": mixed_board,
    "voxel_body": voxel_body,
    "fixed_faces": fixed_faces,
    "parabola": parabola,
    "seeded_board_24x30": lambda ns: seeded_board(ns, 24, 30, seed=3),
}
