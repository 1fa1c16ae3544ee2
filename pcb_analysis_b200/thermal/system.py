"""Host preparation of a conduction problem into the arrays the device system takes.

This is the problem model, not the solve: masks, lumped Robin conductances and
loads, computed with the same operation order as the reference's NumPy
operator (src/thermal/matrix_free_mpir_fem/operator.py:86-128, 374-387) and
its C++ ThermalSystem (cpp/src/thermal/thermal_system.cpp:146-172, 218-245,
290-326), so that every array carries the reference's bits.  The diagonal and
every operator action are computed on the device.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .mesh import corner_views, flat_index
from .problem import ThermalConductionProblem


@dataclass
class PreparedSystem:
    node_shape: tuple[int, int, int]
    element_shape: tuple[int, int, int]
    active_nodes: np.ndarray          # node grid, bool
    fixed_nodes: np.ndarray           # fixed mask | not active
    free_nodes: np.ndarray            # ~fixed_nodes
    fixed_temperature_k: np.ndarray   # node grid, fixed value on active fixed nodes, else 0
    robin_weights: list[np.ndarray] = field(default_factory=list)      # per boundary, flat
    robin_rhs_weights: list[np.ndarray] = field(default_factory=list)  # per boundary, flat
    robin_ambient_k: list[float] = field(default_factory=list)
    robin_only: np.ndarray | None = None     # sum of the boundary conductances, flat
    capacity: np.ndarray | None = None       # C / dt, flat
    robin_total: np.ndarray | None = None    # robin_only + capacity, flat
    robin_rhs: np.ndarray | None = None      # sum of R T_amb, flat
    load: np.ndarray | None = None           # nodal heat input in W, flat

    @property
    def size(self) -> int:
        return int(np.prod(self.node_shape))


def nodal_load(problem: ThermalConductionProblem) -> np.ndarray:
    """Heat per node: nodal heat, plus element heat / 8 on each corner, plus each
    source's power split equally over its nodes (reference operator.py:374-387)."""

    mesh = problem.mesh
    load = problem.nodal_heat_w.copy()
    share = problem.element_heat_w / 8.0
    for target in corner_views(load):
        target[...] += share
    for source in problem.heat_sources:
        per_node = float(source.power_w) / len(source.nodes)
        for node in source.nodes:
            load.flat[flat_index(node, mesh.node_shape)] += per_node
    return load.reshape(-1)


def prepare(problem: ThermalConductionProblem, capacity_per_s: np.ndarray | None = None) -> PreparedSystem:
    mesh = problem.mesh
    size = mesh.size
    active = mesh.active_nodes
    fixed = problem.fixed_temperature_mask | ~active
    prepared = PreparedSystem(
        node_shape=mesh.node_shape,
        element_shape=mesh.element_grid_shape,
        active_nodes=active,
        fixed_nodes=fixed,
        free_nodes=~fixed,
        fixed_temperature_k=np.where(problem.fixed_temperature_mask & active, problem.fixed_temperature_k, 0.0),
    )
    for boundary in problem.convection:
        weights, rhs_weights = boundary.lumped_nodal_weights(mesh)
        prepared.robin_weights.append(weights)
        prepared.robin_rhs_weights.append(rhs_weights)
        prepared.robin_ambient_k.append(boundary.mean_ambient_k())
    prepared.robin_only = (
        np.sum(prepared.robin_weights, axis=0) if prepared.robin_weights else np.zeros(size, dtype=np.float64)
    )
    if capacity_per_s is None:
        prepared.capacity = np.zeros(size, dtype=np.float64)
    else:
        capacity = np.asarray(capacity_per_s, dtype=np.float64).reshape(-1)
        if capacity.size != size:
            raise ValueError("capacity_per_s must hold one value per node")
        if not np.all(np.isfinite(capacity)) or np.any(capacity < 0.0):
            raise ValueError("capacity_per_s must be finite and non-negative")
        prepared.capacity = capacity.copy()
    prepared.robin_total = prepared.robin_only + prepared.capacity
    prepared.robin_rhs = (
        np.sum(prepared.robin_rhs_weights, axis=0) if prepared.robin_rhs_weights else np.zeros(size, dtype=np.float64)
    )
    prepared.load = nodal_load(problem)
    return prepared
