"""A conduction problem as the device takes it, and its host preparation.

:func:`problem_inputs` describes a ``ThermalConductionProblem`` to
``DeviceSystem.from_problem``: the mesh arrays, masks, loads, heat-source
entries and convection boundaries, from which the device prepares the system
(node masks, lumped Robin terms, loads, right-hand side, post-processing).

:func:`prepare` is the same preparation on the host with NumPy, in the
operation order of the reference's NumPy operator
(src/thermal/matrix_free_mpir_fem/operator.py:86-128, 374-387) and its C++
ThermalSystem (cpp/src/thermal/thermal_system.cpp:146-172, 218-245, 290-326),
so that every array carries the reference's bits.  It serves callers that
build prepared arrays without a device (the CPU reference arm of the
benchmark, the host-model tests).
"""

from __future__ import annotations

import os

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


def convection_specs(convection) -> list[dict]:
    """Convection boundaries as ``DeviceSystem`` takes them (scalars stay
    scalars; fields keep their shape)."""

    from .boundaries import ConvectionBoundary

    specs = []
    for boundary in convection:
        coefficient = np.asarray(boundary.coefficient_w_per_m2_k, dtype=np.float64)
        ambient = np.asarray(boundary.ambient_temperature_k, dtype=np.float64)
        spec = dict(coefficient=float(coefficient) if coefficient.ndim == 0 else coefficient,
                    ambient=float(ambient) if ambient.ndim == 0 else ambient)
        if isinstance(boundary, ConvectionBoundary):
            spec.update(kind="face", side=boundary.side)
        else:
            spec.update(kind="exposed", directions=tuple(boundary.directions))
        specs.append(spec)
    return specs


_SCAN_CHUNK = 1 << 23  # values per chunk of the parallel scan (64 MB)


def _any_bits(words: np.ndarray) -> bool:
    """Whether any 64-bit word is nonzero: chunks of a large array scanned by
    several host threads (NumPy's reductions run without the GIL), so that a
    c3-sized field (71 M values, 571 MB) takes milliseconds instead of the
    tenths of a second one thread needs."""

    n = words.size
    if n <= 2 * _SCAN_CHUNK:
        return bool(np.any(words))
    from concurrent.futures import ThreadPoolExecutor

    bounds = range(0, n, _SCAN_CHUNK)
    workers = max(1, min(8, os.cpu_count() or 1, len(bounds)))
    with ThreadPoolExecutor(max_workers=workers) as pool:
        return any(pool.map(lambda lo: bool(np.any(words[lo:lo + _SCAN_CHUNK])), bounds))


def _optional(values: np.ndarray) -> np.ndarray | None:
    """None for an array of +0.0 only, which the device takes as absent.  One
    pass over the raw bits: +0.0 is the only float64 whose bits are all zero
    (-0.0 has the sign bit set)."""

    flat = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
    if _any_bits(flat.view(np.uint64)):
        return values
    return None


def problem_inputs(problem: ThermalConductionProblem, capacity_per_s: np.ndarray | None = None) -> dict:
    """Keyword arguments of ``DeviceSystem.from_problem`` for ``problem``."""

    mesh = problem.mesh
    node_shape = mesh.node_shape
    sources = []
    for source in problem.heat_sources:
        nodes = np.asarray(source.nodes, dtype=np.int64).reshape(-1, 3)
        flat = np.ravel_multi_index((nodes[:, 0], nodes[:, 1], nodes[:, 2]), node_shape)
        sources.append((flat, float(source.power_w) / len(source.nodes)))
    mask = problem.fixed_temperature_mask
    fixed = bool(np.any(mask))
    return dict(
        slab_thickness_m=np.asarray(mesh.slab_thickness_m, dtype=np.float64),
        pitch_x_m=np.asarray(mesh.pitch_x_m, dtype=np.float64),
        pitch_y_m=np.asarray(mesh.pitch_y_m, dtype=np.float64),
        k_in=mesh.conductivity_w_per_m_k,
        k_z=mesh.through_plane_conductivity_w_per_m_k,
        active=None if mesh.is_full else mesh.active,
        fixed_mask=mask if fixed else None,
        fixed_temperature_k=problem.fixed_temperature_k if fixed else None,
        nodal_heat_w=_optional(problem.nodal_heat_w),
        element_heat_w=_optional(problem.element_heat_w),
        sources=sources,
        convection=convection_specs(problem.convection),
        capacity_per_s=capacity_per_s,
    )


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
