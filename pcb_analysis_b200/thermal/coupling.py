"""Joule loss of a DC solve placed as thermal load (reference
thermal/matrix_free_mpir_fem/coupling.py:24-142).

The electrical mesh holds copper layers only; the thermal mesh holds every
slab of the stack.  ``layer_slabs[L]`` is the thermal slab that holds
electrical layer ``L``.  The two meshes share the in-plane element grid, so a
loss moves from one grid to the other without interpolation.
"""

from __future__ import annotations

from typing import Sequence

import numpy as np

from .boundaries import HeatSource
from .mesh import LayeredThermalMesh


def _layer_slabs(layer_slabs: Sequence[int], layers: int, slabs: int) -> tuple[int, ...]:
    """Validated layer → slab map (reference coupling.py:24-35)."""
    mapping = tuple(int(s) for s in layer_slabs)
    if len(mapping) != layers:
        raise ValueError(f"layer_slabs has {len(mapping)} entries for {layers} electrical layers")
    if any(not 0 <= s < slabs for s in mapping):
        raise ValueError(f"layer_slabs must lie in [0, {slabs - 1}]")
    return mapping


def element_heat_from_losses(
    element_loss_w: np.ndarray, thermal_mesh: LayeredThermalMesh, layer_slabs: Sequence[int]
) -> np.ndarray:
    """Per-element copper loss ``(layers, rows, cols)`` added into the thermal
    element grid ``(slabs, rows, cols)`` (reference coupling.py:38-57).  Two
    layers mapped to one slab add up there."""
    loss = np.asarray(element_loss_w, dtype=np.float64)
    slabs, rows, cols = thermal_mesh.element_grid_shape
    if loss.ndim != 3 or loss.shape[1:] != (rows, cols):
        raise ValueError("the electrical element grid must match the thermal (rows, cols) footprint")
    mapping = _layer_slabs(layer_slabs, loss.shape[0], slabs)
    heat = np.zeros((slabs, rows, cols), dtype=np.float64)
    for layer, slab in enumerate(mapping):
        heat[slab] += loss[layer]
    return heat


def element_joule_heat_w(solution, thermal_mesh: LayeredThermalMesh, layer_slabs: Sequence[int]) -> np.ndarray:
    """The element Joule loss of a DC solution as ``element_heat_w`` of a
    thermal problem (reference coupling.py:60-74).  Via losses are nodal and
    go through :func:`via_joule_heat_sources`."""
    return element_heat_from_losses(solution.element_joule_loss_w, thermal_mesh, layer_slabs)


def via_heat_sources(
    vias: Sequence,
    via_loss_w: np.ndarray,
    layer_count: int,
    thermal_mesh: LayeredThermalMesh,
    layer_slabs: Sequence[int],
) -> tuple[HeatSource, ...]:
    """Each via's loss as two heat sources, half at each end (reference
    coupling.py:77-111).  An end on electrical layer ``L`` heats the node pair
    (slab face, row, col) and (slab face + 1, row, col) of slab
    ``layer_slabs[L]``, so the heat enters the copper slab itself."""
    slabs, rows, cols = thermal_mesh.element_grid_shape
    mapping = _layer_slabs(layer_slabs, layer_count, slabs)
    losses = np.asarray(via_loss_w, dtype=np.float64)
    if losses.shape != (len(vias),):
        raise ValueError("via_loss_w must hold one value per via")
    sources: list[HeatSource] = []
    for index, (via, loss) in enumerate(zip(vias, losses)):
        for end, (layer, row, col) in (("lower", via.lower), ("upper", via.upper)):
            if row > rows or col > cols:
                raise ValueError(f"via node {(layer, row, col)!r} lies outside the thermal footprint")
            slab = mapping[layer]
            sources.append(
                HeatSource(nodes=((slab, row, col), (slab + 1, row, col)), power_w=0.5 * float(loss),
                           name=f"via{index}-{end}")
            )
    return tuple(sources)


def via_joule_heat_sources(
    problem, solution, thermal_mesh: LayeredThermalMesh, layer_slabs: Sequence[int]
) -> tuple[HeatSource, ...]:
    """Nodal heat of every via of a DC problem's solution (reference
    coupling.py:114-131)."""
    return via_heat_sources(problem.vias, solution.via_joule_loss_w, problem.mesh.node_shape[0],
                            thermal_mesh, layer_slabs)
