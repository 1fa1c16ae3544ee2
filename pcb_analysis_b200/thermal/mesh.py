"""Layered hexahedral Q1 mesh of a board stack.

Mirrors ``thermal.matrix_free_mpir_fem.mesh`` of pcb-analysis
(src/thermal/matrix_free_mpir_fem/mesh.py:127-343): the same constructor
arguments, validation messages, derived properties and element factors, so a
problem built for the reference builds here unchanged.

Node (z, y, x) of a mesh with S slabs, R rows and C columns has flat index
(z * (R + 1) + y) * (C + 1) + x; z = 0 is the bottom face.  The local corner
order of an element is 4 dz + 2 dy + dx.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Literal, Sequence

import numpy as np

COPPER_THERMAL_CONDUCTIVITY_W_PER_M_K = 385.0
FR4_IN_PLANE_THERMAL_CONDUCTIVITY_W_PER_M_K = 0.8
FR4_THROUGH_PLANE_THERMAL_CONDUCTIVITY_W_PER_M_K = 0.3

Node = tuple[int, int, int]
Side = Literal["top", "bottom"]
Preconditioner = Literal["two-level", "jacobi", "multilevel"]
FaceDirection = Literal["-x", "+x", "-y", "+y", "-z", "+z"]
FACE_DIRECTIONS: tuple[FaceDirection, ...] = ("-x", "+x", "-y", "+y", "-z", "+z")

# Corners (4 dz + 2 dy + dx) lying on each element face (mesh.py:44-51).
FACE_CORNERS: dict[str, tuple[int, int, int, int]] = {
    "-x": (0, 2, 4, 6),
    "+x": (1, 3, 5, 7),
    "-y": (0, 1, 4, 5),
    "+y": (2, 3, 6, 7),
    "-z": (0, 1, 2, 3),
    "+z": (4, 5, 6, 7),
}


def corner_views(grid: Any) -> tuple[Any, ...]:
    """The eight (slabs, rows, cols) windows of a node grid, corner order 4dz+2dy+dx.

    Window ``c`` holds, at element (s, r, c'), the node of that element's corner ``c``
    (reference mesh.py:28-37).
    """

    slabs, rows, cols = (axis - 1 for axis in grid.shape)
    out = []
    for corner in range(8):
        dz, dy, dx = corner >> 2, (corner >> 1) & 1, corner & 1
        out.append(grid[dz : dz + slabs, dy : dy + rows, dx : dx + cols])
    return tuple(out)


def exposed_element_faces(active: np.ndarray) -> dict[FaceDirection, np.ndarray]:
    """Faces of active elements whose neighbour across the face is void or outside.

    One boolean element-grid array per direction (reference mesh.py:54-77).
    """

    mask = np.asarray(active, dtype=bool)
    if mask.ndim != 3:
        raise ValueError("active must have shape (slabs, rows, cols)")
    faces: dict[FaceDirection, np.ndarray] = {}
    for direction in FACE_DIRECTIONS:
        axis = {"x": 2, "y": 1, "z": 0}[direction[1]]
        step = 1 if direction[0] == "+" else -1
        padded = np.pad(mask, [(1, 1) if a == axis else (0, 0) for a in range(3)])
        # neighbour[i] = padded[i + 1 + step] along the axis
        start = 1 + step
        index = [slice(None)] * 3
        index[axis] = slice(start, start + mask.shape[axis])
        faces[direction] = mask & ~padded[tuple(index)]
    return faces


def lump_faces_onto_nodes(face_weight: np.ndarray, direction: str, node_shape: tuple[int, int, int]) -> np.ndarray:
    """Spread one weight per element face equally over the face's four nodes.

    Corners are visited in the order of ``FACE_CORNERS`` and each adds
    ``weight / 4`` (reference mesh.py:80-92), which fixes the rounding.
    """

    weights = np.zeros(node_shape, dtype=np.float64)
    targets = corner_views(weights)
    share = face_weight / 4.0
    for corner in FACE_CORNERS[direction]:
        targets[corner][...] += share
    return weights


def face_area_m2(mesh: "LayeredThermalMesh", direction: str) -> np.ndarray:
    """Area of each element's face normal to ``direction`` (reference mesh.py:95-106)."""

    shape = mesh.element_grid_shape
    hz = np.asarray(mesh.slab_thickness_m, dtype=np.float64)[:, None, None]
    hx = mesh.pitch_x_m[None, None, :]
    hy = mesh.pitch_y_m[None, :, None]
    axis = direction[1]
    if axis == "z":
        area = hx * hy
    elif axis == "y":
        area = hx * hz
    else:
        area = hy * hz
    return np.array(np.broadcast_to(area, shape), dtype=np.float64)


def check_pitch_axis(value: object, count: int, name: str) -> np.ndarray:
    """A scalar or per-cell pitch as a ``(count,)`` array of positive lengths
    (reference electrical/matrix_free_mpir_fem/grid.py:223-233)."""

    pitch = np.asarray(value, dtype=np.float64)
    if pitch.ndim == 0:
        pitch = np.full(count, float(pitch))
    elif pitch.shape != (count,):
        raise ValueError(f"{name} must be a scalar or hold one value per cell ({count})")
    if not np.all(np.isfinite(pitch)) or np.any(pitch <= 0.0):
        raise ValueError(f"{name} must be finite and positive")
    return pitch.copy()


def _element_field(value: Any, shape: tuple[int, int, int], name: str) -> np.ndarray:
    array = np.asarray(value, dtype=np.float64)
    if array.ndim == 0:
        return np.full(shape, float(array), dtype=np.float64)
    if array.shape == (shape[0],):
        return np.repeat(array, shape[1] * shape[2]).reshape(shape)
    if array.shape == shape:
        return array.copy()
    raise ValueError(f"{name} must be a scalar, one value per slab, or match shape {shape}")


@dataclass(frozen=True)
class LayeredThermalMesh:
    """Structured hexahedral Q1 mesh of a PCB stack (reference mesh.py:127-343).

    ``slab_thickness_m`` lists the element slabs from the bottom up.  The
    in-plane pitches are one width or one width per column / row.
    Conductivities are a scalar, one value per slab or one per element;
    through-plane conductivity defaults to the in-plane one.  ``active`` marks
    the elements that exist; void elements carry no conductivity.
    """

    slab_thickness_m: Sequence[float]
    pitch_x_m: float | Sequence[float] | np.ndarray
    pitch_y_m: float | Sequence[float] | np.ndarray
    conductivity_w_per_m_k: float | Sequence[float] | np.ndarray
    element_shape: tuple[int, int] | None = None
    through_plane_conductivity_w_per_m_k: float | Sequence[float] | np.ndarray | None = None
    active: np.ndarray | None = None
    volumetric_heat_capacity_j_per_m3_k: float | Sequence[float] | np.ndarray | None = None

    def __post_init__(self) -> None:
        thickness = np.asarray(self.slab_thickness_m, dtype=np.float64)
        if thickness.ndim != 1 or thickness.size < 1:
            raise ValueError("slab_thickness_m must list at least one slab")
        if not np.all(np.isfinite(thickness)) or np.any(thickness <= 0.0):
            raise ValueError("slab thicknesses must be finite and positive")
        k_in = np.asarray(self.conductivity_w_per_m_k, dtype=np.float64)
        pitch_x = np.asarray(self.pitch_x_m, dtype=np.float64)
        pitch_y = np.asarray(self.pitch_y_m, dtype=np.float64)
        if self.element_shape is not None:
            rows, cols = (int(v) for v in self.element_shape)
        elif k_in.ndim == 3:
            rows, cols = int(k_in.shape[1]), int(k_in.shape[2])
        elif pitch_x.ndim == 1 and pitch_y.ndim == 1:
            rows, cols = int(pitch_y.size), int(pitch_x.size)
        else:
            raise ValueError(
                "element_shape is required unless conductivity has shape "
                "(slabs, rows, cols) or both pitches are per-cell arrays"
            )
        if rows < 1 or cols < 1:
            raise ValueError("element_shape must have positive axes")
        shape = (int(thickness.size), rows, cols)
        object.__setattr__(self, "pitch_x_m", check_pitch_axis(pitch_x, cols, "pitch_x_m"))
        object.__setattr__(self, "pitch_y_m", check_pitch_axis(pitch_y, rows, "pitch_y_m"))

        k_in = _element_field(k_in, shape, "conductivity_w_per_m_k")
        if self.through_plane_conductivity_w_per_m_k is None:
            k_z = k_in.copy()
        else:
            k_z = _element_field(
                self.through_plane_conductivity_w_per_m_k, shape, "through_plane_conductivity_w_per_m_k"
            )
        if self.active is None:
            active = np.ones(shape, dtype=bool)
        else:
            active = np.asarray(self.active, dtype=bool)
            if active.shape != shape:
                raise ValueError("active must match (slabs, rows, cols)")
            if not np.any(active):
                raise ValueError("at least one element must be active")
            active = active.copy()
        for name, array in (
            ("conductivity_w_per_m_k", k_in),
            ("through_plane_conductivity_w_per_m_k", k_z),
        ):
            if not np.all(np.isfinite(array)) or np.any(array[active] <= 0.0):
                raise ValueError(f"{name} must be finite and positive on active elements")
        k_in = np.where(active, k_in, 0.0)
        k_z = np.where(active, k_z, 0.0)
        capacity = None
        if self.volumetric_heat_capacity_j_per_m3_k is not None:
            capacity = _element_field(
                self.volumetric_heat_capacity_j_per_m3_k, shape, "volumetric_heat_capacity_j_per_m3_k"
            )
            if not np.all(np.isfinite(capacity)) or np.any(capacity[active] <= 0.0):
                raise ValueError(
                    "volumetric_heat_capacity_j_per_m3_k must be finite and positive on active elements"
                )
            capacity = np.where(active, capacity, 0.0)
        object.__setattr__(self, "slab_thickness_m", tuple(thickness.tolist()))
        object.__setattr__(self, "volumetric_heat_capacity_j_per_m3_k", capacity)
        object.__setattr__(self, "element_shape", (rows, cols))
        object.__setattr__(self, "conductivity_w_per_m_k", k_in)
        object.__setattr__(self, "through_plane_conductivity_w_per_m_k", k_z)
        object.__setattr__(self, "active", active)

    @property
    def element_grid_shape(self) -> tuple[int, int, int]:
        rows, cols = self.element_shape  # type: ignore[misc]
        return len(self.slab_thickness_m), rows, cols

    @property
    def node_shape(self) -> tuple[int, int, int]:
        slabs, rows, cols = self.element_grid_shape
        return slabs + 1, rows + 1, cols + 1

    @property
    def size(self) -> int:
        slabs, rows, cols = self.node_shape
        return slabs * rows * cols

    @property
    def uniform_pitch(self) -> bool:
        return bool(np.all(self.pitch_x_m == self.pitch_x_m[0]) and np.all(self.pitch_y_m == self.pitch_y_m[0]))

    @property
    def cell_area_m2(self) -> np.ndarray:
        return np.outer(self.pitch_y_m, self.pitch_x_m)

    @property
    def x_edges_m(self) -> np.ndarray:
        return np.concatenate(([0.0], np.cumsum(self.pitch_x_m)))

    @property
    def y_edges_m(self) -> np.ndarray:
        return np.concatenate(([0.0], np.cumsum(self.pitch_y_m)))

    @property
    def element_volume_m3(self) -> np.ndarray:
        hz = np.asarray(self.slab_thickness_m, dtype=np.float64)
        return hz[:, None, None] * self.cell_area_m2[None, :, :]

    def element_coefficients(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """a_x = k_in h_y h_z / h_x, a_y = k_in h_x h_z / h_y, a_z = k_z h_x h_y / h_z.

        Evaluated left to right as the reference does (mesh.py:276-293), so the
        FP64 factors carry the same bits.
        """

        hz = np.asarray(self.slab_thickness_m, dtype=np.float64)[:, None, None]
        hx = self.pitch_x_m[None, None, :]
        hy = self.pitch_y_m[None, :, None]
        k_in = self.conductivity_w_per_m_k
        k_z = self.through_plane_conductivity_w_per_m_k
        return (
            np.ascontiguousarray(k_in * hy * hz / hx),
            np.ascontiguousarray(k_in * hx * hz / hy),
            np.ascontiguousarray(k_z * hx * hy / hz),
        )

    @property
    def has_heat_capacity(self) -> bool:
        return self.volumetric_heat_capacity_j_per_m3_k is not None

    def nodal_heat_capacity_j_per_k(self) -> np.ndarray:
        """Element heat capacity rho c V lumped equally onto its eight corners."""

        if self.volumetric_heat_capacity_j_per_m3_k is None:
            raise ValueError("the mesh has no volumetric_heat_capacity_j_per_m3_k; a transient solve needs one")
        element = self.volumetric_heat_capacity_j_per_m3_k * self.element_volume_m3 / 8.0
        nodal = np.zeros(self.node_shape, dtype=np.float64)
        for view in corner_views(nodal):
            view[...] += element
        return nodal

    @property
    def is_full(self) -> bool:
        return bool(np.all(self.active))

    @property
    def active_nodes(self) -> np.ndarray:
        """Nodes of at least one active element."""

        nodes = np.zeros(self.node_shape, dtype=bool)
        for view in corner_views(nodes):
            view |= self.active  # type: ignore[operator]
        return nodes

    def exposed_faces(self) -> dict[FaceDirection, np.ndarray]:
        return exposed_element_faces(self.active)  # type: ignore[arg-type]


def flat_index(node: Node, shape: tuple[int, int, int]) -> int:
    """Flat index of a (z, y, x) node (reference mesh.py:318-325)."""

    if len(node) != 3 or any(index < 0 for index in node):
        raise ValueError(f"invalid node {node!r}")
    try:
        return int(np.ravel_multi_index(node, shape))
    except ValueError as exc:
        raise ValueError(f"node {node!r} lies outside mesh shape {shape}") from exc


STIFFNESS_1D = np.array([[1.0, -1.0], [-1.0, 1.0]])
MASS_1D = np.array([[2.0, 1.0], [1.0, 2.0]]) / 6.0


def unit_hexahedron_matrices() -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """U_x = M (x) M (x) S, U_y = M (x) S (x) M, U_z = S (x) M (x) M (reference mesh.py:346-359)."""

    unit_x = np.kron(MASS_1D, np.kron(MASS_1D, STIFFNESS_1D))
    unit_y = np.kron(MASS_1D, np.kron(STIFFNESS_1D, MASS_1D))
    unit_z = np.kron(STIFFNESS_1D, np.kron(MASS_1D, MASS_1D))
    return unit_x, unit_y, unit_z
