"""Grey radiation of board faces to an ambient, as Newton-linearised Robin faces.

The public names, fields and messages are those of pcb-analysis's
src/thermal/matrix_free_mpir_fem/radiation.py.  A face at T that sees an
ambient T_a with emissivity e loses e sigma (T^4 - T_a^4).  About a field
T_k that loss is, to first order, h_k (T - T_eff) with

    h_k = 4 e sigma T_k^3,   T_eff = T_k - (T_k^4 - T_a^4) / (4 T_k^3),

an ordinary convection face; the solve repeats with the faces taken at the
new field (Newton's method, since conduction is linear).
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any

import numpy as np

from .boundaries import ConvectionBoundary, ExposedFaceConvection
from .mesh import FACE_DIRECTIONS, FaceDirection, LayeredThermalMesh, Side, corner_views

STEFAN_BOLTZMANN_W_PER_M2_K4 = 5.670374419e-8


def _face_values(value: Any, ranks: tuple[int, ...], what: str, ok, message: str):
    """A scalar or an array of one of `ranks`, every entry passing `ok`."""

    array = np.asarray(value, dtype=np.float64)
    if array.ndim not in ranks:
        raise ValueError(f"{what} must be a scalar or an array matching the faces")
    if not ok(array):
        raise ValueError(message)
    return float(array) if array.ndim == 0 else array.copy()


def _emissivity_ok(e: np.ndarray) -> bool:
    return bool(np.isfinite(e).all() and (e >= 0.0).all() and (e <= 1.0).all())


def _ambient_ok(t: np.ndarray) -> bool:
    return bool(np.isfinite(t).all() and (t > 0.0).all())


def newton_linearisation(emissivity, surface_temperature_k, ambient_temperature_k) -> tuple[np.ndarray, np.ndarray]:
    """(h_k, T_eff) of the Newton step about the given surface temperature;
    a surface value that is not a positive number is taken at the ambient."""

    ambient = np.asarray(ambient_temperature_k, dtype=np.float64)
    about = np.asarray(surface_temperature_k, dtype=np.float64)
    about = np.where(np.isfinite(about) & (about > 0.0), about, ambient)
    t3 = about**3
    h = 4.0 * np.asarray(emissivity) * STEFAN_BOLTZMANN_W_PER_M2_K4 * t3
    t_eff = about - (about**4 - ambient**4) / (4.0 * t3)
    return h, np.array(np.broadcast_to(t_eff, about.shape))


def face_temperature_k(mesh: LayeredThermalMesh, temperature_k: np.ndarray, side: Side) -> np.ndarray:
    """Mean of the four corner temperatures of each top or bottom face, (rows, cols)."""

    grid = np.asarray(temperature_k, dtype=np.float64).reshape(mesh.node_shape)
    nodes = grid[-1 if side == "top" else 0]
    return 0.25 * (nodes[:-1, :-1] + nodes[:-1, 1:] + nodes[1:, :-1] + nodes[1:, 1:])


def element_temperature_k(mesh: LayeredThermalMesh, temperature_k: np.ndarray) -> np.ndarray:
    """Mean of the eight corner temperatures of each element."""

    grid = np.asarray(temperature_k, dtype=np.float64).reshape(mesh.node_shape)
    return sum(corner_views(grid), np.zeros(mesh.element_grid_shape)) / 8.0


class _Radiating:
    """What both radiating boundaries share: their two face fields, the
    checks on them, and the linearisation about a node field."""

    _face_rank = 0  # rank of a per-face array: 2 for the top/bottom faces, 3 for element faces

    def _check_fields(self) -> None:
        ranks = (0, self._face_rank)
        object.__setattr__(self, "emissivity", _face_values(
            self.emissivity, ranks, "emissivity", _emissivity_ok, "emissivity must lie in [0, 1]"))
        object.__setattr__(self, "ambient_temperature_k", _face_values(
            self.ambient_temperature_k, ranks, "ambient", _ambient_ok,
            "radiative ambient temperature must be finite and positive (kelvin)"))

    def _faces_shape(self, mesh: LayeredThermalMesh) -> tuple[int, ...]:
        raise NotImplementedError

    def _surface_k(self, mesh: LayeredThermalMesh, temperature_k: np.ndarray) -> np.ndarray:
        raise NotImplementedError

    def check_shape(self, mesh: LayeredThermalMesh) -> None:
        shape = self._faces_shape(mesh)
        axes = "(rows, cols)" if len(shape) == 2 else "(slabs, rows, cols)"
        for name in ("emissivity", "ambient_temperature_k"):
            value = np.asarray(getattr(self, name))
            if value.ndim == len(shape) and value.shape != shape:
                raise ValueError(f"{name} array must match {axes} of the mesh")

    @property
    def radiates(self) -> bool:
        return bool((np.asarray(self.emissivity) > 0.0).any())

    def mean_ambient_k(self) -> float:
        return float(np.mean(self.ambient_temperature_k))

    def _tangent(self, mesh: LayeredThermalMesh, temperature_k: np.ndarray):
        ambient = np.broadcast_to(self.ambient_temperature_k, self._faces_shape(mesh))
        return newton_linearisation(self.emissivity, self._surface_k(mesh, temperature_k), ambient)


@dataclass(frozen=True)
class RadiationBoundary(_Radiating):
    """Radiation of the top or bottom face to an ambient; scalars or (rows, cols) arrays."""

    side: Side
    emissivity: float | np.ndarray
    ambient_temperature_k: float | np.ndarray
    _face_rank = 2

    def __post_init__(self) -> None:
        if self.side not in ("top", "bottom"):
            raise ValueError("side must be 'top' or 'bottom'")
        self._check_fields()

    def _faces_shape(self, mesh: LayeredThermalMesh) -> tuple[int, ...]:
        return tuple(mesh.element_grid_shape[1:])

    def _surface_k(self, mesh: LayeredThermalMesh, temperature_k: np.ndarray) -> np.ndarray:
        return face_temperature_k(mesh, temperature_k, self.side)

    def linearize(self, mesh: LayeredThermalMesh, temperature_k: np.ndarray) -> ConvectionBoundary:
        h, t_eff = self._tangent(mesh, temperature_k)
        return ConvectionBoundary(self.side, h, t_eff)


@dataclass(frozen=True)
class ExposedFaceRadiation(_Radiating):
    """Radiation of every exposed face of the active elements to an ambient."""

    emissivity: float | np.ndarray
    ambient_temperature_k: float | np.ndarray
    directions: tuple[FaceDirection, ...] = FACE_DIRECTIONS
    _face_rank = 3

    def __post_init__(self) -> None:
        chosen = tuple(self.directions)
        if not chosen or not set(chosen) <= set(FACE_DIRECTIONS):
            raise ValueError(f"directions must be drawn from {FACE_DIRECTIONS}")
        if len(set(chosen)) != len(chosen):
            raise ValueError("directions must be unique")
        object.__setattr__(self, "directions", chosen)
        self._check_fields()

    def _faces_shape(self, mesh: LayeredThermalMesh) -> tuple[int, ...]:
        return tuple(mesh.element_grid_shape)

    def _surface_k(self, mesh: LayeredThermalMesh, temperature_k: np.ndarray) -> np.ndarray:
        return element_temperature_k(mesh, temperature_k)

    def linearize(self, mesh: LayeredThermalMesh, temperature_k: np.ndarray) -> ExposedFaceConvection:
        h, t_eff = self._tangent(mesh, temperature_k)
        return ExposedFaceConvection(h, t_eff, directions=self.directions)


Radiation = RadiationBoundary | ExposedFaceRadiation
