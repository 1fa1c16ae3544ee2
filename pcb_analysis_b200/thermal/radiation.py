"""Grey surface-to-ambient radiation, handled as a Newton-linearised Robin face.

Mirrors src/thermal/matrix_free_mpir_fem/radiation.py of pcb-analysis.  A
surface at T facing an ambient T_a with emissivity e loses
q = e sigma (T^4 - T_a^4).  Linearised at the iterate T_k this is the Robin
face q = h_k (T - T_eff) with h_k = 4 e sigma T_k^3 and
T_eff = T_k - (T_k^4 - T_a^4) / (4 T_k^3); since conduction is linear, solving
the linear problem with these faces and repeating is Newton's method.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .boundaries import ConvectionBoundary, ExposedFaceConvection
from .mesh import FACE_DIRECTIONS, FaceDirection, LayeredThermalMesh, Side, corner_views

STEFAN_BOLTZMANN_W_PER_M2_K4 = 5.670374419e-8


def _emissivity(value, ndim: tuple[int, ...]):
    e = np.asarray(value, dtype=np.float64)
    if e.ndim not in ndim:
        raise ValueError("emissivity must be a scalar or an array matching the faces")
    if not np.all(np.isfinite(e)) or np.any(e < 0.0) or np.any(e > 1.0):
        raise ValueError("emissivity must lie in [0, 1]")
    return float(e) if e.ndim == 0 else e.copy()


def _ambient(value, ndim: tuple[int, ...]):
    a = np.asarray(value, dtype=np.float64)
    if a.ndim not in ndim:
        raise ValueError("ambient must be a scalar or an array matching the faces")
    if not np.all(np.isfinite(a)) or np.any(a <= 0.0):
        raise ValueError("radiative ambient temperature must be finite and positive (kelvin)")
    return float(a) if a.ndim == 0 else a.copy()


def newton_linearisation(emissivity, surface_temperature_k, ambient_temperature_k) -> tuple[np.ndarray, np.ndarray]:
    """(h_k, T_eff) of the Newton step at the given surface temperature."""

    surface = np.asarray(surface_temperature_k, dtype=np.float64)
    ambient = np.asarray(ambient_temperature_k, dtype=np.float64)
    surface = np.where(np.isfinite(surface) & (surface > 0.0), surface, ambient)
    cubic = surface**3
    coefficient = 4.0 * np.asarray(emissivity) * STEFAN_BOLTZMANN_W_PER_M2_K4 * cubic
    effective = surface - (surface**4 - ambient**4) / (4.0 * cubic)
    return coefficient, np.broadcast_to(effective, surface.shape).copy()


def face_temperature_k(mesh: LayeredThermalMesh, temperature_k: np.ndarray, side: Side) -> np.ndarray:
    """Mean of the four corner temperatures of each top or bottom face, (rows, cols)."""

    grid = np.asarray(temperature_k, dtype=np.float64).reshape(mesh.node_shape)
    layer = grid[-1] if side == "top" else grid[0]
    return 0.25 * (layer[:-1, :-1] + layer[:-1, 1:] + layer[1:, :-1] + layer[1:, 1:])


def element_temperature_k(mesh: LayeredThermalMesh, temperature_k: np.ndarray) -> np.ndarray:
    """Mean of the eight corner temperatures of each element."""

    grid = np.asarray(temperature_k, dtype=np.float64).reshape(mesh.node_shape)
    total = np.zeros(mesh.element_grid_shape, dtype=np.float64)
    for view in corner_views(grid):
        total += view
    return total / 8.0


@dataclass(frozen=True)
class RadiationBoundary:
    """Radiation of the top or bottom face to an ambient; scalars or (rows, cols) arrays."""

    side: Side
    emissivity: float | np.ndarray
    ambient_temperature_k: float | np.ndarray

    def __post_init__(self) -> None:
        if self.side not in ("top", "bottom"):
            raise ValueError("side must be 'top' or 'bottom'")
        object.__setattr__(self, "emissivity", _emissivity(self.emissivity, (0, 2)))
        object.__setattr__(self, "ambient_temperature_k", _ambient(self.ambient_temperature_k, (0, 2)))

    def check_shape(self, mesh: LayeredThermalMesh) -> None:
        shape = mesh.element_grid_shape[1:]
        for name in ("emissivity", "ambient_temperature_k"):
            value = np.asarray(getattr(self, name))
            if value.ndim == 2 and value.shape != shape:
                raise ValueError(f"{name} array must match (rows, cols) of the mesh")

    @property
    def radiates(self) -> bool:
        return bool(np.any(np.asarray(self.emissivity) > 0.0))

    def mean_ambient_k(self) -> float:
        return float(np.mean(self.ambient_temperature_k))

    def linearize(self, mesh: LayeredThermalMesh, temperature_k: np.ndarray) -> ConvectionBoundary:
        shape = mesh.element_grid_shape[1:]
        surface = face_temperature_k(mesh, temperature_k, self.side)
        h, t_eff = newton_linearisation(self.emissivity, surface, np.broadcast_to(self.ambient_temperature_k, shape))
        return ConvectionBoundary(self.side, h, t_eff)


@dataclass(frozen=True)
class ExposedFaceRadiation:
    """Radiation of every exposed face of the active elements to an ambient."""

    emissivity: float | np.ndarray
    ambient_temperature_k: float | np.ndarray
    directions: tuple[FaceDirection, ...] = FACE_DIRECTIONS

    def __post_init__(self) -> None:
        directions = tuple(self.directions)
        if not directions or any(d not in FACE_DIRECTIONS for d in directions):
            raise ValueError(f"directions must be drawn from {FACE_DIRECTIONS}")
        if len(set(directions)) != len(directions):
            raise ValueError("directions must be unique")
        object.__setattr__(self, "emissivity", _emissivity(self.emissivity, (0, 3)))
        object.__setattr__(self, "ambient_temperature_k", _ambient(self.ambient_temperature_k, (0, 3)))
        object.__setattr__(self, "directions", directions)

    def check_shape(self, mesh: LayeredThermalMesh) -> None:
        shape = mesh.element_grid_shape
        for name in ("emissivity", "ambient_temperature_k"):
            value = np.asarray(getattr(self, name))
            if value.ndim == 3 and value.shape != shape:
                raise ValueError(f"{name} array must match (slabs, rows, cols) of the mesh")

    @property
    def radiates(self) -> bool:
        return bool(np.any(np.asarray(self.emissivity) > 0.0))

    def mean_ambient_k(self) -> float:
        return float(np.mean(self.ambient_temperature_k))

    def linearize(self, mesh: LayeredThermalMesh, temperature_k: np.ndarray) -> ExposedFaceConvection:
        shape = mesh.element_grid_shape
        surface = element_temperature_k(mesh, temperature_k)
        h, t_eff = newton_linearisation(self.emissivity, surface, np.broadcast_to(self.ambient_temperature_k, shape))
        return ExposedFaceConvection(h, t_eff, directions=self.directions)


Radiation = RadiationBoundary | ExposedFaceRadiation
