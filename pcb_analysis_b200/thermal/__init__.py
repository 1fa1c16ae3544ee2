"""Steady Q1 heat conduction of a layered board, solved on a B200.

Mirrors the public surface of pcb-analysis's ``thermal.matrix_free_mpir_fem``
(src/thermal/matrix_free_mpir_fem/__init__.py) for the steady solve.
"""

from .boundaries import Convection, ConvectionBoundary, ExposedFaceConvection, HeatSource
from .mesh import (
    COPPER_THERMAL_CONDUCTIVITY_W_PER_M_K,
    FACE_DIRECTIONS,
    FR4_IN_PLANE_THERMAL_CONDUCTIVITY_W_PER_M_K,
    FR4_THROUGH_PLANE_THERMAL_CONDUCTIVITY_W_PER_M_K,
    LayeredThermalMesh,
    exposed_element_faces,
    unit_hexahedron_matrices,
)
from .operator import B200Float32Runtime, MatrixFreeThermalOperator
from .problem import ThermalConductionProblem
from .radiation import (
    STEFAN_BOLTZMANN_W_PER_M2_K4,
    ExposedFaceRadiation,
    Radiation,
    RadiationBoundary,
    newton_linearisation,
)
from .solve import ThermalConductionSolution, solve_thermal_conduction
from .transient import TimeSchedule, TransientStep, TransientThermalSolution, solve_thermal_transient

__all__ = [
    "B200Float32Runtime",
    "COPPER_THERMAL_CONDUCTIVITY_W_PER_M_K",
    "Convection",
    "ConvectionBoundary",
    "ExposedFaceConvection",
    "ExposedFaceRadiation",
    "FACE_DIRECTIONS",
    "FR4_IN_PLANE_THERMAL_CONDUCTIVITY_W_PER_M_K",
    "FR4_THROUGH_PLANE_THERMAL_CONDUCTIVITY_W_PER_M_K",
    "HeatSource",
    "LayeredThermalMesh",
    "MatrixFreeThermalOperator",
    "Radiation",
    "RadiationBoundary",
    "STEFAN_BOLTZMANN_W_PER_M2_K4",
    "ThermalConductionProblem",
    "ThermalConductionSolution",
    "TimeSchedule",
    "TransientStep",
    "TransientThermalSolution",
    "exposed_element_faces",
    "newton_linearisation",
    "solve_thermal_conduction",
    "solve_thermal_transient",
    "unit_hexahedron_matrices",
]
