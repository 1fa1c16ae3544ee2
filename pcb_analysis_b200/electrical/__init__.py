"""DC conduction in layered PCB copper, solved on a B200.

Mirrors the layered DC surface of pcb-analysis's
``electrical.matrix_free_mpir_fem`` (src/electrical/matrix_free_mpir_fem/pcb.py):
the problem records, ``MatrixFreePCBOperator`` and ``solve_pcb_dc``.
"""

from ..mpir import MPIRConfig, MPIRResult, solve_mpir
from .pcb import (
    COPPER_CONDUCTIVITY_S_PER_M,
    CurrentTerminal,
    LayeredPCBMesh,
    MatrixFreePCBOperator,
    PCBConductionProblem,
    PCBConductionSolution,
    ViaConnection,
    VoltageTerminal,
    solve_pcb_dc,
    unit_sheet_matrices,
)

__all__ = [
    "COPPER_CONDUCTIVITY_S_PER_M",
    "CurrentTerminal",
    "LayeredPCBMesh",
    "MPIRConfig",
    "MPIRResult",
    "MatrixFreePCBOperator",
    "PCBConductionProblem",
    "PCBConductionSolution",
    "ViaConnection",
    "VoltageTerminal",
    "solve_mpir",
    "solve_pcb_dc",
    "unit_sheet_matrices",
]
