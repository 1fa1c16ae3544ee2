"""B200-native steady Q1 thermal solve of pcb-analysis's thermal package.

The package keeps the reference's Python call surface (``thermal``
subpackage, ``MPIRConfig``/``MPIRResult``/``solve_mpir``) and runs the
operator, the Jacobi PCG and the MPIR refinement in hand-written sm_100a
kernels of ``libthermal_b200.so`` (C ABI: include/thermal_b200.h).
"""

from .mpir import MPIRConfig, MPIRResult, MPIRStep, solve_mpir

__all__ = ["MPIRConfig", "MPIRResult", "MPIRStep", "solve_mpir"]
__version__ = "0.1.0"
