"""Split-precision matrix-free conduction operator, resident on a B200.

Drop-in for ``MatrixFreeThermalOperator`` of pcb-analysis
(src/thermal/matrix_free_mpir_fem/operator.py:30-525): same constructor,
attributes and methods.  Rows of fixed nodes (and of nodes of void elements
only) are the identity; the lumped Robin conductance sits on the diagonal.
Every action runs on the device through libthermal_b200.so: the FP32 low
action, the FP64 high action, the unconstrained stiffness action of the right
hand side and the heat budget, and the whole MPIR solve (native_solve_mpir).
"""

from __future__ import annotations

from typing import Any

import numpy as np

from .. import _native
from ..mpir import LOW_RUNTIME_NAME, MPIRConfig
from .mesh import Preconditioner
from .problem import ThermalConductionProblem
from .system import convection_specs, problem_inputs

KERNEL_NAME = "b200-haar-zmarch-hex-q1"
HIGH_KERNEL_NAME = "b200-haar-zmarch-hex-q1-fp64"


class B200Float32Runtime:
    """The low-precision runtime of this package: FP32 vectors in B200 HBM.

    Stands where the reference passes a NumPy or CuPy runtime
    (src/electrical/matrix_free_mpir_fem/runtime.py:20-44); device arrays are
    torch CUDA tensors, host arrays NumPy.
    """

    name = LOW_RUNTIME_NAME
    dtype = np.float32
    is_cuda = True

    def __init__(self, device_id: int = 0) -> None:
        _native.require_device(device_id)
        self.device_id = int(device_id)

    def from_host(self, value: np.ndarray) -> Any:
        import torch

        return torch.as_tensor(np.asarray(value, dtype=np.float32), device=f"cuda:{self.device_id}")

    def to_host(self, value: Any) -> np.ndarray:
        if hasattr(value, "detach"):
            return value.detach().cpu().numpy().astype(np.float64)
        return np.asarray(value, dtype=np.float64)

    def synchronize(self) -> None:
        import torch

        torch.cuda.synchronize(self.device_id)


def _check_backend(runtime: Any, backend: Any, native: Any) -> None:
    if runtime is not None and backend is not None:
        raise ValueError("pass either runtime or backend, not both")
    if backend not in (None, "cuda", "auto"):
        raise NotImplementedError(
            f"backend={backend!r}: the B200 build runs only on the GPU (use backend='cuda' or leave it unset)"
        )
    if runtime is not None and not isinstance(runtime, B200Float32Runtime):
        raise NotImplementedError("the B200 build takes only its own B200Float32Runtime")
    if native is False:
        # The reference uses native=False to pick its NumPy path; there is no
        # such path here, so the request cannot be honoured.
        raise NotImplementedError("native=False asks for a host implementation; the B200 build has none")


class MatrixFreeThermalOperator:
    """Split FP64/FP32 element-by-element heat-conduction operator on the device.

    ``preconditioner="two-level"`` (the reference default) adds the
    patch-constant coarse correction of reference two_level.py to the Jacobi
    scaling, assembled and inverted on the device; ``coarse_block_nodes`` sets
    the patch width (``None``: the smallest width whose coarse grid has at most
    2048 patches).  ``preconditioner="jacobi"`` is the diagonal scaling alone.
    ``preconditioner="multilevel"`` (no reference counterpart) solves each
    node column's z coupling exactly and corrects with one V-cycle over
    Galerkin grids (4 x 4 patches of the fine grid, then 2 x 2 patches per
    level), so that its iteration count stays nearly flat on boards far
    larger than the two-level patches can serve.
    """

    def __init__(
        self,
        problem: ThermalConductionProblem,
        *,
        runtime: B200Float32Runtime | None = None,
        backend: str | None = None,
        device_id: int = 0,
        preconditioner: Preconditioner = "two-level",
        coarse_block_nodes: int | None = None,
        native: bool | None = None,
        capacity_per_s: np.ndarray | None = None,
    ) -> None:
        _check_backend(runtime, backend, native)
        if preconditioner not in ("two-level", "jacobi", "multilevel"):
            raise ValueError("preconditioner must be 'two-level', 'jacobi' or 'multilevel'")
        if coarse_block_nodes is not None and int(coarse_block_nodes) < 1:
            raise ValueError("coarse_block_nodes must be a positive node count")
        self.high_dtype = np.float64
        self.inner_solver = "pcg"
        self.problem = problem
        self.mesh = problem.mesh
        self.size = self.mesh.size
        self.preconditioner = preconditioner
        self.runtime = runtime or B200Float32Runtime(device_id)
        self.coarse_correction = None
        self._capacity = None if capacity_per_s is None else _capacity_array(capacity_per_s, self.size)
        self._masks: dict[str, np.ndarray] = {}
        self._diagonal: np.ndarray | None = None
        # The problem is prepared on the device: masks, lumped Robin terms,
        # loads, then the solver arrays and the diagonal.
        self.device_system = _native.DeviceSystem.from_problem(
            **problem_inputs(problem, self._capacity), device=self.runtime.device_id)
        if preconditioner != "jacobi":
            try:
                self.device_system.set_preconditioner(preconditioner, coarse_block_nodes)
            except Exception:
                self.device_system.close()
                raise
            self.coarse_correction = self.device_system.preconditioner()
        self.low_operator_backend = KERNEL_NAME
        self.high_operator_backend = HIGH_KERNEL_NAME

    # ----------------------------------------------------------------- masks
    # Host copies of the node masks (reference operator.py:89-96), made on
    # first use: the device holds its own.
    # Each is computed on first use only: a solve needs the free mask alone.
    def _mask(self, name: str) -> np.ndarray:
        if name not in self._masks:
            problem = self.problem
            if name == "active_nodes":
                value = self.mesh.active_nodes
            elif name == "fixed_nodes":
                value = problem.fixed_temperature_mask | ~self._mask("active_nodes")
            elif name == "free_nodes":
                value = ~self._mask("fixed_nodes")
            elif name == "fixed_temperature_k":
                value = np.where(problem.fixed_temperature_mask & self._mask("active_nodes"),
                                 problem.fixed_temperature_k, 0.0)
            else:
                raise KeyError(name)
            self._masks[name] = value
        return self._masks[name]

    @property
    def active_nodes(self) -> np.ndarray:
        return self._mask("active_nodes")

    @property
    def fixed_nodes(self) -> np.ndarray:
        return self._mask("fixed_nodes")

    @property
    def free_nodes(self) -> np.ndarray:
        return self._mask("free_nodes")

    @property
    def fixed_temperature_k(self) -> np.ndarray:
        return self._mask("fixed_temperature_k")

    def system_arrays(self) -> dict[str, np.ndarray]:
        """The prepared board as ``DeviceSystem`` takes it: geometry, element
        conductivities, lumped Robin totals and the free-node mask (the last
        two read back from the device)."""

        mesh = self.mesh
        prepared = self.device_system.prepared()
        return dict(
            slab_thickness_m=np.asarray(mesh.slab_thickness_m, dtype=np.float64),
            pitch_x_m=np.asarray(mesh.pitch_x_m, dtype=np.float64),
            pitch_y_m=np.asarray(mesh.pitch_y_m, dtype=np.float64),
            k_in=np.asarray(mesh.conductivity_w_per_m_k, dtype=np.float64),
            k_z=np.asarray(mesh.through_plane_conductivity_w_per_m_k, dtype=np.float64),
            robin_total=prepared["robin_total"],
            free_nodes=prepared["free_nodes"],
        )

    def close(self) -> None:
        """Release the device memory of this operator."""

        self.device_system.close()

    # ---------------------------------------------------------------- actions
    def _flat(self, values: Any, name: str = "vector") -> np.ndarray:
        flat = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        if flat.size != self.size:
            raise ValueError(f"{name} has size {flat.size}, expected {self.size}")
        return flat

    def apply_high(self, vector: np.ndarray) -> np.ndarray:
        """FP64 action y = A x on the device (reference operator.py:308-316)."""

        return self.device_system.apply_f64(self._flat(vector))

    def apply_low(self, vector: Any) -> Any:
        """FP32 action on the device; a torch CUDA tensor stays on the device."""

        if hasattr(vector, "is_cuda") and vector.is_cuda:
            import torch

            x = vector.reshape(-1).to(torch.float32).contiguous()
            if x.numel() != self.size:
                raise ValueError(f"vector has size {x.numel()}, expected {self.size}")
            y = torch.empty_like(x)
            self.device_system.apply_f32_device(x, y)
            return y.reshape(vector.shape)
        flat = np.ascontiguousarray(vector, dtype=np.float32).reshape(-1)
        if flat.size != self.size:
            raise ValueError(f"vector has size {flat.size}, expected {self.size}")
        return self.device_system.apply_f32(flat)

    def stiffness_high(self, vector: np.ndarray) -> np.ndarray:
        """Unconstrained conduction action K x in FP64 (reference operator.py:243-269)."""

        return self.device_system.stiffness_f64(self._flat(vector))

    def diagonal_high(self) -> np.ndarray:
        if self._diagonal is None:
            self._diagonal = self.device_system.diagonal()
        return self._diagonal

    def diagonal_low(self) -> np.ndarray:
        return self.diagonal_high().astype(np.float32)

    def _refreshed(self) -> None:
        self._diagonal = None
        if self.coarse_correction is not None:
            self.coarse_correction = self.device_system.preconditioner()

    def replace_boundaries(self, problem: ThermalConductionProblem) -> None:
        """Take the convection boundaries of `problem`, the same board with
        other Robin boundaries (the Newton linearisation of its radiation), on
        the resident system: the lumped terms, the diagonal and the coarse
        operator are rebuilt on the device."""

        same_board = (
            problem.mesh is self.mesh
            or (problem.mesh.element_grid_shape == self.mesh.element_grid_shape
                and np.array_equal(problem.mesh.active, self.mesh.active))
        )
        if not (same_board
                and np.array_equal(problem.fixed_temperature_mask, self.problem.fixed_temperature_mask)
                and np.array_equal(problem.fixed_temperature_k, self.problem.fixed_temperature_k)):
            raise ValueError("replace_boundaries needs the same board with the same fixed nodes")
        self.device_system.set_convection(convection_specs(problem.convection))
        self.problem = problem
        self._refreshed()

    def set_capacity_per_s(self, capacity_per_s: np.ndarray) -> None:
        """Replace the lumped C / dt term of a backward-Euler step on the
        resident system (the Robin totals, the diagonal and the two-level
        coarse operator are rebuilt on the device)."""

        self._capacity = _capacity_array(capacity_per_s, self.size)
        self.device_system.set_capacity(self._capacity)
        self._refreshed()

    def precondition_low(self, vector: Any) -> np.ndarray:
        """FP32 preconditioner action of the inner PCG (reference operator.py:366-371)."""

        if self.coarse_correction is None:
            return (np.asarray(vector, dtype=np.float32).reshape(-1) / self.diagonal_low()).astype(np.float32)
        return self.device_system.precondition_f32(self._flat(vector))

    def native_solve_mpir(
        self, rhs_high: np.ndarray, config: MPIRConfig, initial_guess: np.ndarray | None = None
    ) -> tuple:
        """The whole MPIR solve on the device (reference hook, operator.py:318-347)."""

        result = self.device_system.solve_mpir(self._flat(rhs_high, "rhs"), config, initial_guess)
        return (
            result["solution"],
            result["converged"],
            result["outer_iterations"],
            result["inner_iterations"],
            result["relative_residual"],
            result["high_operator_applications"],
            result["low_operator_applications"],
            result["history"],
        )

    # ------------------------------------------------------------------ loads
    def nodal_load(self) -> np.ndarray:
        """Heat per node, W (reference operator.py:374-387), prepared on the device."""

        return self.device_system.prepared_array("load")

    def default_reference_temperature(self) -> float:
        """Ambient of the first convective face, else the mean fixed value (operator.py:389-397)."""

        if self.problem.convection:
            return float(self.problem.convection[0].mean_ambient_k())
        mask = self.problem.fixed_temperature_mask & self.active_nodes
        return float(np.mean(self.problem.fixed_temperature_k[mask]))

    def build_rhs(self, reference_temperature_k: float = 0.0, previous_temperature_k: np.ndarray | None = None) -> np.ndarray:
        """Right-hand side for the rise above ``reference_temperature_k`` (operator.py:411-440),
        built on the device: fixed temperatures move onto the free rows through
        the unconstrained stiffness action; fixed rows carry the shifted value."""

        return self.device_system.build_rhs(float(reference_temperature_k), previous_temperature_k)

    # ---------------------------------------------------------- post-process
    def postprocess(self, temperature_k: np.ndarray, previous_temperature_k: np.ndarray | None = None) -> dict:
        """-k grad T per element, heat removed per boundary and the heat budget
        of a temperature field (reference operator.py:443-525, solve.py:255-280),
        in one pass on the device."""

        return self.device_system.postprocess(temperature_k, previous_temperature_k)

    def stored_heat_w(self, temperature_k: np.ndarray, previous_temperature_k: np.ndarray | None) -> np.ndarray:
        flat = np.asarray(temperature_k, dtype=np.float64).reshape(-1)
        if previous_temperature_k is None or self._capacity is None:
            return np.zeros(self.size, dtype=np.float64)
        previous = np.asarray(previous_temperature_k, dtype=np.float64).reshape(-1)
        finite = np.isfinite(flat) & np.isfinite(previous)
        return np.where(finite, self._capacity * (flat - previous), 0.0)

    def unconstrained_residual(self, temperature_k: np.ndarray, previous_temperature_k: np.ndarray | None = None) -> np.ndarray:
        """K T + R (T - T_amb) + C/dt (T - T_n) - q at every node (operator.py:458-482)."""

        out = self.device_system.postprocess(temperature_k, previous_temperature_k, flux=False, residual=True)
        return out["residual"]

    def convective_heat(self, temperature_k: np.ndarray) -> np.ndarray:
        """Heat removed by each convection boundary, W, in problem order."""

        return self.device_system.postprocess(temperature_k, flux=False)["convective_heat_w"]

    def element_heat_flux(self, temperature_k: np.ndarray) -> np.ndarray:
        """-k grad T at each element centre, W/m^2, as (x, y, z) (operator.py:500-525)."""

        return self.device_system.postprocess(temperature_k)["heat_flux"]


def _capacity_array(capacity_per_s: Any, size: int) -> np.ndarray:
    capacity = np.asarray(capacity_per_s, dtype=np.float64).reshape(-1)
    if capacity.size != size:
        raise ValueError("capacity_per_s must hold one value per node")
    if not np.all(np.isfinite(capacity)) or np.any(capacity < 0.0):
        raise ValueError("capacity_per_s must be finite and non-negative")
    return capacity.copy()
