"""DC conduction in layered PCB copper, solved on a B200.

Mirrors ``electrical.matrix_free_mpir_fem.pcb`` of pcb-analysis
(src/electrical/matrix_free_mpir_fem/pcb.py:1-978): the same mesh, via,
terminal and problem records with their validation messages, the operator
protocol of ``MatrixFreePCBOperator`` and ``solve_pcb_dc`` with its solution
fields.  Each copper layer is a sheet of bilinear (Q1) quadrilaterals of
conductance sigma t, and plated vias are conductance links between layer
nodes.  The operator, its diagonal and the whole MPIR solve (Jacobi or the
two-level preconditioner) run on the device through libthermal_b200.so
(``tb_dc_system_create``); the right-hand side and the post-processing follow
the reference's formulas on the host, with the unconstrained conductance
action on the device.
"""

from __future__ import annotations

import dataclasses
from dataclasses import dataclass
from typing import Any, Literal, Sequence

import numpy as np

from .. import _native
from ..mpir import MPIRConfig, MPIRResult, solve_mpir
from ..thermal.mesh import check_pitch_axis
from ..thermal.operator import B200Float32Runtime, _check_backend

Preconditioner = Literal["two-level", "jacobi"]

COPPER_CONDUCTIVITY_S_PER_M = 1.0 / 1.724e-8
Node = tuple[int, int, int]

KERNEL_NAME = "b200-haar-sheet-q1-vias"
HIGH_KERNEL_NAME = "b200-haar-sheet-q1-vias-fp64"


@dataclass(frozen=True)
class ViaConnection:
    """One resistive vertical connection between two nodal layer locations."""

    lower: Node
    upper: Node
    resistance_ohm: float

    def __post_init__(self) -> None:
        lower = tuple(int(index) for index in self.lower)
        upper = tuple(int(index) for index in self.upper)
        if len(lower) != 3 or len(upper) != 3:
            raise ValueError("via endpoints must be (layer, row, column) nodes")
        if lower == upper:
            raise ValueError("a via must connect two different nodes")
        if lower[0] == upper[0]:
            raise ValueError("a via must connect different layers")
        if not np.isfinite(self.resistance_ohm) or self.resistance_ohm <= 0.0:
            raise ValueError("via resistance must be finite and positive")
        object.__setattr__(self, "lower", lower)
        object.__setattr__(self, "upper", upper)

    @property
    def conductance_s(self) -> float:
        return 1.0 / float(self.resistance_ohm)


def _nodes(nodes: Sequence[Node]) -> tuple[Node, ...]:
    out = tuple(tuple(int(index) for index in node) for node in nodes)
    return out  # type: ignore[return-value]


@dataclass(frozen=True)
class CurrentTerminal:
    """A total current spread equally over a set of nodes."""

    nodes: tuple[Node, ...]
    current_a: float
    name: str = "terminal"

    def __post_init__(self) -> None:
        nodes = _nodes(self.nodes)
        if not nodes:
            raise ValueError("a current terminal needs at least one node")
        if len(set(nodes)) != len(nodes):
            raise ValueError("terminal nodes must be unique")
        if not np.isfinite(self.current_a):
            raise ValueError("terminal current must be finite")
        object.__setattr__(self, "nodes", nodes)


@dataclass(frozen=True)
class VoltageTerminal:
    """A set of nodes held at one potential (an ideal voltage source)."""

    nodes: tuple[Node, ...]
    voltage_v: float
    name: str = "terminal"

    def __post_init__(self) -> None:
        nodes = _nodes(self.nodes)
        if not nodes:
            raise ValueError("a voltage terminal needs at least one node")
        if len(set(nodes)) != len(nodes):
            raise ValueError("terminal nodes must be unique")
        if not np.isfinite(self.voltage_v):
            raise ValueError("terminal voltage must be finite")
        object.__setattr__(self, "nodes", nodes)


@dataclass(frozen=True)
class LayeredPCBMesh:
    """Structured Q1 sheet mesh of one conductor role (reference pcb.py:105-186).

    ``element_active`` has shape (layers, node_rows - 1, node_cols - 1); the
    pitches are one width or one per column / row; the conductivity is a
    scalar, one value per layer or one per element.
    """

    element_active: np.ndarray
    layer_thickness_m: Sequence[float]
    pitch_x_m: float | Sequence[float] | np.ndarray
    pitch_y_m: float | Sequence[float] | np.ndarray
    conductivity_s_per_m: float | Sequence[float] | np.ndarray = COPPER_CONDUCTIVITY_S_PER_M

    def __post_init__(self) -> None:
        active = np.asarray(self.element_active, dtype=bool)
        if active.ndim != 3 or active.shape[1] < 1 or active.shape[2] < 1:
            raise ValueError("element_active must have shape (layers, rows, cols) with positive axes")
        thickness = np.asarray(self.layer_thickness_m, dtype=np.float64)
        if thickness.shape != (active.shape[0],):
            raise ValueError("layer_thickness_m must contain one value per layer")
        if not np.all(np.isfinite(thickness)) or np.any(thickness <= 0.0):
            raise ValueError("layer thicknesses must be finite and positive")
        object.__setattr__(self, "pitch_x_m", check_pitch_axis(self.pitch_x_m, active.shape[2], "pitch_x_m"))
        object.__setattr__(self, "pitch_y_m", check_pitch_axis(self.pitch_y_m, active.shape[1], "pitch_y_m"))
        conductivity = np.asarray(self.conductivity_s_per_m, dtype=np.float64)
        if conductivity.ndim == 0:
            conductivity = np.full(active.shape, conductivity, dtype=np.float64)
        elif conductivity.shape == (active.shape[0],):
            conductivity = np.broadcast_to(conductivity[:, None, None], active.shape).copy()
        elif conductivity.shape != active.shape:
            raise ValueError("conductivity must be scalar, per-layer, or match element_active")
        if not np.all(np.isfinite(conductivity)) or np.any(conductivity <= 0.0):
            raise ValueError("conductivity must be finite and positive")
        object.__setattr__(self, "element_active", active.copy())
        object.__setattr__(self, "layer_thickness_m", tuple(thickness.tolist()))
        object.__setattr__(self, "conductivity_s_per_m", conductivity.copy())

    @property
    def node_shape(self) -> tuple[int, int, int]:
        layers, rows, cols = self.element_active.shape
        return layers, rows + 1, cols + 1

    @property
    def size(self) -> int:
        return int(np.prod(self.node_shape))

    @property
    def uniform_pitch(self) -> bool:
        return bool(np.all(self.pitch_x_m == self.pitch_x_m[0]) and np.all(self.pitch_y_m == self.pitch_y_m[0]))

    @property
    def cell_area_m2(self) -> np.ndarray:
        return self.pitch_y_m[:, None] * self.pitch_x_m[None, :]

    def element_coefficients(self) -> tuple[np.ndarray, np.ndarray]:
        """c_x = sigma t h_y / h_x and c_y = sigma t h_x / h_y, zero on void elements
        (reference pcb.py:171-186; the device rebuilds them in this order)."""

        conductivity = np.asarray(self.conductivity_s_per_m, dtype=np.float64)
        thickness = np.asarray(self.layer_thickness_m, dtype=np.float64)[:, None, None]
        sheet = conductivity * thickness * self.element_active.astype(np.float64)
        hx = self.pitch_x_m[None, None, :]
        hy = self.pitch_y_m[None, :, None]
        return np.ascontiguousarray(sheet * hy / hx), np.ascontiguousarray(sheet * hx / hy)


@dataclass(frozen=True)
class PCBConductionProblem:
    """One conductor role and its drive (reference pcb.py:189-246).

    Current-driven: balanced ``terminals`` with a ``reference_node`` for the
    gauge.  Voltage-driven: ``voltage_terminals`` fix the potential and
    ``reference_node`` stays None.  A node belongs to at most one terminal.
    """

    mesh: LayeredPCBMesh
    terminals: tuple[CurrentTerminal, ...] = ()
    reference_node: Node | None = None
    vias: tuple[ViaConnection, ...] = ()
    voltage_terminals: tuple[VoltageTerminal, ...] = ()

    def __post_init__(self) -> None:
        terminals = tuple(self.terminals)
        voltage_terminals = tuple(self.voltage_terminals)
        if voltage_terminals:
            if self.reference_node is not None:
                raise ValueError("voltage terminals fix the potential; reference_node must be None")
        else:
            if not terminals:
                raise ValueError("a PCB conduction problem needs current or voltage terminals")
            if self.reference_node is None:
                raise ValueError("a current-driven problem needs a reference_node")
            total = float(sum(t.current_a for t in terminals))
            magnitude = float(sum(abs(t.current_a) for t in terminals))
            if abs(total) > 1.0e-12 * max(1.0, magnitude):
                raise ValueError(f"terminal currents must sum to zero, got {total:.6g} A")
        owner: dict[Node, str] = {}
        for terminal in (*terminals, *voltage_terminals):
            for node in terminal.nodes:
                if node in owner:
                    raise ValueError(f"node {node!r} belongs to terminals {owner[node]!r} and {terminal.name!r}")
                owner[node] = terminal.name
        object.__setattr__(self, "terminals", terminals)
        object.__setattr__(self, "voltage_terminals", voltage_terminals)
        object.__setattr__(self, "vias", tuple(self.vias))
        if self.reference_node is not None:
            object.__setattr__(self, "reference_node", tuple(int(v) for v in self.reference_node))

    @property
    def voltage_driven(self) -> bool:
        return bool(self.voltage_terminals)


_STIFFNESS_1D = np.array([[1.0, -1.0], [-1.0, 1.0]])
_MASS_1D = np.array([[2.0, 1.0], [1.0, 2.0]]) / 6.0


def unit_sheet_matrices() -> tuple[np.ndarray, np.ndarray]:
    """U_x = M (x) S and U_y = S (x) M, local node order 2 dy + dx (reference pcb.py:249-256)."""

    return np.kron(_MASS_1D, _STIFFNESS_1D), np.kron(_STIFFNESS_1D, _MASS_1D)


def _flat_index(node: Node, shape: tuple[int, int, int]) -> int:
    if len(node) != 3 or any(index < 0 for index in node):
        raise ValueError(f"invalid node {node!r}")
    try:
        return int(np.ravel_multi_index(node, shape))
    except ValueError as exc:
        raise ValueError(f"node {node!r} lies outside mesh shape {shape}") from exc


def _element_views(grid: Any) -> tuple[Any, Any, Any, Any]:
    return grid[:, :-1, :-1], grid[:, :-1, 1:], grid[:, 1:, :-1], grid[:, 1:, 1:]


class MatrixFreePCBOperator:
    """Split FP64/FP32 sheet-conductance operator on the device (reference pcb.py:275-878).

    Fixed nodes are the inactive nodes, the ``reference_node`` and every
    ``dirichlet_nodes`` entry; the operator is the identity on fixed rows and
    ignores fixed columns.  ``preconditioner="two-level"`` (the default) adds
    the patch-constant coarse correction on the (layers, rows, cols) node grid.
    """

    def __init__(
        self,
        mesh: LayeredPCBMesh,
        *,
        reference_node: Node | None = None,
        dirichlet_nodes: Sequence[Node] = (),
        vias: Sequence[ViaConnection] = (),
        runtime: B200Float32Runtime | None = None,
        backend: str | None = None,
        device_id: int = 0,
        preconditioner: Preconditioner = "two-level",
        coarse_block_nodes: int | None = None,
        native: bool | None = None,
    ) -> None:
        _check_backend(runtime, backend, native)
        if preconditioner not in ("two-level", "jacobi"):
            raise ValueError("preconditioner must be 'two-level' or 'jacobi'")
        if coarse_block_nodes is not None and int(coarse_block_nodes) < 1:
            raise ValueError("coarse_block_nodes must be a positive node count")
        self.high_dtype = np.float64
        self.inner_solver = "pcg"
        self.mesh = mesh
        self.size = mesh.size
        self.runtime = runtime or B200Float32Runtime(device_id)
        self.vias = tuple(vias)
        self.preconditioner = preconditioner
        self.reference_node = None if reference_node is None else tuple(reference_node)
        if reference_node is None and not dirichlet_nodes:
            raise ValueError("pass a reference_node or dirichlet_nodes to fix the potential")
        shape = mesh.node_shape
        self._via_a = np.asarray([_flat_index(v.lower, shape) for v in self.vias], dtype=np.int64)
        self._via_b = np.asarray([_flat_index(v.upper, shape) for v in self.vias], dtype=np.int64)
        self._via_g = np.asarray([v.conductance_s for v in self.vias], dtype=np.float64)
        reference = -1 if reference_node is None else _flat_index(reference_node, shape)
        dirichlet = np.asarray([_flat_index(node, shape) for node in dirichlet_nodes], dtype=np.int64)
        self.device_system = _native.DeviceSystem.from_dc(
            layer_thickness_m=np.asarray(mesh.layer_thickness_m, dtype=np.float64),
            pitch_x_m=mesh.pitch_x_m,
            pitch_y_m=mesh.pitch_y_m,
            conductivity_s_per_m=mesh.conductivity_s_per_m,
            element_active=mesh.element_active,
            via_lower=self._via_a,
            via_upper=self._via_b,
            via_conductance_s=self._via_g,
            reference_node=reference,
            dirichlet_nodes=dirichlet,
            device=self.runtime.device_id,
        )
        active, free = self.device_system.dc_masks()
        self.active_nodes = active.reshape(shape)
        self.free_nodes = free.reshape(shape)
        self._diagonal: np.ndarray | None = None
        self.coarse_correction = None
        if preconditioner == "two-level":
            try:
                self.device_system.set_preconditioner("two-level", coarse_block_nodes)
            except Exception:
                self.device_system.close()
                raise
            self.coarse_correction = self.device_system.preconditioner()
        self.low_operator_backend = KERNEL_NAME
        self.high_operator_backend = HIGH_KERNEL_NAME

    def close(self) -> None:
        """Release the device memory of this operator."""

        self.device_system.close()

    # ---------------------------------------------------------------- actions
    def _flat(self, values: Any) -> np.ndarray:
        flat = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        if flat.size != self.size:
            raise ValueError(f"vector has size {flat.size}, expected {self.size}")
        return flat

    def apply_high(self, vector: np.ndarray) -> np.ndarray:
        """FP64 action y = where(free, K (x * free) + vias, x) (reference pcb.py:619-633)."""

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

    def apply_full_high(self, vector: np.ndarray) -> np.ndarray:
        """Unconstrained conductance action K v: the current leaving each node (reference pcb.py:702-724)."""

        return self.device_system.stiffness_f64(self._flat(vector))

    def diagonal_high(self) -> np.ndarray:
        if self._diagonal is None:
            self._diagonal = self.device_system.diagonal()
        return self._diagonal

    def diagonal_low(self) -> np.ndarray:
        return self.diagonal_high().astype(np.float32)

    def precondition_low(self, vector: Any) -> np.ndarray:
        if self.coarse_correction is None:
            return (np.asarray(vector, dtype=np.float32).reshape(-1) / self.diagonal_low()).astype(np.float32)
        return self.device_system.precondition_f32(self._flat(vector))

    def native_solve_mpir(self, rhs_high: np.ndarray, config: MPIRConfig, initial_guess: np.ndarray | None = None) -> tuple:
        """The whole MPIR solve on the device (reference hook, pcb.py:635-667)."""

        result = self.device_system.solve_mpir(self._flat(rhs_high), config, initial_guess)
        return (
            result["solution"], result["converged"], result["outer_iterations"], result["inner_iterations"],
            result["relative_residual"], result["high_operator_applications"],
            result["low_operator_applications"], result["history"],
        )

    # ------------------------------------------------------------- terminals
    def _node_index(self, node: Node) -> int:
        return _flat_index(node, self.mesh.node_shape)

    def dirichlet_potential(self, voltage_terminals: Sequence[VoltageTerminal] = ()) -> np.ndarray:
        """Potential vector holding each voltage terminal's value, zero elsewhere (reference pcb.py:726-745)."""

        potential = np.zeros(self.size, dtype=np.float64)
        free = self.free_nodes.reshape(-1)
        active = self.active_nodes.reshape(-1)
        for terminal in voltage_terminals:
            for node in terminal.nodes:
                index = self._node_index(node)
                if free[index] or not active[index]:
                    raise ValueError(
                        f"voltage terminal {terminal.name!r} node {node!r} is not a Dirichlet node of this operator"
                    )
                potential[index] = float(terminal.voltage_v)
        return potential

    def terminal_currents(self, potential_v: np.ndarray, voltage_terminals: Sequence[VoltageTerminal]) -> np.ndarray:
        """Current each voltage terminal drives into the copper, A (reference pcb.py:747-768)."""

        injected = self.apply_full_high(np.nan_to_num(np.asarray(potential_v, dtype=np.float64), nan=0.0))
        return np.asarray(
            [float(np.sum(injected[[self._node_index(node) for node in t.nodes]])) for t in voltage_terminals],
            dtype=np.float64,
        )

    def build_rhs(self, terminals: Sequence[CurrentTerminal], voltage_terminals: Sequence[VoltageTerminal] = ()) -> np.ndarray:
        """Current injections, the gauge rows, and the lifted voltage terminals (reference pcb.py:770-808)."""

        rhs = np.zeros(self.mesh.node_shape, dtype=np.float64)
        active = self.active_nodes.reshape(-1)
        for terminal in terminals:
            share = float(terminal.current_a) / len(terminal.nodes)
            for node in terminal.nodes:
                index = self._node_index(node)
                if not active[index]:
                    raise ValueError(f"terminal {terminal.name!r} contains inactive node {node!r}")
                rhs.flat[index] += share
        # the gauge equation V_ref = 0 replaces the redundant balanced row
        rhs[~self.free_nodes] = 0.0
        rhs = rhs.reshape(-1)
        if voltage_terminals:
            fixed = self.dirichlet_potential(voltage_terminals)
            lifted = self.apply_full_high(fixed)
            rhs = np.where(self.free_nodes.reshape(-1), rhs - lifted, fixed)
        return rhs

    # --------------------------------------------------------- post-process
    def element_post(self, potential_v: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """(E at each element centre, V/m, (x, y); Joule loss per element, W), both
        computed on the device in one pass (reference pcb.py:810-848)."""

        return self.device_system.dc_post(self._flat(potential_v))

    def element_electric_field(self, potential_v: np.ndarray) -> np.ndarray:
        """E at each element centre, V/m, (x, y), zero on void elements (reference pcb.py:810-822)."""

        return self.element_post(potential_v)[0]

    def via_currents(self, potential_v: np.ndarray) -> np.ndarray:
        flat = np.asarray(potential_v, dtype=np.float64).reshape(-1)
        return self._via_g * (flat[self._via_a] - flat[self._via_b])

    def element_joule_loss(self, potential_v: np.ndarray) -> np.ndarray:
        """c_x v^T U_x v + c_y v^T U_y v per element, W (reference pcb.py:830-848)."""

        return self.element_post(potential_v)[1]

    def via_joule_loss(self, potential_v: np.ndarray) -> np.ndarray:
        flat = np.asarray(potential_v, dtype=np.float64).reshape(-1)
        drop = flat[self._via_a] - flat[self._via_b]
        return self._via_g * drop * drop

    def joule_loss(self, potential_v: np.ndarray) -> float:
        return float(np.sum(self.element_joule_loss(potential_v)) + np.sum(self.via_joule_loss(potential_v)))


@dataclass(frozen=True)
class PCBConductionSolution:
    potential_v: np.ndarray
    current_density_a_per_m2: np.ndarray
    via_current_a: np.ndarray
    joule_loss_w: float
    element_joule_loss_w: np.ndarray
    via_joule_loss_w: np.ndarray
    max_current_density_a_per_m2: float
    solve: MPIRResult
    voltage_terminal_current_a: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, dtype=np.float64))


def solve_pcb_dc(
    problem: PCBConductionProblem,
    *,
    config: MPIRConfig | None = None,
    runtime: B200Float32Runtime | None = None,
    backend: str | None = None,
    device_id: int = 0,
    initial_potential_v: np.ndarray | None = None,
    preconditioner: Preconditioner = "two-level",
    coarse_block_nodes: int | None = None,
    native: bool | None = None,
) -> PCBConductionSolution:
    """Solve a layered PCB's DC conduction problem with matrix-free MPIR on the
    device (reference pcb.py:896-978).  ``initial_potential_v`` warm-starts the
    outer refinement; its NaN entries count as zero."""

    operator = MatrixFreePCBOperator(
        problem.mesh,
        reference_node=problem.reference_node,
        dirichlet_nodes=tuple(node for terminal in problem.voltage_terminals for node in terminal.nodes),
        vias=problem.vias,
        runtime=runtime,
        backend=backend,
        device_id=device_id,
        preconditioner=preconditioner,
        coarse_block_nodes=coarse_block_nodes,
        native=native,
    )
    try:
        rhs = operator.build_rhs(problem.terminals, problem.voltage_terminals)
        fixed = operator.dirichlet_potential(problem.voltage_terminals)
        initial = None
        if initial_potential_v is not None:
            initial = np.nan_to_num(np.asarray(initial_potential_v, dtype=np.float64).reshape(-1), nan=0.0)
            if initial.size != operator.size:
                raise ValueError("initial_potential_v must hold one value per node")
            initial = np.where(operator.free_nodes.reshape(-1), initial, fixed)
        elif problem.voltage_terminals:
            initial = fixed
        result = solve_mpir(operator, rhs, config=config, initial_guess=initial)
        potential = result.solution.reshape(problem.mesh.node_shape)
        reported = np.where(operator.active_nodes, potential, np.nan)
        terminal_current = operator.terminal_currents(potential, problem.voltage_terminals)
        field, element_loss = operator.element_post(potential)
        via_loss = operator.via_joule_loss(potential)
        conductivity = np.asarray(problem.mesh.conductivity_s_per_m, dtype=np.float64)
        current_density = conductivity[..., None] * field
        magnitudes = np.linalg.norm(current_density, axis=-1)
        active = magnitudes[problem.mesh.element_active]
        maximum = float(np.max(active)) if active.size else 0.0
        return PCBConductionSolution(
            potential_v=reported,
            current_density_a_per_m2=current_density,
            via_current_a=operator.via_currents(potential),
            joule_loss_w=float(np.sum(element_loss) + np.sum(via_loss)),
            element_joule_loss_w=element_loss,
            via_joule_loss_w=via_loss,
            max_current_density_a_per_m2=maximum,
            solve=result,
            voltage_terminal_current_a=terminal_current,
        )
    finally:
        operator.close()
