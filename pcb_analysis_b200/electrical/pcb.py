"""DC conduction in layered PCB copper, solved on a B200.

The call surface is that of pcb-analysis's
``electrical.matrix_free_mpir_fem.pcb`` (src/electrical/matrix_free_mpir_fem/
pcb.py:105-978): the mesh, via, terminal and problem records with their
validation messages, the operator protocol of ``MatrixFreePCBOperator`` and
``solve_pcb_dc`` with its solution fields.  Each copper layer is a sheet of
bilinear (Q1) quadrilaterals of conductance sigma t, and plated vias are
conductance links between layer nodes.  The operator, its diagonal, the whole
MPIR solve (Jacobi or the two-level preconditioner) and the element field and
loss run on the device through libthermal_b200.so (``tb_dc_system_create``,
``tb_dc_post``); the host gathers terminal and via quantities by index.
"""

from __future__ import annotations

import dataclasses
import math
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


def _as_node(node: Sequence[int]) -> Node:
    return tuple(int(i) for i in node)  # type: ignore[return-value]


# ------------------------------------------------------------------ records
@dataclass(frozen=True)
class ViaConnection:
    """One resistive vertical connection between two nodal layer locations."""

    lower: Node
    upper: Node
    resistance_ohm: float

    def __post_init__(self) -> None:
        a, b = _as_node(self.lower), _as_node(self.upper)
        if len(a) != 3 or len(b) != 3:
            raise ValueError("via endpoints must be (layer, row, column) nodes")
        if a == b:
            raise ValueError("a via must connect two different nodes")
        if a[0] == b[0]:
            raise ValueError("a via must connect different layers")
        if not (math.isfinite(self.resistance_ohm) and self.resistance_ohm > 0.0):
            raise ValueError("via resistance must be finite and positive")
        object.__setattr__(self, "lower", a)
        object.__setattr__(self, "upper", b)

    @property
    def conductance_s(self) -> float:
        return 1.0 / float(self.resistance_ohm)


class _TerminalNodes:
    """Node-set checks shared by the two terminal kinds."""

    _kind = "terminal"
    _value_field = ""
    _value_message = ""

    def _check_nodes(self) -> None:
        nodes = tuple(_as_node(node) for node in self.nodes)
        if not nodes:
            raise ValueError(f"a {self._kind} needs at least one node")
        if len(set(nodes)) < len(nodes):
            raise ValueError("terminal nodes must be unique")
        if not math.isfinite(getattr(self, self._value_field)):
            raise ValueError(self._value_message)
        object.__setattr__(self, "nodes", nodes)


@dataclass(frozen=True)
class CurrentTerminal(_TerminalNodes):
    """A total current spread equally over a set of nodes."""

    nodes: tuple[Node, ...]
    current_a: float
    name: str = "terminal"
    _kind = "current terminal"
    _value_field = "current_a"
    _value_message = "terminal current must be finite"

    def __post_init__(self) -> None:
        self._check_nodes()


@dataclass(frozen=True)
class VoltageTerminal(_TerminalNodes):
    """A set of nodes held at one potential (an ideal voltage source)."""

    nodes: tuple[Node, ...]
    voltage_v: float
    name: str = "terminal"
    _kind = "voltage terminal"
    _value_field = "voltage_v"
    _value_message = "terminal voltage must be finite"

    def __post_init__(self) -> None:
        self._check_nodes()


def _sheet_conductivity(value: Any, shape: tuple[int, int, int]) -> np.ndarray:
    """Conductivity per element from a scalar, one value per layer or a full field."""

    sigma = np.asarray(value, dtype=np.float64)
    if sigma.ndim == 0 or sigma.shape == (shape[0],):
        sigma = np.broadcast_to(sigma.reshape((-1, 1, 1)) if sigma.ndim else sigma, shape)
    elif sigma.shape != shape:
        raise ValueError("conductivity must be scalar, per-layer, or match element_active")
    if not (np.isfinite(sigma).all() and (sigma > 0.0).all()):
        raise ValueError("conductivity must be finite and positive")
    return np.array(sigma, dtype=np.float64)


@dataclass(frozen=True)
class LayeredPCBMesh:
    """Structured Q1 sheet mesh of one conductor role.

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
        active = np.array(self.element_active, dtype=bool)
        if active.ndim != 3 or min(active.shape[1:], default=0) < 1:
            raise ValueError("element_active must have shape (layers, rows, cols) with positive axes")
        thickness = np.asarray(self.layer_thickness_m, dtype=np.float64)
        if thickness.shape != active.shape[:1]:
            raise ValueError("layer_thickness_m must contain one value per layer")
        if not (np.isfinite(thickness).all() and (thickness > 0.0).all()):
            raise ValueError("layer thicknesses must be finite and positive")
        layers, rows, cols = active.shape
        object.__setattr__(self, "pitch_x_m", check_pitch_axis(self.pitch_x_m, cols, "pitch_x_m"))
        object.__setattr__(self, "pitch_y_m", check_pitch_axis(self.pitch_y_m, rows, "pitch_y_m"))
        object.__setattr__(self, "conductivity_s_per_m", _sheet_conductivity(self.conductivity_s_per_m, active.shape))
        object.__setattr__(self, "element_active", active)
        object.__setattr__(self, "layer_thickness_m", tuple(float(t) for t in thickness))

    @property
    def node_shape(self) -> tuple[int, int, int]:
        layers, rows, cols = self.element_active.shape
        return layers, rows + 1, cols + 1

    @property
    def size(self) -> int:
        return int(np.prod(self.node_shape))

    @property
    def uniform_pitch(self) -> bool:
        return bool((self.pitch_x_m == self.pitch_x_m[0]).all() and (self.pitch_y_m == self.pitch_y_m[0]).all())

    @property
    def cell_area_m2(self) -> np.ndarray:
        return np.outer(self.pitch_y_m, self.pitch_x_m)

    def element_coefficients(self) -> tuple[np.ndarray, np.ndarray]:
        """c_x = sigma t h_y / h_x and c_y = sigma t h_x / h_y, zero on void
        elements, each evaluated ((sigma t) active) h / h in that order (the
        order the device rebuilds them in)."""

        sheet = (np.asarray(self.conductivity_s_per_m, dtype=np.float64)
                 * np.asarray(self.layer_thickness_m, dtype=np.float64).reshape(-1, 1, 1)
                 * self.element_active.astype(np.float64))
        along_x = self.pitch_x_m.reshape(1, 1, -1)
        along_y = self.pitch_y_m.reshape(1, -1, 1)
        return np.ascontiguousarray(sheet * along_y / along_x), np.ascontiguousarray(sheet * along_x / along_y)


def _check_drive(terminals: tuple, voltage_terminals: tuple, reference_node) -> None:
    if voltage_terminals:
        if reference_node is not None:
            raise ValueError("voltage terminals fix the potential; reference_node must be None")
        return
    if not terminals:
        raise ValueError("a PCB conduction problem needs current or voltage terminals")
    if reference_node is None:
        raise ValueError("a current-driven problem needs a reference_node")
    currents = np.asarray([t.current_a for t in terminals], dtype=np.float64)
    net = float(currents.sum())
    if abs(net) > 1.0e-12 * max(1.0, float(np.abs(currents).sum())):
        raise ValueError(f"terminal currents must sum to zero, got {net:.6g} A")


def _check_ownership(terminals: Sequence) -> None:
    seen: dict[Node, str] = {}
    for terminal in terminals:
        for node in terminal.nodes:
            if node in seen:
                raise ValueError(f"node {node!r} belongs to terminals {seen[node]!r} and {terminal.name!r}")
            seen[node] = terminal.name


@dataclass(frozen=True)
class PCBConductionProblem:
    """One conductor role and its drive.

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
        for name in ("terminals", "voltage_terminals", "vias"):
            object.__setattr__(self, name, tuple(getattr(self, name)))
        _check_drive(self.terminals, self.voltage_terminals, self.reference_node)
        _check_ownership(self.terminals + self.voltage_terminals)
        if self.reference_node is not None:
            object.__setattr__(self, "reference_node", _as_node(self.reference_node))

    @property
    def voltage_driven(self) -> bool:
        return len(self.voltage_terminals) > 0


def unit_sheet_matrices() -> tuple[np.ndarray, np.ndarray]:
    """U_x = M (x) S and U_y = S (x) M, local node order 2 dy + dx."""

    stiffness = np.array([[1.0, -1.0], [-1.0, 1.0]])
    mass = np.array([[2.0, 1.0], [1.0, 2.0]]) / 6.0
    return np.kron(mass, stiffness), np.kron(stiffness, mass)


def _flat_index(node: Node, shape: tuple[int, int, int]) -> int:
    if len(node) != 3 or min(node) < 0:
        raise ValueError(f"invalid node {node!r}")
    if any(i >= n for i, n in zip(node, shape)):
        raise ValueError(f"node {node!r} lies outside mesh shape {shape}")
    return int(np.ravel_multi_index(node, shape))


# ------------------------------------------------------------------ operator
class MatrixFreePCBOperator:
    """Split FP64/FP32 sheet-conductance operator on the device.

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
        if reference_node is None and not len(dirichlet_nodes):
            raise ValueError("pass a reference_node or dirichlet_nodes to fix the potential")
        self.high_dtype = np.float64
        self.inner_solver = "pcg"
        self.mesh = mesh
        self.size = mesh.size
        self.runtime = runtime or B200Float32Runtime(device_id)
        self.vias = tuple(vias)
        self.preconditioner = preconditioner
        self.reference_node = None if reference_node is None else _as_node(reference_node)
        shape = mesh.node_shape
        ends = np.asarray([[_flat_index(v.lower, shape), _flat_index(v.upper, shape)] for v in self.vias],
                          dtype=np.int64).reshape(-1, 2)
        self._via_a, self._via_b = ends[:, 0].copy(), ends[:, 1].copy()
        self._via_g = np.asarray([v.conductance_s for v in self.vias], dtype=np.float64)
        self.device_system = _native.DeviceSystem.from_dc(
            layer_thickness_m=np.asarray(mesh.layer_thickness_m, dtype=np.float64),
            pitch_x_m=mesh.pitch_x_m,
            pitch_y_m=mesh.pitch_y_m,
            conductivity_s_per_m=mesh.conductivity_s_per_m,
            element_active=mesh.element_active,
            via_lower=self._via_a,
            via_upper=self._via_b,
            via_conductance_s=self._via_g,
            reference_node=-1 if reference_node is None else _flat_index(self.reference_node, shape),
            dirichlet_nodes=np.asarray([_flat_index(_as_node(n), shape) for n in dirichlet_nodes], dtype=np.int64),
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

    def __enter__(self) -> "MatrixFreePCBOperator":
        return self

    def __exit__(self, *exc: object) -> None:
        self.close()

    # ---------------------------------------------------------------- actions
    def _flat(self, values: Any) -> np.ndarray:
        flat = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        if flat.size != self.size:
            raise ValueError(f"vector has size {flat.size}, expected {self.size}")
        return flat

    def apply_high(self, vector: np.ndarray) -> np.ndarray:
        """FP64 action y = where(free, K (x * free) + vias, x)."""

        return self.device_system.apply_f64(self._flat(vector))

    def apply_low(self, vector: Any) -> Any:
        """FP32 action on the device; a torch CUDA tensor stays on the device."""

        if getattr(vector, "is_cuda", False):
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
        """Unconstrained conductance action K v: the current leaving each node."""

        return self.device_system.stiffness_f64(self._flat(vector))

    def diagonal_high(self) -> np.ndarray:
        if self._diagonal is None:
            self._diagonal = self.device_system.diagonal()
        return self._diagonal

    def diagonal_low(self) -> np.ndarray:
        return self.diagonal_high().astype(np.float32)

    def precondition_low(self, vector: Any) -> np.ndarray:
        if self.coarse_correction is not None:
            return self.device_system.precondition_f32(self._flat(vector))
        return (np.asarray(vector, dtype=np.float32).reshape(-1) / self.diagonal_low()).astype(np.float32)

    def native_solve_mpir(self, rhs_high: np.ndarray, config: MPIRConfig, initial_guess: np.ndarray | None = None) -> tuple:
        """The whole MPIR solve on the device (the reference solver's native hook)."""

        out = self.device_system.solve_mpir(self._flat(rhs_high), config, initial_guess)
        keys = ("solution", "converged", "outer_iterations", "inner_iterations", "relative_residual",
                "high_operator_applications", "low_operator_applications", "history")
        return tuple(out[k] for k in keys)

    # ------------------------------------------------------------- terminals
    def _node_index(self, node: Node) -> int:
        return _flat_index(_as_node(node), self.mesh.node_shape)

    def _terminal_indices(self, terminal) -> np.ndarray:
        return np.asarray([self._node_index(node) for node in terminal.nodes], dtype=np.int64)

    def dirichlet_potential(self, voltage_terminals: Sequence[VoltageTerminal] = ()) -> np.ndarray:
        """Potential vector holding each voltage terminal's value, zero elsewhere."""

        potential = np.zeros(self.size, dtype=np.float64)
        held = ~self.free_nodes.reshape(-1) & self.active_nodes.reshape(-1)
        for terminal in voltage_terminals:
            where = self._terminal_indices(terminal)
            stray = np.flatnonzero(~held[where])
            if stray.size:
                node = terminal.nodes[int(stray[0])]
                raise ValueError(
                    f"voltage terminal {terminal.name!r} node {node!r} is not a Dirichlet node of this operator")
            potential[where] = float(terminal.voltage_v)
        return potential

    def terminal_currents(self, potential_v: np.ndarray, voltage_terminals: Sequence[VoltageTerminal]) -> np.ndarray:
        """Current each voltage terminal drives into the copper, A."""

        leaving = self.apply_full_high(np.nan_to_num(np.asarray(potential_v, dtype=np.float64), nan=0.0))
        return np.asarray([float(np.sum(leaving[self._terminal_indices(t)])) for t in voltage_terminals],
                          dtype=np.float64)

    def build_rhs(self, terminals: Sequence[CurrentTerminal],
                  voltage_terminals: Sequence[VoltageTerminal] = ()) -> np.ndarray:
        """Current injections, zero on the fixed (gauge) rows, and the lifted voltage terminals."""

        injected = np.zeros(self.size, dtype=np.float64)
        active = self.active_nodes.reshape(-1)
        for terminal in terminals:
            where = self._terminal_indices(terminal)
            dead = np.flatnonzero(~active[where])
            if dead.size:
                raise ValueError(f"terminal {terminal.name!r} contains inactive node {terminal.nodes[int(dead[0])]!r}")
            injected[where] += float(terminal.current_a) / len(terminal.nodes)
        free = self.free_nodes.reshape(-1)
        injected[~free] = 0.0  # the gauge equation V_ref = 0 takes the redundant balanced row
        if not voltage_terminals:
            return injected
        held = self.dirichlet_potential(voltage_terminals)
        return np.where(free, injected - self.apply_full_high(held), held)

    # --------------------------------------------------------- post-process
    def element_post(self, potential_v: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """(E at each element centre, V/m, (x, y); Joule loss per element, W),
        both computed on the device in one pass."""

        return self.device_system.dc_post(self._flat(potential_v))

    def element_electric_field(self, potential_v: np.ndarray) -> np.ndarray:
        """E at each element centre, V/m, (x, y), zero on void elements."""

        return self.element_post(potential_v)[0]

    def _via_drop(self, potential_v: np.ndarray) -> np.ndarray:
        flat = np.asarray(potential_v, dtype=np.float64).reshape(-1)
        return flat[self._via_a] - flat[self._via_b]

    def via_currents(self, potential_v: np.ndarray) -> np.ndarray:
        return self._via_g * self._via_drop(potential_v)

    def element_joule_loss(self, potential_v: np.ndarray) -> np.ndarray:
        """c_x v^T U_x v + c_y v^T U_y v per element, W."""

        return self.element_post(potential_v)[1]

    def via_joule_loss(self, potential_v: np.ndarray) -> np.ndarray:
        drop = self._via_drop(potential_v)
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


def _warm_start(operator: MatrixFreePCBOperator, guess: Any, held: np.ndarray, voltage_driven: bool):
    """Initial potential of the refinement: the guess (NaN as 0) on free
    nodes and the terminal values on held ones; the terminal values alone
    without a guess under voltage drive."""

    if guess is None:
        return held if voltage_driven else None
    flat = np.nan_to_num(np.asarray(guess, dtype=np.float64).reshape(-1), nan=0.0)
    if flat.size != operator.size:
        raise ValueError("initial_potential_v must hold one value per node")
    return np.where(operator.free_nodes.reshape(-1), flat, held)


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
    """Solve a layered PCB's DC conduction problem with matrix-free MPIR on
    the device.  ``initial_potential_v`` warm-starts the outer refinement;
    its NaN entries count as zero."""

    held_nodes = tuple(node for terminal in problem.voltage_terminals for node in terminal.nodes)
    with MatrixFreePCBOperator(
        problem.mesh, reference_node=problem.reference_node, dirichlet_nodes=held_nodes, vias=problem.vias,
        runtime=runtime, backend=backend, device_id=device_id, preconditioner=preconditioner,
        coarse_block_nodes=coarse_block_nodes, native=native,
    ) as operator:
        rhs = operator.build_rhs(problem.terminals, problem.voltage_terminals)
        held = operator.dirichlet_potential(problem.voltage_terminals)
        start = _warm_start(operator, initial_potential_v, held, problem.voltage_driven)
        record = solve_mpir(operator, rhs, config=config, initial_guess=start)
        potential = record.solution.reshape(problem.mesh.node_shape)
        field, element_loss = operator.element_post(potential)
        via_loss = operator.via_joule_loss(potential)
        density = np.asarray(problem.mesh.conductivity_s_per_m, dtype=np.float64)[..., None] * field
        live = np.linalg.norm(density, axis=-1)[problem.mesh.element_active]
        return PCBConductionSolution(
            potential_v=np.where(operator.active_nodes, potential, np.nan),
            current_density_a_per_m2=density,
            via_current_a=operator.via_currents(potential),
            joule_loss_w=float(np.sum(element_loss) + np.sum(via_loss)),
            element_joule_loss_w=element_loss,
            via_joule_loss_w=via_loss,
            max_current_density_a_per_m2=float(live.max()) if live.size else 0.0,
            solve=record,
            voltage_terminal_current_a=operator.terminal_currents(potential, problem.voltage_terminals),
        )
