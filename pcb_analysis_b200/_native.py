"""ctypes binding of libthermal_b200.so (C ABI in include/thermal_b200.h).

The library is the only implementation of the operator and the solve: if it
is not built, or no CUDA device answers, every call raises instead of falling
back to a CPU path.
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path
from typing import Any, Sequence

import numpy as np

LIBRARY_PATH = Path(__file__).resolve().parent / "libthermal_b200.so"

TB_OK = 0
TB_EINVAL = 1
TB_ENOTSPD = 2
TB_ECUDA = 3
TB_ETIMEOUT = 4
TB_ENOMEM = 5
TB_ENONFINITE = 6
TB_ENOTSUP = 7

_EXCEPTIONS: dict[int, type[Exception]] = {
    TB_EINVAL: ValueError,
    TB_ENOTSPD: RuntimeError,
    TB_ECUDA: RuntimeError,
    TB_ETIMEOUT: TimeoutError,
    TB_ENOMEM: MemoryError,
    TB_ENONFINITE: FloatingPointError,
    TB_ENOTSUP: NotImplementedError,
}

_c_double_p = ctypes.POINTER(ctypes.c_double)
_c_float_p = ctypes.POINTER(ctypes.c_float)
_c_uint8_p = ctypes.POINTER(ctypes.c_uint8)


class SystemDesc(ctypes.Structure):
    _fields_ = [
        ("slabs", ctypes.c_int32),
        ("rows", ctypes.c_int32),
        ("cols", ctypes.c_int32),
        ("slab_thickness_m", _c_double_p),
        ("pitch_x_m", _c_double_p),
        ("pitch_y_m", _c_double_p),
        ("k_in", _c_double_p),
        ("k_z", _c_double_p),
        ("robin_total", _c_double_p),
        ("free_nodes", _c_uint8_p),
    ]


class MPIRConfigC(ctypes.Structure):
    _fields_ = [
        ("relative_tolerance", ctypes.c_double),
        ("absolute_tolerance", ctypes.c_double),
        ("inner_relative_tolerance", ctypes.c_double),
        ("max_outer_iterations", ctypes.c_int32),
        ("max_inner_iterations", ctypes.c_int32),
    ]


class MPIRResultC(ctypes.Structure):
    _fields_ = [
        ("converged", ctypes.c_int32),
        ("outer_iterations", ctypes.c_int32),
        ("inner_iterations", ctypes.c_int32),
        ("high_operator_applications", ctypes.c_int32),
        ("low_operator_applications", ctypes.c_int32),
        ("history_length", ctypes.c_int32),
        ("relative_residual", ctypes.c_double),
    ]


class MPIRStepC(ctypes.Structure):
    _fields_ = [
        ("outer_iteration", ctypes.c_int32),
        ("inner_iterations", ctypes.c_int32),
        ("high_relative_residual", ctypes.c_double),
        ("inner_relative_residual", ctypes.c_double),
    ]


class PCGResultC(ctypes.Structure):
    _fields_ = [
        ("converged", ctypes.c_int32),
        ("iterations", ctypes.c_int32),
        ("relative_residual", ctypes.c_double),
    ]


class EngineConfigC(ctypes.Structure):
    _fields_ = [
        ("capacity", ctypes.c_int32),
        ("max_slabs", ctypes.c_int32),
        ("tile_rows", ctypes.c_int32),
        ("preconditioner", ctypes.c_int32),
        ("budget_bytes", ctypes.c_int64),
        ("staging", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class ConvectionDescC(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("side", ctypes.c_int32),
        ("direction_count", ctypes.c_int32),
        ("directions", ctypes.c_int32 * 6),
        ("coefficient_w_per_m2_k", ctypes.c_double),
        ("ambient_temperature_k", ctypes.c_double),
        ("coefficient_field", _c_double_p),
        ("ambient_field", _c_double_p),
    ]


class ProblemDescC(ctypes.Structure):
    _fields_ = [
        ("slabs", ctypes.c_int32),
        ("rows", ctypes.c_int32),
        ("cols", ctypes.c_int32),
        ("slab_thickness_m", _c_double_p),
        ("pitch_x_m", _c_double_p),
        ("pitch_y_m", _c_double_p),
        ("k_in", _c_double_p),
        ("k_z", _c_double_p),
        ("active", _c_uint8_p),
        ("fixed_mask", _c_uint8_p),
        ("fixed_temperature_k", _c_double_p),
        ("nodal_heat_w", _c_double_p),
        ("element_heat_w", _c_double_p),
        ("source_entries", ctypes.c_int32),
        ("source_nodes", ctypes.POINTER(ctypes.c_int64)),
        ("source_node_w", _c_double_p),
        ("convection_count", ctypes.c_int32),
        ("convection", ctypes.POINTER(ConvectionDescC)),
        ("capacity_per_s", _c_double_p),
    ]


class DcDescC(ctypes.Structure):
    _fields_ = [
        ("layers", ctypes.c_int32),
        ("rows", ctypes.c_int32),
        ("cols", ctypes.c_int32),
        ("layer_thickness_m", _c_double_p),
        ("pitch_x_m", _c_double_p),
        ("pitch_y_m", _c_double_p),
        ("conductivity_s_per_m", _c_double_p),
        ("element_active", _c_uint8_p),
        ("via_count", ctypes.c_int32),
        ("via_lower", ctypes.POINTER(ctypes.c_int64)),
        ("via_upper", ctypes.POINTER(ctypes.c_int64)),
        ("via_conductance_s", _c_double_p),
        ("reference_node", ctypes.c_int64),
        ("dirichlet_count", ctypes.c_int32),
        ("dirichlet_nodes", ctypes.POINTER(ctypes.c_int64)),
    ]


TB_CONVECTION_FACE = 0
TB_CONVECTION_EXPOSED = 1
DIRECTION_CODES = {"-x": 0, "+x": 1, "-y": 2, "+y": 3, "-z": 4, "+z": 5}

_VP = ctypes.c_void_p
_I32 = ctypes.c_int32
_SIGNATURES: dict[str, tuple[Any, list[Any]]] = {
    "tb_version": (ctypes.c_char_p, []),
    "tb_last_error": (ctypes.c_char_p, []),
    "tb_device_count": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int32)]),
    "tb_system_create": (ctypes.c_int, [ctypes.POINTER(SystemDesc), _I32, ctypes.POINTER(_VP)]),
    "tb_system_destroy": (ctypes.c_int, [_VP]),
    "tb_system_info": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
    "tb_apply_f32": (ctypes.c_int, [_VP, _VP, _VP]),
    "tb_apply_f64": (ctypes.c_int, [_VP, _VP, _VP]),
    "tb_apply_f32_device": (ctypes.c_int, [_VP, _VP, _VP]),
    "tb_apply_f64_device": (ctypes.c_int, [_VP, _VP, _VP]),
    "tb_residual_f64_device_static": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "tb_set_robin": (ctypes.c_int, [_VP, _VP]),
    "tb_set_preconditioner": (ctypes.c_int, [_VP, _I32, _I32]),
    "tb_get_preconditioner": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int32)]),
    "tb_get_coarse": (ctypes.c_int, [_VP, _VP, _VP]),
    "tb_precondition_f32": (ctypes.c_int, [_VP, _VP, _VP]),
    "tb_get_multilevel": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int32), _I32, ctypes.POINTER(ctypes.c_int32)]),
    "tb_get_multilevel_stencil": (ctypes.c_int, [_VP, _I32, _VP]),
    "tb_engine_create": (ctypes.c_int, [_I32, ctypes.POINTER(EngineConfigC), ctypes.POINTER(_VP)]),
    "tb_engine_destroy": (ctypes.c_int, [_VP]),
    "tb_engine_footprint": (
        ctypes.c_int,
        [ctypes.POINTER(SystemDesc), _I32, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)],
    ),
    "tb_engine_submit": (
        ctypes.c_int, [_VP, ctypes.POINTER(SystemDesc), _VP, _VP, ctypes.POINTER(MPIRConfigC), ctypes.POINTER(ctypes.c_int64)]
    ),
    "tb_engine_step": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int32)]),
    "tb_engine_finished": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64), _I32, ctypes.POINTER(ctypes.c_int32)]),
    "tb_engine_collect": (
        ctypes.c_int, [_VP, ctypes.c_int64, _VP, ctypes.POINTER(MPIRResultC), ctypes.POINTER(MPIRStepC), _I32]
    ),
    "tb_engine_info": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64)]),
    "tb_engine_staging": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int32)]),
    "tb_engine_stream": (ctypes.c_int, [_VP, ctypes.POINTER(_VP)]),
    "tb_engine_time_apply": (ctypes.c_int, [_VP, _I32, ctypes.POINTER(ctypes.c_double)]),
    "tb_stiffness_f64": (ctypes.c_int, [_VP, _VP, _VP]),
    "tb_diagonal": (ctypes.c_int, [_VP, _VP]),
    "tb_solve_mpir": (
        ctypes.c_int,
        [_VP, _VP, _VP, ctypes.POINTER(MPIRConfigC), ctypes.POINTER(MPIRResultC), ctypes.POINTER(MPIRStepC), _I32],
    ),
    "tb_solve_mpir_device": (
        ctypes.c_int,
        [_VP, _VP, _VP, ctypes.POINTER(MPIRConfigC), ctypes.POINTER(MPIRResultC), ctypes.POINTER(MPIRStepC), _I32],
    ),
    "tb_solve_pcg_f64": (
        ctypes.c_int,
        [_VP, _VP, _VP, ctypes.c_double, ctypes.c_double, _I32, ctypes.POINTER(PCGResultC)],
    ),
    "tb_solve_pcg_f64_device": (
        ctypes.c_int,
        [_VP, _VP, _VP, ctypes.c_double, ctypes.c_double, _I32, ctypes.POINTER(PCGResultC)],
    ),
    "tb_solve_pcg_f64_ml": (
        ctypes.c_int,
        [_VP, _VP, _VP, ctypes.c_double, ctypes.c_double, _I32, ctypes.POINTER(PCGResultC)],
    ),
    "tb_solve_pcg_f64_ml_device": (
        ctypes.c_int,
        [_VP, _VP, _VP, ctypes.c_double, ctypes.c_double, _I32, ctypes.POINTER(PCGResultC)],
    ),
    "tb_set_timing": (ctypes.c_int, [_VP, _I32]),
    "tb_set_stage_test": (ctypes.c_int, [_VP, _I32]),
    "tb_set_ml_staging": (ctypes.c_int, [_VP, _I32]),
    "tb_get_ml_staging": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int32)]),
    "tb_get_timing": (ctypes.c_int, [_VP, _c_double_p, ctypes.POINTER(ctypes.c_int64)]),
    "tb_get_kernel_clock": (ctypes.c_int, [_VP, _c_double_p, ctypes.POINTER(ctypes.c_int64)]),
    "tb_get_kernel_clocks": (ctypes.c_int, [_VP, _I32, _c_double_p, ctypes.POINTER(ctypes.c_int64)]),
    "tb_set_apply_plan": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int32)]),
    "tb_get_apply_plan": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int32)]),
    "tb_set_tile_rows": (ctypes.c_int, [_VP, _I32]),
    "tb_get_tile_rows": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int32)]),
    "tb_system_stream": (ctypes.c_int, [_VP, ctypes.POINTER(_VP)]),
    "tb_get_launch_count": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64)]),
    "tb_system_create_problem": (ctypes.c_int, [ctypes.POINTER(ProblemDescC), _I32, ctypes.POINTER(_VP)]),
    "tb_dc_system_create": (ctypes.c_int, [ctypes.POINTER(DcDescC), _I32, ctypes.POINTER(_VP)]),
    "tb_dc_get_masks": (ctypes.c_int, [_VP, _VP, _VP]),
    "tb_dc_post": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "tb_set_convection": (ctypes.c_int, [_VP, ctypes.POINTER(ConvectionDescC), _I32]),
    "tb_set_capacity": (ctypes.c_int, [_VP, _VP]),
    "tb_get_prepared": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "tb_get_boundary_weights": (ctypes.c_int, [_VP, _I32, _VP, _VP]),
    "tb_build_rhs": (ctypes.c_int, [_VP, ctypes.c_double, _VP, _VP]),
    "tb_postprocess": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "tb_build_rhs_device": (ctypes.c_int, [_VP, ctypes.c_double, _VP, _VP]),
    "tb_postprocess_rise_device": (ctypes.c_int, [_VP, _VP, ctypes.c_double, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "tb_download": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_size_t]),
}

PRECONDITIONER_KINDS = {"jacobi": 0, "two-level": 1, "multilevel": 2}  # tb_set_preconditioner kinds

_lock = threading.Lock()
_lib: ctypes.CDLL | None = None


def library_path() -> Path:
    return LIBRARY_PATH


def load() -> ctypes.CDLL:
    """Load the library (once) and declare the signatures of its entry points."""

    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIBRARY_PATH.exists():
            raise ImportError(
                f"{LIBRARY_PATH.name} is not built; run `python -m pcb_analysis_b200.build` "
                "(nvcc with sm_100a) before using the B200 thermal solver"
            )
        lib = ctypes.CDLL(str(LIBRARY_PATH))
        for name, (restype, argtypes) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
        return lib


def exported_names() -> list[str]:
    return list(_SIGNATURES)


def check(status: int) -> None:
    if status == TB_OK:
        return
    message = load().tb_last_error().decode(errors="replace")
    raise _EXCEPTIONS.get(status, RuntimeError)(message or f"libthermal_b200 status {status}")


def device_count() -> int:
    n = ctypes.c_int32(0)
    check(load().tb_device_count(ctypes.byref(n)))
    return int(n.value)


def require_device(device: int = 0) -> None:
    count = device_count()
    if count < 1:
        raise RuntimeError("no CUDA device is visible; the B200 thermal solver has no CPU fallback")
    if device < 0 or device >= count:
        raise ValueError(f"CUDA device_id {device} is outside the visible range [0, {count - 1}]")


def _ptr(array: np.ndarray) -> int:
    return array.ctypes.data


def _tensor_ptr(tensor: Any, dtype: Any, size: int, name: str) -> int:
    if not tensor.is_cuda or not tensor.is_contiguous() or tensor.dtype != dtype or tensor.numel() != size:
        raise ValueError(f"{name} must be a contiguous CUDA tensor of {size} {dtype} values")
    return int(tensor.data_ptr())


def system_desc(
    *,
    slab_thickness_m: np.ndarray,
    pitch_x_m: np.ndarray,
    pitch_y_m: np.ndarray,
    k_in: np.ndarray,
    k_z: np.ndarray,
    robin_total: np.ndarray,
    free_nodes: np.ndarray,
) -> tuple[SystemDesc, tuple[np.ndarray, ...], tuple[int, int, int]]:
    """The C description of one board, the arrays it points into (keep them
    alive while the description is used) and the element shape."""

    thickness = np.ascontiguousarray(slab_thickness_m, dtype=np.float64)
    px = np.ascontiguousarray(pitch_x_m, dtype=np.float64)
    py = np.ascontiguousarray(pitch_y_m, dtype=np.float64)
    shape = (thickness.size, py.size, px.size)
    kin = np.ascontiguousarray(k_in, dtype=np.float64).reshape(-1)
    kz = np.ascontiguousarray(k_z, dtype=np.float64).reshape(-1)
    nodes = (shape[0] + 1) * (shape[1] + 1) * (shape[2] + 1)
    robin = np.ascontiguousarray(robin_total, dtype=np.float64).reshape(-1)
    free = np.ascontiguousarray(free_nodes, dtype=np.uint8).reshape(-1)
    if kin.size != np.prod(shape) or kz.size != np.prod(shape):
        raise ValueError("conductivity arrays must hold one value per element")
    if robin.size != nodes or free.size != nodes:
        raise ValueError("robin_total and free_nodes must hold one value per node")
    keep = (thickness, px, py, kin, kz, robin, free)
    desc = SystemDesc(
        shape[0],
        shape[1],
        shape[2],
        thickness.ctypes.data_as(_c_double_p),
        px.ctypes.data_as(_c_double_p),
        py.ctypes.data_as(_c_double_p),
        kin.ctypes.data_as(_c_double_p),
        kz.ctypes.data_as(_c_double_p),
        robin.ctypes.data_as(_c_double_p),
        free.ctypes.data_as(_c_uint8_p),
    )
    return desc, keep, shape


def convection_descs(convection: Sequence[dict[str, Any]], shape: tuple[int, int, int]) -> tuple[Any, list[Any]]:
    """C descriptions of convection boundaries and the arrays they point into."""

    count = len(convection)
    array = (ConvectionDescC * max(count, 1))()
    keep: list[Any] = [array]
    for i, spec in enumerate(convection):
        d = array[i]
        kind = spec["kind"]
        if kind == "face":
            d.kind = TB_CONVECTION_FACE
            side = spec["side"]
            if side not in ("bottom", "top"):
                raise ValueError("side must be 'bottom' or 'top'")
            d.side = 1 if side == "top" else 0
            field_shape: tuple[int, ...] = shape[1:]
        elif kind == "exposed":
            d.kind = TB_CONVECTION_EXPOSED
            directions = tuple(spec["directions"])
            if not 1 <= len(directions) <= 6 or any(k not in DIRECTION_CODES for k in directions):
                raise ValueError(f"directions must be drawn from {tuple(DIRECTION_CODES)}")
            d.direction_count = len(directions)
            for k, name in enumerate(directions):
                d.directions[k] = DIRECTION_CODES[name]
            field_shape = shape
        else:
            raise ValueError("convection kind must be 'face' or 'exposed'")
        for value, scalar, field in (
            (spec["coefficient"], "coefficient_w_per_m2_k", "coefficient_field"),
            (spec["ambient"], "ambient_temperature_k", "ambient_field"),
        ):
            a = np.asarray(value, dtype=np.float64)
            if a.ndim == 0:
                setattr(d, scalar, float(a))
                setattr(d, field, None)
                continue
            if a.shape != field_shape:
                raise ValueError(f"{field} must have shape {field_shape}")
            flat = np.ascontiguousarray(a).reshape(-1)
            keep.append(flat)
            setattr(d, field, flat.ctypes.data_as(_c_double_p))
    return array, keep


def mpir_config_c(config: Any) -> MPIRConfigC:
    return MPIRConfigC(
        float(config.relative_tolerance),
        float(config.absolute_tolerance),
        float(config.inner_relative_tolerance),
        int(config.max_outer_iterations),
        int(config.max_inner_iterations),
    )


class DeviceSystem:
    """One prepared board resident on a CUDA device (tb_system)."""

    def __init__(
        self,
        *,
        slab_thickness_m: np.ndarray,
        pitch_x_m: np.ndarray,
        pitch_y_m: np.ndarray,
        k_in: np.ndarray,
        k_z: np.ndarray,
        robin_total: np.ndarray,
        free_nodes: np.ndarray,
        device: int = 0,
    ) -> None:
        lib = load()
        require_device(device)
        desc, self._keep, shape = system_desc(
            slab_thickness_m=slab_thickness_m, pitch_x_m=pitch_x_m, pitch_y_m=pitch_y_m, k_in=k_in, k_z=k_z,
            robin_total=robin_total, free_nodes=free_nodes,
        )
        handle = ctypes.c_void_p()
        check(lib.tb_system_create(ctypes.byref(desc), int(device), ctypes.byref(handle)))
        self._adopt(lib, handle, shape, device)
        self._keep = None

    def _adopt(self, lib: ctypes.CDLL, handle: ctypes.c_void_p, shape: tuple[int, int, int], device: int) -> None:
        self._handle = handle
        self._lib = lib
        self.device = int(device)
        self.element_shape = shape
        self.node_shape = (shape[0] + 1, shape[1] + 1, shape[2] + 1)
        self.size = self.node_shape[0] * self.node_shape[1] * self.node_shape[2]
        self.convection_count = 0

    @classmethod
    def from_problem(
        cls,
        *,
        slab_thickness_m: np.ndarray,
        pitch_x_m: np.ndarray,
        pitch_y_m: np.ndarray,
        k_in: np.ndarray,
        k_z: np.ndarray,
        active: np.ndarray | None = None,
        fixed_mask: np.ndarray | None = None,
        fixed_temperature_k: np.ndarray | None = None,
        nodal_heat_w: np.ndarray | None = None,
        element_heat_w: np.ndarray | None = None,
        sources: Sequence[tuple[np.ndarray, float]] = (),
        convection: Sequence[dict[str, Any]] = (),
        capacity_per_s: np.ndarray | None = None,
        device: int = 0,
    ) -> "DeviceSystem":
        """A board given as its conduction problem, prepared on the device
        (tb_system_create_problem).  ``sources`` lists (flat node indices,
        power per node) per heat source in order; ``convection`` lists dicts
        ``kind`` ("face" or "exposed"), ``side`` ("bottom" / "top", face
        kind), ``directions`` (exposed kind), ``coefficient`` and ``ambient``
        (scalars or fields)."""

        lib = load()
        require_device(device)
        thickness = np.ascontiguousarray(slab_thickness_m, dtype=np.float64)
        px = np.ascontiguousarray(pitch_x_m, dtype=np.float64)
        py = np.ascontiguousarray(pitch_y_m, dtype=np.float64)
        shape = (thickness.size, py.size, px.size)
        elements = shape[0] * shape[1] * shape[2]
        nodes = (shape[0] + 1) * (shape[1] + 1) * (shape[2] + 1)
        keep: list[Any] = [thickness, px, py]

        def f64(array: Any, count: int, name: str) -> Any:
            if array is None:
                return None
            flat = np.ascontiguousarray(array, dtype=np.float64).reshape(-1)
            if flat.size != count:
                raise ValueError(f"{name} must hold {count} values")
            keep.append(flat)
            return flat.ctypes.data_as(_c_double_p)

        def u8(array: Any, count: int, name: str) -> Any:
            if array is None:
                return None
            flat = np.ascontiguousarray(array).reshape(-1)
            flat = flat.view(np.uint8) if flat.dtype == np.bool_ else np.ascontiguousarray(flat, dtype=np.uint8)
            if flat.size != count:
                raise ValueError(f"{name} must hold {count} values")
            keep.append(flat)
            return flat.ctypes.data_as(_c_uint8_p)

        if sources:
            src_nodes = np.ascontiguousarray(np.concatenate([np.asarray(n, dtype=np.int64).reshape(-1) for n, _ in sources]))
            src_w = np.ascontiguousarray(np.concatenate(
                [np.full(np.asarray(n).size, float(w), dtype=np.float64) for n, w in sources]))
        else:
            src_nodes = np.zeros(1, dtype=np.int64)
            src_w = np.zeros(1, dtype=np.float64)
        keep += [src_nodes, src_w]
        conv, conv_keep = convection_descs(convection, shape)
        keep.append(conv_keep)
        desc = ProblemDescC(
            shape[0], shape[1], shape[2],
            thickness.ctypes.data_as(_c_double_p), px.ctypes.data_as(_c_double_p), py.ctypes.data_as(_c_double_p),
            f64(k_in, elements, "k_in"), f64(k_z, elements, "k_z"),
            u8(active, elements, "active"), u8(fixed_mask, nodes, "fixed_mask"),
            f64(fixed_temperature_k, nodes, "fixed_temperature_k"), f64(nodal_heat_w, nodes, "nodal_heat_w"),
            f64(element_heat_w, elements, "element_heat_w"),
            int(src_nodes.size if sources else 0), src_nodes.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            src_w.ctypes.data_as(_c_double_p),
            len(convection), conv,
            f64(capacity_per_s, nodes, "capacity_per_s"),
        )
        handle = ctypes.c_void_p()
        check(lib.tb_system_create_problem(ctypes.byref(desc), int(device), ctypes.byref(handle)))
        self = cls.__new__(cls)
        self._adopt(lib, handle, shape, device)
        self.convection_count = len(convection)
        self._keep = None
        return self

    # ------------------------------------------------------------ lifetime
    def close(self) -> None:
        handle = getattr(self, "_handle", None)
        if handle is not None and handle.value:
            self._lib.tb_system_destroy(handle)
            self._handle = None

    def __del__(self) -> None:  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self) -> "DeviceSystem":
        return self

    def __exit__(self, *exc: object) -> None:
        self.close()

    @property
    def handle(self) -> ctypes.c_void_p:
        if self._handle is None:
            raise RuntimeError("the device system was closed")
        return self._handle

    def info(self) -> tuple[int, int]:
        nodes = ctypes.c_int64()
        nbytes = ctypes.c_int64()
        check(self._lib.tb_system_info(self.handle, ctypes.byref(nodes), ctypes.byref(nbytes)))
        return int(nodes.value), int(nbytes.value)

    # --------------------------------------------------------------- timing
    def set_stage_test(self, polls: int) -> None:
        """Test only: make the tensor-copy stage waits run out (tb_set_stage_test)."""

        check(self._lib.tb_set_stage_test(self.handle, int(polls)))

    @property
    def ml_staging(self) -> bool:
        """Whether the inner PCG's multilevel fine pass runs as the staged (tensor-copy fed) kernel."""

        out = ctypes.c_int32()
        check(self._lib.tb_get_ml_staging(self.handle, ctypes.byref(out)))
        return bool(out.value)

    @ml_staging.setter
    def ml_staging(self, staged: bool) -> None:
        check(self._lib.tb_set_ml_staging(self.handle, 1 if staged else 0))

    def set_timing(self, enabled: bool) -> None:
        check(self._lib.tb_set_timing(self.handle, 1 if enabled else 0))

    def timing(self) -> dict[str, tuple[float, int]]:
        ms = (ctypes.c_double * 4)()
        n = (ctypes.c_int64 * 4)()
        check(self._lib.tb_get_timing(self.handle, ms, n))
        keys = ("apply_f32", "apply_f64", "vector", "call")
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(keys)}

    def kernel_clock(self) -> dict[str, tuple[float, int]]:
        """Running device-time totals (ms, launches) of the FP32 and FP64 operator kernels and of the
        multilevel fine pass."""

        ns = (ctypes.c_double * 3)()
        n = (ctypes.c_int64 * 3)()
        check(self._lib.tb_get_kernel_clocks(self.handle, 3, ns, n))
        keys = ("apply_f32", "apply_f64", "ml_update")
        return {k: (ns[i] * 1e-6, int(n[i])) for i, k in enumerate(keys)}

    @property
    def tile_rows(self) -> int:
        out = ctypes.c_int32()
        check(self._lib.tb_get_tile_rows(self.handle, ctypes.byref(out)))
        return int(out.value)

    @tile_rows.setter
    def tile_rows(self, rows: int) -> None:
        check(self._lib.tb_set_tile_rows(self.handle, int(rows)))

    @property
    def apply_plan(self) -> tuple[int, int, int, int, int]:
        """(kind, rows, zw, sl, band): kind 0 z-march tiles, 1 warp march, 2 one balanced wave of z-march tiles."""

        out = (ctypes.c_int32 * 5)()
        check(self._lib.tb_get_apply_plan(self.handle, out))
        return tuple(int(v) for v in out)

    @apply_plan.setter
    def apply_plan(self, plan) -> None:
        arr = (ctypes.c_int32 * 5)(*[int(v) for v in plan])
        check(self._lib.tb_set_apply_plan(self.handle, arr))

    def stream_handle(self) -> int:
        out = ctypes.c_void_p()
        check(self._lib.tb_system_stream(self.handle, ctypes.byref(out)))
        return int(out.value or 0)

    def launch_count(self) -> int:
        out = ctypes.c_int64()
        check(self._lib.tb_get_launch_count(self.handle, ctypes.byref(out)))
        return int(out.value)

    # -------------------------------------------------------------- actions
    def _vector(self, vector: Any, dtype: Any, name: str = "vector") -> np.ndarray:
        flat = np.ascontiguousarray(vector, dtype=dtype).reshape(-1)
        if flat.size != self.size:
            raise ValueError(f"{name} has size {flat.size}, expected {self.size}")
        return flat

    def apply_f32(self, vector: Any) -> np.ndarray:
        x = self._vector(vector, np.float32)
        y = np.empty_like(x)
        check(self._lib.tb_apply_f32(self.handle, _ptr(x), _ptr(y)))
        return y

    def apply_f64(self, vector: Any) -> np.ndarray:
        x = self._vector(vector, np.float64)
        y = np.empty_like(x)
        check(self._lib.tb_apply_f64(self.handle, _ptr(x), _ptr(y)))
        return y

    def apply_f32_device(self, x: Any, y: Any) -> None:
        import torch

        torch.cuda.synchronize(self.device)
        check(
            self._lib.tb_apply_f32_device(
                self.handle, _tensor_ptr(x, torch.float32, self.size, "x"), _tensor_ptr(y, torch.float32, self.size, "y")
            )
        )

    def apply_f64_device(self, x: Any, y: Any) -> None:
        import torch

        torch.cuda.synchronize(self.device)
        check(
            self._lib.tb_apply_f64_device(
                self.handle, _tensor_ptr(x, torch.float64, self.size, "x"), _tensor_ptr(y, torch.float64, self.size, "y")
            )
        )

    def residual_f64_device_static(self, x: Any, b: Any, r: Any) -> tuple[float, float]:
        """r = b - A x in FP64 on device tensors through the allocation-free
        entry point; returns (||r||^2, max |r|)."""
        import torch

        torch.cuda.synchronize(self.device)
        norms = (ctypes.c_double * 2)()
        check(
            self._lib.tb_residual_f64_device_static(
                self.handle,
                _tensor_ptr(x, torch.float64, self.size, "x"),
                _tensor_ptr(b, torch.float64, self.size, "b"),
                _tensor_ptr(r, torch.float64, self.size, "r"),
                ctypes.cast(norms, _VP),
            )
        )
        return float(norms[0]), float(norms[1])

    def set_robin(self, robin_total: Any) -> None:
        """New lumped Robin totals (node order) on the resident system."""

        robin = self._vector(robin_total, np.float64, "robin_total")
        check(self._lib.tb_set_robin(self.handle, _ptr(robin)))

    # -------------------------------------------------------- preconditioner
    def set_preconditioner(self, kind: str, coarse_block_nodes: int | None = None) -> None:
        """``"jacobi"``, ``"two-level"`` or ``"multilevel"`` for the inner FP32 PCG."""

        if kind not in PRECONDITIONER_KINDS:
            raise ValueError("preconditioner must be 'two-level', 'jacobi' or 'multilevel'")
        check(self._lib.tb_set_preconditioner(self.handle, PRECONDITIONER_KINDS[kind], int(coarse_block_nodes or 0)))

    def preconditioner(self) -> dict[str, Any]:
        out = (ctypes.c_int32 * 5)()
        check(self._lib.tb_get_preconditioner(self.handle, out))
        kind = {v: k for k, v in PRECONDITIONER_KINDS.items()}[int(out[0])]
        shape = (int(out[2]), int(out[3]), int(out[4]))
        info = {"kind": kind, "block": int(out[1]), "coarse_shape": shape, "coarse_size": int(np.prod(shape))}
        if kind == "multilevel":
            info["levels"] = self.multilevel_grids()
        return info

    def multilevel_grids(self) -> list[tuple[int, int, int]]:
        """Shapes (node layers, rows, columns) of the multilevel coarse grids, level 1 first."""

        dims = (ctypes.c_int32 * (3 * 16))()
        count = ctypes.c_int32(0)
        check(self._lib.tb_get_multilevel(self.handle, dims, 16, ctypes.byref(count)))
        return [(int(dims[3 * l]), int(dims[3 * l + 1]), int(dims[3 * l + 2])) for l in range(min(count.value, 16))]

    def multilevel_stencil(self, level: int) -> np.ndarray:
        """FP32 stencil (14, layers, rows, columns) of multilevel coarse grid `level` (1-based)."""

        shape = self.multilevel_grids()[level - 1]
        out = np.empty((14,) + shape, dtype=np.float32)
        check(self._lib.tb_get_multilevel_stencil(self.handle, int(level), _ptr(out)))
        return out

    def coarse(self) -> tuple[np.ndarray, np.ndarray]:
        """(Z^T A Z, its symmetrised inverse) of the two-level preconditioner."""

        n = self.preconditioner()["coarse_size"]
        matrix = np.empty((n, n))
        inverse = np.empty((n, n))
        check(self._lib.tb_get_coarse(self.handle, _ptr(matrix), _ptr(inverse)))
        return matrix, inverse

    def precondition_f32(self, vector: Any) -> np.ndarray:
        x = self._vector(vector, np.float32)
        y = np.empty_like(x)
        check(self._lib.tb_precondition_f32(self.handle, _ptr(x), _ptr(y)))
        return y

    @classmethod
    def from_dc(
        cls,
        *,
        layer_thickness_m: np.ndarray,
        pitch_x_m: np.ndarray,
        pitch_y_m: np.ndarray,
        conductivity_s_per_m: np.ndarray,
        element_active: np.ndarray,
        via_lower: Sequence[int] = (),
        via_upper: Sequence[int] = (),
        via_conductance_s: Sequence[float] = (),
        reference_node: int = -1,
        dirichlet_nodes: Sequence[int] = (),
        device: int = 0,
    ) -> "DeviceSystem":
        """A layered DC system (tb_dc_system_create): sheets of layers x rows x
        cols elements, vias between flat node indices, a reference node (-1:
        none) and Dirichlet nodes."""

        lib = load()
        require_device(device)
        active = np.ascontiguousarray(element_active, dtype=bool)
        if active.ndim != 3:
            raise ValueError("element_active must have shape (layers, rows, cols)")
        layers, rows, cols = active.shape
        active8 = active.view(np.uint8)
        thickness = np.ascontiguousarray(layer_thickness_m, dtype=np.float64)
        px = np.ascontiguousarray(pitch_x_m, dtype=np.float64)
        py = np.ascontiguousarray(pitch_y_m, dtype=np.float64)
        sigma = np.ascontiguousarray(conductivity_s_per_m, dtype=np.float64).reshape(-1)
        if thickness.size != layers or px.size != cols or py.size != rows or sigma.size != active.size:
            raise ValueError("mesh arrays do not match element_active")
        lower = np.ascontiguousarray(via_lower, dtype=np.int64).reshape(-1)
        upper = np.ascontiguousarray(via_upper, dtype=np.int64).reshape(-1)
        g = np.ascontiguousarray(via_conductance_s, dtype=np.float64).reshape(-1)
        if not lower.size == upper.size == g.size:
            raise ValueError("via arrays must have one entry per via")
        dirichlet = np.ascontiguousarray(dirichlet_nodes, dtype=np.int64).reshape(-1)
        keep = (active8, thickness, px, py, sigma, lower, upper, g, dirichlet)
        i64 = ctypes.POINTER(ctypes.c_int64)
        desc = DcDescC(
            layers, rows, cols,
            thickness.ctypes.data_as(_c_double_p), px.ctypes.data_as(_c_double_p), py.ctypes.data_as(_c_double_p),
            sigma.ctypes.data_as(_c_double_p), active8.ctypes.data_as(_c_uint8_p),
            int(g.size), lower.ctypes.data_as(i64), upper.ctypes.data_as(i64), g.ctypes.data_as(_c_double_p),
            int(reference_node), int(dirichlet.size), dirichlet.ctypes.data_as(i64),
        )
        handle = ctypes.c_void_p()
        check(lib.tb_dc_system_create(ctypes.byref(desc), int(device), ctypes.byref(handle)))
        del keep
        self = cls.__new__(cls)
        self._adopt(lib, handle, (layers - 1, rows, cols), device)
        self._keep = None
        return self

    def dc_masks(self) -> tuple[np.ndarray, np.ndarray]:
        """(active, free) node masks of a layered DC system, as booleans."""

        active = np.empty(self.size, dtype=np.uint8)
        free = np.empty(self.size, dtype=np.uint8)
        check(self._lib.tb_dc_get_masks(self.handle, _ptr(active), _ptr(free)))
        return active.astype(bool), free.astype(bool)

    def dc_post(self, potential: Any) -> tuple[np.ndarray, np.ndarray]:
        """(field (layers, rows, cols, 2), element Joule loss (layers, rows, cols))
        of a layered DC system's potential, computed on the device."""

        x = self._vector(potential, np.float64)
        shape = (self.element_shape[0] + 1,) + tuple(self.element_shape[1:])  # sheet layers
        field = np.empty(shape + (2,), dtype=np.float64)
        loss = np.empty(shape, dtype=np.float64)
        check(self._lib.tb_dc_post(self.handle, _ptr(x), _ptr(field), _ptr(loss)))
        return field, loss

    # --------------------------------------------------- problem systems
    def set_convection(self, convection: Sequence[dict[str, Any]]) -> None:
        conv, _keep = convection_descs(convection, self.element_shape)
        check(self._lib.tb_set_convection(self.handle, conv, len(convection)))
        self.convection_count = len(convection)

    def set_capacity(self, capacity_per_s: Any | None) -> None:
        if capacity_per_s is None:
            check(self._lib.tb_set_capacity(self.handle, None))
            return
        cap = self._vector(capacity_per_s, np.float64, "capacity_per_s")
        check(self._lib.tb_set_capacity(self.handle, _ptr(cap)))

    def prepared(self) -> dict[str, np.ndarray]:
        """Robin conductance / total / R T_amb, nodal load, free and active masks."""

        out = {k: np.empty(self.size, dtype=np.float64) for k in ("robin_only", "robin_total", "robin_rhs", "load")}
        free = np.empty(self.size, dtype=np.uint8)
        active = np.empty(self.size, dtype=np.uint8)
        check(self._lib.tb_get_prepared(self.handle, _ptr(out["robin_only"]), _ptr(out["robin_total"]),
                                        _ptr(out["robin_rhs"]), _ptr(out["load"]), _ptr(free), _ptr(active)))
        out["free_nodes"] = free
        out["active_nodes"] = active
        return out

    def prepared_array(self, name: str) -> np.ndarray:
        """One of the prepared flat arrays: robin_only, robin_total, robin_rhs, load."""

        order = ("robin_only", "robin_total", "robin_rhs", "load")
        if name not in order:
            raise ValueError(f"name must be one of {order}")
        out = np.empty(self.size, dtype=np.float64)
        args = [None] * 6
        args[order.index(name)] = _ptr(out)
        check(self._lib.tb_get_prepared(self.handle, *args))
        return out

    def boundary_weights(self, index: int) -> tuple[np.ndarray, np.ndarray]:
        w = np.empty(self.size, dtype=np.float64)
        rw = np.empty(self.size, dtype=np.float64)
        check(self._lib.tb_get_boundary_weights(self.handle, int(index), _ptr(w), _ptr(rw)))
        return w, rw

    def build_rhs(self, reference_temperature_k: float, previous_temperature_k: Any | None = None) -> np.ndarray:
        prev = None if previous_temperature_k is None else self._vector(previous_temperature_k, np.float64,
                                                                        "previous_temperature_k")
        rhs = np.empty(self.size, dtype=np.float64)
        check(self._lib.tb_build_rhs(self.handle, float(reference_temperature_k),
                                     None if prev is None else _ptr(prev), _ptr(rhs)))
        return rhs

    def postprocess(self, temperature_k: Any, previous_temperature_k: Any | None = None, *, flux: bool = True,
                    residual: bool = False) -> dict[str, Any]:
        """Flux, per-boundary removed heat and the heat budget of a temperature field."""

        t = self._vector(temperature_k, np.float64, "temperature_k")
        return self._postprocess(lambda *out: self._lib.tb_postprocess(self.handle, _ptr(t), *out),
                                 previous_temperature_k, flux, residual)

    def postprocess_rise_device(self, rise: Any, reference_temperature_k: float,
                                previous_temperature_k: Any | None = None, *, flux: bool = True,
                                residual: bool = False, temperature: bool = False) -> dict[str, Any]:
        """``postprocess`` of T = rise + reference, ``rise`` being the flat FP64
        CUDA tensor a device solve left (tb_postprocess_rise_device): the field
        stays in HBM; the outputs are host arrays, with T itself under
        "temperature" when asked for, and its (min, max) over the active nodes
        under "temperature_extrema"."""

        import torch

        rise_ptr = self._device_tensor(rise, "rise")
        field = np.empty(self.size, dtype=np.float64) if temperature else None
        extrema = np.empty(2, dtype=np.float64)
        torch.cuda.synchronize(self.device)
        out = self._postprocess(
            lambda *arrays: self._lib.tb_postprocess_rise_device(
                self.handle, rise_ptr, float(reference_temperature_k), *arrays,
                None if field is None else _ptr(field), _ptr(extrema)),
            previous_temperature_k, flux, residual)
        out["temperature"] = field
        out["temperature_extrema"] = (float(extrema[0]), float(extrema[1]))
        return out

    def download(self, tensor: Any) -> np.ndarray:
        """A flat FP64 CUDA tensor of this system's device as a new host array
        (tb_download: the host side of the copy spread over host threads)."""

        import torch

        ptr = self._device_tensor(tensor, "tensor")
        out = np.empty(self.size, dtype=np.float64)
        torch.cuda.synchronize(self.device)
        check(self._lib.tb_download(self.handle, _ptr(out), ptr, out.nbytes))
        return out

    def _postprocess(self, call: Any, previous_temperature_k: Any | None, flux: bool, residual: bool
                     ) -> dict[str, Any]:
        prev = None if previous_temperature_k is None else self._vector(previous_temperature_k, np.float64,
                                                                        "previous_temperature_k")
        heat_flux = np.empty(self.element_shape + (3,), dtype=np.float64) if flux else None
        res = np.empty(self.size, dtype=np.float64) if residual else None
        convective = np.empty(max(self.convection_count, 1), dtype=np.float64)
        budget = np.empty(3, dtype=np.float64)
        check(call(None if prev is None else _ptr(prev), None if heat_flux is None else _ptr(heat_flux),
                   _ptr(convective), _ptr(budget), None if res is None else _ptr(res)))
        return dict(heat_flux=heat_flux, convective_heat_w=convective[: self.convection_count].copy(),
                    total_heat_input_w=float(budget[0]), fixed_temperature_heat_w=float(budget[1]),
                    stored_heat_w=float(budget[2]), residual=res)

    def build_rhs_device(self, reference_temperature_k: float, rhs: Any,
                         previous_temperature_k: Any | None = None) -> None:
        """``build_rhs`` into the flat FP64 CUDA tensor ``rhs`` (tb_build_rhs_device);
        ``previous_temperature_k`` is a flat FP64 CUDA tensor or None."""

        import torch

        rhs_ptr = self._device_tensor(rhs, "rhs")
        prev_ptr = None if previous_temperature_k is None else self._device_tensor(previous_temperature_k,
                                                                                  "previous_temperature_k")
        torch.cuda.synchronize(self.device)
        check(self._lib.tb_build_rhs_device(self.handle, float(reference_temperature_k), prev_ptr, rhs_ptr))

    def _device_tensor(self, tensor: Any, name: str) -> int:
        import torch

        ptr = _tensor_ptr(tensor, torch.float64, self.size, name)
        if tensor.device.index != self.device:
            raise ValueError(f"{name} must be on cuda:{self.device}")
        return ptr

    def stiffness_f64(self, vector: Any) -> np.ndarray:
        x = self._vector(vector, np.float64)
        y = np.empty_like(x)
        check(self._lib.tb_stiffness_f64(self.handle, _ptr(x), _ptr(y)))
        return y

    def diagonal(self) -> np.ndarray:
        out = np.empty(self.size, dtype=np.float64)
        check(self._lib.tb_diagonal(self.handle, _ptr(out)))
        return out

    # --------------------------------------------------------------- solves
    @staticmethod
    def _config(config: Any) -> MPIRConfigC:
        return mpir_config_c(config)

    def solve_mpir(self, rhs: Any, config: Any, initial_guess: Any | None = None) -> dict[str, Any]:
        b = self._vector(rhs, np.float64, "rhs")
        x = np.zeros(self.size) if initial_guess is None else self._vector(initial_guess, np.float64, "initial_guess").copy()
        cap = int(config.max_outer_iterations) + 1
        history = (MPIRStepC * cap)()
        result = MPIRResultC()
        check(
            self._lib.tb_solve_mpir(
                self.handle, _ptr(b), _ptr(x), ctypes.byref(self._config(config)), ctypes.byref(result), history, cap
            )
        )
        return _mpir_dict(result, history, x)

    def solve_mpir_device(self, rhs: Any, x: Any, config: Any) -> dict[str, Any]:
        """MPIR on device-resident flat FP64 tensors; ``x`` is the guess in and the solution out."""

        import torch

        torch.cuda.synchronize(self.device)
        cap = int(config.max_outer_iterations) + 1
        history = (MPIRStepC * cap)()
        result = MPIRResultC()
        check(
            self._lib.tb_solve_mpir_device(
                self.handle,
                _tensor_ptr(rhs, torch.float64, self.size, "rhs"),
                _tensor_ptr(x, torch.float64, self.size, "x"),
                ctypes.byref(self._config(config)),
                ctypes.byref(result),
                history,
                cap,
            )
        )
        return _mpir_dict(result, history, None)

    def solve_pcg_f64(
        self, rhs: Any, *, relative_tolerance: float, absolute_tolerance: float = 0.0, max_iterations: int,
        initial_guess: Any | None = None, multilevel: bool = False,
    ) -> dict[str, Any]:
        """Plain FP64 PCG: Jacobi, or (``multilevel``) the system's multilevel preconditioner."""

        b = self._vector(rhs, np.float64, "rhs")
        x = np.zeros(self.size) if initial_guess is None else self._vector(initial_guess, np.float64, "initial_guess").copy()
        result = PCGResultC()
        entry = self._lib.tb_solve_pcg_f64_ml if multilevel else self._lib.tb_solve_pcg_f64
        check(
            entry(
                self.handle, _ptr(b), _ptr(x), float(relative_tolerance), float(absolute_tolerance),
                int(max_iterations), ctypes.byref(result),
            )
        )
        return {
            "solution": x,
            "converged": bool(result.converged),
            "iterations": int(result.iterations),
            "relative_residual": float(result.relative_residual),
        }

    def solve_pcg_f64_device(
        self, rhs: Any, x: Any, *, relative_tolerance: float, absolute_tolerance: float = 0.0, max_iterations: int,
        multilevel: bool = False,
    ) -> dict[str, Any]:
        import torch

        torch.cuda.synchronize(self.device)
        result = PCGResultC()
        entry = self._lib.tb_solve_pcg_f64_ml_device if multilevel else self._lib.tb_solve_pcg_f64_device
        check(
            entry(
                self.handle,
                _tensor_ptr(rhs, torch.float64, self.size, "rhs"),
                _tensor_ptr(x, torch.float64, self.size, "x"),
                float(relative_tolerance),
                float(absolute_tolerance),
                int(max_iterations),
                ctypes.byref(result),
            )
        )
        return {
            "converged": bool(result.converged),
            "iterations": int(result.iterations),
            "relative_residual": float(result.relative_residual),
        }


def _mpir_dict(result: MPIRResultC, history: Any, solution: np.ndarray | None) -> dict[str, Any]:
    steps = [
        (
            int(history[i].outer_iteration),
            float(history[i].high_relative_residual),
            int(history[i].inner_iterations),
            float(history[i].inner_relative_residual),
        )
        for i in range(int(result.history_length))
    ]
    return {
        "solution": solution,
        "converged": bool(result.converged),
        "outer_iterations": int(result.outer_iterations),
        "inner_iterations": int(result.inner_iterations),
        "relative_residual": float(result.relative_residual),
        "high_operator_applications": int(result.high_operator_applications),
        "low_operator_applications": int(result.low_operator_applications),
        "history": steps,
    }


_PRECONDITIONERS = {"jacobi": 0, "two-level": 1}  # the batch engine's kinds


def engine_footprint(arrays: dict[str, Any], preconditioner: str = "jacobi") -> tuple[int, int]:
    """(resident, transient) device bytes of one board in a BatchEngine."""

    desc, keep, _ = system_desc(**arrays)
    resident = ctypes.c_int64()
    transient = ctypes.c_int64()
    check(load().tb_engine_footprint(ctypes.byref(desc), _PRECONDITIONERS[preconditioner], ctypes.byref(resident),
                                     ctypes.byref(transient)))
    del keep
    return int(resident.value), int(transient.value)


class BatchEngine:
    """Many boards resident on one device, solved together (tb_engine)."""

    _STAGINGS = {"auto": 0, "cp.async": 1, "tensor": 2}

    def __init__(self, *, capacity: int = 64, max_slabs: int = 32, tile_rows: int = 0,
                 budget_bytes: int = 80 * 10**9, device: int = 0, preconditioner: str = "jacobi",
                 staging: str = "auto") -> None:
        lib = load()
        require_device(device)
        if preconditioner not in _PRECONDITIONERS:
            raise ValueError("preconditioner must be 'two-level' or 'jacobi'")
        if staging not in self._STAGINGS:
            raise ValueError("staging must be 'auto', 'cp.async' or 'tensor'")
        cfg = EngineConfigC(int(capacity), int(max_slabs), int(tile_rows), _PRECONDITIONERS[preconditioner],
                            int(budget_bytes), self._STAGINGS[staging], 0)
        self.preconditioner = preconditioner
        handle = ctypes.c_void_p()
        check(lib.tb_engine_create(int(device), ctypes.byref(cfg), ctypes.byref(handle)))
        self._lib = lib
        self._handle = handle
        self.device = int(device)
        self._sizes: dict[int, tuple[int, int]] = {}  # ticket -> (nodes, max outer iterations)

    def close(self) -> None:
        handle = getattr(self, "_handle", None)
        if handle is not None and handle.value:
            self._lib.tb_engine_destroy(handle)
            self._handle = None

    def __del__(self) -> None:  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self) -> "BatchEngine":
        return self

    def __exit__(self, *exc: object) -> None:
        self.close()

    @property
    def handle(self) -> ctypes.c_void_p:
        if self._handle is None:
            raise RuntimeError("the engine was closed")
        return self._handle

    def submit(self, arrays: dict[str, Any], rhs: Any, config: Any, initial_guess: Any | None = None) -> int | None:
        """Admit one board; returns its ticket, or None when the engine has no
        room for it now (no free slot or not enough of the byte budget)."""

        desc, keep, shape = system_desc(**arrays)
        nodes = (shape[0] + 1) * (shape[1] + 1) * (shape[2] + 1)
        b = np.ascontiguousarray(rhs, dtype=np.float64).reshape(-1)
        if b.size != nodes:
            raise ValueError(f"rhs has size {b.size}, expected {nodes}")
        x0 = None
        if initial_guess is not None:
            x0 = np.ascontiguousarray(initial_guess, dtype=np.float64).reshape(-1)
            if x0.size != nodes:
                raise ValueError(f"initial_guess has size {x0.size}, expected {nodes}")
        ticket = ctypes.c_int64()
        status = self._lib.tb_engine_submit(
            self.handle, ctypes.byref(desc), _ptr(b), None if x0 is None else _ptr(x0),
            ctypes.byref(mpir_config_c(config)), ctypes.byref(ticket),
        )
        del keep
        if status == TB_ENOMEM:
            return None
        check(status)
        self._sizes[int(ticket.value)] = (nodes, int(config.max_outer_iterations))
        return int(ticket.value)

    def step(self) -> int:
        """Run one graph chunk over the resident boards; returns how many finished boards await collection."""

        n = ctypes.c_int32()
        check(self._lib.tb_engine_step(self.handle, ctypes.byref(n)))
        return int(n.value)

    def finished(self) -> list[int]:
        count = ctypes.c_int32()
        check(self._lib.tb_engine_finished(self.handle, None, 0, ctypes.byref(count)))
        if count.value == 0:
            return []
        out = (ctypes.c_int64 * count.value)()
        check(self._lib.tb_engine_finished(self.handle, out, count.value, ctypes.byref(count)))
        return [int(v) for v in out]

    def collect(self, ticket: int) -> dict[str, Any]:
        nodes, max_outer = self._sizes[int(ticket)]
        x = np.empty(nodes, dtype=np.float64)
        cap = max_outer + 1
        history = (MPIRStepC * cap)()
        result = MPIRResultC()
        status = self._lib.tb_engine_collect(self.handle, int(ticket), _ptr(x), ctypes.byref(result), history, cap)
        del self._sizes[int(ticket)]
        check(status)
        return _mpir_dict(result, history, x)

    def time_apply(self, launches: int = 5) -> float:
        """Milliseconds of one batched FP32 operator launch over the resident boards."""

        ms = ctypes.c_double()
        check(self._lib.tb_engine_time_apply(self.handle, int(launches), ctypes.byref(ms)))
        return float(ms.value)

    def stream_handle(self) -> int:
        out = _VP()
        check(self._lib.tb_engine_stream(self.handle, ctypes.byref(out)))
        return int(out.value or 0)

    def info(self) -> dict[str, int]:
        out = (ctypes.c_int64 * 8)()
        check(self._lib.tb_engine_info(self.handle, out))
        keys = ("resident", "scheduled", "bytes_in_use", "budget_bytes", "chunks", "kernel_launches", "tile_rows",
                "capacity")
        info = {k: int(out[i]) for i, k in enumerate(keys)}
        staging = ctypes.c_int32()
        check(self._lib.tb_engine_staging(self.handle, ctypes.byref(staging)))
        info["staging"] = {1: "cp.async", 2: "tensor"}.get(int(staging.value), "auto")
        return info
