"""ctypes wrapper of the CPU oracle (liboracle_cpu.so built from thermal_oracle.c).

TEST INFRASTRUCTURE: the oracle is the checker of the device kernels and the
timed CPU baseline; only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline import it.  It takes the reference's own prepared arrays (element
factors (3, S, R, C), Robin total, free mask) so that it can be pinned against
the golden vectors recorded from the reference (tests/golden).
"""

from __future__ import annotations

import ctypes
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle_cpu.so"
_lib = None


class _View(ctypes.Structure):
    _fields_ = [
        ("slabs", ctypes.c_int32),
        ("rows", ctypes.c_int32),
        ("cols", ctypes.c_int32),
        ("coef", ctypes.c_void_p),
        ("robin", ctypes.c_void_p),
        ("free_nodes", ctypes.c_void_p),
    ]


class _MpirResult(ctypes.Structure):
    _fields_ = [
        ("converged", ctypes.c_int32),
        ("outer_iterations", ctypes.c_int32),
        ("inner_iterations", ctypes.c_int32),
        ("high_applications", ctypes.c_int32),
        ("low_applications", ctypes.c_int32),
        ("history_length", ctypes.c_int32),
        ("relative_residual", ctypes.c_double),
    ]


class _MpirStep(ctypes.Structure):
    _fields_ = [
        ("outer_iteration", ctypes.c_int32),
        ("inner_iterations", ctypes.c_int32),
        ("high_relative_residual", ctypes.c_double),
        ("inner_relative_residual", ctypes.c_double),
    ]


def build(force: bool = False) -> Path:
    """Compile the oracle with the Makefile beside this file."""

    source = HERE / "thermal_oracle.c"
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < source.stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "-B"], check=True, capture_output=True)
    return LIB_PATH


def load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(LIB_PATH))
        vp = ctypes.c_void_p
        i32 = ctypes.c_int
        lib.or_apply_f64.argtypes = [ctypes.POINTER(_View), vp, vp, i32]
        lib.or_apply_fast_f64.argtypes = [ctypes.POINTER(_View), vp, vp, i32]
        lib.or_stiffness_f64.argtypes = [ctypes.POINTER(_View), vp, vp, i32]
        lib.or_apply_f32.argtypes = [ctypes.POINTER(_View), vp, vp, vp, vp, i32]
        lib.or_apply_fast_f32.argtypes = [ctypes.POINTER(_View), vp, vp, vp, vp, i32]
        lib.or_diagonal.argtypes = [ctypes.POINTER(_View), vp]
        lib.or_unit_matrices.argtypes = [vp]
        lib.or_pcg_f64.argtypes = [
            ctypes.POINTER(_View), vp, vp, vp, ctypes.c_double, ctypes.c_double, i32, i32,
            ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double),
        ]
        lib.or_pcg_f64.restype = i32
        lib.or_solve_mpir.argtypes = [
            ctypes.POINTER(_View), vp, vp, vp, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
            i32, i32, i32, ctypes.POINTER(_MpirResult), vp, i32,
        ]
        lib.or_solve_mpir.restype = i32
        lib.or_inner_iterations.argtypes = [ctypes.POINTER(_View), vp, vp, vp, vp, i32, i32, ctypes.POINTER(ctypes.c_double)]
        lib.or_inner_iterations.restype = i32
        lib.or_max_threads.restype = i32
        _lib = lib
    return _lib


def max_threads() -> int:
    return int(load().or_max_threads())


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


@dataclass
class OracleSystem:
    """The reference's prepared operator: element factors, Robin total, free mask."""

    coef: np.ndarray         # (3, S, R, C) float64
    robin_total: np.ndarray  # (N,) float64
    free: np.ndarray         # (N,) uint8
    threads: int = 0

    def __post_init__(self) -> None:
        self.coef = np.ascontiguousarray(self.coef, dtype=np.float64)
        _, s, r, c = self.coef.shape
        self.element_shape = (s, r, c)
        self.node_shape = (s + 1, r + 1, c + 1)
        self.size = int(np.prod(self.node_shape))
        self.robin_total = np.ascontiguousarray(self.robin_total, dtype=np.float64).reshape(-1)
        self.free = np.ascontiguousarray(self.free, dtype=np.uint8).reshape(-1)
        self.coef32 = self.coef.astype(np.float32)
        self.robin32 = self.robin_total.astype(np.float32)
        self.threads = self.threads or max_threads()
        self._view = _View(s, r, c, _p(self.coef), _p(self.robin_total), _p(self.free))
        self._diag = None

    @classmethod
    def from_arrays(cls, *, slab_thickness_m, pitch_x_m, pitch_y_m, k_in, k_z, robin_total, free, threads: int = 0):
        """Element factors computed as the reference does (mesh.py:276-293)."""

        hz = np.asarray(slab_thickness_m, dtype=np.float64)[:, None, None]
        hx = np.asarray(pitch_x_m, dtype=np.float64)[None, None, :]
        hy = np.asarray(pitch_y_m, dtype=np.float64)[None, :, None]
        k_in = np.asarray(k_in, dtype=np.float64)
        k_z = np.asarray(k_z, dtype=np.float64)
        coef = np.stack((k_in * hy * hz / hx, k_in * hx * hz / hy, k_z * hx * hy / hz))
        return cls(coef, robin_total, free, threads)

    def _vec(self, v, dtype) -> np.ndarray:
        out = np.ascontiguousarray(v, dtype=dtype).reshape(-1)
        if out.size != self.size:
            raise ValueError("vector size mismatch")
        return out

    def apply_f64(self, x, fast: bool = False) -> np.ndarray:
        x = self._vec(x, np.float64)
        y = np.empty_like(x)
        fn = load().or_apply_fast_f64 if fast else load().or_apply_f64
        fn(ctypes.byref(self._view), _p(x), _p(y), self.threads)
        return y

    def stiffness_f64(self, x) -> np.ndarray:
        x = self._vec(x, np.float64)
        y = np.empty_like(x)
        load().or_stiffness_f64(ctypes.byref(self._view), _p(x), _p(y), self.threads)
        return y

    def apply_f32(self, x, fast: bool = False) -> np.ndarray:
        x = self._vec(x, np.float32)
        y = np.empty_like(x)
        fn = load().or_apply_fast_f32 if fast else load().or_apply_f32
        fn(ctypes.byref(self._view), _p(self.coef32), _p(self.robin32), _p(x), _p(y), self.threads)
        return y

    def diagonal(self) -> np.ndarray:
        if self._diag is None:
            d = np.empty(self.size, dtype=np.float64)
            load().or_diagonal(ctypes.byref(self._view), _p(d))
            self._diag = d
        return self._diag

    def dinv32(self) -> np.ndarray:
        return (1.0 / self.diagonal()).astype(np.float32)

    def pcg_f64(self, b, x0=None, *, rtol: float = 1e-10, atol: float = 0.0, max_iterations: int = 1_000_000):
        b = self._vec(b, np.float64)
        x = np.zeros(self.size) if x0 is None else self._vec(x0, np.float64).copy()
        its = ctypes.c_int32()
        rel = ctypes.c_double()
        st = load().or_pcg_f64(
            ctypes.byref(self._view), _p(self.diagonal()), _p(b), _p(x), rtol, atol, int(max_iterations),
            self.threads, ctypes.byref(its), ctypes.byref(rel),
        )
        if st:
            raise RuntimeError("PCG requires a finite symmetric positive-definite operator")
        return x, int(its.value), float(rel.value)

    def solve_mpir(self, b, x0=None, *, rtol=1e-10, atol=0.0, inner_rtol=1e-4, max_outer=40, max_inner=200000):
        b = self._vec(b, np.float64)
        x = np.zeros(self.size) if x0 is None else self._vec(x0, np.float64).copy()
        res = _MpirResult()
        cap = max_outer + 1
        hist = (_MpirStep * cap)()
        dinv = self.dinv32()
        st = load().or_solve_mpir(
            ctypes.byref(self._view), _p(self.coef32), _p(self.robin32), _p(dinv), _p(b), _p(x), rtol, atol,
            inner_rtol, int(max_outer), int(max_inner), self.threads, ctypes.byref(res), ctypes.addressof(hist), cap,
        )
        if st:
            raise RuntimeError("inner PCG requires a finite symmetric positive-definite operator")
        steps = [
            (hist[i].outer_iteration, hist[i].high_relative_residual, hist[i].inner_iterations, hist[i].inner_relative_residual)
            for i in range(res.history_length)
        ]
        return {
            "solution": x,
            "converged": bool(res.converged),
            "outer_iterations": res.outer_iterations,
            "inner_iterations": res.inner_iterations,
            "relative_residual": res.relative_residual,
            "history": steps,
        }

    def inner_iterations(self, rhs, iterations: int) -> float:
        """Run exactly ``iterations`` FP32 PCG iterations on ``rhs``; returns the relative residual."""

        rhs = self._vec(rhs, np.float64)
        rel = ctypes.c_double()
        load().or_inner_iterations(
            ctypes.byref(self._view), _p(self.coef32), _p(self.robin32), _p(self.dinv32()), _p(rhs),
            int(iterations), self.threads, ctypes.byref(rel),
        )
        return float(rel.value)


# ------------------------------------------------------------ two-level
def choose_block_size(node_shape, max_coarse_size: int = 2048, minimum: int = 4) -> int:
    """Smallest patch width >= ``minimum`` whose coarse grid has at most
    ``max_coarse_size`` patches (reference two_level.py:36-50)."""

    layers, rows, cols = node_shape
    block = max(1, int(minimum))
    while layers * -(-rows // block) * -(-cols // block) > max_coarse_size and block < max(rows, cols):
        block += 1
    return block


class CoarseSpaceOracle:
    """Jacobi plus patch-constant coarse correction (reference
    src/electrical/matrix_free_mpir_fem/two_level.py:62-229), restated.

    A patch is ``block x block`` nodes of one node layer; Z^T sums a free-node
    field over patches, Z copies a patch value onto its free nodes.  Z^T A Z is
    exact from 27 FP64 actions: patches whose (layer, row, col) indices agree
    modulo 3 never share an element, so the action of one colour's indicator,
    summed over patch I, is the coupling of I with the single patch of that
    colour within one patch of I in every direction.  Patches without free
    nodes get a unit diagonal.  The inverse comes from a Cholesky factor and
    is symmetrised, as the reference does.
    """

    def __init__(self, system: OracleSystem, block: int | None = None, max_coarse_size: int = 2048) -> None:
        self.system = system
        layers, rows, cols = system.node_shape
        self.block = int(block) if block else choose_block_size(system.node_shape, max_coarse_size)
        b = self.block
        self.coarse_shape = (layers, -(-rows // b), -(-cols // b))
        self.coarse_size = int(np.prod(self.coarse_shape))
        self.free = system.free.reshape(system.node_shape).astype(bool)
        self._flat = None
        counts = self.restrict(self.free.astype(np.float64))
        matrix = self._galerkin()
        empty = counts <= 0.0
        matrix[empty, :] = 0.0
        matrix[:, empty] = 0.0
        matrix[empty, empty] = 1.0
        self.coarse_matrix = matrix
        factor = np.linalg.cholesky(matrix)
        inverse = np.linalg.solve(factor.T, np.linalg.solve(factor, np.eye(self.coarse_size)))
        self.coarse_inverse = 0.5 * (inverse + inverse.T)

    def _flat_patch(self) -> np.ndarray:
        """Flat coarse index of every node's patch (computed once)."""

        if getattr(self, "_flat", None) is None:
            layers, rows, cols = self.system.node_shape
            z, y, x = np.meshgrid(np.arange(layers), np.arange(rows), np.arange(cols), indexing="ij")
            self._flat = np.ravel_multi_index((z, y // self.block, x // self.block), self.coarse_shape).reshape(-1)
            self._free_flat = self.free.reshape(-1)
        return self._flat

    def restrict(self, grid: np.ndarray) -> np.ndarray:
        flat = self._flat_patch()
        values = np.where(self._free_flat, np.asarray(grid, dtype=np.float64).reshape(-1), 0.0)
        return np.bincount(flat, weights=values, minlength=self.coarse_size)

    def prolong(self, coarse: np.ndarray) -> np.ndarray:
        flat = self._flat_patch()
        return np.where(self._free_flat, np.asarray(coarse, dtype=np.float64).reshape(-1)[flat], 0.0)

    @staticmethod
    def _colour(l, r, c):
        return (l % 3) * 9 + (r % 3) * 3 + (c % 3)

    def _galerkin(self) -> np.ndarray:
        nc = self.coarse_size
        L, R, C = np.meshgrid(*[np.arange(n) for n in self.coarse_shape], indexing="ij")
        colours = self._colour(L, R, C).reshape(-1)
        matrix = np.zeros((nc, nc))
        rows = np.arange(nc)
        coords = (L.reshape(-1), R.reshape(-1), C.reshape(-1))
        for colour in range(27):
            indicator = (colours == colour).astype(np.float64)
            if not indicator.any():
                continue
            action = self.system.apply_f64(self.prolong(indicator))
            summed = self.restrict(action)
            # the same-coloured patch J next to each row patch I
            target = np.full(nc, -1)
            for d in np.ndindex(3, 3, 3):
                j = [a + o - 1 for a, o in zip(coords, d)]
                inside = np.ones(nc, dtype=bool)
                for a, n in zip(j, self.coarse_shape):
                    inside &= (a >= 0) & (a < n)
                hit = inside & (self._colour(*[np.where(inside, a, 0) for a in j]) == colour)
                target[hit] = np.ravel_multi_index([a[hit] for a in j], self.coarse_shape)
            ok = target >= 0
            matrix[rows[ok], target[ok]] = summed[ok]
        return matrix

    def precondition_f64(self, v: np.ndarray) -> np.ndarray:
        v = np.asarray(v, dtype=np.float64).reshape(-1)
        coarse = self.coarse_inverse @ self.restrict(v)
        return v / self.system.diagonal() + self.prolong(coarse)

    def pcg_f64(self, b: np.ndarray, *, rtol: float = 1e-10, max_iterations: int = 100000):
        """FP64 PCG with this preconditioner (small cases: NumPy loop)."""

        b = np.asarray(b, dtype=np.float64).reshape(-1)
        x = np.zeros_like(b)
        r = b.copy()
        bn = np.linalg.norm(b)
        if bn == 0.0:
            return x, 0, 0.0
        z = self.precondition_f64(r)
        p = z.copy()
        rz = float(r @ z)
        rel = 1.0
        for it in range(1, max_iterations + 1):
            q = self.system.apply_f64(p)
            alpha = rz / float(p @ q)
            x += alpha * p
            r -= alpha * q
            rel = float(np.linalg.norm(r)) / bn
            if rel <= rtol:
                return x, it, rel
            z = self.precondition_f64(r)
            rz_new = float(r @ z)
            p = z + (rz_new / rz) * p
            rz = rz_new
        return x, max_iterations, rel
