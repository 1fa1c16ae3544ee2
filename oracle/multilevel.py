"""CPU restatement of the multilevel preconditioner (scipy, FP64).

TEST INFRASTRUCTURE: the checker of the device's multilevel preconditioner
(pcb_analysis_b200/csrc/tb_multilevel.cuh); only tests/ and bench.py's CPU
legs use it.  It has no counterpart in the reference: it extends the
reference's two-level preconditioner (src/electrical/matrix_free_mpir_fem/
two_level.py:62-229: patch-constant coarse functions on b x b nodes of one
node layer, Galerkin coarse matrix, Jacobi fine scaling), whose patch width
must grow with the board, by

    M^-1 r = T^-1 r + Z_1 V_1(Z_1^T r)

* T: the z-line block of the operator (each node column's tridiagonal
  coupling along z), solved exactly;
* Z_l: aggregation of b x b non-empty nodes of one node layer, b = 4 from
  the fine grid to level 1, below it 2 on every level when the first coarse
  grid is more than 200 node columns across, else 4 (aggregate_width);
* A_{l+1} = Z_l^T A_l Z_l down to at most 2048 unknowns (dense solve there);
* V_l: one symmetric V-cycle, x = w T_l^-1 R, R_{l+1} = Z_l^T (R - A_l x),
  y' = x + Z_l V_{l+1}(R_{l+1}), y = y' + w T_l^-1 (R - A_l y'), w = 2/3.

A coarse node whose aggregate holds no non-empty node is empty: a unit row,
left out of the next restriction and of the prolongation.

The fine operator is assembled from the reference's element factors (3, S,
R, C), Robin totals and free mask exactly as the reference's operator acts
(operator.py:243-316): y = where(free, K (x * free) + R x, x) with
K_e = a_x M(x)M(x)S + a_y M(x)S(x)M + a_z S(x)M(x)M in the corner order
4 dz + 2 dy + dx (mesh.py:28-37, 346-359).
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl

AGGREGATE = 4  # aggregate width from the fine grid to level 1
WIDE_SIDE = 200  # a first coarse grid wider than this makes every coarse level aggregate 2 x 2
MAX_COARSE = 2048


def aggregate_width(level: int, first: tuple[int, int, int]) -> int:
    """Width of the aggregates that form level + 1 from level (0 = fine);
    `first` is the node shape of level 1."""

    if level == 0:
        return AGGREGATE
    return 2 if max(first[1], first[2]) > WIDE_SIDE else 4
OMEGA = 2.0 / 3.0

_M = np.array([[2.0, 1.0], [1.0, 2.0]]) / 6.0
_S = np.array([[1.0, -1.0], [-1.0, 1.0]])
UNIT = (np.kron(_M, np.kron(_M, _S)), np.kron(_M, np.kron(_S, _M)), np.kron(_S, np.kron(_M, _M)))


def assemble(coef: np.ndarray, robin_total: np.ndarray, free: np.ndarray) -> sp.csr_matrix:
    """The constrained FP64 operator as a sparse matrix (node order (z, y, x))."""

    coef = np.asarray(coef, dtype=np.float64)
    _, S, R, C = coef.shape
    shape = (S + 1, R + 1, C + 1)
    n = int(np.prod(shape))
    index = np.arange(n).reshape(shape)
    rows, cols, vals = [], [], []
    for i in range(8):
        iz, iy, ix = (i >> 2) & 1, (i >> 1) & 1, i & 1
        ni = index[iz:iz + S, iy:iy + R, ix:ix + C].reshape(-1)
        for j in range(8):
            jz, jy, jx = (j >> 2) & 1, (j >> 1) & 1, j & 1
            nj = index[jz:jz + S, jy:jy + R, jx:jx + C].reshape(-1)
            v = (coef[0] * UNIT[0][i, j] + coef[1] * UNIT[1][i, j] + coef[2] * UNIT[2][i, j]).reshape(-1)
            rows.append(ni)
            cols.append(nj)
            vals.append(v)
    K = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    f = np.asarray(free, dtype=bool).reshape(-1).astype(np.float64)
    P = sp.diags(f)
    A = P @ (K + sp.diags(np.asarray(robin_total, dtype=np.float64).reshape(-1))) @ P + sp.diags(1.0 - f)
    return A.tocsr()


class ZLine:
    """Exact solve of each node column's tridiagonal block (LDL^T)."""

    def __init__(self, A: sp.csr_matrix, shape: tuple[int, int, int]) -> None:
        L = shape[0]
        plane = shape[1] * shape[2]
        self.L, self.plane = L, plane
        d = A.diagonal().reshape(L, plane)
        up = A.diagonal(plane)  # A[i, i + plane]
        e = np.zeros((L, plane))
        e[:-1] = up.reshape(L - 1, plane)
        p = np.empty((L, plane))
        l = np.zeros((L, plane))
        p[0] = d[0]
        for z in range(1, L):
            l[z] = e[z - 1] / p[z - 1]
            p[z] = d[z] - l[z] * e[z - 1]
        self.l, self.p = l, p

    def __call__(self, r: np.ndarray) -> np.ndarray:
        L, l, p = self.L, self.l, self.p
        g = np.asarray(r, dtype=np.float64).reshape(L, self.plane).copy()
        for z in range(1, L):
            g[z] -= l[z] * g[z - 1]
        w = g / p
        for z in range(L - 2, -1, -1):
            w[z] -= l[z + 1] * w[z + 1]
        return w.reshape(-1)


def _aggregation(shape: tuple[int, int, int], keep: np.ndarray, width: int
                 ) -> tuple[sp.csr_matrix, tuple[int, int, int]]:
    L, ny, nx = shape
    cshape = (L, -(-ny // width), -(-nx // width))
    z, y, x = np.meshgrid(np.arange(L), np.arange(ny), np.arange(nx), indexing="ij")
    target = np.ravel_multi_index((z, y // width, x // width), cshape).reshape(-1)
    rows = np.flatnonzero(keep)
    Z = sp.csr_matrix((np.ones(rows.size), (rows, target[rows])), shape=(int(np.prod(shape)), int(np.prod(cshape))))
    return Z, cshape


class MultilevelOracle:
    """The hierarchy of the device's multilevel preconditioner, in FP64."""

    def __init__(self, coef: np.ndarray, robin_total: np.ndarray, free: np.ndarray) -> None:
        _, S, R, C = np.asarray(coef).shape
        self.node_shape = (S + 1, R + 1, C + 1)
        self.A = [assemble(coef, robin_total, free)]
        self.shapes = [self.node_shape]
        self.keep = [np.asarray(free, dtype=bool).reshape(-1)]
        self.Z: list[sp.csr_matrix] = []
        while True:
            Z, cshape = _aggregation(self.shapes[-1], self.keep[-1],
                                     aggregate_width(len(self.Z), self.shapes[min(1, len(self.shapes) - 1)]))
            Ac = (Z.T @ self.A[-1] @ Z).tocsr()
            empty = Ac.diagonal() == 0.0
            Ac = (Ac + sp.diags(empty.astype(np.float64))).tocsr()
            self.Z.append(Z)
            self.A.append(Ac)
            self.shapes.append(cshape)
            self.keep.append(~empty)
            if Ac.shape[0] <= MAX_COARSE or (cshape[1] == 1 and cshape[2] == 1):
                break
        self.smoothers = [ZLine(A, shape) for A, shape in zip(self.A[:-1], self.shapes[:-1])]
        self.coarsest = spl.splu(self.A[-1].tocsc())

    @property
    def grids(self) -> list[tuple[int, int, int]]:
        """Coarse grid shapes, level 1 first."""

        return list(self.shapes[1:])

    def stencil(self, level: int) -> np.ndarray:
        """Upper 27-point stencil (14, *shape) of coarse level `level` >= 1 in the
        device's layout (array k: A(i, i + d(13 + k)); empty nodes: centre 1)."""

        A = self.A[level].tocsr()
        L, ny, nx = self.shapes[level]
        out = np.zeros((14, L, ny, nx))
        z, y, x = np.meshgrid(np.arange(L), np.arange(ny), np.arange(nx), indexing="ij")
        i = np.ravel_multi_index((z, y, x), (L, ny, nx))
        for k in range(14):
            o = 13 + k
            dz, dy, dx = o // 9 - 1, (o // 3) % 3 - 1, o % 3 - 1
            jz, jy, jx = z + dz, y + dy, x + dx
            inside = (jz >= 0) & (jz < L) & (jy >= 0) & (jy < ny) & (jx >= 0) & (jx < nx)
            j = np.ravel_multi_index((np.clip(jz, 0, L - 1), np.clip(jy, 0, ny - 1), np.clip(jx, 0, nx - 1)),
                                     (L, ny, nx))
            vals = np.asarray(A[i.reshape(-1), j.reshape(-1)]).reshape(i.shape)
            out[k] = np.where(inside, vals, 0.0)
        return out

    def _vcycle(self, level: int, rhs: np.ndarray) -> np.ndarray:
        if level == len(self.A) - 1:
            return self.coarsest.solve(rhs)
        A, T = self.A[level], self.smoothers[level]
        x = OMEGA * T(rhs)
        coarse = self.Z[level].T @ (rhs - A @ x)
        y = x + self.Z[level] @ self._vcycle(level + 1, coarse)
        return y + OMEGA * T(rhs - A @ y)

    def precondition(self, r: np.ndarray) -> np.ndarray:
        r = np.asarray(r, dtype=np.float64).reshape(-1)
        return self.smoothers[0](r) + self.Z[0] @ self._vcycle(1, self.Z[0].T @ r)

    def pcg(self, b: np.ndarray, *, rtol: float = 1e-10, max_iterations: int = 100000):
        """FP64 PCG with this preconditioner; returns (x, iterations, relative residual)."""

        A = self.A[0]
        b = np.asarray(b, dtype=np.float64).reshape(-1)
        x = np.zeros_like(b)
        r = b.copy()
        bn = float(np.linalg.norm(b))
        if bn == 0.0:
            return x, 0, 0.0
        z = self.precondition(r)
        p = z.copy()
        rz = float(r @ z)
        rel = 1.0
        for it in range(1, max_iterations + 1):
            q = A @ p
            alpha = rz / float(p @ q)
            x += alpha * p
            r -= alpha * q
            rel = float(np.linalg.norm(r)) / bn
            if rel <= rtol:
                return x, it, rel
            z = self.precondition(r)
            rz_new = float(r @ z)
            p = z + (rz_new / rz) * p
            rz = rz_new
        return x, max_iterations, rel
