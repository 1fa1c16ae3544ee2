"""CPU oracle of the layered DC operator (NumPy restatement).

TEST INFRASTRUCTURE: the checker of the device's layered DC kernels; only
tests/ import it.  It restates the reference's NumPy operator
(src/electrical/matrix_free_mpir_fem/pcb.py): element coefficients
(:171-186), masks (:333-370), the element action with vias (:575-596), the
diagonal (:598-617), the unconstrained action (:702-724) and the right-hand
side (:770-808), and is pinned to the golden vectors recorded from the
reference (tests/golden/dc).  Plain NumPy over whole grids: it is meant for
boards of at most some 10^5 nodes.
"""

from __future__ import annotations

import numpy as np

_S = np.array([[1.0, -1.0], [-1.0, 1.0]])
_M = np.array([[2.0, 1.0], [1.0, 2.0]]) / 6.0
UNIT = np.stack((np.kron(_M, _S), np.kron(_S, _M)))  # U_x, U_y in local order 2 dy + dx


def _views(grid: np.ndarray) -> tuple[np.ndarray, ...]:
    return grid[:, :-1, :-1], grid[:, :-1, 1:], grid[:, 1:, :-1], grid[:, 1:, 1:]


class DcOracle:
    """The reference's layered DC operator on the host, from plain arrays.

    ``active`` (L, R, C) elements, ``thickness`` (L), ``px`` (C), ``py`` (R),
    ``sigma`` (L, R, C); vias as flat node index arrays and conductances;
    ``reference`` flat node or -1; ``dirichlet`` flat nodes.
    """

    def __init__(self, active, thickness, px, py, sigma, via_a=(), via_b=(), via_g=(), reference=-1, dirichlet=()):
        self.active = np.asarray(active, dtype=bool)
        layers, rows, cols = self.active.shape
        self.node_shape = (layers, rows + 1, cols + 1)
        self.size = int(np.prod(self.node_shape))
        thickness = np.asarray(thickness, dtype=np.float64)[:, None, None]
        sheet = np.asarray(sigma, dtype=np.float64) * thickness * self.active.astype(np.float64)
        hx = np.asarray(px, dtype=np.float64)[None, None, :]
        hy = np.asarray(py, dtype=np.float64)[None, :, None]
        self.coef = np.stack((sheet * hy / hx, sheet * hx / hy))
        self.via_a = np.asarray(via_a, dtype=np.int64)
        self.via_b = np.asarray(via_b, dtype=np.int64)
        self.via_g = np.asarray(via_g, dtype=np.float64)
        active_nodes = np.zeros(self.node_shape, dtype=bool)
        for view in _views(active_nodes):
            view |= self.active
        active_nodes.flat[self.via_a] = True
        active_nodes.flat[self.via_b] = True
        fixed = ~active_nodes
        if reference >= 0:
            fixed.flat[int(reference)] = True
        fixed.flat[np.asarray(dirichlet, dtype=np.int64)] = True
        self.active_nodes = active_nodes
        self.free = ~fixed

    def _action(self, vector: np.ndarray, free: np.ndarray) -> np.ndarray:
        grid = np.asarray(vector, dtype=np.float64).reshape(self.node_shape)
        working = np.where(free, grid, 0.0)
        values = _views(working)
        out = np.zeros_like(working)
        targets = _views(out)
        for row in range(4):
            contribution = np.zeros_like(self.coef[0])
            for column in range(4):
                weight = self.coef[0] * UNIT[0, row, column] + self.coef[1] * UNIT[1, row, column]
                contribution = contribution + weight * values[column]
            targets[row][...] += contribution
        flat_w = working.reshape(-1)
        flat_out = out.reshape(-1)
        if self.via_a.size:
            delta = self.via_g * (flat_w[self.via_a] - flat_w[self.via_b])
            np.add.at(flat_out, self.via_a, delta)
            np.add.at(flat_out, self.via_b, -delta)
        return np.where(free.reshape(-1), flat_out, np.asarray(vector, dtype=np.float64).reshape(-1))

    def apply_f64(self, vector: np.ndarray) -> np.ndarray:
        """where(free, K (x * free) + vias, x)."""

        return self._action(vector, self.free)

    def apply_full(self, vector: np.ndarray) -> np.ndarray:
        """K x with every node free (the current leaving each node)."""

        return self._action(vector, np.ones(self.node_shape, dtype=bool))

    def diagonal(self) -> np.ndarray:
        diag = np.zeros(self.node_shape)
        for index, target in enumerate(_views(diag)):
            target[...] += self.coef[0] * UNIT[0, index, index] + self.coef[1] * UNIT[1, index, index]
        flat = diag.reshape(-1)
        if self.via_a.size:
            np.add.at(flat, self.via_a, self.via_g)
            np.add.at(flat, self.via_b, self.via_g)
        return np.where(self.free.reshape(-1), flat, 1.0)

    def dense(self) -> np.ndarray:
        """The operator as a dense matrix (small boards)."""

        eye = np.eye(self.size)
        return np.column_stack([self.apply_f64(eye[:, j]) for j in range(self.size)])

    def solve(self, rhs: np.ndarray) -> np.ndarray:
        """Direct FP64 solve of the constrained system (small boards)."""

        return np.linalg.solve(self.dense(), np.asarray(rhs, dtype=np.float64))


def from_problem(problem) -> DcOracle:
    """The oracle of a PCBConductionProblem (either implementation's records)."""

    mesh = problem.mesh
    shape = mesh.node_shape
    flat = lambda node: int(np.ravel_multi_index(node, shape))  # noqa: E731
    return DcOracle(
        mesh.element_active, mesh.layer_thickness_m, mesh.pitch_x_m, mesh.pitch_y_m, mesh.conductivity_s_per_m,
        [flat(v.lower) for v in problem.vias], [flat(v.upper) for v in problem.vias],
        [v.conductance_s for v in problem.vias],
        -1 if problem.reference_node is None else flat(problem.reference_node),
        [flat(node) for t in problem.voltage_terminals for node in t.nodes],
    )
