"""The multilevel preconditioner's CPU restatement (oracle/multilevel.py).

* Its assembled operator is the oracle's matrix-free action (itself pinned to
  the reference's apply_high on the golden cases): within 64 eps of ||y||.
* Its preconditioner is a symmetric positive-definite linear map (within
  1e-12 relative), as a plain PCG needs.
* On a copper stack it takes far fewer PCG iterations than Jacobi and than
  the reference's two-level preconditioner at its own patch width.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle.multilevel import MultilevelOracle, assemble
from oracle.oracle import CoarseSpaceOracle, OracleSystem
from tests.conftest import golden_cases, load_golden


def _board(slabs, rows, cols, seed, fixed=0.0):
    rng = np.random.default_rng(seed)
    k_in = np.where(rng.random((slabs, rows, cols)) < 0.6, 385.0, 0.3)
    k_in[1::2] = 0.3  # copper slabs between FR-4 slabs
    node_shape = (slabs + 1, rows + 1, cols + 1)
    robin = np.zeros(node_shape)
    robin[-1] = 25.0 * 0.0625e-6
    robin[0] = 5.0 * 0.0625e-6
    free = np.ones(node_shape, dtype=np.uint8)
    if fixed:
        free[0, :, : max(1, int(fixed * (cols + 1)))] = 0
    thick = np.where(np.arange(slabs) % 2 == 0, 35e-6, 0.16e-3)
    return OracleSystem.from_arrays(slab_thickness_m=thick, pitch_x_m=np.full(cols, 0.25e-3),
                                    pitch_y_m=np.full(rows, 0.25e-3), k_in=k_in, k_z=k_in,
                                    robin_total=robin.reshape(-1), free=free.reshape(-1))


@pytest.mark.parametrize("name", golden_cases())
def test_assembled_operator_is_the_oracle_action(name: str) -> None:
    g = load_golden(name)
    oracle = OracleSystem(g["coef"], g["robin_total"], g["free"])
    A = assemble(g["coef"], g["robin_total"], g["free"])
    x = np.random.default_rng(1).standard_normal(oracle.size)
    y = oracle.apply_f64(x)
    assert np.linalg.norm(A @ x - y) <= 64 * np.finfo(np.float64).eps * np.linalg.norm(y)


def test_preconditioner_is_symmetric_positive_definite() -> None:
    oracle = _board(7, 72, 84, seed=3, fixed=0.1)
    ml = MultilevelOracle(oracle.coef, oracle.robin_total, oracle.free)
    assert len(ml.grids) >= 2  # a V-cycle level above the dense grid
    rng = np.random.default_rng(5)
    u, v = rng.standard_normal(oracle.size), rng.standard_normal(oracle.size)
    mu, mv = ml.precondition(u), ml.precondition(v)
    assert abs(u @ mv - v @ mu) <= 1e-12 * np.linalg.norm(u) * np.linalg.norm(mv)
    assert u @ mu > 0 and v @ mv > 0


def test_iterations_are_far_below_jacobi_and_two_level() -> None:
    oracle = _board(9, 120, 120, seed=7, fixed=0.05)
    b = np.where(oracle.free.astype(bool), np.random.default_rng(2).random(oracle.size), 0.0)
    ml = MultilevelOracle(oracle.coef, oracle.robin_total, oracle.free)
    x_ml, it_ml, rel = ml.pcg(b, rtol=1e-8)
    _, it_2l, _ = CoarseSpaceOracle(oracle).pcg_f64(b, rtol=1e-8)
    x_j, it_j, _ = oracle.pcg_f64(b, rtol=1e-8)
    assert rel <= 1e-8
    assert it_ml * 3 < it_2l and it_ml * 10 < it_j, (it_ml, it_2l, it_j)
    np.testing.assert_allclose(x_ml, x_j, rtol=0, atol=1e-6 * np.abs(x_j).max())
