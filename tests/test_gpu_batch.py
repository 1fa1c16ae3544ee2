"""The batch engine (many boards in one set of graph-captured kernels) against
single-board solves, the oracle, and itself alone versus in a mix.

* every board converges to relative residual 1e-10, checked with the oracle's
  FP64 action (the engine's own residual is not trusted for this);
* temperatures agree with the single-board MPIR solve within rtol 1e-8
  (the two paths reduce in different orders, so bits differ);
* a board's solution, counts and history are bit-identical whether it is
  solved alone or admitted into a running mix of other boards;
* admission refuses boards beyond the byte budget or the slot count.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import OracleSystem
from pcb_analysis_b200.mpir import MPIRConfig

pytestmark = pytest.mark.gpu

CONFIG = MPIRConfig(inner_relative_tolerance=1e-4, max_outer_iterations=30, max_inner_iterations=100000)


def _board(seed: int, slabs: int, rows: int, cols: int, *, voids: bool = False, fixed: float = 0.0):
    rng = np.random.default_rng(seed)
    k_in = np.where(rng.random((slabs, rows, cols)) < 0.5, 385.0, 0.3)
    k_z = k_in * rng.uniform(0.5, 1.0, k_in.shape)
    if voids:
        void = rng.random(k_in.shape) < 0.08
        k_in = np.where(void, 0.0, k_in)
        k_z = np.where(void, 0.0, k_z)
    node_shape = (slabs + 1, rows + 1, cols + 1)
    robin = np.zeros(node_shape)
    robin[-1] = rng.uniform(0.5e-6, 2e-6, robin[-1].shape)
    robin[0] = rng.uniform(0.1e-6, 1e-6, robin[0].shape)
    free = np.ones(node_shape, dtype=np.uint8)
    if fixed > 0.0:
        free[0][rng.random(free[0].shape) < fixed] = 0
    if voids:
        live = k_in > 0
        touched = np.zeros(node_shape, dtype=bool)
        for dz in (0, 1):
            for dy in (0, 1):
                for dx in (0, 1):
                    touched[dz : dz + slabs, dy : dy + rows, dx : dx + cols] |= live
        free &= touched.astype(np.uint8)
    rhs = np.zeros(node_shape)
    rhs[-1] = rng.uniform(0.0, 1e-3, rhs[-1].shape) * (rng.random(rhs[-1].shape) < 0.05)
    rhs = rhs.reshape(-1)
    flat_free = free.reshape(-1)
    rhs[flat_free == 0] = rng.uniform(-2.0, 2.0, int((flat_free == 0).sum()))
    arrays = dict(
        slab_thickness_m=rng.uniform(0.035e-3, 0.4e-3, slabs), pitch_x_m=np.full(cols, 0.25e-3),
        pitch_y_m=np.full(rows, 0.25e-3), k_in=k_in, k_z=k_z, robin_total=robin.reshape(-1), free_nodes=flat_free,
    )
    return arrays, rhs


BOARDS = [
    dict(seed=1, slabs=3, rows=20, cols=33),
    dict(seed=2, slabs=5, rows=41, cols=17, fixed=0.2),
    dict(seed=3, slabs=8, rows=64, cols=64, voids=True),
    dict(seed=4, slabs=2, rows=7, cols=130),
    dict(seed=5, slabs=12, rows=30, cols=45, fixed=0.05),
    dict(seed=6, slabs=4, rows=96, cols=70),
]


def _drain(engine, count: int) -> dict[int, dict]:
    done: dict[int, dict] = {}
    for _ in range(200000):
        if len(done) >= count:
            break
        engine.step()
        for ticket in engine.finished():
            done[ticket] = engine.collect(ticket)
    assert len(done) == count
    return done


def _true_relative_residual(arrays, rhs, x) -> float:
    oracle = OracleSystem.from_arrays(free=arrays["free_nodes"], **{k: v for k, v in arrays.items() if k != "free_nodes"})
    return float(np.linalg.norm(rhs - oracle.apply_f64(x)) / np.linalg.norm(rhs))


def test_batched_boards_match_single_solves_and_converge() -> None:
    from pcb_analysis_b200._native import BatchEngine, DeviceSystem

    boards = [_board(**spec) for spec in BOARDS]
    with BatchEngine(capacity=8, max_slabs=16, tile_rows=16) as engine:
        tickets = [engine.submit(arrays, rhs, CONFIG) for arrays, rhs in boards]
        assert all(t is not None for t in tickets)
        results = _drain(engine, len(boards))
        assert engine.info()["resident"] == 0
    for (arrays, rhs), ticket in zip(boards, tickets):
        got = results[ticket]
        assert got["converged"]
        assert got["relative_residual"] <= 1e-10
        assert _true_relative_residual(arrays, rhs, got["solution"]) <= 1.0000001e-10
        assert len(got["history"]) == got["outer_iterations"]
        assert sum(step[2] for step in got["history"]) == got["inner_iterations"]
        assert got["high_operator_applications"] == got["outer_iterations"] + 1
        with DeviceSystem(**arrays) as dev:
            single = dev.solve_mpir(rhs, CONFIG)
        scale = np.abs(single["solution"]).max()
        np.testing.assert_allclose(got["solution"], single["solution"], rtol=1e-8, atol=1e-9 * scale)


def test_a_board_gives_the_same_bits_alone_and_in_a_mix() -> None:
    from pcb_analysis_b200._native import BatchEngine

    boards = [_board(**spec) for spec in BOARDS]
    target = 2
    with BatchEngine(capacity=8, max_slabs=16, tile_rows=16) as engine:
        alone = _drain_one(engine, *boards[target])
        early = [engine.submit(*boards[i], CONFIG) for i in (0, 4)]
        for _ in range(3):
            engine.step()
        mine = engine.submit(*boards[target], CONFIG)
        engine.step()
        late = [engine.submit(*boards[i], CONFIG) for i in (1, 3, 5)]
        results = _drain(engine, 6)
    mixed = results[mine]
    np.testing.assert_array_equal(mixed["solution"], alone["solution"])
    assert mixed["history"] == alone["history"]
    for key in ("outer_iterations", "inner_iterations", "relative_residual", "low_operator_applications"):
        assert mixed[key] == alone[key]
    assert all(t in results for t in early + late)


def _drain_one(engine, arrays, rhs):
    ticket = engine.submit(arrays, rhs, CONFIG)
    return _drain(engine, 1)[ticket]


def test_admission_refuses_what_does_not_fit_and_admits_after_collection() -> None:
    from pcb_analysis_b200._native import BatchEngine, engine_footprint

    a0, b0 = _board(**BOARDS[2])
    a1, b1 = _board(**BOARDS[5])
    r0, t0 = engine_footprint(a0)
    r1, t1 = engine_footprint(a1)
    budget = r0 + max(t0, t1) + r1 // 2  # room for board 0, not for board 1 beside it
    with BatchEngine(capacity=4, max_slabs=16, tile_rows=16, budget_bytes=budget) as engine:
        first = engine.submit(a0, b0, CONFIG)
        assert first is not None
        assert engine.info()["bytes_in_use"] == r0
        assert engine.submit(a1, b1, CONFIG) is None
        done = _drain(engine, 1)
        assert done[first]["converged"]
        second = engine.submit(a1, b1, CONFIG)
        assert second is not None
        assert _drain(engine, 1)[second]["converged"]
    with BatchEngine(capacity=1, max_slabs=16, tile_rows=16) as engine:
        assert engine.submit(a0, b0, CONFIG) is not None
        assert engine.submit(a1, b1, CONFIG) is None


def test_autotuned_tile_height_and_a_zero_right_hand_side() -> None:
    from pcb_analysis_b200._native import BatchEngine

    boards = [_board(**spec) for spec in BOARDS[:4]]
    with BatchEngine(capacity=8, max_slabs=16, tile_rows=0) as engine:
        tickets = [engine.submit(arrays, rhs, CONFIG) for arrays, rhs in boards]
        zero = engine.submit(boards[0][0], np.zeros_like(boards[0][1]), CONFIG)
        results = _drain(engine, len(tickets) + 1)
        assert engine.info()["tile_rows"] in (8, 16, 32)
    for (arrays, rhs), ticket in zip(boards, tickets):
        assert results[ticket]["converged"]
        assert _true_relative_residual(arrays, rhs, results[ticket]["solution"]) <= 1.0000001e-10
    assert results[zero]["converged"] and results[zero]["inner_iterations"] == 0
    assert not np.any(results[zero]["solution"])


def test_two_level_batch_matches_single_two_level_solves() -> None:
    from pcb_analysis_b200._native import BatchEngine, DeviceSystem

    boards = [_board(**spec) for spec in BOARDS]
    with BatchEngine(capacity=8, max_slabs=16, tile_rows=16, preconditioner="two-level") as engine:
        tickets = [engine.submit(arrays, rhs, CONFIG) for arrays, rhs in boards]
        results = _drain(engine, len(boards))
    for (arrays, rhs), ticket in zip(boards, tickets):
        got = results[ticket]
        assert got["converged"] and got["relative_residual"] <= 1e-10
        assert _true_relative_residual(arrays, rhs, got["solution"]) <= 1.0000001e-10
        with DeviceSystem(**arrays) as dev:
            dev.set_preconditioner("two-level")
            single = dev.solve_mpir(rhs, CONFIG)
            dev.set_preconditioner("jacobi")
            jacobi = dev.solve_mpir(rhs, CONFIG)
        assert got["inner_iterations"] <= jacobi["inner_iterations"]
        scale = np.abs(single["solution"]).max()
        np.testing.assert_allclose(got["solution"], single["solution"], rtol=1e-8, atol=1e-9 * scale)


def test_two_level_board_gives_the_same_bits_alone_and_in_a_mix() -> None:
    from pcb_analysis_b200._native import BatchEngine

    boards = [_board(**spec) for spec in BOARDS]
    with BatchEngine(capacity=8, max_slabs=16, tile_rows=16, preconditioner="two-level") as engine:
        alone = _drain_one(engine, *boards[4])
        first = [engine.submit(*boards[i], CONFIG) for i in (0, 2)]
        engine.step()
        mine = engine.submit(*boards[4], CONFIG)
        late = [engine.submit(*boards[i], CONFIG) for i in (1, 5)]
        results = _drain(engine, 5)
    np.testing.assert_array_equal(results[mine]["solution"], alone["solution"])
    assert results[mine]["history"] == alone["history"]
    assert all(t in results for t in first + late)


@pytest.mark.parametrize("preconditioner", ["jacobi", "two-level"])
def test_tensor_copy_staging_gives_the_batch_the_same_bits(preconditioner: str) -> None:
    """The batched operator fed by tensor copies (each board's maps in the
    engine's device memory, acquired before use) reproduces the cp.async-fed
    engine bit for bit: solutions, counts and histories of every board, also
    after slots are reused by later boards."""

    from pcb_analysis_b200._native import BatchEngine

    boards = [_board(**spec) for spec in BOARDS]
    runs = {}
    for staging in ("cp.async", "tensor"):
        with BatchEngine(capacity=3, max_slabs=16, tile_rows=8, preconditioner=preconditioner,
                         staging=staging) as engine:
            assert engine.info()["staging"] == staging
            first = [engine.submit(*boards[i], CONFIG) for i in range(3)]
            done = _drain(engine, 3)
            later = [engine.submit(*boards[i], CONFIG) for i in range(3, 6)]  # the freed slots, new maps
            done.update(_drain(engine, 3))
        runs[staging] = [done[t] for t in first + later]
    for plain, staged in zip(runs["cp.async"], runs["tensor"]):
        assert staged["converged"]
        np.testing.assert_array_equal(staged["solution"], plain["solution"])
        assert staged["history"] == plain["history"]
        assert staged["inner_iterations"] == plain["inner_iterations"]


def test_autotuned_engine_reports_its_staging() -> None:
    from pcb_analysis_b200._native import BatchEngine

    arrays, rhs = _board(**BOARDS[2])
    with BatchEngine(capacity=2, max_slabs=16) as engine:
        got = _drain_one(engine, arrays, rhs)
        info = engine.info()
        assert info["tile_rows"] in (8, 16, 32) and info["staging"] in ("cp.async", "tensor")
    assert got["converged"] and _true_relative_residual(arrays, rhs, got["solution"]) <= 1.0000001e-10


# Boards of different slab counts with more tiles than the 592 resident blocks
# of the 8-row operator, so that a block walks tiles of several boards.
WALK_BOARDS = [
    dict(seed=11, slabs=3, rows=200, cols=300),
    dict(seed=12, slabs=7, rows=300, cols=300),
    dict(seed=13, slabs=12, rows=250, cols=400, fixed=0.02),
    dict(seed=14, slabs=5, rows=350, cols=280),
]


def test_tensor_copy_staging_across_boards_of_different_slab_counts() -> None:
    """A block of the batched operator that moves from a tile of one board to
    a tile of another keeps its stage barriers (their place does not depend on
    the slab count) and its phase count: the tensor-copy engine reproduces the
    cp.async engine bit for bit when blocks walk boards of 3, 5, 7 and 12
    slabs."""

    from pcb_analysis_b200._native import BatchEngine

    boards = [_board(**spec) for spec in WALK_BOARDS]
    runs = {}
    for staging in ("cp.async", "tensor"):
        with BatchEngine(capacity=4, max_slabs=16, tile_rows=8, staging=staging) as engine:
            tickets = [engine.submit(arrays, rhs, CONFIG) for arrays, rhs in boards]
            launch_ms = engine.time_apply(2)  # the store-epilogue launch walks the boards too
            done = _drain(engine, len(boards))
        assert launch_ms > 0.0
        runs[staging] = [done[t] for t in tickets]
    for plain, staged in zip(runs["cp.async"], runs["tensor"]):
        assert staged["converged"] and staged["relative_residual"] <= 1e-10
        np.testing.assert_array_equal(staged["solution"], plain["solution"])
        assert staged["inner_iterations"] == plain["inner_iterations"]
