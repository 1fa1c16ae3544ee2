"""Device operator actions against the CPU oracle and the reference's golden vectors.

Tolerances:
* FP64 action and unconstrained stiffness: ||y - y_ref|| <= 64 eps64 ||y_ref||
  (the reference's native parity bound, tests/test_native_thermal.py:94);
* FP32 action: ||y32 - A64 x|| <= 16 eps32 ||A64 x||, against the exact FP64
  action of the same FP32 input (the device kernel rounds differently from the
  reference's FP32 gather, so it is held to the FP64 truth instead);
* fixed rows are copied exactly; the Jacobi diagonal is bit-identical to the
  reference's; repeated actions are bit-identical (node-owned, no atomics).
"""

from __future__ import annotations

import numpy as np
import pytest

import pcb_analysis_b200.thermal as ns
from oracle.oracle import OracleSystem
from pcb_analysis_b200.thermal.system import prepare
from tests.conftest import golden_cases, load_golden
from tests.problems import CASES

pytestmark = pytest.mark.gpu

EPS64 = np.finfo(np.float64).eps
EPS32 = np.finfo(np.float32).eps


def _operator(problem):
    return ns.MatrixFreeThermalOperator(problem, preconditioner="jacobi")


@pytest.mark.parametrize("name", golden_cases())
def test_device_actions_match_the_golden_vectors(name: str) -> None:
    g = load_golden(name)
    op = _operator(CASES[name](ns))
    try:
        assert op.low_operator_backend == "b200-haar-zmarch-hex-q1"
        y64 = op.apply_high(g["v64"])
        assert np.linalg.norm(y64 - g["apply_high"]) <= 64 * EPS64 * np.linalg.norm(g["apply_high"])
        fixed = g["free"] == 0
        np.testing.assert_array_equal(y64[fixed], g["v64"][fixed])
        k64 = op.stiffness_high(g["v64"])
        assert np.linalg.norm(k64 - g["stiffness"]) <= 64 * EPS64 * np.linalg.norm(g["stiffness"])
        np.testing.assert_array_equal(op.diagonal_high(), g["diagonal"])

        oracle = OracleSystem(g["coef"], g["robin_total"], g["free"])
        exact = oracle.apply_f64(g["v32"].astype(np.float64))
        y32 = op.apply_low(g["v32"])
        assert y32.dtype == np.float32
        assert np.linalg.norm(y32 - exact) <= 16 * EPS32 * np.linalg.norm(exact)
        np.testing.assert_array_equal(y32[fixed], g["v32"][fixed])
        np.testing.assert_array_equal(op.apply_low(g["v32"]), y32)
        np.testing.assert_array_equal(op.apply_high(g["v64"]), y64)
    finally:
        op.close()


def _random_system(slabs, rows, cols, seed, voids=False, fixed_frac=0.05, robin_planes="tb"):
    rng = np.random.default_rng(seed)
    thickness = rng.uniform(0.03e-3, 0.5e-3, slabs)
    px = rng.uniform(0.1e-3, 0.4e-3, cols)
    py = rng.uniform(0.1e-3, 0.4e-3, rows)
    k_in = np.where(rng.random((slabs, rows, cols)) < 0.5, 385.0, 0.3)
    k_z = k_in * rng.uniform(0.5, 1.0, k_in.shape)
    if voids:
        void = rng.random(k_in.shape) < 0.1
        k_in = np.where(void, 0.0, k_in)
        k_z = np.where(void, 0.0, k_z)
    n = (slabs + 1) * (rows + 1) * (cols + 1)
    robin = np.zeros((slabs + 1, rows + 1, cols + 1))
    if "t" in robin_planes:
        robin[-1] = rng.uniform(0.0, 1e-5, robin[-1].shape)
    if "b" in robin_planes:
        robin[0] = rng.uniform(0.0, 1e-5, robin[0].shape)
    if "a" in robin_planes:
        robin += rng.uniform(0.0, 1e-6, robin.shape)
    free = (rng.random(n) >= fixed_frac).astype(np.uint8)
    if voids:
        # nodes touched by no conducting element are fixed, as the front end does
        touched = np.zeros((slabs + 1, rows + 1, cols + 1), dtype=bool)
        live = k_in > 0
        for dz in (0, 1):
            for dy in (0, 1):
                for dx in (0, 1):
                    touched[dz : dz + slabs, dy : dy + rows, dx : dx + cols] |= live
        free &= touched.reshape(-1).astype(np.uint8)
    free = free.reshape(-1)
    robin = robin.reshape(-1)
    return dict(slab_thickness_m=thickness, pitch_x_m=px, pitch_y_m=py, k_in=k_in, k_z=k_z,
                robin_total=robin, free=free)


# Shapes straddling the 60 x 15 output tile of the kernel and its halos.
SHAPES = [
    (1, 1, 1), (1, 1, 2), (2, 3, 1), (1, 14, 59), (2, 15, 60), (3, 16, 61), (1, 13, 58),
    (4, 29, 119), (5, 30, 120), (2, 31, 121), (6, 46, 200), (9, 17, 63), (1, 1, 300), (3, 200, 1),
]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("variant", ["plain", "voids_allrobin"])
def test_device_actions_match_the_oracle_on_ragged_shapes(shape, variant) -> None:
    from pcb_analysis_b200._native import DeviceSystem

    slabs, rows, cols = shape
    arrays = _random_system(slabs, rows, cols, seed=sum(shape),
                            voids=variant != "plain", robin_planes="tba" if variant != "plain" else "tb")
    free = arrays.pop("free")
    oracle = OracleSystem.from_arrays(free=free, **arrays)
    dev = DeviceSystem(free_nodes=free, **arrays)
    try:
        assert dev.tile_rows in (8, 16, 32)
        rng = np.random.default_rng(7)
        x = rng.standard_normal(oracle.size)
        ref = oracle.apply_f64(x)
        ks = oracle.stiffness_f64(x)
        x32 = x.astype(np.float32)
        exact = oracle.apply_f64(x32.astype(np.float64))
        np.testing.assert_array_equal(dev.diagonal(), oracle.diagonal())
        outputs = []
        for rows in (8, 16, 32):  # every tile height of the kernel
            dev.tile_rows = rows
            y = dev.apply_f64(x)
            assert np.linalg.norm(y - ref) <= 64 * EPS64 * np.linalg.norm(ref)
            np.testing.assert_array_equal(y[free == 0], x[free == 0])
            assert np.linalg.norm(dev.stiffness_f64(x) - ks) <= 64 * EPS64 * np.linalg.norm(ks)
            y32 = dev.apply_f32(x32)
            assert np.linalg.norm(y32 - exact) <= 16 * EPS32 * np.linalg.norm(exact)
            np.testing.assert_array_equal(y32[free == 0], x32[free == 0])
            outputs.append(y32)
        # the element arithmetic does not depend on the tiling: same bits
        np.testing.assert_array_equal(outputs[0], outputs[1])
        np.testing.assert_array_equal(outputs[1], outputs[2])
    finally:
        dev.close()


def test_constant_field_maps_to_the_robin_term_exactly() -> None:
    """K 1 = 0: with no fixed nodes only the lumped Robin conductance survives
    (tests/test_thermal_conduction.py:60-68), here without round-off at all."""

    problem = ns.ThermalConductionProblem(
        ns.LayeredThermalMesh((35e-6, 0.4e-3), 0.2e-3, 0.3e-3, np.array(
            [[[385.0, 385.0], [0.8, 385.0]], [[0.8, 0.8], [0.8, 385.0]]]), through_plane_conductivity_w_per_m_k=(385.0, 0.3)),
        convection=(ns.ConvectionBoundary("top", 12.0, 300.0),),
    )
    op = _operator(problem)
    try:
        ones = np.ones(op.size)
        action = op.apply_high(ones).reshape(problem.mesh.node_shape)
        assert np.all(action[:-1] == 0.0)
        np.testing.assert_array_equal(action[-1].reshape(-1), prepare(problem).robin_total.reshape(problem.mesh.node_shape)[-1].reshape(-1))
        low = op.apply_low(ones.astype(np.float32)).reshape(problem.mesh.node_shape)
        assert np.all(low[:-1] == 0.0)
    finally:
        op.close()


def test_device_pointer_entry_points_match_the_host_ones() -> None:
    import torch

    g = load_golden("mixed_board")
    op = _operator(CASES["mixed_board"](ns))
    try:
        x = torch.as_tensor(g["v32"], device="cuda")
        y = op.apply_low(x)
        assert y.is_cuda and y.dtype == torch.float32
        np.testing.assert_array_equal(y.cpu().numpy(), op.apply_low(g["v32"]))
        x64 = torch.as_tensor(g["v64"], device="cuda")
        y64 = torch.empty_like(x64)
        op.device_system.apply_f64_device(x64, y64)
        np.testing.assert_array_equal(y64.cpu().numpy(), op.apply_high(g["v64"]))
    finally:
        op.close()


def _faces_only_system(slabs, rows, cols, seed):
    """Robin terms and fixed nodes on the bottom and top planes only (a plain board)."""

    arrays = _random_system(slabs, rows, cols, seed, fixed_frac=0.0)
    rng = np.random.default_rng(seed + 1)
    free = np.ones((slabs + 1, rows + 1, cols + 1), dtype=np.uint8)
    free[0][rng.random(free[0].shape) < 0.1] = 0
    free[-1][rng.random(free[-1].shape) < 0.05] = 0
    arrays["free"] = free.reshape(-1)
    return arrays


WARP_SHAPES = [(1, 1, 1), (1, 3, 40), (2, 17, 33), (3, 16, 61), (5, 30, 120), (8, 40, 90), (12, 37, 70),
               (13, 21, 45), (16, 33, 65), (4, 200, 3), (7, 5, 300)]


@pytest.mark.parametrize("shape", WARP_SHAPES)
def test_warp_march_kernel_matches_the_oracle_in_every_decomposition(shape) -> None:
    """Every (z groups, slabs per lane, band) launch shape of the warp-marching
    kernel gives the oracle's action, and all of them the same bits (the sum
    at a node runs in one order whatever the decomposition)."""

    from pcb_analysis_b200._native import DeviceSystem

    slabs, rows, cols = shape
    arrays = _faces_only_system(slabs, rows, cols, seed=sum(shape) + 11)
    free = arrays.pop("free")
    oracle = OracleSystem.from_arrays(free=free, **arrays)
    dev = DeviceSystem(free_nodes=free, **arrays)
    try:
        x32 = np.random.default_rng(5).standard_normal(oracle.size).astype(np.float32)
        exact = oracle.apply_f64(x32.astype(np.float64))
        dev.apply_plan = (0, 16, 0, 0, 0)
        tiles = dev.apply_f32(x32)
        assert np.linalg.norm(tiles - exact) <= 16 * EPS32 * np.linalg.norm(exact)
        tried = 0
        first = None
        for zw in (1, 2, 4):
            for sl in range(-(-slabs // zw), 9):
                for band in (4, 8, 64):
                    try:
                        dev.apply_plan = (1, 16, zw, sl, band)
                    except ValueError:
                        continue
                    y32 = dev.apply_f32(x32)
                    assert np.linalg.norm(y32 - exact) <= 16 * EPS32 * np.linalg.norm(exact), (zw, sl, band)
                    np.testing.assert_array_equal(y32[free == 0], x32[free == 0])
                    if first is None:
                        first = y32
                    np.testing.assert_array_equal(y32, first)
                    tried += 1
                break  # the smallest slab count per lane that exists for this group count
        assert tried >= 3 or slabs > 32
    finally:
        dev.close()


# Boards whose tile count sits just above a wave (c2-like), far below one, and
# with fewer (tile, plane) pairs than resident blocks.
SPLIT_SHAPES = [(1, 1, 1), (1, 3, 5), (2, 15, 60), (12, 40, 130), (3, 70, 61), (12, 200, 300), (16, 90, 33),
                (12, 512, 512)]


@pytest.mark.parametrize("shape", SPLIT_SHAPES)
def test_balanced_launch_writes_the_same_bits_as_one_block_per_tile(shape) -> None:
    """The one-wave launch that splits the board's tile planes evenly over the
    blocks (plan kind 2) writes every node with the operations of the
    one-block-per-tile launch, so the outputs agree bit for bit, with Robin
    terms and fixed nodes on every plane and with void elements."""

    from pcb_analysis_b200._native import DeviceSystem

    slabs, rows, cols = shape
    arrays = _random_system(slabs, rows, cols, seed=sum(shape) + 3, voids=True, robin_planes="tba")
    free = arrays.pop("free")
    dev = DeviceSystem(free_nodes=free, **arrays)
    try:
        x32 = np.random.default_rng(7).standard_normal(dev.size).astype(np.float32)
        for rows_variant in (8, 16, 32):
            dev.apply_plan = (0, rows_variant, 0, 0, 0)
            tiles = dev.apply_f32(x32)
            dev.apply_plan = (2, rows_variant, 0, 0, 0)
            balanced = dev.apply_f32(x32)
            np.testing.assert_array_equal(balanced, tiles)
            assert dev.apply_plan[0] == 2
        if slabs * rows * cols <= 200_000:
            oracle = OracleSystem.from_arrays(free=free, **arrays)
            exact = oracle.apply_f64(x32.astype(np.float64))
            assert np.linalg.norm(balanced - exact) <= 16 * EPS32 * np.linalg.norm(exact)
    finally:
        dev.close()


# Ragged shapes for the tensor-copy staging: tiles cut by every edge, one and
# many slabs, Robin terms and fixed nodes on every plane, void elements.
TMA_SHAPES = [(1, 1, 1), (1, 3, 5), (2, 15, 60), (3, 16, 61), (12, 40, 130), (5, 70, 200), (16, 33, 64),
              (12, 200, 300)]


@pytest.mark.parametrize("shape", TMA_SHAPES)
def test_tensor_copy_staging_writes_the_same_bits_as_cp_async(shape) -> None:
    """The z-march kernels fed by tensor copies (one thread per block issues
    the plane's tiles onto an mbarrier; plan5[2] = 1) compute with the
    operations of the cp.async-fed kernels, so every tile height and both
    launch kinds give the same bits, and the oracle's action; so do the
    five-stage tensor-copy tiles (plan5[3] = 5, three planes in flight)."""

    from pcb_analysis_b200._native import DeviceSystem

    slabs, rows, cols = shape
    arrays = _random_system(slabs, rows, cols, seed=sum(shape) + 23, voids=True, robin_planes="tba")
    free = arrays.pop("free")
    dev = DeviceSystem(free_nodes=free, **arrays)
    try:
        x32 = np.random.default_rng(13).standard_normal(dev.size).astype(np.float32)
        for kind in (0, 2):
            for rows_variant in (8, 16, 32):
                dev.apply_plan = (kind, rows_variant, 0, 0, 0)
                plain = dev.apply_f32(x32)
                dev.apply_plan = (kind, rows_variant, 1, 0, 0)
                assert tuple(dev.apply_plan) == (kind, rows_variant, 1, 0, 0)
                staged = dev.apply_f32(x32)
                np.testing.assert_array_equal(staged, plain, err_msg=f"kind {kind}, {rows_variant} rows")
                np.testing.assert_array_equal(dev.apply_f32(x32), staged)
                if kind == 0 and rows_variant <= 16:  # three planes in flight instead of two
                    dev.apply_plan = (0, rows_variant, 1, 5, 0)
                    assert tuple(dev.apply_plan) == (0, rows_variant, 1, 5, 0)
                    np.testing.assert_array_equal(dev.apply_f32(x32), plain, err_msg=f"5 stages, {rows_variant} rows")
                    np.testing.assert_array_equal(dev.apply_f32(x32), plain)
        if slabs * rows * cols <= 200_000:
            oracle = OracleSystem.from_arrays(free=free, **arrays)
            exact = oracle.apply_f64(x32.astype(np.float64))
            assert np.linalg.norm(staged - exact) <= 16 * EPS32 * np.linalg.norm(exact)
            np.testing.assert_array_equal(staged[free == 0], x32[free == 0])
        with pytest.raises(ValueError):
            dev.apply_plan = (0, 16, 2, 0, 0)
        for plan in ((2, 16, 1, 5, 0), (0, 32, 1, 5, 0), (0, 16, 0, 5, 0), (0, 16, 1, 6, 0)):
            with pytest.raises(ValueError):
                dev.apply_plan = plan
    finally:
        dev.close()
