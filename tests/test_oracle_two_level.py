"""The oracle's two-level coarse space against the reference's
(tests/golden/coarse, recorded by make_golden_coarse.py)."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import CoarseSpaceOracle, OracleSystem, choose_block_size
from tests.conftest import load_golden

COARSE = Path(__file__).resolve().parent / "golden" / "coarse"
CASES = sorted(p.stem for p in COARSE.glob("*.npz"))


def _case(tag: str):
    name, _, block = tag.rpartition("_b")
    if not name or not block.isdigit():
        name, block = tag, ""
    return name, (int(block) if block else None)


@pytest.mark.parametrize("tag", CASES)
def test_coarse_space_matches_the_reference(tag: str) -> None:
    name, block = _case(tag)
    g = load_golden(name)
    ref = np.load(COARSE / f"{tag}.npz")
    oracle = OracleSystem(g["coef"], g["robin_total"], g["free"])
    cs = CoarseSpaceOracle(oracle, block=block)
    assert cs.block == int(ref["block"])
    assert tuple(cs.coarse_shape) == tuple(ref["coarse_shape"])
    scale = np.abs(ref["coarse_matrix"]).max()
    np.testing.assert_allclose(cs.coarse_matrix, ref["coarse_matrix"], rtol=0, atol=64 * np.finfo(float).eps * scale)
    inv_scale = np.abs(ref["coarse_inverse"]).max()
    np.testing.assert_allclose(cs.coarse_inverse, ref["coarse_inverse"], rtol=0, atol=1e-9 * inv_scale)
    y = cs.precondition_f64(g["v64"])
    np.testing.assert_allclose(y, ref["precondition_high"], rtol=0, atol=1e-9 * np.abs(ref["precondition_high"]).max())


def test_block_choice_follows_the_size_cap() -> None:
    assert choose_block_size((5, 25, 31)) == 4
    assert choose_block_size((5, 81, 81)) == 5
    assert choose_block_size((13, 513, 513)) == 43
    assert choose_block_size((17, 2049, 2049)) == 205


def test_two_level_pcg_reaches_the_reference_temperatures() -> None:
    g = load_golden("seeded_board_24x30")
    oracle = OracleSystem(g["coef"], g["robin_total"], g["free"])
    cs = CoarseSpaceOracle(oracle)
    x, its, rel = cs.pcg_f64(g["rhs"], rtol=1e-11)
    _, jacobi_its, _ = oracle.pcg_f64(g["rhs"], rtol=1e-11)
    assert rel <= 1e-11 and its < jacobi_its
    t = x + float(g["reference_temperature"])
    ref = g["two_level_temperature"]
    finite = np.isfinite(ref)
    np.testing.assert_allclose(t[finite], ref[finite], rtol=1e-8, atol=1e-7)
