"""The CPU oracle against the golden vectors recorded from the reference.

Pins oracle/thermal_oracle.c before it is trusted as the checker of the device
kernels: the FP64 and FP32 actions within the reference's own native-parity
tolerances (tests/test_native_thermal.py:72,94 of pcb-analysis), the
diagonal to the bit, and the solves within the cross-implementation tolerance
of tests/test_cuda_thermal_conduction.py:101 (rtol 1e-8, atol 1e-7 K).
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import OracleSystem
from tests.conftest import golden_cases, load_golden

EPS64 = np.finfo(np.float64).eps
EPS32 = np.finfo(np.float32).eps
CASES = golden_cases()


def _system(g) -> OracleSystem:
    return OracleSystem(g["coef"], g["robin_total"], g["free"], threads=3)


def test_fixtures_present() -> None:
    assert len(CASES) >= 10


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("fast", [False, True])
def test_oracle_fp64_action_matches_reference(name: str, fast: bool) -> None:
    g = load_golden(name)
    system = _system(g)
    expected = g["apply_high"]
    actual = system.apply_f64(g["v64"], fast=fast)
    assert np.linalg.norm(actual - expected) <= 64.0 * EPS64 * np.linalg.norm(expected)
    fixed = g["free"] == 0
    np.testing.assert_array_equal(actual[fixed], g["v64"][fixed])


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("fast", [False, True])
def test_oracle_fp32_action_matches_reference(name: str, fast: bool) -> None:
    g = load_golden(name)
    system = _system(g)
    expected = g["apply_low"].astype(np.float64)
    actual = system.apply_f32(g["v32"], fast=fast)
    assert actual.dtype == np.float32
    assert np.linalg.norm(actual - expected) <= 8.0 * EPS32 * np.linalg.norm(expected)
    fixed = g["free"] == 0
    np.testing.assert_array_equal(actual[fixed], g["v32"][fixed])


@pytest.mark.parametrize("name", CASES)
def test_oracle_stiffness_matches_reference(name: str) -> None:
    g = load_golden(name)
    actual = _system(g).stiffness_f64(g["v64"])
    expected = g["stiffness"]
    assert np.linalg.norm(actual - expected) <= 64.0 * EPS64 * np.linalg.norm(expected)


@pytest.mark.parametrize("name", CASES)
def test_oracle_diagonal_is_bit_identical(name: str) -> None:
    g = load_golden(name)
    np.testing.assert_array_equal(_system(g).diagonal(), g["diagonal"])


def _temperature(g, theta: np.ndarray) -> np.ndarray:
    t = theta + float(g["reference_temperature"])
    return np.where(g["active_nodes"] == 1, t, np.nan)


@pytest.mark.parametrize("name", CASES)
def test_oracle_fp64_pcg_reaches_the_reference_temperatures(name: str) -> None:
    g = load_golden(name)
    system = _system(g)
    theta, iterations, rel = system.pcg_f64(g["rhs"], rtol=1e-10)
    # True residual after restarts from the iterate.  The stiffest stacks hit
    # the FP64 floor eps ||A|| ||x|| of the residual itself at about 2e-10.
    assert rel <= 5e-10
    t = _temperature(g, theta)
    for tag in ("fp64_pcg", "two_level"):
        ref = g[f"{tag}_temperature"]
        finite = np.isfinite(ref)
        np.testing.assert_array_equal(finite, np.isfinite(t))
        np.testing.assert_allclose(t[finite], ref[finite], rtol=1e-8, atol=1e-7)


@pytest.mark.parametrize("name", CASES)
def test_oracle_mpir_reaches_the_reference_temperatures(name: str) -> None:
    g = load_golden(name)
    system = _system(g)
    out = system.solve_mpir(g["rhs"], inner_rtol=1e-4, max_outer=20, max_inner=100000)
    # 1e-10, or the FP64 floor of the residual (~1.4e-10 on the 1 x 4 copper
    # stack), which the facade's re-reference restart handles
    assert out["converged"] or out["relative_residual"] <= 3e-10
    t = _temperature(g, out["solution"])
    ref = g["fp64_pcg_temperature"]
    finite = np.isfinite(ref)
    np.testing.assert_allclose(t[finite], ref[finite], rtol=1e-8, atol=1e-7)
    steps = out["history"]
    assert len(steps) == out["outer_iterations"]
    assert [s[0] for s in steps] == list(range(1, len(steps) + 1))


def test_oracle_is_thread_count_independent() -> None:
    g = load_golden("stack_12x20_fixed")
    a = OracleSystem(g["coef"], g["robin_total"], g["free"], threads=1)
    b = OracleSystem(g["coef"], g["robin_total"], g["free"], threads=4)
    np.testing.assert_array_equal(a.apply_f64(g["v64"], fast=True), b.apply_f64(g["v64"], fast=True))
    ra = a.solve_mpir(g["rhs"], inner_rtol=1e-4)
    rb = b.solve_mpir(g["rhs"], inner_rtol=1e-4)
    np.testing.assert_array_equal(ra["solution"], rb["solution"])
