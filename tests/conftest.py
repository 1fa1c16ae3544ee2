"""Shared test setup: the ``gpu`` marker and the golden fixtures.

Tests marked ``gpu`` need a CUDA device and the built libthermal_b200.so; they
are the parity tests proper.  Everything else runs on the CPU.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config: pytest.Config) -> None:
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built sm_100a library")


def golden_cases() -> list[str]:
    return sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load_golden(name: str) -> dict[str, np.ndarray]:
    with np.load(GOLDEN / f"{name}.npz") as data:
        return {k: data[k] for k in data.files}


@pytest.fixture(scope="session")
def ns_local():
    """This package's thermal namespace (for tests.problems builders)."""

    import pcb_analysis_b200.thermal as ns

    return ns
