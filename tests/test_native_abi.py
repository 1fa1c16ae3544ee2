"""The C-ABI library loads and exports every entry point include/thermal_b200.h declares.

No compute call is made here: these run on a machine without a GPU.
"""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

from pcb_analysis_b200 import _native, build

HEADER = Path(__file__).resolve().parent.parent / "include" / "thermal_b200.h"


def _declared() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(tb_\w+)\s*\(", text, flags=re.M)))


def test_library_is_built_for_sm100a() -> None:
    assert build.LIBRARY.exists(), "run python -m pcb_analysis_b200.build"
    assert "sm_100a" in _native.load().tb_version().decode()


def test_every_declared_symbol_is_exported_and_bound() -> None:
    lib = ctypes.CDLL(str(_native.library_path()))
    names = _declared()
    assert len(names) >= 18
    for name in names:
        assert hasattr(lib, name), name
        assert name in _native.exported_names(), name


def test_status_codes_map_to_the_reference_exception_types() -> None:
    assert _native._EXCEPTIONS[_native.TB_EINVAL] is ValueError
    assert _native._EXCEPTIONS[_native.TB_ENOTSPD] is RuntimeError
    assert _native._EXCEPTIONS[_native.TB_ENOMEM] is MemoryError


def test_no_device_means_a_loud_error_not_a_fallback() -> None:
    if _native.device_count() > 0:
        pytest.skip("a CUDA device is visible")
    import pcb_analysis_b200.thermal as ns
    from tests.problems import stack

    with pytest.raises(RuntimeError, match="no CUDA device"):
        ns.MatrixFreeThermalOperator(stack(ns, 2, 3), preconditioner="jacobi")


def test_unsupported_paths_are_refused() -> None:
    import pcb_analysis_b200.thermal as ns
    from tests.problems import stack

    problem = stack(ns, 2, 3)
    with pytest.raises(NotImplementedError, match="GPU"):
        ns.MatrixFreeThermalOperator(problem, backend="cpu", preconditioner="jacobi")
    with pytest.raises(NotImplementedError, match="GPU"):
        ns.MatrixFreeThermalOperator(problem, backend="cpu")
    with pytest.raises(ValueError, match="coarse_block_nodes"):
        ns.MatrixFreeThermalOperator(problem, coarse_block_nodes=0)


def test_engine_footprint_counts_the_resident_fields() -> None:
    """A resident board holds, per padded node, four FP64 and six FP32 fields;
    per padded element, the two conductivities in both precisions."""

    import numpy as np

    def arrays(slabs, rows, cols):
        nodes = (slabs + 1) * (rows + 1) * (cols + 1)
        return dict(slab_thickness_m=np.ones(slabs), pitch_x_m=np.ones(cols), pitch_y_m=np.ones(rows),
                    k_in=np.ones(slabs * rows * cols), k_z=np.ones(slabs * rows * cols),
                    robin_total=np.zeros(nodes), free_nodes=np.ones(nodes, dtype=np.uint8))

    slabs, rows, cols = 8, 300, 203
    resident, transient = _native.engine_footprint(arrays(slabs, rows, cols))
    padded_nodes = (slabs + 1) * (rows + 1) * ((cols + 1 + 3) // 4 * 4)
    padded_elements = slabs * rows * ((cols + 3) // 4 * 4)
    fields = 56 * padded_nodes + 24 * padded_elements
    assert fields <= resident <= fields * 1.02 + 64 * 1024
    assert transient > 0
    bigger, _ = _native.engine_footprint(arrays(slabs, 2 * rows, cols))
    assert bigger > 1.9 * resident
