"""Record the reference's two-level coarse space for every golden case.

Run where the reference's source tree is available:

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_coarse.py /path/to/pcb-analysis/src

For every problem of tests/problems.py CASES it builds the reference's own
NumPy operator with the default two-level preconditioner
(MatrixFreeThermalOperator(preconditioner="two-level", native=False), whose
AggregationCoarseCorrection is src/electrical/matrix_free_mpir_fem/
two_level.py:62-229) and records, in tests/golden/coarse/<case>[_b<block>].npz:

* the patch width and the coarse grid shape;
* the Galerkin matrix Z^T A Z assembled from 27 coloured FP64 actions, with
  empty patches given a unit diagonal, and its symmetrised inverse;
* the FP64 preconditioner action D^-1 v + Z (Z^T A Z)^-1 Z^T v of the seeded
  vector v64 of the case's main fixture.

Besides the default patch width, seeded_board_24x30 is also recorded with a
forced width of 7 (ragged edge patches).
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

EXTRA_BLOCKS = {"seeded_board_24x30": (7,)}


def main(reference_src: str) -> None:
    sys.path.insert(0, reference_src)
    import thermal.matrix_free_mpir_fem as ref

    from tests.problems import CASES

    out = HERE / "coarse"
    out.mkdir(exist_ok=True)
    for name, build in CASES.items():
        v64 = np.load(HERE / f"{name}.npz")["v64"]
        for block in (None,) + EXTRA_BLOCKS.get(name, ()):
            problem = build(ref)
            op = ref.MatrixFreeThermalOperator(problem, preconditioner="two-level", native=False,
                                               coarse_block_nodes=block)
            cc = op.coarse_correction
            record = {
                "block": np.int64(cc.block),
                "coarse_shape": np.array(cc.coarse_shape, dtype=np.int64),
                "coarse_matrix": cc.coarse_matrix,
                "coarse_inverse": cc._coarse_inverse_high,
                "precondition_high": cc.apply_high(v64),
            }
            tag = name if block is None else f"{name}_b{block}"
            np.savez_compressed(out / f"{tag}.npz", **record)
            print(f"{tag}: block {cc.block}, coarse {cc.coarse_shape} = {cc.coarse_size}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(f"usage: python {sys.argv[0]} <path to the reference package's src directory>")
    main(sys.argv[1])
