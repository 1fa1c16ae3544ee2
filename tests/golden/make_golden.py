"""Record golden vectors from the reference implementation (pcb-analysis 0.14.1).

Run in a container where the reference's source tree is available:

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py /path/to/pcb-analysis/src

For every problem of tests/problems.py CASES it builds the reference's own
NumPy operator (MatrixFreeThermalOperator with native=False) and records, in
tests/golden/<case>.npz:

* the prepared arrays: element factors (3, S, R, C), Robin total, free mask,
  diagonal, nodal load, the right-hand side at the default reference
  temperature, the per-boundary Robin weights;
* the FP64 action apply_high and the FP32 action apply_low of seeded random
  vectors, and the unconstrained stiffness action;
* two converged solves of solve_thermal_conduction at relative residual 1e-10:
  the reference default (two-level MPIR) and a plain FP64 Jacobi PCG (the
  reference's own inner PCG driven by an FP64 runtime), with their heat budgets.

The fixtures are the pins of the CPU oracle (oracle/) and of the host problem
model; the device kernels are tested against the oracle and these fixtures.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))


def main(reference_src: str) -> None:
    sys.path.insert(0, reference_src)
    import thermal.matrix_free_mpir_fem as ref
    from electrical.matrix_free_mpir_fem import MPIRConfig
    from electrical.matrix_free_mpir_fem.runtime import NumpyFloat32Runtime

    from tests.problems import CASES

    class NumpyFloat64Runtime(NumpyFloat32Runtime):
        """The reference's NumPy runtime at FP64: turns its inner PCG into a plain FP64 PCG."""

        name = "numpy-fp64"
        dtype = np.float64

        def to_host(self, value):
            return np.asarray(value, dtype=np.float64)

    for name, build in CASES.items():
        problem = build(ref)
        op = ref.MatrixFreeThermalOperator(problem, preconditioner="jacobi", native=False)
        size = op.size
        rng = np.random.default_rng(1234)
        v64 = rng.standard_normal(size)
        v32 = rng.standard_normal(size).astype(np.float32)
        reference = op.default_reference_temperature()
        stiffness = op._stiffness_action(
            v64.reshape(problem.mesh.node_shape), np, op._coefficients_high, op._unit_high
        ).reshape(-1)
        record = {
            "coef": op._coefficients_high,
            "unit": op._unit_high,
            "robin_total": op._robin_total_high,
            "robin_rhs": op._robin_rhs_high,
            "free": op.free_nodes.reshape(-1).astype(np.uint8),
            "active_nodes": op.active_nodes.reshape(-1).astype(np.uint8),
            "diagonal": op._diagonal_high,
            "load": op.nodal_load(),
            "reference_temperature": np.float64(reference),
            "rhs": op.build_rhs(reference),
            "v64": v64,
            "apply_high": op.apply_high(v64),
            "v32": v32,
            "apply_low": np.asarray(op.apply_low(v32), dtype=np.float32),
            "stiffness": stiffness,
            "robin_weights": np.stack(op._robin_weights_high) if op._robin_weights_high else np.zeros((0, size)),
            "robin_rhs_weights": (
                np.stack(op._robin_rhs_weights_high) if op._robin_rhs_weights_high else np.zeros((0, size))
            ),
        }
        config = MPIRConfig(max_outer_iterations=40, max_inner_iterations=5000)
        default = ref.solve_thermal_conduction(problem, config=config)
        assert default.solve.converged, name
        fp64 = ref.solve_thermal_conduction(
            problem,
            runtime=NumpyFloat64Runtime(),
            preconditioner="jacobi",
            native=False,
            config=MPIRConfig(
                relative_tolerance=1e-10,
                inner_relative_tolerance=1e-11,
                max_outer_iterations=16,
                max_inner_iterations=200000,
            ),
        )
        assert fp64.solve.converged, name
        for tag, sol in (("two_level", default), ("fp64_pcg", fp64)):
            record[f"{tag}_temperature"] = sol.temperature_k.reshape(-1)
            record[f"{tag}_flux"] = sol.heat_flux_w_per_m2
            record[f"{tag}_budget"] = np.array(
                [
                    sol.total_heat_input_w,
                    sol.fixed_temperature_heat_w,
                    sol.heat_balance_error_w,
                    sol.max_temperature_k,
                    sol.min_temperature_k,
                    sol.solve.relative_residual,
                ]
            )
            record[f"{tag}_convective"] = sol.convective_heat_w
        np.savez_compressed(HERE / f"{name}.npz", **record)
        print(f"{name}: {size} nodes, two-level {default.solve.inner_iterations} inner, "
              f"fp64 pcg {fp64.solve.inner_iterations} iterations")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(f"usage: python {sys.argv[0]} <path to the reference package's src directory>")
    main(sys.argv[1])
