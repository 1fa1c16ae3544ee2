"""Record golden vectors of the layered DC path from the reference implementation.

Run where the reference's source tree is available:

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_dc.py /path/to/pcb-analysis/src

For every case of tests/dc_cases.py it builds the reference's NumPy operator
(MatrixFreePCBOperator with native=False) and records, in tests/golden/dc/<case>.npz:

* the element coefficients, active and free node masks and the FP64 diagonal;
* the FP64 action apply_high and the unconstrained action apply_full_high of a
  seeded random vector, and the right-hand side of the problem's drive;
* the converged solve_pcb_dc (the reference default: two-level MPIR at
  relative residual 1e-12): potential, current density, via currents, Joule
  losses and the voltage-terminal currents.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))


def main(reference_src: str) -> None:
    sys.path.insert(0, reference_src)
    import electrical.matrix_free_mpir_fem as ref
    from electrical.matrix_free_mpir_fem import MPIRConfig

    from tests.dc_cases import DC_CASES

    out = HERE / "dc"
    out.mkdir(exist_ok=True)
    for name, build in DC_CASES.items():
        problem = build(ref)
        operator = ref.MatrixFreePCBOperator(
            problem.mesh,
            reference_node=problem.reference_node,
            dirichlet_nodes=tuple(node for t in problem.voltage_terminals for node in t.nodes),
            vias=problem.vias,
            native=False,
        )
        rng = np.random.default_rng(11)
        v = rng.standard_normal(operator.size)
        coefficients = np.stack(problem.mesh.element_coefficients())
        record = dict(
            coef=coefficients,
            active_nodes=operator.active_nodes.reshape(-1).astype(np.uint8),
            free=operator.free_nodes.reshape(-1).astype(np.uint8),
            diagonal=operator._diagonal_high,
            v=v,
            apply_high=operator.apply_high(v),
            apply_full=operator.apply_full_high(v),
            rhs=operator.build_rhs(problem.terminals, problem.voltage_terminals),
        )
        solution = ref.solve_pcb_dc(problem, config=MPIRConfig(relative_tolerance=1e-12, max_outer_iterations=40),
                                    native=False)
        assert solution.solve.converged, name
        record.update(
            potential=solution.potential_v.reshape(-1),
            current_density=solution.current_density_a_per_m2,
            via_current=solution.via_current_a,
            joule=np.array([solution.joule_loss_w, solution.max_current_density_a_per_m2]),
            element_joule=solution.element_joule_loss_w,
            via_joule=solution.via_joule_loss_w,
            terminal_current=solution.voltage_terminal_current_a,
        )
        np.savez_compressed(out / f"{name}.npz", **record)
        print(f"{name}: {operator.size} nodes, {len(problem.vias)} vias, inner {solution.solve.inner_iterations}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(f"usage: python {sys.argv[0]} <path to the reference package's src directory>")
    main(sys.argv[1])
