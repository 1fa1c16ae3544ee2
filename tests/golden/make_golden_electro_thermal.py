"""Record golden vectors of the electro-thermal coupling from the reference implementation.

Run where the reference's source tree is available:

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_electro_thermal.py /path/to/pcb-analysis/src

On the voltage-driven loop of tests/electro_thermal_cases.py it records, in
tests/golden/coupling/electro_thermal.npz:

* the reference's run_electro_thermal (multiphysics/staggered_coupling/
  electro_thermal.py:354-478, NumPy solves, default CouplingConfig) with
  Aitken relaxation and without: passes, losses, temperature changes and
  relaxation factors per pass, and the final temperature, potential,
  conductivity, via resistances, layer temperatures and terminal currents;
* the host steps on seeded inputs: heated_electrical_problem at a seeded
  temperature field, element_heat_from_losses and via_heat_sources of
  seeded losses, and five updates of TemperatureFixedPoint on seeded
  proposals.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))


def fixed_point_proposals(shape, seed: int = 5) -> list[np.ndarray]:
    """Five proposals of an oscillating, contracting loop around a seeded field."""
    rng = np.random.default_rng(seed)
    target = 298.15 + 20.0 * rng.random(shape)
    wobble = rng.standard_normal(shape)
    return [target + (-0.55) ** k * 8.0 * wobble for k in range(5)]


def main(reference_src: str) -> None:
    sys.path.insert(0, reference_src)
    import electrical.matrix_free_mpir_fem as ed
    import thermal.matrix_free_mpir_fem as td
    import multiphysics.staggered_coupling.electro_thermal as et
    from thermal.matrix_free_mpir_fem.coupling import element_heat_from_losses, via_heat_sources
    from tests import electro_thermal_cases as cases

    problem = cases.voltage_loop(ed, cases.GOLDEN_VOLTAGE_V)
    scenario = cases.scenario(ed, td, et, problem)
    record: dict[str, np.ndarray] = {}
    for tag, config in (("aitken", et.CouplingConfig()), ("plain", et.CouplingConfig(aitken=False))):
        result = et.run_electro_thermal(scenario, config=config, native=False)
        assert result.converged, tag
        h = result.history
        record[f"{tag}_passes"] = np.array([result.iterations])
        record[f"{tag}_loss"] = np.array([s.joule_loss_w for s in h])
        record[f"{tag}_change"] = np.array([s.temperature_change_k for s in h])
        record[f"{tag}_relaxation"] = np.array([s.relaxation for s in h])
        record[f"{tag}_cold_loss"] = np.array([result.cold_joule_loss_w])
        record[f"{tag}_temperature"] = result.thermal.temperature_k.reshape(-1)
        record[f"{tag}_potential"] = result.electrical.potential_v.reshape(-1)
        record[f"{tag}_conductivity"] = result.conductivity_s_per_m
        record[f"{tag}_via_resistance"] = result.via_resistance_ohm
        record[f"{tag}_layer_temperature"] = result.element_temperature_k
        record[f"{tag}_terminal_current"] = result.electrical.voltage_terminal_current_a
        record[f"{tag}_heat_input"] = np.array([result.thermal.total_heat_input_w])
        print(f"{tag}: {result.iterations} passes, loss {result.electrical.joule_loss_w:.6e} W "
              f"(cold {result.cold_joule_loss_w:.6e}), max T {result.thermal.max_temperature_k:.3f} K")

    rng = np.random.default_rng(3)
    mesh = scenario.thermal_mesh
    temperature = 298.15 + 40.0 * rng.random(mesh.node_shape)
    heated = et.heated_electrical_problem(scenario, temperature)
    record["seeded_temperature"] = temperature
    record["heated_conductivity"] = np.asarray(heated.mesh.conductivity_s_per_m)
    record["heated_via_resistance"] = np.array([v.resistance_ohm for v in heated.vias])
    record["seeded_layer_temperature"] = et.electrical_layer_temperature_k(temperature, mesh, scenario.layer_slabs)

    losses = rng.random((2,) + problem.mesh.element_active.shape[1:])
    via_losses = rng.random(len(problem.vias))
    record["seeded_element_loss"] = losses
    record["seeded_element_heat"] = element_heat_from_losses(losses, mesh, (0, 2))
    record["seeded_via_loss"] = via_losses
    sources = via_heat_sources(problem.vias, via_losses, 2, mesh, (0, 2))
    record["via_source_nodes"] = np.array([s.nodes for s in sources])
    record["via_source_power"] = np.array([s.power_w for s in sources])

    fixed_point = et.TemperatureFixedPoint(scenario, et.CouplingConfig())
    changes, relaxations = [], []
    for proposal in fixed_point_proposals(mesh.node_shape):
        changes.append(fixed_point.update(proposal))
        relaxations.append(fixed_point.relaxation)
    record["fixed_point_change"] = np.array(changes)
    record["fixed_point_relaxation"] = np.array(relaxations)
    record["fixed_point_temperature"] = fixed_point.temperature
    out = HERE / "coupling"
    out.mkdir(exist_ok=True)
    np.savez_compressed(out / "electro_thermal.npz", **record)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(f"usage: python {sys.argv[0]} <path to the reference package's src directory>")
    main(sys.argv[1])
