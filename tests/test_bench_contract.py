"""The bench's roofline arithmetic and reporting helpers (CPU).

The FP32 operator's algorithmic bytes per launch are 4N (x) + 4N (y) + 8E
(k_in, k_z) + 5F (the Robin total and the operand's reread on the two boundary
planes, F = 2 (R+1)(C+1)); the c2 figure is the one the ncu summaries quote.
"""

from __future__ import annotations

import json

import bench


def test_operator_bytes_per_launch_on_c2_and_c3() -> None:
    assert bench.algorithmic_bytes_apply32((12, 512, 512)) == 55_167_090
    n3 = 17 * 2049 * 2049
    e3 = 16 * 2048 * 2048
    assert bench.algorithmic_bytes_apply32((16, 2048, 2048)) == 8 * n3 + 8 * e3 + 5 * 2 * 2049 * 2049


def test_operator_kernel_names_follow_the_launch_plan() -> None:
    assert bench.operator_kernel_name((2, 16, 1, 0, 0)).startswith("apply_split_kernel<float, OPERATOR, DOT, 16>")
    assert "tensor copies" in bench.operator_kernel_name((0, 8, 1, 0, 0))
    assert "cp.async" in bench.operator_kernel_name((0, 32, 0, 0, 0))
    assert bench.operator_kernel_name((1, 16, 2, 4, 8)).startswith("warp_apply_kernel<2, 4, DOT>")


def test_cpu_model_extrapolates_only_beyond_its_measured_anchor() -> None:
    """The reference arm's count model: c1 measured whole, c2 / c3 scaled by
    the board's side and flagged extrapolated."""

    model = bench.CpuModel.__new__(bench.CpuModel)
    model.anchor_s, model.anchor_inner, model.anchor_outer, model.anchor_converged = 90.0, 18_000, 6, True
    model.apply64_s, model.threads = 0.5, 8
    for workload, factor in (("c1", 1), ("c3", 16)):
        model.workload = workload
        model.inner = 18_000 * factor
        model.outer = 6
        model.extrapolated = workload != "c1"
        seconds = model.solve_seconds(3.0)
        parts = model.describe(3.0, 2)
        if workload == "c1":
            assert seconds == 90.0 and parts["model"] is None and not parts["extrapolated"]
        else:
            assert seconds == 3.0 * 18_000 * 16 + 0.5 * 7 and parts["extrapolated"]
            assert "x side 2048 / 128" in parts["model"]["rule"]


def test_reference_arm_of_the_engine_workloads_reports_unavailable(capsys) -> None:
    class Args:
        workload = "c4"

    bench.run_reference_arm(Args(), rank=0)
    line = json.loads(capsys.readouterr().out.strip())
    assert line["impl"] == "reference" and "unavailable" in line
    bench.run_reference_arm(Args(), rank=1)  # other ranks print nothing
    assert capsys.readouterr().out == ""


def test_both_arms_describe_the_single_board_workload_with_the_same_config() -> None:
    """The b200 line and the reference arm's line carry the workload alone in
    `config`, from one helper, so that the two lines' configs compare equal;
    how each arm solves it goes under `solver`."""

    import inspect

    problem, description = bench.build_problem("c1", 0)
    config = bench.single_board_config("c1", description, problem)
    assert config == bench.single_board_config("c1", description, problem)
    assert set(config) == {"workload", "nodes", "elements", "l2"}
    assert config["nodes"] == problem.mesh.size
    for arm in (bench.run_reference_arm, bench.run_single):
        source = inspect.getsource(arm)
        assert '"config": single_board_config(args.workload, description, problem)' in source
        assert '"solver":' in source
