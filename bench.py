"""Benchmark of the steady Q1 thermal solve on B200: solves/s of the MPIR solve.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload c3|c2|c1|c4|c5|dc] [--preconditioner multilevel|two-level|jacobi]

One step = one complete MPIR solve (FP32 PCG inner to 1e-4, FP64 residual,
update and norm to a relative residual of 1e-10) of the seeded synthetic board
of the workload, from zero.  The default is c3, the largest single-board
configuration: 2048 x 2048 cells x 16 slabs, 71,372,817 nodes, with the
multilevel preconditioner.  The board, its coefficients and the right-hand
side are resident in HBM when the timed region starts; the PCG working set
(~5 GB at c3) is far larger than the 126 MB L2, so no flush is needed between
steps.  With N GPUs every rank solves its own board (replicas: boards are
independent, there is no collective); the value is the total solves/s, timed
on the device (CUDA events on the solver's stream), max over ranks.

Printed as one JSON line on rank 0, with:
* ``latency_ms``: p50/p99 of the per-step device time; ``iterations``;
* ``accuracy``: final relative residual and max |dT| (K) against an FP64 PCG
  of the same board on the GPU converged to 1e-10 (``fp64_pcg``: with the same
  preconditioner, the like-for-like FP64 baseline); ``fp64_jacobi_pcg``: the
  plain FP64 Jacobi PCG (c1, c2, or with --fp64-jacobi);
* ``roofline``: the FP32 operator apply, algorithmic bytes
  B = 4N + 4N + 8E + 5F per launch (F = 2 (R+1)(C+1)) over its average device
  time inside the timed solves (each launch stamps %globaltimer at its first
  block's start and last block's end), against MEASURED_PEAKS.json hbm_gbs;
* ``e2e``: the same metric through the public call solve_thermal_conduction
  with host NumPy inputs (upload, preparation, solve, heat budget, download);
* ``cpu_baseline``: the CPU port of the reference's Jacobi MPIR on the host
  cores: a complete c1 solve and a sample of the board's PCG iterations,
  measured; the board's full solve modelled from them (``extrapolated``);
* ``c4`` / ``c5`` (c3 only): the batched and served workloads condensed;
* ``clocks``: nvidia-smi samples taken during the timed region.

``--impl reference`` runs only the CPU port (rank 0; other ranks exit).
"""

from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "Q1 thermal solves/s + p50/p99 latency at 1e-10 rel resid vs FP64 PCG, 1 B200"
UNIT = "solves/s"

# Boards sides (cells) of the single-board workloads, for the CPU count model.
SIDE_CELLS = {"c1": 128, "c2": 512, "c3": 2048}


def _env_int(name: str, default: int) -> int:
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def build_problem(workload: str, seed: int, cells: int = 0):
    """The board of a single-board workload; `cells` (> 0) narrows it to that
    many cells per side with the same rules (a smaller case for profiling)."""

    from pcb_analysis_b200 import workloads

    if cells > 0:
        maker = {"c1": workloads.board_c1, "c2": workloads.board_c2, "c3": workloads.board_c3}[workload]
        return maker(seed, rows=cells, cols=cells), f"{workload} rules at {cells}x{cells} cells (profiling case)"
    if workload == "c3":
        return workloads.board_c3(seed), (
            "c3: 2048x2048 cells x 16 slabs (6 Cu, 40-90% fill), 64 sources U(0.05,5) W, h=25/5, "
            "fixed 25 C bottom strip (columns 0..40)")
    if workload == "c1":
        return workloads.board_c1(seed), "c1: 128x128 cells x 8 slabs (Cu, 6 FR-4, Cu), 60% copper, 4 x 1 W pads, h=10/10"
    if workload == "c2":
        return workloads.board_c2(seed), (
            "c2: 512x512 cells x 12 slabs (4 Cu), inner planes ~85% copper, outer traces, "
            "16 sources U(0.1,2) W, h=10/10"
        )
    raise SystemExit(f"unknown workload {workload}")


def mpir_config():
    from pcb_analysis_b200.mpir import MPIRConfig

    return MPIRConfig(
        relative_tolerance=1e-10,
        inner_relative_tolerance=1e-4,
        max_outer_iterations=60,
        max_inner_iterations=2_000_000,
    )


def algorithmic_bytes_apply32(shape) -> int:
    s, r, c = shape
    n = (s + 1) * (r + 1) * (c + 1)
    e = s * r * c
    f = 2 * (r + 1) * (c + 1)
    return 4 * n + 4 * n + 8 * e + 5 * f


DC_METRIC = "layered DC solves/s at 1e-10 rel resid vs FP64 PCG, 1 B200"


def algorithmic_bytes_dc32(mesh) -> int:
    """One FP32 layered DC action: read x (4N), the node bits (1N) and the sheet
    conductance (4E), write y (4N)."""

    layers, rows, cols = mesh.element_active.shape
    n = layers * (rows + 1) * (cols + 1)
    return 4 * n + n + 4 * layers * rows * cols + 4 * n


def run_dc(args, device: int) -> dict:
    """The layered DC workload: solve_pcb_dc's MPIR solve of a 4.2 M-node
    power net, resident, against the plain FP64 PCG on the same system."""

    import torch

    from pcb_analysis_b200 import electrical as ed
    from pcb_analysis_b200.workloads import dc_power_net

    problem = dc_power_net(0)
    mesh = problem.mesh
    op = ed.MatrixFreePCBOperator(
        mesh, dirichlet_nodes=tuple(node for t in problem.voltage_terminals for node in t.nodes), vias=problem.vias,
        preconditioner=args.preconditioner, device_id=device)
    dev = op.device_system
    rhs_host = op.build_rhs(problem.terminals, problem.voltage_terminals)
    fixed = op.dirichlet_potential(problem.voltage_terminals)
    rhs = torch.as_tensor(rhs_host, device=f"cuda:{device}")
    x0 = torch.as_tensor(fixed, device=f"cuda:{device}")
    x = torch.empty_like(rhs)
    config = mpir_config()
    stream = torch.cuda.ExternalStream(dev.stream_handle(), device=f"cuda:{device}")

    def step() -> dict:
        x.copy_(x0)
        torch.cuda.synchronize(device)
        return dev.solve_mpir_device(rhs, x, config)

    for _ in range(args.warmup):
        result = step()
    sampler = ClockSampler(device)
    sampler.start()
    clock0 = dev.kernel_clock()
    step_ms = []
    for _ in range(args.steps):
        x.copy_(x0)
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        result = dev.solve_mpir_device(rhs, x, config)
        e1.record(stream)
        torch.cuda.synchronize(device)
        step_ms.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    clock1 = dev.kernel_clock()
    apply_ms = clock1["apply_f32"][0] - clock0["apply_f32"][0]
    apply_n = clock1["apply_f32"][1] - clock0["apply_f32"][1]
    ms = float(np.median(step_ms))
    solution = x.detach().cpu().numpy()

    x64 = x0.clone()
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    pcg = dev.solve_pcg_f64_device(rhs, x64, relative_tolerance=1e-10, max_iterations=4_000_000)
    pcg_s = time.perf_counter() - t0
    pcg_solution = x64.detach().cpu().numpy()
    free = op.free_nodes.reshape(-1)
    max_dv = float(np.max(np.abs(solution[free] - pcg_solution[free])))

    bytes_apply = algorithmic_bytes_dc32(mesh)
    peak, peak_kind = measured_peak()
    avg_ms = apply_ms / apply_n if apply_n else None
    achieved = bytes_apply / (avg_ms * 1e-3) / 1e9 if avg_ms else None

    e2e = None
    if args.e2e_steps > 0:
        samples = []
        for _ in range(args.e2e_steps):
            t0 = time.perf_counter()
            sol = ed.solve_pcb_dc(problem, preconditioner=args.preconditioner, config=config, device_id=device)
            samples.append(time.perf_counter() - t0)
        n, e = mesh.size, int(mesh.element_active.size)
        # up: element mask, conductivity, pitches, vias; the rhs, initial potential and the lifting vector;
        # the potential for the terminal currents.  Down: the lifted action, the solution, the K v of the currents.
        h2d = e + 8 * e + 24 * len(problem.vias) + 8 * n * 4
        d2h = 8 * n * 3 + 2 * n
        e2e = {"value": 1.0 / float(np.median(samples)), "unit": "solves/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "statistic": f"median of {len(samples)} calls",
               "samples_s": [round(v, 4) for v in samples], "converged": bool(sol.solve.converged),
               "joule_loss_w": sol.joule_loss_w}

    cpu = None
    if not args.no_cpu_baseline:
        from oracle.dc_oracle import from_problem

        oracle = from_problem(problem)
        v = rhs_host.copy()
        oracle.apply_f64(v)  # first touch
        t0 = time.perf_counter()
        reps = 3
        for _ in range(reps):
            oracle.apply_f64(v)
        per_apply = (time.perf_counter() - t0) / reps
        solve_s = per_apply * (result["inner_iterations"] + result["outer_iterations"] + 1)
        cpu = {"value": 1.0 / solve_s, "unit": "solves/s", "cores": 1, "kind": "port",
               "sample": (f"{reps} FP64 actions of the NumPy restatement of the reference operator "
                          f"({per_apply * 1e3:.0f} ms each, one core), extrapolated to the "
                          f"{result['inner_iterations']} inner + {result['outer_iterations'] + 1} outer actions of "
                          "the GPU solve; the vector updates are not counted, so this bounds the CPU time from below")}

    return {
        "metric": DC_METRIC,
        "value": 1000.0 / ms,
        "unit": "solves/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 inner / f64 outer",
        "data": "synthetic",
        "config": {"workload": ("dc: 4-layer power net, 1024 x 1024 cells at 0.25 mm, planes with voids, "
                                "2000 vias, 1 V regulator, 16 loads"),
                   "nodes": mesh.size, "elements": int(mesh.element_active.size), "vias": len(problem.vias),
                   "preconditioner": args.preconditioner, "parallelism": "replicas x1",
                   "l2": "working set ~130 MB > 126 MB L2: no flush between steps"},
        "latency_ms": {"p50": ms, "steps": [round(v, 3) for v in step_ms]},
        "iterations": {"outer": result["outer_iterations"], "inner": result["inner_iterations"]},
        "accuracy": {"relative_residual": result["relative_residual"], "converged": result["converged"],
                     "max_abs_dV_vs_fp64_pcg": max_dv},
        "fp64_pcg": {"solve_s": pcg_s, "iterations": pcg["iterations"], "converged": pcg["converged"],
                     "relative_residual": pcg["relative_residual"], "speedup_of_mpir": pcg_s / (ms * 1e-3)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind, "traffic": None,
                     "kernel": "dc_march_kernel<float, OPERATOR, DOT> (FP32 sheet + via action + p.Ap, y-marching)",
                     "bytes_per_launch": bytes_apply, "avg_launch_ms": avg_ms, "launches": apply_n},
        "clocks": clocks,
        "e2e": e2e,
        "cpu_baseline": cpu,
    }


def operator_kernel_name(plan) -> str:
    """The FP32 operator kernel a launch plan (kind, rows, staging or zw, sl, band) runs."""

    kind, rows = int(plan[0]), int(plan[1])
    if kind == 1:
        return f"warp_apply_kernel<{plan[2]}, {plan[3]}, DOT> (FP32 Q1 action + p.Ap, warp march)"
    staging = "tensor copies" if int(plan[2]) == 1 else "cp.async"
    name = "apply_split_kernel" if kind == 2 else "apply_kernel"
    stages = int(plan[3]) if len(plan) > 3 and int(plan[3]) > 0 else 4
    return (f"{name}<float, OPERATOR, DOT, {rows}> (FP32 Q1 action + p.Ap, {stages} stages filled by {staging}, "
            f"{stages - 2} planes in flight)")


def measured_peak() -> tuple[float, str]:
    path = REPO / "MEASURED_PEAKS.json"
    try:
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(workload: str, kernel: str = "apply_f32", nodes: int = 0) -> int | None:
    """dram__bytes_read.sum + dram__bytes_write.sum per launch of `kernel`, from
    the committed ncu summary of this workload: its measured figure
    (profiles/<kernel>_<workload>.md, "traffic_bytes_per_launch"), or, for a
    board too large to capture, the figure per node of a smaller case of the
    same rules (profiles/<kernel>_<workload>_<cells>.md,
    "traffic_bytes_per_node") times this board's nodes: the traffic of these
    kernels grows in proportion to the nodes."""

    path = REPO / "profiles" / f"{kernel}_{workload}.md"
    if path.exists():
        match = re.search(r"traffic_bytes_per_launch:\s*([0-9]+)", path.read_text())
        if match:
            return int(match.group(1))
    if nodes > 0:
        for small in sorted((REPO / "profiles").glob(f"{kernel}_{workload}_*.md")):
            match = re.search(r"traffic_bytes_per_node:\s*([0-9.]+)", small.read_text())
            if match:
                return int(round(float(match.group(1)) * nodes))
    return None


class ClockSampler:
    """nvidia-smi SM clocks and throttle reasons, sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int) -> None:
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self) -> None:
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
            )
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(mx) if mx else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def coarse_step_model_seconds(nodes: int, coarse: int, reps: int = 3) -> float:
    """CPU time of one coarse correction for a board of `nodes` nodes and
    `coarse` coarse unknowns, without its set-up: a patch restriction of the
    node field (bincount), the FP32 dense matvec and the prolongation."""

    rng = np.random.default_rng(0)
    inv = rng.standard_normal((coarse, coarse)).astype(np.float32)
    patch = rng.integers(0, coarse, nodes)
    v = rng.standard_normal(nodes).astype(np.float32)
    t0 = time.perf_counter()
    for _ in range(reps):
        c = inv @ np.bincount(patch, weights=v, minlength=coarse).astype(np.float32)
        _ = c[patch]
    return (time.perf_counter() - t0) / reps


def oracle_system(problem):
    """The CPU port of the reference operator for a board (test infrastructure),
    with the right-hand side the facade builds for it."""

    from oracle.oracle import OracleSystem
    from pcb_analysis_b200.thermal.system import prepare

    host = prepare(problem)
    oracle = OracleSystem(np.stack(problem.mesh.element_coefficients()), host.robin_total,
                          host.free_nodes.reshape(-1).astype(np.uint8))
    reference = host.robin_ambient_k[0] if host.robin_ambient_k else 0.0
    fixed = host.fixed_nodes.reshape(-1)
    shifted = np.where(fixed & host.active_nodes.reshape(-1), host.fixed_temperature_k.reshape(-1) - reference, 0.0)
    rhs = host.load + (host.robin_rhs - host.robin_total * reference) - oracle.stiffness_f64(shifted)
    rhs[fixed] = shifted[fixed]
    return oracle, rhs


class CpuModel:
    """The reference's CPU solve of this path (the CPU port of its Jacobi MPIR:
    FP32 Jacobi PCG inner to 1e-4, FP64 residual to 1e-10, OpenMP over the
    host cores), measured where it fits in a run and modelled where it does not.

    * Anchor, measured: one complete solve of the c1 board (128 x 128 x 8, the
      reference's CPU-runnable configuration), with its own inner and outer
      counts.
    * Sample, measured: FP32 Jacobi-PCG iterations and an FP64 apply of the
      workload's own board on the same cores.
    * Model, for c2 / c3: the inner count grows with the board's side (Jacobi
      PCG needs ~sqrt(cond) ~ 1/h iterations; the stack is alike), so
      inner(w) = inner(c1) x side(w) / side(c1), and the outer count is c1's.
      Such an estimate is flagged ``extrapolated``.
    """

    def __init__(self, workload: str, problem) -> None:
        from pcb_analysis_b200.workloads import board_c1

        self.workload = workload
        anchor, rhs1 = oracle_system(board_c1(0))
        t0 = time.perf_counter()
        out = anchor.solve_mpir(rhs1, rtol=1e-10, inner_rtol=1e-4, max_outer=60, max_inner=2_000_000)
        self.anchor_s = time.perf_counter() - t0
        self.anchor_inner = int(out["inner_iterations"])
        self.anchor_outer = int(out["outer_iterations"])
        self.anchor_converged = bool(out["converged"])
        self.threads = anchor.threads
        if workload == "c1":
            self.oracle, self.rhs = anchor, rhs1
        else:
            self.oracle, self.rhs = oracle_system(problem)
        peak = float(np.max(np.abs(self.rhs)))
        self.scale = 2.0 ** -np.frexp(peak)[1] if peak > 0 else 1.0
        self.oracle.inner_iterations(self.rhs * self.scale, 1)  # first touch of the work arrays
        t0 = time.perf_counter()
        self.oracle.apply_f64(self.rhs, fast=True)
        self.apply64_s = time.perf_counter() - t0
        factor = SIDE_CELLS[workload] / SIDE_CELLS["c1"]
        self.inner = int(round(self.anchor_inner * factor))
        self.outer = self.anchor_outer
        self.extrapolated = workload != "c1"

    def sample(self, iterations: int) -> float:
        """Seconds per FP32 PCG iteration over `iterations` iterations of the workload."""

        t0 = time.perf_counter()
        self.oracle.inner_iterations(self.rhs * self.scale, iterations)
        return (time.perf_counter() - t0) / iterations

    def solve_seconds(self, per_iteration: float) -> float:
        if not self.extrapolated:
            return self.anchor_s
        return per_iteration * self.inner + self.apply64_s * (self.outer + 1)

    def describe(self, per_iteration: float, iterations: int) -> dict:
        return {
            "anchor": {"board": "c1 (128x128x8)", "solve_s": round(self.anchor_s, 3), "inner": self.anchor_inner,
                       "outer": self.anchor_outer, "converged": self.anchor_converged, "measured": True},
            "sample": {"board": self.workload, "fp32_pcg_iterations": iterations,
                       "s_per_iteration": per_iteration, "fp64_apply_s": self.apply64_s, "measured": True},
            "model": (None if not self.extrapolated else
                      {"inner": self.inner, "outer": self.outer,
                       "rule": f"inner = {self.anchor_inner} (c1, measured) x side {SIDE_CELLS[self.workload]} / 128; "
                               "outer as c1; time = inner x s_per_iteration + (outer + 1) x fp64_apply_s"}),
            "extrapolated": self.extrapolated,
        }


def cpu_baseline(model: CpuModel, iterations: int = 2) -> dict:
    per_iteration = model.sample(iterations)
    solve_s = model.solve_seconds(per_iteration)
    return {
        "value": 1.0 / solve_s,
        "unit": UNIT,
        "cores": model.threads,
        "kind": "port",
        "sample": (f"CPU port of the reference's Jacobi MPIR on {model.threads} threads: complete c1 solve measured "
                   f"({model.anchor_s:.1f} s, {model.anchor_inner} inner / {model.anchor_outer} outer), "
                   f"{iterations} FP32 PCG iterations of this board measured ({per_iteration:.3f} s each)"
                   + (f"; this board's solve modelled at {model.inner} inner iterations" if model.extrapolated else "")),
        "extrapolated": model.extrapolated,
        "solve_s": solve_s,
        "parts": model.describe(per_iteration, iterations),
    }


def single_board_config(workload: str, description: str, problem) -> dict:
    """The workload of a single-board line (c1, c2, c3): what both arms solve."""

    return {"workload": description, "nodes": problem.mesh.size,
            "elements": int(np.prod(problem.mesh.element_grid_shape)),
            "l2": "PCG working set > 126 MB L2 (c3: ~5 GB): no flush between steps"}


def run_reference_arm(args, rank: int) -> None:
    """The reference's CPU solve of the workload on the host cores (rank 0)."""

    if rank != 0:
        return
    if args.workload == "dc":
        print(json.dumps({"impl": "reference", "metric": DC_METRIC, "unavailable": (
            "the layered DC workload reports its CPU baseline (the oracle's NumPy restatement of the reference "
            "operator, sampled and extrapolated) in the b200 arm's cpu_baseline")}), flush=True)
        return
    if args.workload not in SIDE_CELLS:
        print(json.dumps({"impl": "reference", "metric": METRIC, "unavailable": (
            "the CPU port is timed on the single-board workloads c1, c2 and c3; the batched and served workloads "
            "are compared with serial plain FP64 solves on the GPU in the b200 arm")}), flush=True)
        return
    problem, description = build_problem(args.workload, 0)
    model = CpuModel(args.workload, problem)
    iterations = 2 if args.workload == "c3" else 10
    for _ in range(args.warmup):
        model.sample(iterations)
    times = [model.sample(iterations) for _ in range(args.steps)]
    per_iteration = statistics.median(times)
    solve_s = model.solve_seconds(per_iteration)
    value = 1.0 / solve_s
    line = {
        "metric": METRIC,
        "impl": "reference",
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        # what each timed step measured: a sample of FP32 PCG iterations
        "ms_per_step": per_iteration * iterations * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 inner / f64 outer",
        "data": "synthetic",
        "config": single_board_config(args.workload, description, problem),
        "solver": {"method": "MPIR: FP32 Jacobi PCG inner rtol 1e-4, FP64 residual/update/norm to rtol 1e-10 "
                             "(the CPU port of the reference's solve)", "preconditioner": {"kind": "jacobi"}},
        "parallelism": "rank 0 alone, on the host cores",
        "extrapolated": model.extrapolated,
        "solve_s_estimate": solve_s,
        "sample_per_step": f"{iterations} FP32 Jacobi-PCG iterations of the {args.workload} board",
        "cpu_baseline": {
            "value": value, "unit": UNIT, "cores": model.threads, "kind": "port",
            "sample": (f"c1 solved completely ({model.anchor_s:.1f} s); per step {iterations} PCG iterations of this "
                       "board; the reference's C++ core needs Eigen/SuperLU and does not build offline"),
            "extrapolated": model.extrapolated,
            "parts": model.describe(per_iteration, iterations),
        },
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def whole_job_rate(local_ms: float, units_per_rank: int, world: int, dist=None, device=None) -> tuple[float, float]:
    """Whole-job throughput of `world` replicas: every rank processed
    `units_per_rank` units; the job took as long as its slowest rank."""

    slowest = float(local_ms)
    if dist is not None and world > 1:
        import torch

        t = torch.tensor([slowest], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        slowest = float(t.item())
    return world * units_per_rank / (slowest * 1e-3), slowest


# ------------------------------------------------------------ batched / served
ENGINE_WORKLOADS = {
    "c4": "c4: 64 boards, sides log-uniform 96..768 cells, 4..12 slabs, own stackup/occupancy/sources, h=10",
    "c5": ("c5: served stream, sides log-uniform 64..1024 cells, 4..16 slabs, random stackup/sources, h in {5,10,25}, "
           "fixed bottom strip on half the boards, Poisson arrivals"),
}


def engine_requests(workload: str, count: int):
    from pcb_analysis_b200 import workloads
    from pcb_analysis_b200.serve import board_request

    if workload == "c4":
        problems = workloads.batch_c4(0, count)
    else:
        problems = [workloads.request_c5(i) for i in range(count)]
    return [board_request(p, tag=i) for i, p in enumerate(problems)]


def board_bytes_apply32(arrays) -> int:
    shape = (len(arrays["slab_thickness_m"]), len(arrays["pitch_y_m"]), len(arrays["pitch_x_m"]))
    return algorithmic_bytes_apply32(shape)


def engine_cpu_baseline(requests, results, budget_s: float = 15.0, two_level: bool = False) -> dict:
    """The CPU oracle on a bounded sample of every board's solve, extrapolated
    by the iteration counts the board needed on the GPU."""

    from oracle.oracle import OracleSystem

    total_s, sampled, sample_s, threads = 0.0, 0, 0.0, 1
    per_board = max(2, int(budget_s / max(1, len(requests)) / 0.02))
    for q, r in zip(requests, results):
        a = q.arrays
        oracle = OracleSystem.from_arrays(free=a["free_nodes"], **{k: v for k, v in a.items() if k != "free_nodes"})
        threads = oracle.threads
        rhs = q.rhs
        peak = float(np.max(np.abs(rhs)))
        scale = 2.0 ** -np.frexp(peak)[1] if peak > 0 else 1.0
        iters = max(2, min(per_board, 50))
        oracle.inner_iterations(rhs * scale, 1)
        t0 = time.perf_counter()
        oracle.inner_iterations(rhs * scale, iters)
        per_iteration = (time.perf_counter() - t0) / iters
        t0 = time.perf_counter()
        oracle.apply_f64(rhs, fast=True)
        per_apply64 = time.perf_counter() - t0
        sample_s += per_iteration * iters + per_apply64
        sampled += iters
        if two_level:
            from oracle.oracle import choose_block_size

            layers, rows, cols = oracle.node_shape
            b = choose_block_size(oracle.node_shape)
            per_iteration += coarse_step_model_seconds(oracle.size, layers * -(-rows // b) * -(-cols // b))
        total_s += per_iteration * r["inner_iterations"] + per_apply64 * (r["outer_iterations"] + 1)
    return {
        "value": len(requests) / total_s,
        "unit": UNIT,
        "cores": threads,
        "kind": "port",
        "sample": (f"{sampled} FP32 Jacobi-PCG iterations and one FP64 apply per board over all {len(requests)} "
                   f"boards ({sample_s:.1f} s on {threads} threads)"
                   + (", plus a modelled two-level coarse correction per iteration (restriction, FP32 inverse "
                      "matvec, prolongation of the board's coarse size)" if two_level else "")
                   + ", each extrapolated to the inner iterations and FP64 residuals that board needed"),
        "solve_s_extrapolated": total_s,
    }


def run_engine(args, device: int) -> dict:
    """Batched (c4) or served (c5) solves through the batch engine."""

    import torch

    from pcb_analysis_b200._native import BatchEngine, DeviceSystem
    from pcb_analysis_b200.serve import poisson_arrivals, serve

    count = args.boards or (64 if args.workload == "c4" else 32)
    requests = engine_requests(args.workload, count)
    config = mpir_config()
    n = len(requests)
    max_slabs = max(len(q.arrays["slab_thickness_m"]) for q in requests)
    engine = BatchEngine(capacity=min(256, n), max_slabs=max_slabs, tile_rows=args.tile_rows, staging=args.staging,
                         budget_bytes=int(80e9), device=device, preconditioner=args.preconditioner)
    stream = torch.cuda.ExternalStream(engine.stream_handle(), device=f"cuda:{device}")
    apply_ms = None

    def resident_pass(timed: bool, time_apply: bool = False):
        nonlocal apply_ms
        tickets = [engine.submit(q.arrays, q.rhs, config) for q in requests]
        if any(t is None for t in tickets):
            raise SystemExit("the engine refused a board of the batch")
        if time_apply:
            apply_ms = engine.time_apply(5)
        torch.cuda.synchronize(device)
        launches0 = engine.info()["kernel_launches"]
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        t0 = time.perf_counter()
        seen: dict[int, float] = {}
        while len(seen) < n:
            engine.step()
            for t in engine.finished():
                seen.setdefault(t, time.perf_counter() - t0)
        end.record(stream)
        torch.cuda.synchronize(device)
        launches = engine.info()["kernel_launches"] - launches0
        wall = time.perf_counter() - t0
        results = [engine.collect(t) for t in tickets]
        return results, start.elapsed_time(end), [seen[t] for t in tickets], wall, launches

    for w in range(args.warmup):
        resident_pass(False, time_apply=(w == 0))
    sampler = ClockSampler(device)
    sampler.start()
    device_ms, latencies, launches, results = 0.0, [], 0, None
    for _ in range(args.steps):
        results, ms, done_at, _, launched = resident_pass(True)
        device_ms += ms
        latencies += done_at
        launches += launched
    clocks = sampler.stop()
    value = args.steps * n / (device_ms * 1e-3)
    tile_rows = engine.info()["tile_rows"]
    staging = engine.info()["staging"]

    # ---- e2e: the served stream from host arrays (upload, prepare, solve, download)
    rate = args.rate if args.workload == "c5" else None
    arrivals = poisson_arrivals(n, rate, seed=1) if rate else [0.0] * n
    report = serve(requests, arrivals, config, engine=engine)
    served_lat = [r.latency_s for r in report.results]
    e2e = {
        "value": report.solves_per_s, "unit": UNIT,
        "h2d_bytes_per_step": int(sum(16 * q.arrays["k_in"].size + 17 * q.nodes for q in requests)),
        "d2h_bytes_per_step": int(sum(8 * q.nodes for q in requests)),
        "requests": n, "wall_s": report.wall_s,
        "arrivals": f"Poisson {rate}/s" if rate else "all at t=0",
        "latency_s": {"p50": float(np.percentile(served_lat, 50)), "p99": float(np.percentile(served_lat, 99))},
        "converged": all(r.result.converged for r in report.results),
    }
    engine.close()

    # ---- serial single-board baselines on the same boards (inputs resident)
    fp64_s, mpir_s, max_dt, max_rel_dt, fp64_iters = 0.0, 0.0, 0.0, 0.0, []
    mpir_serial = not args.no_serial_mpir
    for q, r in zip(requests, results):
        with DeviceSystem(**q.arrays, device=device) as dev:
            rhs = torch.as_tensor(q.rhs, device=f"cuda:{device}")
            x64 = torch.zeros_like(rhs)
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            pcg = dev.solve_pcg_f64_device(rhs, x64, relative_tolerance=1e-10, max_iterations=4_000_000)
            fp64_s += time.perf_counter() - t0
            fp64_iters.append(pcg["iterations"])
            if mpir_serial:
                dev.set_preconditioner(args.preconditioner)
                x = torch.zeros_like(rhs)
                torch.cuda.synchronize(device)
                t0 = time.perf_counter()
                dev.solve_mpir_device(rhs, x, config)
                mpir_s += time.perf_counter() - t0
        ref = x64.cpu().numpy()
        free = q.arrays["free_nodes"].astype(bool)
        dt = float(np.max(np.abs(r["solution"][free] - ref[free]))) if free.any() else 0.0
        max_dt = max(max_dt, dt)
        rise = float(np.max(np.abs(ref[free]))) if free.any() else 0.0
        max_rel_dt = max(max_rel_dt, dt / rise if rise > 0 else 0.0)

    cpu = None if args.no_cpu_baseline else engine_cpu_baseline(requests, results,
                                                                two_level=args.preconditioner == "two-level")
    peak, peak_kind = measured_peak()
    bytes_apply = sum(board_bytes_apply32(q.arrays) for q in requests)
    achieved = bytes_apply / (apply_ms * 1e-3) / 1e9 if apply_ms else None
    nodes = [q.nodes for q in requests]
    return {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": device_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 inner / f64 outer",
        "data": "synthetic",
        "config": {
            "workload": ENGINE_WORKLOADS[args.workload],
            "boards_per_step": n,
            "nodes_total": int(sum(nodes)),
            "nodes_min_max": [int(min(nodes)), int(max(nodes))],
            "solver": (f"MPIR: FP32 PCG ({args.preconditioner} preconditioner) inner rtol 1e-4, FP64 residual/update "
                       "to rtol 1e-10, all boards in one graph-captured kernel set with per-board masks"),
            "tile_rows": tile_rows,
            "staging": staging,
            "step": "every board of the batch admitted (resident in HBM), then run until all have converged",
            "l2": "working set of the batch >> 126 MB L2: no flush between steps",
            "parallelism": "replicas x1",
        },
        "latency_ms": {"p50": float(np.percentile(latencies, 50)) * 1e3, "p99": float(np.percentile(latencies, 99)) * 1e3,
                       "of": "completion time of each board from the start of its batch, resident inputs"},
        "accuracy": {
            "converged": all(r["converged"] for r in results),
            "max_relative_residual": max(r["relative_residual"] for r in results),
            "max_abs_dT_K_vs_fp64_pcg": max_dt,
            "max_rel_dT_vs_fp64_pcg": max_rel_dt,
        },
        "iterations": {"inner_total": int(sum(r["inner_iterations"] for r in results)),
                       "inner_max": int(max(r["inner_iterations"] for r in results)),
                       "fp64_pcg_total": int(sum(fp64_iters))},
        "fp64_serial": {"solves_per_s": n / fp64_s, "solve_s_total": fp64_s, "speedup_of_batched": value * fp64_s / n,
                        "speedup_of_served_e2e": e2e["value"] * fp64_s / n,
                        "timing": "one DeviceSystem per board, tb_solve_pcg_f64_device from resident inputs"},
        "mpir_serial": ({"solves_per_s": n / mpir_s, "solve_s_total": mpir_s, "speedup_of_batched": value * mpir_s / n}
                        if mpir_serial else None),
        "roofline": {
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None,
            "peak_kind": peak_kind,
            "traffic": profiled_traffic(args.workload),
            "kernel": (f"batch_apply32<{tile_rows}> (FP32 Q1 action over every board of the batch, stages filled by "
                       f"{'tensor copies' if staging == 'tensor' else 'cp.async'})"),
            "bytes_per_launch": bytes_apply,
            "avg_launch_ms": apply_ms,
            "timing": "store-epilogue launches over all boards, CUDA events, between chunks",
        },
        "gpu_launches": launches,
        "clocks": clocks,
        "e2e": e2e,
        "cpu_baseline": cpu,
    }


def engine_summary(args, device: int, workload: str) -> dict:
    """The batched (c4) or served (c5) measurement, condensed for the
    single-board line: solves/s, latency, the serial FP64 PCG ratio, accuracy
    and the served stream from host arrays."""

    sub = argparse.Namespace(**vars(args))
    sub.workload = workload
    sub.boards = 64 if workload == "c4" else 32
    sub.steps, sub.warmup = 2, 1
    sub.preconditioner = "two-level"
    sub.no_cpu_baseline = True
    sub.no_serial_mpir = True
    t0 = time.perf_counter()
    line = run_engine(sub, device)
    return {
        "workload": line["config"]["workload"],
        "boards": line["config"]["boards_per_step"],
        "solves_per_s": line["value"],
        "latency_ms": {k: line["latency_ms"][k] for k in ("p50", "p99")},
        "fp64_serial_solves_per_s": line["fp64_serial"]["solves_per_s"],
        "speedup_vs_fp64_serial": line["fp64_serial"]["speedup_of_batched"],
        "served_e2e": {k: line["e2e"][k] for k in ("value", "arrivals", "latency_s", "converged")},
        "speedup_served_e2e_vs_fp64_serial": line["fp64_serial"]["speedup_of_served_e2e"],
        "accuracy": line["accuracy"],
        "solver": line["config"]["solver"],
        "steps": sub.steps, "warmup": sub.warmup,
        "roofline_frac": line["roofline"]["frac"],
        "clocks": line["clocks"],
        "wall_s": round(time.perf_counter() - t0, 1),
    }


def run_single(args, device: int, rank: int, world: int, dist) -> dict | None:
    """One board (c1, c2, c3): MPIR solves from zero with the board resident."""

    import torch

    import pcb_analysis_b200.thermal as ns
    from pcb_analysis_b200.thermal.operator import MatrixFreeThermalOperator

    problem, description = build_problem(args.workload, rank, args.cells)
    op = MatrixFreeThermalOperator(problem, preconditioner=args.preconditioner, device_id=device)
    dev = op.device_system
    if args.apply_plan:
        dev.apply_plan = tuple(int(v) for v in args.apply_plan.split(","))
    if args.ml_fine != "auto" and args.preconditioner == "multilevel":
        dev.ml_staging = args.ml_fine == "staged"
    config = mpir_config()
    rhs_host = op.build_rhs(op.default_reference_temperature())
    rhs = torch.as_tensor(rhs_host, device=f"cuda:{device}")
    x = torch.zeros_like(rhs)
    stream = torch.cuda.ExternalStream(dev.stream_handle(), device=f"cuda:{device}")

    def step() -> dict:
        x.zero_()
        return dev.solve_mpir_device(rhs, x, config)

    for _ in range(args.warmup):
        step()

    # ---------------------------------------------------------------- timed
    sampler = ClockSampler(device)
    sampler.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(device)
    launches0 = dev.launch_count()
    clock0 = dev.kernel_clock()
    events = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    events[0].record(stream)
    results = []
    for k in range(args.steps):
        results.append(step())
        events[k + 1].record(stream)
    torch.cuda.synchronize(device)
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    launches = dev.launch_count() - launches0
    clock1 = dev.kernel_clock()
    step_ms = [events[k].elapsed_time(events[k + 1]) for k in range(args.steps)]
    total_ms = events[0].elapsed_time(events[-1])
    apply_ms = clock1["apply_f32"][0] - clock0["apply_f32"][0]
    apply_n = clock1["apply_f32"][1] - clock0["apply_f32"][1]
    apply64_ms = clock1["apply_f64"][0] - clock0["apply_f64"][0]
    fine_ms = clock1["ml_update"][0] - clock0["ml_update"][0]
    fine_n = clock1["ml_update"][1] - clock0["ml_update"][1]
    value, slowest_ms = whole_job_rate(total_ms / args.steps, 1, world, dist, f"cuda:{device}")
    total_ms = slowest_ms * args.steps
    result = results[-1]
    solution = x.detach().cpu().numpy()
    free = op.free_nodes.reshape(-1)

    # ------------------------------- FP64 PCG baselines on the same board
    def fp64(multilevel: bool) -> tuple[dict, np.ndarray, float]:
        x64 = torch.zeros_like(rhs)
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        out = dev.solve_pcg_f64_device(rhs, x64, relative_tolerance=1e-10, max_iterations=4_000_000,
                                       multilevel=multilevel)
        torch.cuda.synchronize(device)
        seconds = time.perf_counter() - t0  # the solve alone; its solution is read back after the clock stops
        return out, x64.detach().cpu().numpy(), seconds

    same = args.preconditioner == "multilevel"
    fp64(same)  # warm-up: the FP64 chunk graphs are captured on first use, as the MPIR ones were in its warm-up
    pcg, pcg_solution, pcg_s = fp64(same)
    fp64_same = {"preconditioner": "multilevel" if same else "jacobi", "solve_s": pcg_s, "solves_per_s": 1.0 / pcg_s,
                 "iterations": pcg["iterations"], "relative_residual": pcg["relative_residual"],
                 "converged": pcg["converged"], "speedup_of_mpir": value * pcg_s,
                 "like_for_like": same or args.preconditioner == "jacobi"}
    fp64_jacobi = None
    if same and (args.fp64_jacobi or args.workload in ("c1", "c2")):
        fp64(False)
        jac, _, jac_s = fp64(False)
        fp64_jacobi = {"preconditioner": "jacobi", "solve_s": jac_s, "solves_per_s": 1.0 / jac_s,
                       "iterations": jac["iterations"], "relative_residual": jac["relative_residual"],
                       "converged": jac["converged"], "speedup_of_mpir": value * jac_s}
    max_dt = float(np.max(np.abs(solution[free] - pcg_solution[free])))
    max_rise = float(np.max(np.abs(pcg_solution[free])))

    # ------------------------------------------------------------ roofline
    shape = problem.mesh.element_grid_shape
    bytes_apply = algorithmic_bytes_apply32(shape)
    peak, peak_kind = measured_peak()
    achieved = bytes_apply / (apply_ms / apply_n * 1e-3) / 1e9 if apply_n > 0 else None
    operator_roofline = {
        "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
        "traffic": profiled_traffic(args.workload, "apply_f32", problem.mesh.size), "bytes_per_launch": bytes_apply,
        "avg_launch_ms": apply_ms / apply_n if apply_n > 0 else None, "launches": apply_n,
        "share_of_solve_time": apply_ms / total_ms if total_ms > 0 else None,
    }
    fine_roofline = None
    if fine_n > 0:
        # ml_update, iteration form: read q, r, l, 1/p and write r, T^-1 r: 24 B per node
        fine_bytes = 24 * problem.mesh.size
        fine_achieved = fine_bytes / (fine_ms / fine_n * 1e-3) / 1e9
        fine_roofline = {
            "bound": "hbm", "achieved": fine_achieved, "peak": peak, "unit": "GB/s", "frac": fine_achieved / peak,
            "peak_kind": peak_kind, "traffic": profiled_traffic(args.workload, "ml_update", problem.mesh.size),
            "bytes_per_launch": fine_bytes,
            "avg_launch_ms": fine_ms / fine_n, "launches": fine_n, "share_of_solve_time": fine_ms / total_ms,
            "kernel": ("ml_update_staged<NP> (PCG update, z-line column solve, restriction, r.r and r.z; column "
                       "boxes staged by tensor copies)" if dev.ml_staging else
                       "ml_update<NP, ML_ITER> (PCG update, z-line column solve, restriction, r.r and r.z)"),
        }

    # ------------------------------------------------------------------ e2e
    e2e = None
    if rank == 0 and args.e2e_steps > 0:
        samples = []
        sol = None
        for _ in range(args.e2e_steps):
            t0 = time.perf_counter()
            sol = ns.solve_thermal_conduction(problem, preconditioner=args.preconditioner, config=config,
                                              device_id=device)
            samples.append(time.perf_counter() - t0)
        e2e_s = float(np.median(samples))
        n, e = problem.mesh.size, int(np.prod(shape))
        # The board goes up as its problem and is prepared on the device; the
        # right-hand side, the solve and the post-processing stay in HBM.
        # Uploaded: k_in, k_z, pitches, heat-source entries, the fixed mask
        # and values when there are fixed nodes.  Downloaded: the solution
        # and the heat flux.
        entries = sum(len(src.nodes) for src in problem.heat_sources)
        fixed_bytes = 9 * n if problem.fixed_temperature_mask.any() else 0
        h2d = 2 * 8 * e + 8 * (sum(shape)) + 16 * entries + fixed_bytes
        d2h = 8 * n + 3 * 8 * e
        e2e = {"value": 1.0 / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "statistic": f"median of {len(samples)} calls", "samples_s": [round(v, 4) for v in samples],
               "converged": bool(sol.solve.converged), "heat_balance_error_w": sol.heat_balance_error_w,
               "path": "solve_thermal_conduction from host NumPy arrays: upload, device preparation, "
                       "preconditioner set-up, MPIR, heat budget and flux, downloads"}

    # -------------------------------------------------- CPU baseline, extras
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(CpuModel(args.workload, problem), iterations=2 if args.workload == "c3" else 10)
    preconditioner_info = dev.preconditioner()
    apply_plan = list(dev.apply_plan)
    ml_fine = ("staged" if dev.ml_staging else "loading") if args.preconditioner == "multilevel" else None
    op.close()
    extras = {}
    if rank == 0 and world == 1 and args.workload == "c3" and not args.no_engine:
        for workload in ("c4", "c5"):
            extras[workload] = engine_summary(args, device, workload)
    if rank != 0:
        return None
    ordered = sorted(step_ms)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 inner / f64 outer",
        "data": "synthetic",
        # the workload alone, the same object in the reference arm's line; how
        # each arm solves it is under "solver"
        "config": single_board_config(args.workload, description, problem),
        "solver": {
            "method": (f"MPIR: FP32 PCG ({args.preconditioner} preconditioner) inner rtol 1e-4, FP64 "
                       "residual/update/norm to rtol 1e-10, every solve complete"),
            "preconditioner": preconditioner_info,
        },
        "parallelism": f"replicas x{world}",
        "latency_ms": {"p50": float(np.percentile(ordered, 50)), "p99": float(np.percentile(ordered, 99)),
                       "steps": [round(v, 3) for v in step_ms]},
        "iterations": {"outer": result["outer_iterations"], "inner": result["inner_iterations"],
                       "history": [list(h) for h in result["history"]]},
        "accuracy": {
            "relative_residual": result["relative_residual"],
            "converged": result["converged"],
            "max_abs_dT_K_vs_fp64_pcg": max_dt,
            "max_rel_dT_vs_fp64_pcg": max_dt / max_rise if max_rise > 0 else 0.0,
            "max_rise_K": max_rise,
            "against": f"FP64 PCG ({fp64_same['preconditioner']}) on the same board, rtol 1e-10",
        },
        "fp64_pcg": fp64_same,
        "fp64_jacobi_pcg": fp64_jacobi,
        # the dominant kernel of the timed solves, by device time
        "roofline": (fine_roofline if fine_roofline is not None and fine_ms > apply_ms
                     else dict(operator_roofline, kernel=operator_kernel_name(apply_plan))),
        "roofline_operator": dict(operator_roofline, kernel=operator_kernel_name(apply_plan)),
        "roofline_fine_pass": fine_roofline,
        "kernel_time_ms": {"apply_f32": apply_ms, "ml_update": fine_ms, "apply_f64": apply64_ms, "total": total_ms},
        "apply_plan": apply_plan,
        "ml_fine_pass": ml_fine,
        "gpu_launches": launches,
        "clocks": clocks,
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    line.update(extras)
    return line


def run_profile_case(args, device: int) -> None:
    """Profiling harness, not a bench line: the board's system and one MPIR
    solve, so that a launch list under ncu stays a few tens of thousands of
    launches long (a bench run, with its warm-up solves and the FP64 PCG,
    makes about five times as many)."""

    import torch

    from pcb_analysis_b200.thermal.operator import MatrixFreeThermalOperator

    problem, description = build_problem(args.workload, 0, args.cells)
    op = MatrixFreeThermalOperator(problem, preconditioner=args.preconditioner, device_id=device)
    try:
        dev = op.device_system
        if args.apply_plan:
            dev.apply_plan = tuple(int(v) for v in args.apply_plan.split(","))
        rhs = torch.as_tensor(op.build_rhs(op.default_reference_temperature()), device=f"cuda:{device}")
        x = torch.zeros_like(rhs)
        launches0 = dev.launch_count()
        out = dev.solve_mpir_device(rhs, x, mpir_config())
        torch.cuda.synchronize(device)
        print(json.dumps({"profile_case": description, "converged": out["converged"],
                          "inner_iterations": out["inner_iterations"], "history": out["history"],
                          "set_up_launches": launches0, "solve_launches": dev.launch_count() - launches0}),
              flush=True)
    finally:
        op.close()


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=5)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=["b200", "reference"], default="b200")
    parser.add_argument("--workload", choices=["c3", "c2", "c1", "c4", "c5", "dc"], default="c3")
    parser.add_argument("--e2e-steps", type=int, default=5)
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--no-engine", action="store_true", help="c3: leave out the c4 / c5 sub-objects")
    parser.add_argument("--fp64-jacobi", action="store_true",
                        help="also time the plain FP64 Jacobi PCG (always on c1 and c2)")
    parser.add_argument("--boards", type=int, default=0, help="boards per batch (c4) or requests (c5)")
    parser.add_argument("--rate", type=float, default=4.0, help="c5 Poisson arrival rate, requests/s")
    parser.add_argument("--tile-rows", type=int, default=0, help="batched FP32 tile height (0: autotuned)")
    parser.add_argument("--staging", choices=["auto", "cp.async", "tensor"], default="auto",
                        help="batched FP32 operator staging (auto: timed with the tile height)")
    parser.add_argument("--no-serial-mpir", action="store_true")
    parser.add_argument("--preconditioner", choices=["multilevel", "two-level", "jacobi"], default=None,
                        help="inner PCG preconditioner (default: multilevel for one board, two-level for the "
                             "batch engine)")
    parser.add_argument("--apply-plan", default="", help="FP32 operator launch plan kind,rows,zw,sl,band "
                        "(default: the one the autotuner picks)")
    parser.add_argument("--ml-fine", choices=["auto", "staged", "loading"], default="auto",
                        help="multilevel fine pass: the tensor-copy fed kernel or the one that loads its columns "
                             "(default: the library's default, the loading kernel)")
    parser.add_argument("--profile-case", action="store_true",
                        help="profiling harness: set up the board and run one solve (prints no bench line)")
    parser.add_argument("--cells", type=int, default=0,
                        help="c1/c2/c3: a board of this many cells per side with the same rules (profiling cases)")
    args = parser.parse_args()
    if args.warmup < 3:
        parser.error("--warmup must be at least 3")
    if args.preconditioner is None:
        args.preconditioner = "two-level" if args.workload in ("c4", "c5", "dc") else "multilevel"

    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local_rank = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    if args.profile_case:
        run_profile_case(args, local_rank)
        return

    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    device = local_rank if world > 1 else 0
    torch.cuda.set_device(device)

    if args.workload == "dc":
        line = run_dc(args, device)
    elif args.workload in ENGINE_WORKLOADS:
        line = run_engine(args, device)
        if world > 1:
            value, slowest = whole_job_rate(line["ms_per_step"], line["config"]["boards_per_step"], world, dist,
                                            f"cuda:{device}")
            line["value"], line["ms_per_step"] = value, slowest
            line["n_gpus"] = world
            line["config"]["parallelism"] = f"replicas x{world}"
    else:
        line = run_single(args, device, rank, world, dist)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
