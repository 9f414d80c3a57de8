"""Benchmark: cell-solves/s of the Rosenbrock chemistry solve on the GPU.

Workload (the metric's configuration): seeded 210-species / 440-reaction
mechanism, 1,048,576 grid cells, half of them at night (photolysis off),
T ~ U(200, 310) K, four-stage Rosenbrock, one Solve(dt = 600 s) per step,
per-cell step control.  A step restores the initial concentrations (device
copy) and solves every cell; inputs (1.8 GB state + 3.7 GB rate constants)
exceed the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
    python bench.py --workload c600     # 600 species / 1,500 reactions, 262,144 cells
    python bench.py --workload ts1      # micm's TS1 benchmark mechanism, 1,048,576 cells, dt = 30 s
    python bench.py --workload chapman  # micm_bench's default mechanism (Chapman), 1,048,576 cells

N > 1 runs under torchrun: each rank solves its own 1M-cell shard (weak
scaling; cells are independent, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-solves/s @1M cells, FP64 rtol1e-6 (fused vs plain); adjoint/forward time"
UNIT = "cell-solves/s"
KERNEL_OF_VARIANT = {0: "k_fused_stream", 1: "k_fused", 2: "k_fused_thread"}
# workload -> cells per GPU, description, the adjoint timing that goes with it
# (configuration, cells, checkpoints per cell), host-CPU sample, ncu capture of
# the fused kernel whose DRAM bytes per cell-solve scale the traffic figure
WORKLOADS = {
    "c210_uneven": dict(cells=1048576, cpu_sample=65536,
                        text="210 species, 440 reactions, {cells} cells per GPU, half night, T~U(200,310) K, "
                             "4-stage Rosenbrock, dt=600 s, per-cell step control, fused persistent kernel",
                        l2="inputs exceed L2 (1.8 GB state + 3.7 GB rate constants); no flush",
                        adjoint=("c60_adjoint", 131072, 256),
                        profile="k_fused_thread_c210_65536cells.md"),
    "c600": dict(cells=262144, cpu_sample=16384,
                 text="600 species, 1,500 reactions, {cells} cells per GPU, 4-stage Rosenbrock, dt=600 s, "
                      "per-cell step control, fused persistent kernel (LU factor of 11,304 entries per cell, "
                      "beyond shared memory)",
                 l2="inputs exceed L2 (1.3 GB state + 3.1 GB rate constants); no flush",
                 adjoint=("c600", 262144, 160),
                 profile="k_fused_thread_c600_65536cells.md"),
    "chapman": dict(cells=1048576, cpu_sample=262144,
                    text="micm's Chapman benchmark mechanism (9 species, 7 reactions) on {cells} cells per GPU, "
                         "micm_bench's initial state on every cell, 3-stage Rosenbrock, dt=30 s, fused persistent "
                         "kernel",
                    l2="inputs exceed L2 (75 MB state + 59 MB rate constants + 25 MB parameters); no flush",
                    adjoint=None, profile=None),
    "ts1": dict(cells=1048576, cpu_sample=65536,
                text="micm's TS1 benchmark mechanism (209 species, 547 reactions) on {cells} cells per GPU, "
                     "micm_bench's initial state on every cell, 3-stage Rosenbrock, dt=30 s, fused persistent kernel",
                l2="inputs exceed L2 (1.8 GB state + 4.6 GB rate constants); no flush",
                adjoint=None, profile="k_fused_thread_ts1_65536cells.md"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c210_uneven", choices=sorted(WORKLOADS))
    ap.add_argument("--cells", type=int, default=None, help="cells per GPU (default: the workload's)")
    ap.add_argument("--plain-cells", type=int, default=None,
                    help="cells per GPU for the plain-method comparison (0 = skip; default: --cells)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward timing")
    ap.add_argument("--no-autotune", action="store_true",
                    help="fixed fused configuration (one cell per thread) instead of the autotuner")
    ap.add_argument("--cpu-sample", type=int, default=None, help="cells timed on the host CPU")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if args.cells is None:
        args.cells = w["cells"]
    if args.plain_cells is None:
        args.plain_cells = args.cells
    if args.cpu_sample is None:
        args.cpu_sample = w["cpu_sample"]
    return args


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def max_over_ranks(values, dist, device):
    """Element-wise maximum of per-rank timings (the slowest rank sets the job time)."""
    if not dist:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def job_throughput(cells_per_rank: int, world: int, steps: int, seconds: float) -> float:
    """Cell-solves per second of the whole job: every rank solves its own shard."""
    return cells_per_rank * world * steps / seconds


def workload(name: str, cells: int, rank: int = 0):
    from micm_b200 import synthetic
    if name in ("ts1", "chapman"):
        # micm_bench's cases: the benchmark's initial state on every cell
        from micm_b200 import micm_bench
        cfg = dict(stages=micm_bench.TABLEAU, dt=micm_bench.DT, seed=0, inputs={})
        return cfg, micm_bench.mechanism(name), micm_bench.inputs(name, cells)
    cfg = synthetic.CONFIGS[name]
    mech = cfg["mech"]()
    inputs = synthetic.cell_inputs(mech, cells, cfg["seed"] + 1000 * rank, **cfg["inputs"])
    return cfg, mech, inputs


def cpu_reference(mech, cfg, inputs, sample: int, uniform: bool = False):
    """micm's own CPU solver (oracle/_ref) over a bounded sample of the workload.

    The baseline figure is micm built for speed (libmicm_ref_fast.so: -O3,
    AVX2, multiply-add contraction); the bit-exact parity build (no
    contraction) is timed beside it, and its results are returned for the
    parity check of the GPU's results on the same cells.

    Cells that share their inputs (micm_bench's TS1 case) are timed in micm's
    fastest CPU layout, vector ordering with L = 128 (one State and step size
    per 128 cells), which solves them exactly as per-cell control does.  Cells
    with their own inputs need one step size each, so the baseline is one
    1-cell State per cell (micm's idiom for independent cells); the grouped
    layout is reported beside it for a smaller sample, as it solves a
    different problem there (each group steps at its hardest cell's pace).

    Returns (baseline dict, parity build's final concentrations, its per-cell
    accepted-step counts), or (None, None, None) without the reference."""
    import oracle
    if not oracle.reference_available():
        return None, None, None
    fast = oracle.reference_available(fast=True)
    n = min(sample, len(inputs["temperature"]))
    sub = {k: v[:n] for k, v in inputs.items()}
    threads = os.cpu_count() or 1
    layout_v128 = (f"micm CpuSolverBuilderInPlace with vector ordering L=128 (in-place Mozart LU), one State "
                   f"per 128 cells over {threads} host threads")
    layout_cell = (f"one 1-cell micm State per cell over {threads} host threads, micm CpuSolverBuilderInPlace "
                   "(vector ordering L=1, in-place Mozart LU)")
    build_fast = "micm built -O3 -march=x86-64-v3 (FMA contraction on)"
    build_exact = "micm built -O3 -march=x86-64-v3 -ffp-contract=off (the bit-exact parity build)"

    def timed(fast_build):
        ref = oracle.Reference(mech, tableau=cfg["stages"], fast=fast_build)
        t0 = time.perf_counter()
        if uniform:
            y, st = ref.solve_groups_v128(sub, cfg["dt"], group=128, threads=threads)
        else:
            y, st = ref.solve_per_cell(sub, cfg["dt"], threads=threads)
        return time.perf_counter() - t0, y, st

    t_exact, y_ref, st_ref = timed(False)
    t_base, build = (timed(True)[0], build_fast) if fast else (t_exact, build_exact)
    layout = layout_v128 if uniform else layout_cell
    out = {"value": n / t_base, "unit": UNIT, "cores": threads, "kind": "reference",
           "sample": f"{n} cells of the workload, {layout}, {build}, {t_base:.1f} s",
           "parity_build": {"value": n / t_exact, "unit": UNIT, "sample": f"same cells, {build_exact}, "
                                                                          f"{t_exact:.1f} s"}}
    if not uniform:
        ng = min(n, 16384)
        ref = oracle.Reference(mech, tableau=cfg["stages"], fast=fast)
        t0 = time.perf_counter()
        ref.solve_groups_v128({k: v[:ng] for k, v in inputs.items()}, cfg["dt"], group=128, threads=threads)
        tg = time.perf_counter() - t0
        out["vector128_groups"] = {"value": ng / tg, "unit": UNIT,
                                   "sample": f"{ng} cells, {layout_v128}, {build if fast else build_exact}, "
                                             f"{tg:.1f} s; one step size per group, so not the per-cell solve"}
    return out, y_ref, np.asarray(st_ref)[:, 3]


def parity_summary(y_gpu, acc_gpu, y_ref, acc_ref, rtol=1e-6, atol=1e-12):
    """The GPU's final concentrations and accepted-step counts against micm's on
    the same cells: the parity criterion (every species within rtol / atol,
    identical step counts in at least 99.9 % of cells)."""
    d = np.abs(y_gpu - y_ref)
    bound = atol + rtol * np.abs(y_ref)
    sig = np.abs(y_ref) >= atol
    return {"cells": int(len(y_ref)), "rtol": rtol, "atol": atol,
            "frac_cells_within_rtol_atol": float(np.mean(np.all(d <= bound, axis=1))),
            "max_err_over_bound": float(np.max(d / bound)),
            "max_rel_err": float(np.max(d[sig] / np.abs(y_ref[sig]))) if sig.any() else 0.0,
            "frac_identical_accepted": float(np.mean(np.asarray(acc_gpu) == np.asarray(acc_ref))),
            "frac_bitwise_identical_cells": float(np.mean(np.all(y_gpu == y_ref, axis=1)))}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg, mech, inputs = workload(args.workload, min(args.cells, args.cpu_sample * max(1, args.steps + args.warmup)))
    import oracle
    if not oracle.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmicm_ref.so was not built"}))
        return
    fast = oracle.reference_available(fast=True)
    ref = oracle.Reference(mech, tableau=cfg["stages"], fast=fast)
    build = ("micm built -O3 -march=x86-64-v3 (FMA contraction on)" if fast
             else "micm built -O3 -march=x86-64-v3 -ffp-contract=off")
    threads = os.cpu_count() or 1
    n = args.cpu_sample
    # identical cells (micm_bench's TS1 case): micm's vector-128 layout; else one 1-cell State per cell
    uniform = args.workload in ("ts1", "chapman")
    layout = ("vector ordering L=128, one State per 128 cells" if uniform else "1-cell micm States")
    times = []
    for i in range(args.warmup + args.steps):
        sub = {k: v[(i * n) % len(v):(i * n) % len(v) + n] for k, v in inputs.items()}
        t0 = time.perf_counter()
        if uniform:
            ref.solve_groups_v128(sub, cfg["dt"], group=128, threads=threads)
        else:
            ref.solve_per_cell(sub, cfg["dt"], threads=threads)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    t = float(np.sum(times))
    value = n * args.steps / t
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "impl": "reference",
            "config": {"workload": f"{args.workload}: "
                                   + WORKLOADS[args.workload]["text"].format(cells=args.cells)
                                   + f"; each step a {n}-cell sample on the host",
                       "cells_per_step": n},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"{n} cells per step, {layout} over {threads} threads, {build}"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def flops_per_solve_unit(mech, solver, stages):
    """Algorithmic FP64 operations of one unit of each kind of work (the
    operations the exact-order formulation performs; padding excluded)."""
    info = solver.compiled.info
    st = solver.compiled.stream_stats()
    S = mech.n_species
    react = [sum(1 for x in r.reactants if x >= 0) for r in mech.reactions]
    f_force = sum(react) + 2 * info["n_forcing_terms"]                 # w_r products, sum of nu w
    f_jac = sum(n * (n - 1) for n in react) + 2 * info["n_jacobian_terms"] + S   # dw products, sum, alpha
    f_lu = 2 * info["lu_updates"] + info["lu_lower"] + S                 # updates, pivot scalings, 1/a_kk
    f_solve = 2 * (st["forward"]["terms"] + st["backward"]["terms"]) + S  # both sweeps, diagonal divides
    f_attempt = 2 * S * (stages * (stages - 1) // 2) * 2 + 4 * S * stages + 6 * S  # stage sums, m/e sums, norm
    return dict(force=f_force, jac=f_jac, lu=f_lu, solve=f_solve, attempt=f_attempt)


def bytes_per_solve_unit(mech, solver, stages):
    """Compulsory HBM bytes of one unit of each kind of work when every working
    set lives in HBM (the plain kernels and the one-cell-per-thread kernel):
    -J assembly writes the factor (zeroed, then read-modify-written), the LU
    reads and writes it, each stage solve reads it once and its vector twice,
    a forcing evaluation reads the rate constants and three state-sized
    vectors, and each attempt's stage sums and error norm stream state-sized
    vectors."""
    info = solver.compiled.info
    S, R, nnz = mech.n_species, mech.n_reactions, info["jacobian_nnz"]
    n_axpy = stages * (stages - 1) + 2
    return dict(force=8 * (R + 3 * S), jac=8 * 3 * nnz, lu=8 * (2 * nnz + 2 * S), solve=8 * (nnz + 2 * S),
                attempt=8 * (3 * S * n_axpy + 4 * S))


def solve_bytes(units, stats):
    return (stats["function_calls"] * units["force"] + stats["jacobian_updates"] * units["jac"]
            + stats["decompositions"] * units["lu"] + stats["solves"] * units["solve"]
            + stats["number_of_steps"] * units["attempt"])


def hbm_peak():
    """HBM copy bandwidth measured on this pool (MEASURED_PEAKS.json), else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s"


def measured_traffic(profile, cells):
    """DRAM bytes of one fused launch over `cells` cells, scaled from the committed capture
    (None when the workload has no capture)."""
    if not profile:
        return None
    path = os.path.join(ROOT, "profiles", profile)
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_cell_solve:"):
                    return float(line.split(":")[1]) * cells
    except OSError:
        pass
    return None


def solve_flops(units, stats):
    return (stats["function_calls"] * units["force"] + stats["jacobian_updates"] * units["jac"]
            + stats["decompositions"] * units["lu"] + stats["solves"] * units["solve"]
            + stats["number_of_steps"] * units["attempt"])


def fp64_peak():
    """Nominal dense FP64 rate of the device: SMs x 64 FMA/clock x 2 x max SM clock
    (no FP64 figure is measured by the pool's peak probe)."""
    import torch
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    mhz = 1965.0
    try:
        out = subprocess.run(["nvidia-smi", "--query-gpu=clocks.max.sm", "--format=csv,noheader,nounits",
                              f"--id={torch.cuda.current_device()}"], capture_output=True, text=True, timeout=20)
        mhz = float(out.stdout.strip().splitlines()[0])
    except Exception:
        pass
    return p.multi_processor_count * 64 * 2 * mhz * 1e6 / 1e12


def adjoint_ratio(torch, rank, name, n, max_checkpoints, fused_config=None):
    """Adjoint/forward time of `n` cells of configuration `name` (autotuned
    unless the fused configuration is given)."""
    from micm_b200 import Solver, synthetic
    cfg = synthetic.CONFIGS[name]
    mech = cfg["mech"]()
    inputs = synthetic.cell_inputs(mech, n, cfg["seed"] + 1000 * rank, **cfg["inputs"])
    solver = Solver(mech, cfg["stages"], vector_length=128)
    st = solver.get_state(n)
    st.set_inputs(inputs)
    st.sync_inputs_to_device()
    solver.update_state_parameters(st)
    if fused_config:
        solver.set_fused_config(**fused_config)
        tuned = solver.get_fused_config()
    else:
        tuned = solver.autotune(cfg["dt"], st)
    rng = np.random.default_rng(cfg["seed"])
    target = rng.random(n) * 1e-9
    cols = solver.compiled.species_columns

    def forward():
        st.sync_inputs_to_device()
        solver.update_state_parameters(st)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = solver.solve(cfg["dt"], st, method="fused", step_control="per_cell")
        torch.cuda.synchronize()
        return time.perf_counter() - t0, r

    def adjoint(y_final):
        # the incoming gradient is prepared (vector layout, pinned host memory)
        # before the clock starts, as the forward's inputs are; the call and
        # the download of dL/dy0 and dL/dlog k are timed
        import ctypes
        from micm_b200._native import check, lib
        from micm_b200._abi import SolverStats
        from micm_b200.mechanism import to_vector_layout
        g = np.zeros((n, mech.n_species))
        g[:, cols[0]] = 2.0 * (y_final[:, cols[0]] - target)
        g_vec = torch.from_numpy(to_vector_layout(g, st.L)).pin_memory().numpy()
        dy0 = torch.empty(g_vec.shape[0], dtype=torch.float64).pin_memory().numpy()
        dk = np.zeros(max(mech.n_reactions, 1))
        stats = SolverStats()
        f64 = ctypes.POINTER(ctypes.c_double)
        st.sync_inputs_to_device()
        solver.update_state_parameters(st)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        check(lib().micmb_solve_adjoint(solver.handle, st.handle, float(cfg["dt"]), g_vec.ctypes.data_as(f64),
                                        dy0.ctypes.data_as(f64), dk.ctypes.data_as(f64), int(max_checkpoints),
                                        ctypes.byref(stats)))
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    forward()
    tf, res = forward()
    st.sync_outputs_to_host()
    y_final = st.variables.copy()
    st.set_inputs(inputs)
    adjoint(y_final)
    ta = adjoint(y_final)
    return {"config": f"{name}: {mech.n_species} species, {mech.n_reactions} reactions, {n} cells, "
                      f"{cfg['stages']}-stage, dt={cfg['dt']:g} s, at most {max_checkpoints} accepted steps per cell; "
                      "loss = sum_c (y_c[0] - target_c)^2; gradients w.r.t. all y0 and all log k",
            "forward_ms": 1000 * tf, "adjoint_ms": 1000 * ta, "adjoint_over_forward": ta / tf,
            "accepted_per_cell": res.stats["accepted"] / n, "fused_config": tuned,
            "note": "adjoint time = one micmb_solve_adjoint call (forward solve with checkpoints, reverse sweep, "
                    "upload of dL/dy_final and download of dL/dy0 and dL/dlog k from pinned host memory); forward "
                    "time = one fused Solve, inputs already on the device"}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
        return
    import ctypes
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    # one explicit stream for the whole run: the state's kernels, the restore
    # copies and the timing events must share it (the legacy default stream's
    # handle is 0, which the library reads as "the state's own stream")
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from micm_b200 import Solver
    from micm_b200 import solver as sv
    from micm_b200._native import check, lib
    from micm_b200.mechanism import to_vector_layout

    W = WORKLOADS[args.workload]
    cfg, mech, inputs = workload(args.workload, args.cells, rank)
    L = 128
    solver = Solver(mech, cfg["stages"], vector_length=L)
    state = solver.get_state(args.cells)
    state.set_inputs(inputs)
    state.sync_inputs_to_device()
    solver.update_state_parameters(state)
    if args.no_autotune:
        solver.set_fused_config(variant=2, lu_in_shared=0)
        tuned = solver.get_fused_config()
    else:
        tuned = solver.autotune(cfg["dt"], state)              # cells-per-CTA, LU staging, ring depth, variant
    check(lib().micmb_state_set_stream(state.handle, ctypes.c_void_p(stream.cuda_stream)))
    y0_host = to_vector_layout(state.variables, L)
    y_dev = torch.from_numpy(y0_host).cuda()
    y_view = device_view(state, sv.BUF_VARIABLES)             # torch view of the state's own buffer

    def fused_step():
        y_view.copy_(y_dev)                                    # the step's inputs, already in HBM
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = solver.solve(cfg["dt"], state, method="fused", step_control="per_cell")
        e1.record(stream)
        return r, e0, e1

    for _ in range(args.warmup):
        fused_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    totals = {}
    kernel_ms = 0.0
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        start.record(stream)
        events = []
        for _ in range(args.steps):
            r, e0, e1 = fused_step()
            events.append((e0, e1))
            for key, v in r.stats.items():
                if isinstance(v, (int, float)):
                    totals[key] = totals.get(key, 0) + v
        end.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    kernel_ms = sum(a.elapsed_time(b) for a, b in events)

    # the same steps replayed from a CUDA graph (UpdateStateParameters + the
    # fused Solve captured once per state and time step, micmb_solve_graph)
    y_view.copy_(y_dev)
    solver.solve_graph(cfg["dt"], state, 1)                   # capture (and one run)
    graph_events = []
    torch.cuda.synchronize()
    for _ in range(args.steps):
        y_view.copy_(y_dev)
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        solver.solve_graph(cfg["dt"], state, 1)
        g1.record(stream)
        graph_events.append((g0, g1))
    torch.cuda.synchronize()
    graph_ms = sum(a.elapsed_time(b) for a, b in graph_events)
    ms, kernel_ms, graph_ms = max_over_ranks([ms, kernel_ms, graph_ms], dist, "cuda")

    # parity at the metric's scale: the fused solve's results on the cells the
    # CPU baseline solves (the first cpu_sample cells of this shard)
    n_par = min(args.cpu_sample, args.cells) if (rank == 0 and not args.no_cpu) else 0
    gpu_par = None
    if n_par:
        from micm_b200.mechanism import from_vector_layout, padded_cells
        y_view.copy_(y_dev)
        rpar = solver.solve(cfg["dt"], state, method="fused", step_control="per_cell", per_cell=True)
        torch.cuda.synchronize()
        n_pad = padded_cells(n_par, L)
        yv = y_view[: n_pad * mech.n_species].cpu().numpy()
        y_cols = from_vector_layout(yv, n_par, mech.n_species, L)
        gpu_par = (y_cols[:, solver.compiled.species_columns], rpar.per_cell_accepted[:n_par].copy())
    value = job_throughput(args.cells, world, args.steps, ms / 1000.0)
    attempts_per_cell = totals["number_of_steps"] / (args.cells * args.steps)
    accepted_per_cell = totals["accepted"] / (args.cells * args.steps)

    # roofline of the fused kernel.  One cell per thread keeps every working set
    # in HBM, so the bound is the compulsory traffic of that formulation
    # (bytes_per_solve_unit); the FP64 work is reported beside it.
    bunits = bytes_per_solve_unit(mech, solver, cfg["stages"])
    algo_bytes = solve_bytes(bunits, totals) / args.steps      # per launch (one Solve over the shard)
    kernel_s = kernel_ms / args.steps / 1000.0
    achieved_gbs = algo_bytes / kernel_s / 1e9
    peak_gbs, peak_src = hbm_peak()
    units = flops_per_solve_unit(mech, solver, cfg["stages"])
    flops = solve_flops(units, totals) / args.steps
    traffic = measured_traffic(W["profile"], args.cells)

    # e2e: the public API with host buffers every step (H2D inputs, D2H results)
    h_vars = torch.from_numpy(y0_host).pin_memory().numpy()
    cond = np.stack([state.temperature, state.pressure, state.air_density], axis=1)
    h_cond = torch.from_numpy(to_vector_layout(cond, L)).pin_memory().numpy()
    h_par = torch.from_numpy(to_vector_layout(state.custom_rate_parameters, L)).pin_memory().numpy()
    h_out = torch.empty(h_vars.shape[0], dtype=torch.float64).pin_memory().numpy()
    e2e_steps = max(1, min(args.steps, 2))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        state.upload(sv.BUF_VARIABLES, h_vars)
        state.upload(sv.BUF_CONDITIONS, h_cond)
        state.upload(sv.BUF_CUSTOM_PARAMS, h_par)
        solver.update_state_parameters(state)
        solver.solve(cfg["dt"], state, method="fused", step_control="per_cell")
        check(lib().micmb_state_download(state.handle, sv.BUF_VARIABLES,
                                         h_out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    torch.cuda.synchronize()
    e2e_t = time.perf_counter() - t0
    (e2e_t,) = max_over_ranks([e2e_t], dist, "cuda")
    h2d = h_vars.nbytes + h_cond.nbytes + h_par.nbytes
    d2h = h_out.nbytes

    # plain per-stage kernels on the same shard (one warm-up, one timed solve)
    plain = None
    if args.plain_cells:
        pc = min(args.plain_cells, args.cells)
        y_view.copy_(y_dev)
        pstate = state if pc == args.cells else None
        if pstate is None:
            _, _, pin = workload(args.workload, pc, rank)
            pstate = solver.get_state(pc)
            pstate.set_inputs(pin)
            pstate.sync_inputs_to_device()
        solver.update_state_parameters(pstate)
        pview = device_view(pstate, sv.BUF_VARIABLES)
        p0 = pview.clone()
        solver.solve(cfg["dt"], pstate, method="plain", step_control="per_cell")
        pview.copy_(p0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pres = solver.solve(cfg["dt"], pstate, method="plain", step_control="per_cell")
        torch.cuda.synchronize()
        pt = time.perf_counter() - t0
        (pt,) = max_over_ranks([pt], dist, "cuda")
        plain_gbs = solve_bytes(bytes_per_solve_unit(mech, solver, cfg["stages"]), pres.stats) / pt / 1e9
        plain = {"value": pc * world / pt, "unit": UNIT, "cells_per_gpu": pc, "ms_per_step": 1000 * pt,
                 "attempts_per_cell": pres.stats["number_of_steps"] / pc,
                 "fused_over_plain": value / (pc * world / pt),
                 "roofline": {"bound": "hbm", "achieved": plain_gbs, "peak": peak_gbs, "unit": "GB/s",
                              "frac": plain_gbs / peak_gbs,
                              "note": "algorithmic bytes of the per-stage kernels over the solve's wall time "
                                      "(launches and host synchronisation included)"}}
        # the same kernels with micm's CUDA-path semantics: one step size for
        # all cells from the error norm over all cells (a different step
        # sequence, so not bit-comparable with the per-cell solves); under
        # torchrun the step size is the whole job's: one 8-byte all-gather of
        # the ranks' error sums per attempt (NCCL, on the state's stream)
        if dist:
            def nccl_allgather(send, recv, w, stream_ptr):
                with torch.cuda.stream(torch.cuda.ExternalStream(stream_ptr)):
                    dist.all_gather_into_tensor(torch.as_tensor(_DeviceArray(recv, w), device="cuda"),
                                                torch.as_tensor(_DeviceArray(send, 1), device="cuda"))
                return 0
            pstate.set_global_exchange(nccl_allgather, world, pc * world)
        pview.copy_(p0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gres = solver.solve(cfg["dt"], pstate, method="plain", step_control="global")
        torch.cuda.synchronize()
        gt = time.perf_counter() - t0
        if dist:
            pstate.set_global_exchange(None, 1, 0)
            (gt,) = max_over_ranks([gt], dist, "cuda")
        plain["global_step_size"] = {"value": pc * world / gt, "unit": UNIT, "ms_per_step": 1000 * gt,
                                     "step_size": "one for the whole job" + (f" ({world} ranks, NCCL all-gather "
                                                                             "of the error sums per attempt)"
                                                                             if dist else ""),
                                     "attempts": gres.stats["number_of_steps"], "accepted": gres.stats["accepted"],
                                     "converged": bool(gres.converged),
                                     "fused_over_this": value / (pc * world / gt)}

    # the solve states are released before the adjoint timing, which sizes its
    # checkpoint chunks from the free device memory
    pview = p0 = pstate = y_view = y_dev = None
    state = None
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    adj = None
    if not args.no_adjoint and W["adjoint"]:
        same = W["adjoint"][0] == args.workload            # same mechanism: keep the configuration tuned above
        adj = adjoint_ratio(torch, rank, *W["adjoint"], fused_config=tuned if same else None)

    cpu = parity = None
    if rank == 0 and not args.no_cpu:
        cpu, y_ref, acc_ref = cpu_reference(mech, cfg, inputs, args.cpu_sample,
                                            uniform=args.workload in ("ts1", "chapman"))
        if cpu is not None and gpu_par is not None:
            parity = parity_summary(gpu_par[0], gpu_par[1], y_ref, acc_ref)
            parity["reference"] = ("micm (oracle/_ref parity build) on the same cells, "
                                   + ("micm_bench's vector-128 layout" if args.workload in ("ts1", "chapman")
                                      else "one 1-cell State per cell"))

    if rank == 0:
        info = solver.compiled.info
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": f"{args.workload}: " + W["text"].format(cells=args.cells),
                       "cells_per_gpu": args.cells, "vector_length": L, "fused_config": tuned,
                       "l2": W["l2"],
                       "lu_nnz": info["jacobian_nnz"], "lu_updates": info["lu_updates"],
                       "attempts_per_cell": attempts_per_cell, "accepted_per_cell": accepted_per_cell},
            "clocks": clocks.summary(),
            "e2e": {"value": job_throughput(args.cells, world, e2e_steps, e2e_t), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "calls": "upload variables/conditions/custom params, UpdateStateParameters, Solve, "
                             "download variables (pinned host buffers)"},
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak_gbs, "unit": "GB/s",
                         "frac": achieved_gbs / peak_gbs, "traffic": traffic,
                         "kernel": KERNEL_OF_VARIANT.get(tuned["variant"], "fused") + " (one launch per step)",
                         "algorithmic_bytes_per_launch": algo_bytes, "kernel_ms_per_launch": kernel_ms / args.steps,
                         "peak_source": peak_src,
                         "traffic_source": ("dram__bytes_read.sum + dram__bytes_write.sum of the capture in "
                                            f"profiles/{W['profile']}, scaled by cells") if W["profile"]
                                           else "no capture of this workload",
                         "fp64": {"achieved_tflops": flops / kernel_s / 1e12, "peak_tflops": fp64_peak(),
                                  "frac": flops / kernel_s / 1e12 / fp64_peak(), "flops_per_launch": flops,
                                  "peak_source": "nominal (SMs x 64 FMA/clk x 2 x max SM clock)"}},
            "gpu_launches": args.steps,
            "graph": {"value": job_throughput(args.cells, world, args.steps, graph_ms / 1000.0), "unit": UNIT,
                      "ms_per_step": graph_ms / args.steps,
                      "note": "each step one replay of a CUDA graph holding UpdateStateParameters and the fused "
                              "Solve (micmb_solve_graph), after the same device copy of the initial "
                              "concentrations; rate constants are recomputed inside every replay"},
            "parity": parity,
            "plain": plain,
            "adjoint": adj,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


class _DeviceArray:
    """__cuda_array_interface__ over a state buffer so torch can view it in place."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None}


def device_view(state, buffer):
    import torch
    ptr, count = state.device_buffer(buffer)
    return torch.as_tensor(_DeviceArray(ptr, count), device="cuda")


if __name__ == "__main__":
    main()
