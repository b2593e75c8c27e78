"""Benchmark of the B200 force evaluation: v_xc force-evals/s.

One step = one ``getForceVector`` (Chebyshev-filtered eigensolve -> density ->
block-MINRES adjoint -> projection onto the Q1 v_xc nodes) at a new potential
on the straight path from the Fermi-Amaldi guess towards v_xc*, as an L-BFGS
run visits them.  Default workload: the ethylene-like system of the FP64
configuration (FE order 5, ~1.3e6 DoF, 16 states), synthetic inputs.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--config c1_c2h4] [--precision fp64|mixed] [--ref-budget-s 240]

The reference arm (--impl reference) runs no CUDA: it times whole force
evaluations of the C++/OpenMP restatement of the path (oracle/cpu) on the
host cores, on the same workload, trajectory and knobs.

Multi-GPU: the force evaluation does not shard (one GPU per evaluation), so
N > 1 runs N independent replicas (weak scaling) and reports their summed
throughput, timed as the max over ranks.
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

# the benchmark's headline metric: one getForceVector call is the unit of work
METRIC = "v_xc force-evals/s at fixed \u222b|\u03c1\u2212\u03c1*|: mixed+batched vs FP64, 1 B200; % HBM/TC peak"


def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def _fp64_peak_tflops(device) -> float:
    """FP64 throughput ceiling measured here: cuBLAS DGEMM 8192^3 (2 N^3 flops),
    best of 5 with CUDA events.  On B200 the FP64 tensor-core rate equals the
    FP64 FMA-pipe rate, so this bounds any FP64 kernel."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    torch.matmul(a, b)
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best / 1000.0) / 1e12


def _traffic_from_profiles(name: str):
    path = os.path.join(ROOT, "profiles", "cell_gemm_traffic.json")
    try:
        d = json.load(open(path))
        return d.get(name)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 3 + i and r[3 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def force_knobs(prec: str) -> dict:
    """Hot-path parameters of the benchmark (both arms)."""
    return dict(cheb_degree=0, cheby_tol=1e-6, initial_tol_cheb=1e-6, adjoint_initial_tol=1e-8,
                adjoint_max_iter=5000, max_cheb_passes=100, lanczos_steps=LANCZOS_STEPS,
                precision=0 if prec == "fp64" else 1)


# Steps of the Lanczos run that bounds the spectrum for the Chebyshev filter.
# Its upper bound (largest Ritz value + |beta_k|) settles only after ~40-80
# steps on the 1e6-1e7 DoF meshes: with 20 it is 0.5 % (c1) to 0.9 % (c4) below
# the converged value, and the filter then amplifies the states above it.
LANCZOS_STEPS = 80


def force_params(prec: str):
    from invdft_b200 import native
    return native.default_params(**force_knobs(prec))


TARGET = "superposed neutral-atom Gaussian densities"


def build_workload(name: str):
    """The configuration's mesh, potentials and v_xc mesh, built on the host.

    The target density is the superposition of the atoms' Gaussian clouds, the
    same in both arms (no forward solve, no GPU): every force evaluation costs
    the same whatever the target, and a reachable target only matters for
    runs to convergence (``--converge``)."""
    from invdft_b200.problem.system import build_problem
    t0 = time.time()
    P = build_problem(name, target_solver="atoms")
    return P, dict(t_setup_s=round(time.time() - t0, 1), target_density=TARGET)


_MOLECULE = {"c0_lih": "LiH", "c1_c2h4": "C2H4", "c2_c2h4": "C2H4", "c3_h2o": "H2O", "c4_c8h18": "C8H18"}


def workload_name(config: str, P, precision: str) -> str:
    """The workload both arms name in their JSON line."""
    mol = _MOLECULE.get(config, config)
    return (f"{config}: {mol}-like, FE order {P.p}, {P.n_nodes} DoF, {P.n_cells} cells, {P.n_states} states, "
            f"{P.n_child_cells} v_xc cells / {P.n_child_nodes} nodes, precision {precision}")


def hx_probe(args, dev):
    """``--steps`` Lowdin HX applications of a seeded [n_nodes, width] block on
    the workload's mesh at v_xc = the initial guess: the launch sequence the
    kernel profiles in profiles/ are captured on."""
    import torch
    from invdft_b200.problem.system import build_problem
    from invdft_b200.solver import InverseDFTSolverFunction
    P = build_problem(args.config, target_solver="atoms")
    fn = InverseDFTSolverFunction(P, force_params("fp64"))
    fn.set_potential(P.vxc_init.copy())
    for width in [int(w) for w in str(args.hx_width).split(",")]:
        g = torch.Generator(device=dev).manual_seed(1)
        x = torch.randn(P.n_nodes, width, dtype=torch.float64, device=dev, generator=g)
        for _ in range(max(args.warmup, 1)):   # first use of a width also autotunes the launch shape
            fn.hx(x)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            y = fn.hx(x)
        e1.record()
        torch.cuda.synchronize()
        print(json.dumps({"probe": "hx", "workload": args.config, "n_dofs": P.n_nodes, "n_cells": P.n_cells,
                          "width": width, "warmup": max(args.warmup, 1), "applications": args.steps,
                          "ms_per_hx": e0.elapsed_time(e1) / max(args.steps, 1), "norm": float(y.norm())}))
    fn.close()


def reachable_target(P):
    """rho* from an FP64 forward solve at v_xc* on the GPU (the configurations'
    reachable target); installs it in P."""
    from invdft_b200 import native
    from invdft_b200.problem.system import set_target_density
    from invdft_b200.solver import InverseDFTSolverFunction
    fwd = InverseDFTSolverFunction(P, native.default_params(cheb_degree=0, cheby_tol=1e-9, initial_tol_cheb=1e-9,
                                                            max_cheb_passes=200))
    fwd.solve_eigen(P.vxc_exact.copy())
    _, occ, _ = fwd.eigen()
    psi = fwd.psi()
    rho_q = fwd.density()
    fwd.close()
    set_target_density(P, rho_q, 2.0 * np.sum(occ[None, :] * psi * psi, axis=1))


def converge(args):
    """The metric as defined: L-BFGS (CP line search) from the Fermi-Amaldi
    guess until int |rho - rho*| <= --converge-target, with the reachable target
    of the configuration, in FP64 and in MIXED precision; device time with CUDA
    events.  Reports evaluations, iterations and time to the target, and the
    final v_xc of the two runs against each other."""
    import torch
    from invdft_b200.problem.system import build_problem
    from invdft_b200.solver import InverseDFTSolverFunction, bfgs_run
    P = build_problem(args.config, target_solver="atoms")
    reachable_target(P)
    runs = {}
    for prec in ("fp64", "mixed"):
        fn = InverseDFTSolverFunction(P, force_params(prec))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        v, rep, losses, l1 = bfgs_run(fn, P.vxc_init.copy(), args.converge_max_iter,
                                      density_l1_target=args.converge_target)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        runs[prec] = dict(report=rep, ms=ms, evals_per_s=rep["n_evals"] / (ms / 1000.0),
                          density_l1_first_last=[float(l1[0]), float(l1[-1])], v=v)
        fn.close()
    v64, vmx = runs["fp64"].pop("v"), runs["mixed"].pop("v")
    free = np.ones(P.n_child_nodes, dtype=bool)
    free[P.cons_child.nodes] = False
    out = {"mode": "converge", "workload": workload_name(args.config, P, "fp64 and mixed"),
           "target": f"int |rho - rho*| <= {args.converge_target:g} (reachable rho* from an FP64 forward solve)",
           "runs": runs,
           "time_to_target_speedup_mixed_vs_fp64": runs["fp64"]["ms"] / runs["mixed"]["ms"],
           "evals_per_s_ratio_mixed_vs_fp64": runs["mixed"]["evals_per_s"] / runs["fp64"]["evals_per_s"],
           "final_vxc_rel_l2_mixed_vs_fp64": float(np.linalg.norm((vmx - v64)[free]) / np.linalg.norm(v64[free]))}
    print(json.dumps(out))


def kernel_probe(args):
    """One launch of each kernel of the evaluation on the workload's full-size
    buffers (invdft_kernel_probe): the launch sequence the per-kernel profiles
    in profiles/ are captured on, with few launches before each."""
    from invdft_b200.problem.system import build_problem
    from invdft_b200.solver import InverseDFTSolverFunction, _check
    P = build_problem(args.config, target_solver="atoms")
    fn = InverseDFTSolverFunction(P, force_params("fp64"))
    fn.set_potential(P.vxc_init.copy())
    for _ in range(max(args.steps, 1)):
        _check(fn.lib, fn.ctx, fn.lib.invdft_kernel_probe(fn.ctx))
    print(json.dumps({"probe": "kernels", "workload": args.config, "n_dofs": P.n_nodes, "rounds": max(args.steps, 1)}))
    fn.close()


def aggregate(ms: float, e2e_s: float, steps: int, world: int, dist=None, device="cuda"):
    """Whole-job throughput of ``world`` replicas timed as the max over ranks.

    Returns (force-evals/s on device time, force-evals/s end to end, max ms)."""
    if dist is not None and world > 1:
        import torch
        t = torch.tensor([ms, e2e_s * 1000.0], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, e2e_s = float(t[0]), float(t[1]) / 1000.0
    return steps * world / (ms / 1000.0), steps * world / e2e_s, ms


PATH_START = 0.0   # --path-start


def trajectory(P, k: int, total: int):
    """Point k of total on the straight path guess -> v_xc*: the fraction
    a = s + (1 - s) (k + 1) / (2 total) of the way, s = --path-start."""
    a = PATH_START + (1.0 - PATH_START) * 0.5 * (k + 1) / max(total, 1)
    return P.vxc_init + a * (P.vxc_exact - P.vxc_init)


def cpu_evaluation(P, prec: str, threads: int, k: int, total: int, state=None):
    """One whole getForceVector of the C++/OpenMP restatement (oracle/cpu) on the
    host cores at trajectory point k.  ``state`` (psi, eig, counter, loss_prev,
    tol_cheb, adjoint_tol) hands over the GPU context's state before that
    point, so the CPU repeats exactly the evaluation the GPU timed."""
    from oracle.cpu import CpuForce
    cpu = CpuForce(P, threads=threads, **{**force_knobs("fp64"), "precision": 0})
    if state is not None:
        cpu.set_state(**state)
    pot = trajectory(P, k, total)
    t0 = time.perf_counter()
    f, L, st = cpu.get_force_vector(pot)
    dt = time.perf_counter() - t0
    cpu.close()
    return f, L, st, dt


def run_reference(args, threads: int):
    """The reference arm: the CPU restatement of the path on the host cores,
    whole force evaluations on the same workload, trajectory and knobs as the
    GPU arm.  No CUDA is touched.  One untimed warm-up evaluation stands for
    the GPU arm's warm-up steps (its counter and tolerances are then set as
    after ``--warmup`` evaluations); then evaluations are timed one after
    another until ``--steps`` are done or ``--ref-budget-s`` is spent."""
    from oracle.cpu import CpuForce
    P, info = build_workload(args.config)
    total = args.warmup + args.steps
    cpu = CpuForce(P, threads=threads, **{**force_knobs("fp64"), "precision": 0})
    w0 = time.perf_counter()
    _, Lw, stw = cpu.get_force_vector(trajectory(P, max(args.warmup - 1, 0), total))
    t_warm = time.perf_counter() - w0
    cpu.set_state(counter=max(args.warmup, 1), loss_prev=Lw, tol_cheb=stw["cheb_tol"],
                  adjoint_tol=stw["adjoint_tol"])
    times, stats = [], []
    t_begin = time.perf_counter()
    for k in range(args.warmup, total):
        t0 = time.perf_counter()
        _, L, st = cpu.get_force_vector(trajectory(P, k, total))
        times.append(time.perf_counter() - t0)
        stats.append(st)
        if time.perf_counter() - t_begin + times[-1] > args.ref_budget_s:
            break
    cpu.close()
    n = len(times)
    v = n / sum(times)
    sample = (f"{n} whole FP64 force evaluations (eigensolve, density, block MINRES, projection) of the C++/OpenMP "
              f"restatement on {threads} host threads, at trajectory points {args.warmup}..{args.warmup + n - 1} of "
              f"{total}, after one untimed warm-up evaluation ({t_warm:.1f} s); {n} of the {args.steps} requested "
              f"steps fit the {args.ref_budget_s:.0f} s budget")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "force-evals/s", "n_gpus": args.gpus,
            "steps": n, "steps_requested": args.steps, "warmup": 1, "warmup_requested": args.warmup,
            "ms_per_step": 1000.0 * sum(times) / n, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(args.config, P, "fp64"),
                       "step": "one getForceVector at a new v_xc on the path guess -> v_xc*",
                       "chebyshev_passes": [s["passes"] for s in stats],
                       "minres_iters_max": [s["minres_iters_max"] for s in stats],
                       "hx_columns": [s["n_hx_columns"] for s in stats],
                       "loss": [s["loss"] for s in stats], "s_per_step": times, **info},
            "cpu_baseline": dict(value=v, unit="force-evals/s", kind="port", cores=threads, sample=sample),
            "e2e": {"value": v, "unit": "force-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c1_c2h4")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--ladder-operands", default="fp32", choices=["fp32", "tf32", "bf16"],
                    help="--precision mixed: operands of the low-rung filter products, rounded as a tensor-core "
                         "MMA of that input format would round them (FP32 accumulation)")
    ap.add_argument("--no-fp64-compare", action="store_true",
                    help="do not time the FP64 path on the same trajectory")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU evaluation (profiling runs)")
    ap.add_argument("--ref-budget-s", type=float, default=240.0,
                    help="reference arm: stop timing CPU evaluations once this much time is spent")
    ap.add_argument("--converge", action="store_true",
                    help="L-BFGS to a fixed int |rho - rho*| in FP64 and MIXED precision (the metric as defined)")
    ap.add_argument("--converge-target", type=float, default=1e-5)
    ap.add_argument("--converge-max-iter", type=int, default=300)
    ap.add_argument("--kernel-probe", action="store_true",
                    help="profiling: one launch of each kernel of the evaluation on the workload's buffers")
    ap.add_argument("--hx-width", type=str, default="0",
                    help="kernel probe for profiling: --steps Lowdin HX applications of a seeded block of this "
                         "width at v_xc = the initial guess, timed with CUDA events (no force evaluation)")
    ap.add_argument("--path-start", type=float, default=0.0,
                    help="fraction of the way from the initial guess to v_xc* where the evaluated path starts "
                         "(0: the guess itself)")
    args = ap.parse_args()
    global PATH_START
    PATH_START = args.path_start

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    threads = os.cpu_count() or 1

    if args.impl == "reference":
        # host cores only: rank 0 runs, the others leave without work
        if rank == 0:
            run_reference(args, threads)
        return

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    if args.hx_width != "0":
        hx_probe(args, dev)
        return
    if args.kernel_probe:
        kernel_probe(args)
        return
    if args.converge:
        converge(args)
        return

    P, info = build_workload(args.config)
    from invdft_b200.solver import InverseDFTSolverFunction
    os.environ["INVDFT_LADDER_OPERANDS"] = args.ladder_operands   # read when the context is created
    fn = InverseDFTSolverFunction(P, force_params(args.precision))
    os.environ["INVDFT_LADDER_OPERANDS"] = "fp32"
    lib = fn.lib
    lib.invdft_set_profiling(fn.ctx, 1)
    total = args.warmup + args.steps
    pinned_pot = torch.empty(P.n_child_nodes, dtype=torch.float64).pin_memory()
    pinned_force = torch.empty(P.n_child_nodes, dtype=torch.float64).pin_memory()
    last = None
    for k in range(args.warmup):
        pot = trajectory(P, k, total)
        last = fn.get_force_vector(pot.copy())
    # the context's state before the first timed step, for the CPU repeat of it
    state = None
    if last is not None and rank == 0 and world == 1 and not args.no_cpu_baseline:
        e, _, _ = fn.eigen()
        state = dict(psi=fn.psi(), eig=e, counter=args.warmup, loss_prev=last[1], tol_cheb=last[2]["cheb_tol"],
                     adjoint_tol=last[2]["adjoint_tol"])
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    stats = []
    first_force = None
    t_e2e = 0.0
    with ClockSampler(local) as clk:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        w0 = time.perf_counter()
        torch.cuda.nvtx.range_push("timed")
        for k in range(args.warmup, total):
            pinned_pot.numpy()[:] = trajectory(P, k, total)
            f, L, st = fn.get_force_vector(pinned_pot.numpy())
            pinned_force.numpy()[:] = f
            if first_force is None:
                first_force = f.copy()
            stats.append(st)
        torch.cuda.nvtx.range_pop()
        ev1.record()
        torch.cuda.synchronize()
        t_e2e = time.perf_counter() - w0
    value, e2e, ms = aggregate(ev0.elapsed_time(ev1), t_e2e, args.steps, world, dist)
    n_gemm = sum(s["n_cell_gemm"] for s in stats)
    gemm_ms = sum(s["ms_cell_gemm"] for s in stats)
    gemm_bytes = sum(s["cell_gemm_bytes"] for s in stats)
    gemm_flops = sum(s["cell_gemm_flops"] for s in stats)
    peaks, pk = _peaks()
    # the matrix-free kernel runs in both precisions (its FP32 instance serves
    # the low rungs of the mixed ladder); stored cell matrices only on request
    matrix_free = os.environ.get("INVDFT_HX_KERNEL", "sf") == "sf" and P.p <= 7
    hbm_achieved = gemm_bytes / (gemm_ms / 1000.0) / 1e9 if gemm_ms > 0 else None
    # captured traffic of one launch of a given width, scaled to the mean width
    # of this run's launches (traffic grows with the columns processed)
    cap = _traffic_from_profiles(f"{args.config}:{'sf' if matrix_free else 'dmma'}:fp64")
    mean_cols = sum(s["n_hx_columns"] for s in stats) / max(n_gemm, 1)
    per_launch_traffic = cap["bytes"] * mean_cols / cap["columns"] if isinstance(cap, dict) else cap
    if matrix_free:
        fp64_peak = _fp64_peak_tflops(dev)
        achieved = gemm_flops / (gemm_ms / 1000.0) / 1e12 if gemm_ms > 0 else None
        roofline = {"bound": "tensor", "pipe": "fp64 (DFMA; peak = cuBLAS DGEMM measured live, of measured)",
                    "kernel": "hx_cell_sf (matrix-free FP64 sum-factorised cell products)",
                    "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                    "frac": (achieved / fp64_peak) if achieved else None, "peak_source": "measured",
                    "traffic": per_launch_traffic, "launches": n_gemm, "ms_per_launch": gemm_ms / max(n_gemm, 1),
                    "algorithmic_flops_per_launch": gemm_flops / max(n_gemm, 1),
                    "algorithmic_bytes_per_launch": gemm_bytes / max(n_gemm, 1),
                    "hbm_achieved_gbs": hbm_achieved,
                    "hbm_frac": (hbm_achieved / peaks["hbm_gbs"]) if hbm_achieved else None}
    else:
        roofline = {"bound": "hbm", "kernel": "hx_cell_dmma (FP64 cell-matrix x vector block)",
                    "achieved": hbm_achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": (hbm_achieved / peaks["hbm_gbs"]) if hbm_achieved else None,
                    "peak_source": pk, "traffic": per_launch_traffic,
                    "launches": n_gemm, "ms_per_launch": gemm_ms / max(n_gemm, 1),
                    "algorithmic_bytes_per_launch": gemm_bytes / max(n_gemm, 1)}
    launches = int(sum(s["n_launches"] for s in stats))
    fp64_cmp = None
    if args.precision == "mixed" and not args.no_fp64_compare:
        fn64 = InverseDFTSolverFunction(P, force_params("fp64"))
        for k in range(args.warmup):
            fn64.get_force_vector(trajectory(P, k, total).copy())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        f64_stats = []
        for k in range(args.warmup, total):
            f64_stats.append(fn64.get_force_vector(trajectory(P, k, total).copy())[2])
        e1.record()
        torch.cuda.synchronize()
        v64, _, ms64 = aggregate(e0.elapsed_time(e1), 1.0, args.steps, world, dist)
        fp64_cmp = {"value": v64, "ms_per_step": ms64 / args.steps, "passes": [s["passes"] for s in f64_stats],
                    "minres_iters_max": [s["minres_iters_max"] for s in f64_stats],
                    "stage_ms_mean": {k: float(np.mean([s[f"ms_{k}"] for s in f64_stats]))
                                      for k in ("eigen", "density", "adjoint", "transfer")},
                    "speedup_mixed_vs_fp64": value / v64,
                    "max_abs_loss_diff_vs_fp64": max(abs(a["loss"] - b["loss"]) for a, b in zip(stats, f64_stats))}
        fn64.close()
    if rank == 0:
        if state is None:
            cpu_v, cpu_meta = None, dict(kind="port", cores=threads,
                                         sample="skipped (--no-cpu-baseline, no warm-up, or more than one rank)")
            cpu_check = None
        else:
            f_c, L_c, st_c, dt = cpu_evaluation(P, args.precision, threads, args.warmup, total, state)
            cpu_v = 1.0 / dt
            cpu_meta = dict(kind="port", cores=threads,
                            sample=f"one whole FP64 force evaluation of the C++/OpenMP restatement on {threads} host "
                                   f"threads, repeating the first timed step (trajectory point {args.warmup}) from "
                                   f"the GPU context's state before it: {st_c['passes']} Chebyshev passes, MINRES "
                                   f"max {st_c['minres_iters_max']} iterations, {dt:.1f} s")
            cpu_check = {"force_rel_l2_vs_gpu": float(np.linalg.norm(f_c - first_force) /
                                                      max(np.linalg.norm(f_c), 1e-300)),
                         "loss_cpu": L_c, "loss_gpu": stats[0]["loss"],
                         "passes_cpu_gpu": [st_c["passes"], stats[0]["passes"]],
                         "minres_iters_max_cpu_gpu": [st_c["minres_iters_max"], stats[0]["minres_iters_max"]]}
        line = {
            "metric": METRIC, "value": value, "unit": "force-evals/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else (
                f"f64 + f32 (FP32 matrix-free cell products in the early Chebyshev passes, operands "
                f"{args.ladder_operands}; FP32-operator MINRES in FP64 refinement)" if matrix_free else
                                                          "f64 + f32 (FP32-stored cell matrices in the early "
                                                          "Chebyshev passes)"),
            "data": "synthetic (seeded; see invdft_b200/problem/system.py)",
            "config": {
                "workload": workload_name(args.config, P, args.precision),
                "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (state block + cell results "
                f"{(P.n_nodes + P.n_cells * P.nd) * P.n_states * 8 / 1e9:.2f} GB per HX)",
                "step": "one getForceVector at a new v_xc on the path guess -> v_xc*",
                "chebyshev_passes": [s["passes"] for s in stats],
                "chebyshev_passes_low_precision": [s["passes_low"] for s in stats],
                "fp64_same_trajectory": fp64_cmp,
                "chebyshev_degree": [s["degree"] for s in stats],
                "spectrum_upper_bound": stats[-1]["upper_bound"],
                "minres_iters_max": [s["minres_iters_max"] for s in stats],
                "minres_iters_sum": [s["minres_iters_sum"] for s in stats],
                "adjoint_refinement_steps": [s["refine_steps"] for s in stats],
                "hx_columns": [s["n_hx_columns"] for s in stats],
                "stage_ms_mean": {k: float(np.mean([s[f"ms_{k}"] for s in stats]))
                                  for k in ("eigen", "density", "adjoint", "transfer")},
                "hx_kernel": "matrix-free sum factorisation" if matrix_free else "stored cell matrices (DMMA)",
                "device_bytes_peak": stats[-1]["device_bytes_peak"],
                "cpu_repeat_of_first_step": cpu_check,
                "loss": [s["loss"] for s in stats], **info},
            "e2e": {"value": e2e, "unit": "force-evals/s", "h2d_bytes_per_step": 8 * P.n_child_nodes,
                    "d2h_bytes_per_step": 8 * P.n_child_nodes + 8},
            "gpu_launches": launches,
            "roofline": roofline,
            "cpu_baseline": dict(value=cpu_v, unit="force-evals/s", **cpu_meta),
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    fn.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
