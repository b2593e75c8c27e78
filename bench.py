"""Benchmark of the B200 force evaluation: v_xc force-evals/s.

One step = one ``getForceVector`` (Chebyshev-filtered eigensolve -> density ->
block-MINRES adjoint -> projection onto the Q1 v_xc nodes) at a new potential
on the straight path from the Fermi-Amaldi guess towards v_xc*, as an L-BFGS
run visits them.  Default workload: the ethylene-like system of the FP64
configuration (FE order 5, ~1.3e6 DoF, 16 states), synthetic inputs.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--config c1_c2h4] [--cpu-sample-cells 400]

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


def force_params(prec: str):
    from invdft_b200 import native
    return native.default_params(cheb_degree=0, cheby_tol=1e-6, initial_tol_cheb=1e-6,
                                 adjoint_initial_tol=1e-8, adjoint_max_iter=5000, max_cheb_passes=100,
                                 precision=0 if prec == "fp64" else 1)


def build_workload(name: str, rank: int):
    """Problem with rho* from an FP64 forward solve on the GPU at v_xc*."""
    from invdft_b200.problem.system import build_problem, set_target_density
    from invdft_b200.solver import InverseDFTSolverFunction
    from invdft_b200 import native
    t0 = time.time()
    P = build_problem(name, target_solver="atoms")
    t_mesh = time.time() - t0
    fwd = InverseDFTSolverFunction(P, native.default_params(cheb_degree=0, cheby_tol=1e-9,
                                                            initial_tol_cheb=1e-9, max_cheb_passes=200))
    fwd.solve_eigen(P.vxc_exact.copy())
    e, occ, mu = fwd.eigen()
    psi = fwd.psi()
    rho_q = fwd.density()
    rho_n = 2.0 * np.sum(occ[None, :] * psi * psi, axis=1)
    fwd.close()
    set_target_density(P, rho_q, rho_n)
    P.extras["target_eigenvalues"] = e
    return P, dict(t_mesh_s=round(t_mesh, 1), t_setup_s=round(time.time() - t0, 1))


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


def aggregate(ms: float, e2e_s: float, steps: int, world: int, dist=None, device="cuda"):
    """Whole-job throughput of ``world`` replicas timed as the max over ranks.

    Returns (force-evals/s on device time, force-evals/s end to end, max ms)."""
    if dist is not None and world > 1:
        import torch
        t = torch.tensor([ms, e2e_s * 1000.0], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, e2e_s = float(t[0]), float(t[1]) / 1000.0
    return steps * world / (ms / 1000.0), steps * world / e2e_s, ms


def trajectory(P, k: int, total: int):
    a = 0.5 * (k + 1) / max(total, 1)
    return P.vxc_init + a * (P.vxc_exact - P.vxc_init)


def cpu_sample(P, n_hx_columns: int, N: int, cells: int, threads: int):
    """FP64 oracle HX timed on a bounded sample of cells, scaled to one evaluation."""
    from oracle.fe import CellOps
    import copy
    sub = copy.copy(P)
    n = min(cells, P.n_cells)
    # restrict the cell loop of the oracle's HX to the first n cells
    sub.n_cells = n
    sub.cell_nodes = P.cell_nodes[:n]
    sub.cell_h = P.cell_h[:n]
    sub.jxw = P.jxw[: n * P.nq]
    ops = CellOps(sub)
    ops.cell_hamiltonians(P.v_base[: n * P.nq])
    x = np.random.default_rng(0).standard_normal((P.n_nodes, N))
    ops.hx(x)
    t0 = time.perf_counter()
    reps = 0
    while True:
        ops.hx(x)
        reps += 1
        if time.perf_counter() - t0 > 10.0 or reps >= 50:
            break
    t_hx = (time.perf_counter() - t0) / reps * (P.n_cells / n)
    t_eval = t_hx * n_hx_columns / N
    return 1.0 / t_eval, dict(kind="port", cores=threads,
                              sample=f"oracle FP64 Lowdin HX on {n} of {P.n_cells} cells, {reps} reps of "
                                     f"B={N}, scaled by cells and by the {n_hx_columns} HX columns one "
                                     f"evaluation issues (RR, MINRES vector work and transfers not counted)")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c1_c2h4")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-fp64-compare", action="store_true",
                    help="do not time the FP64 path on the same trajectory")
    ap.add_argument("--cpu-sample-cells", type=int, default=400)
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU sample (profiling runs)")
    ap.add_argument("--hx-width", type=str, default="0",
                    help="kernel probe for profiling: --steps Lowdin HX applications of a seeded block of this "
                         "width at v_xc = the initial guess, timed with CUDA events (no force evaluation)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    threads = os.cpu_count() or 1

    if args.hx_width != "0":
        hx_probe(args, dev)
        return

    if args.impl == "reference":
        if rank != 0:
            if dist:
                dist.destroy_process_group()
            return
        P, info = build_workload(args.config, rank)
        from invdft_b200.solver import InverseDFTSolverFunction
        fn = InverseDFTSolverFunction(P, force_params(args.precision))
        fn.get_force_vector(trajectory(P, 0, 1))
        ncols = fn.last_stats["n_hx_columns"]
        fn.close()
        vals = []
        for _ in range(max(args.steps, 1)):
            v, meta = cpu_sample(P, ncols, P.n_states, args.cpu_sample_cells, threads)
            vals.append(v)
        v = float(np.median(vals))
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "force-evals/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / v,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": workload_name(args.config, P, args.precision),
                           "step": "one getForceVector at a new v_xc on the path guess -> v_xc*"},
                "cpu_baseline": dict(value=v, unit="force-evals/s", **meta),
                "e2e": {"value": v, "unit": "force-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    P, info = build_workload(args.config, rank)
    from invdft_b200.solver import InverseDFTSolverFunction
    fn = InverseDFTSolverFunction(P, force_params(args.precision))
    lib = fn.lib
    lib.invdft_set_profiling(fn.ctx, 1)
    total = args.warmup + args.steps
    pinned_pot = torch.empty(P.n_child_nodes, dtype=torch.float64).pin_memory()
    pinned_force = torch.empty(P.n_child_nodes, dtype=torch.float64).pin_memory()
    for k in range(args.warmup):
        pot = trajectory(P, k, total)
        fn.get_force_vector(pot.copy())
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    stats = []
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
    cap = _traffic_from_profiles(f"{args.config}:{'sf' if matrix_free else 'dmma'}:{args.precision}")
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
                    "speedup_mixed_vs_fp64": value / v64,
                    "max_abs_loss_diff_vs_fp64": max(abs(a["loss"] - b["loss"]) for a, b in zip(stats, f64_stats))}
        fn64.close()
    if rank == 0:
        if args.no_cpu_baseline:
            cpu_v, cpu_meta = None, dict(kind="port", cores=threads, sample="skipped (--no-cpu-baseline)")
        else:
            cpu_v, cpu_meta = cpu_sample(P, int(np.mean([s["n_hx_columns"] for s in stats])), P.n_states,
                                         args.cpu_sample_cells, threads)
        line = {
            "metric": METRIC, "value": value, "unit": "force-evals/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else ("f64 + f32 (FP32 matrix-free cell products in the early "
                                                          "Chebyshev passes)" if matrix_free else
                                                          "f64 + f32 (FP32-stored cell matrices in the early "
                                                          "Chebyshev passes)"),
            "data": "synthetic (seeded; see invdft_b200/problem/system.py)",
            "config": {
                "workload": workload_name(args.config, P, args.precision),
                "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (state block + cell results "
                f"{(P.n_nodes + P.n_cells * P.nd) * P.n_states * 8 / 1e9:.2f} GB per HX)",
                "step": "one getForceVector at a new v_xc on the path guess -> v_xc*",
                "chebyshev_passes": [s["passes"] for s in stats],
                "chebyshev_passes_fp32_stored": [s["passes_low"] for s in stats],
                "fp64_same_trajectory": fp64_cmp,
                "chebyshev_degree": [s["degree"] for s in stats],
                "spectrum_upper_bound": stats[-1]["upper_bound"],
                "minres_iters_max": [s["minres_iters_max"] for s in stats],
                "hx_columns": [s["n_hx_columns"] for s in stats],
                "stage_ms_mean": {k: float(np.mean([s[f"ms_{k}"] for s in stats]))
                                  for k in ("eigen", "density", "adjoint", "transfer")},
                "hx_kernel": "matrix-free sum factorisation" if matrix_free else "stored cell matrices (DMMA)",
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
