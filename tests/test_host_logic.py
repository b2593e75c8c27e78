"""Host-side logic on CPU: the L-BFGS mirror, block partitioning, the
replica aggregation of bench.py over two gloo ranks, and bench.py's reference
arm."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class _Quadratic:
    """L(x) = 1/2 x^T A x - b^T x exposed with the force-evaluation interface."""

    def __init__(self, n=30, seed=0):
        rng = np.random.default_rng(seed)
        Q = rng.standard_normal((n, n))
        self.A = Q @ Q.T / n + np.eye(n)
        self.b = rng.standard_normal(n)
        self.calls = 0

    def get_force_vector(self, x):
        self.calls += 1
        g = self.A @ x - self.b
        return g, 0.5 * x @ self.A @ x - self.b @ x, None

    @staticmethod
    def dot_product(a, b):
        return float(np.dot(a, b))


def test_bfgs_mirror_minimises_a_quadratic():
    from oracle import BFGSInverseDFTSolver
    f = _Quadratic()
    x, g, L = BFGSInverseDFTSolver(max_iter=60, tol=1e-10).solve(f, np.zeros(30))
    xs = np.linalg.solve(f.A, f.b)
    assert np.linalg.norm(x - xs) < 1e-6 * np.linalg.norm(xs)


def test_block_partition_keeps_degenerate_groups_together():
    """The block-size shrink rule of InverseDFTSolverFunction.cpp:927-955."""
    eig = np.array([-1.0, -0.5, -0.4995, -0.2, -0.1999, -0.1998, 0.3])
    tol, block, N = 0.002, 3, len(eig)
    blocks, j = [], 0
    while j < N:
        bs = min(block, N - j)
        while j + bs < N and abs(eig[j + bs - 1] - eig[j + bs]) < tol:
            bs -= 1
        blocks.append((j, bs))
        j += bs
    assert blocks == [(0, 3), (3, 3), (6, 1)]


def _replica_worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    import bench
    ms = 100.0 * (rank + 1)
    v, e2e, tmax = bench.aggregate(ms, ms / 1000.0 * 1.1, steps=4, world=world, dist=dist, device="cpu")
    out.put((rank, v, e2e, tmax))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_replica_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, v, e2e, tmax in res:
        assert tmax == pytest.approx(200.0)
        assert v == pytest.approx(4 * 2 / 0.2)
        assert e2e == pytest.approx(4 * 2 / 0.22)


def test_bench_workload_names_and_profile_traffic():
    """Both bench arms name the workload with the same helper, and the captured
    cell-product traffic of the profiles has the width it was captured at."""
    import importlib.util
    import os
    from types import SimpleNamespace
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(root, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    P = SimpleNamespace(p=5, n_nodes=10, n_cells=2, n_states=16, n_child_cells=3, n_child_nodes=4)
    name = bench.workload_name("c1_c2h4", P, "fp64")
    assert name.startswith("c1_c2h4: C2H4-like, FE order 5, 10 DoF")
    assert bench.workload_name("c0_lih", P, "fp64").startswith("c0_lih: LiH-like")
    cap = bench._traffic_from_profiles("c1_c2h4:sf:fp64")
    assert cap["columns"] == 16 and cap["bytes"] > 0


def test_reference_arm_runs_the_cpu_restatement_without_the_gpu_library():
    """bench.py --impl reference: whole force evaluations of the C++
    restatement on the host cores, one JSON line with the driver's keys, and
    none of the product's CUDA code loaded in the process."""
    import json
    import subprocess
    code = (
        "import sys, json, runpy\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--config', 'tiny_h2', '--steps', '1', '--warmup', '1',"
        " '--ref-budget-s', '5']\n"
        "runpy.run_path('bench.py', run_name='__main__')\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'product_so_loaded': 'libinvdft_b200' in maps}))\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.strip().splitlines() if l.startswith("{")]
    line, probe = lines[-2], lines[-1]
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] >= 1
    assert line["unit"] == "force-evals/s" and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] in ("port", "reference") and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert not probe["product_so_loaded"]
