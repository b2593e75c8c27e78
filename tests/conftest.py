import functools
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@functools.lru_cache(maxsize=None)
def problem(name: str):
    from invdft_b200.problem.system import build_problem
    return build_problem(name)


def oracle_params(**kw):
    from oracle import ForceParams
    kw = {k: v for k, v in kw.items()
          if k not in ("precision", "mixed_residual_floor", "mixed_inner_tol", "mixed_max_refine")}
    base = dict(cheb_degree=30, cheby_tol=1e-10, initial_tol_cheb=1e-10, adjoint_initial_tol=1e-10,
                adaptive_factor_adjoint=1.0,
                adjoint_max_iter=2000, max_cheb_passes=60, lanczos_steps=20)
    base.update(kw)
    return ForceParams(**base)


def native_params(**kw):
    from invdft_b200 import native
    base = dict(cheb_degree=30, cheby_tol=1e-10, initial_tol_cheb=1e-10, adjoint_initial_tol=1e-10,
                adaptive_factor_adjoint=1.0,
                adjoint_max_iter=2000, max_cheb_passes=60, lanczos_steps=20)
    base.update(kw)
    return native.default_params(**base)


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
