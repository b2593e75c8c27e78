"""ctypes binding of the C++/OpenMP restatement (oracle/cpu/force_cpu.cpp).

TEST INFRASTRUCTURE ONLY, like the rest of ``oracle/``: the tests use it as a
fast FP64 checker on meshes too large for the numpy oracle (it is itself
checked against the numpy oracle in tests/test_oracle_cpu.py), and the
benchmark times it as the CPU baseline.  It never loads the CUDA library: the
problem and parameter structs are the C ABI's plain structs, filled here.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from invdft_b200.native import Params, ProblemDesc, Stats, f64, make_desc, ptr

LIB = Path(__file__).resolve().parent / "liboracle_cpu.so"
_lib = None

# the reference's defaults (inverseDFTParameters.cpp:369-445), as in the C ABI
DEFAULTS = dict(cheb_degree=50, max_cheb_passes=100, cheby_tol=1e-6, initial_tol_cheb=1e-6,
                adaptive_factor_cheb=100.0, adjoint_initial_tol=1e-11, adaptive_factor_adjoint=1000.0,
                adjoint_max_iter=5000, degeneracy_tol=0.002, frac_occ_tol=1e-8, additional_states=0,
                block_size=0, inter_block_size=10, factor_lda=0.0, lanczos_steps=20, precision=0,
                mixed_residual_floor=1e-4, mixed_inner_tol=1e-4, mixed_max_refine=12)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        from .build_cpu import build
        build()
    lib = C.CDLL(str(LIB))
    vp = C.c_void_p
    f64p = C.POINTER(C.c_double)
    sig = {
        "ocpu_last_error": (C.c_char_p, []),
        "ocpu_set_threads": (None, [C.c_int]),
        "ocpu_max_threads": (C.c_int, []),
        "ocpu_create": (C.c_int, [C.POINTER(ProblemDesc), C.POINTER(Params), C.POINTER(vp)]),
        "ocpu_destroy": (None, [vp]),
        "ocpu_force_eval": (C.c_int, [vp, f64p, f64p, f64p, C.POINTER(Stats)]),
        "ocpu_solve_eigen": (C.c_int, [vp, f64p, C.POINTER(Stats)]),
        "ocpu_set_potential": (C.c_int, [vp, f64p]),
        "ocpu_hx": (C.c_int, [vp, f64p, f64p, C.c_int]),
        "ocpu_get_eigen": (C.c_int, [vp, f64p, f64p, f64p]),
        "ocpu_get_psi": (C.c_int, [vp, f64p]),
        "ocpu_density": (C.c_int, [vp, f64p]),
        "ocpu_set_state": (C.c_int, [vp, f64p, f64p, C.c_int, C.c_double, C.c_double, C.c_double]),
        "ocpu_lanczos_bounds": (C.c_int, [vp, C.c_int, f64p, f64p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def params(**overrides) -> Params:
    p = Params()
    for k, v in {**DEFAULTS, **overrides}.items():
        setattr(p, k, v)
    return p


class CpuForce:
    """getForceVector on the host cores (FP64, OpenMP)."""

    def __init__(self, prob, threads: int | None = None, **overrides):
        self.lib = load()
        if threads:
            self.lib.ocpu_set_threads(int(threads))
        self.threads = self.lib.ocpu_max_threads()
        self.prob = prob
        self.params = params(**overrides)
        keep: list = []
        desc = make_desc(prob, keep)
        ctx = C.c_void_p()
        self._check(self.lib.ocpu_create(C.byref(desc), C.byref(self.params), C.byref(ctx)))
        self.ctx = ctx

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(f"CPU oracle status {rc}: {self.lib.ocpu_last_error().decode()}")

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.ocpu_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_force_vector(self, pot):
        pot = f64(pot).copy()
        force = np.zeros(self.prob.n_child_nodes)
        loss = C.c_double()
        st = Stats()
        self._check(self.lib.ocpu_force_eval(self.ctx, ptr(pot), ptr(force), C.byref(loss), C.byref(st)))
        return force, float(loss.value), st.as_dict()

    def solve_eigen(self, pot):
        pot = f64(pot).copy()
        st = Stats()
        self._check(self.lib.ocpu_solve_eigen(self.ctx, ptr(pot), C.byref(st)))
        return st.as_dict()

    def set_state(self, psi=None, eig=None, counter: int = 0, loss_prev: float = 0.0, tol_cheb: float = 0.0,
                  adjoint_tol: float = 0.0):
        """Start subspace from nodal eigenvectors (and their Ritz values) and the
        adaptive-tolerance state, so the next evaluation repeats another
        implementation's next one."""
        p = None if psi is None else ptr(f64(psi))
        e = None if eig is None else ptr(f64(eig))
        self._check(self.lib.ocpu_set_state(self.ctx, p, e, int(counter), float(loss_prev), float(tol_cheb),
                                            float(adjoint_tol)))

    def set_potential(self, pot):
        self._check(self.lib.ocpu_set_potential(self.ctx, ptr(f64(pot))))

    def lanczos_bounds(self, steps: int):
        """(lower, upper) spectrum bounds of a `steps`-step Lanczos run at the current potential."""
        lo, hi = C.c_double(), C.c_double()
        self._check(self.lib.ocpu_lanczos_bounds(self.ctx, int(steps), C.byref(lo), C.byref(hi)))
        return lo.value, hi.value

    def hx(self, x):
        x = f64(x)
        B = 1 if x.ndim == 1 else x.shape[1]
        y = np.zeros_like(x)
        self._check(self.lib.ocpu_hx(self.ctx, ptr(x), ptr(y), B))
        return y

    def eigen(self):
        N = self.prob.n_states
        e, o, mu = np.zeros(N), np.zeros(N), C.c_double()
        self._check(self.lib.ocpu_get_eigen(self.ctx, ptr(e), ptr(o), C.byref(mu)))
        return e, o, mu.value

    def psi(self):
        out = np.zeros((self.prob.n_nodes, self.prob.n_states))
        self._check(self.lib.ocpu_get_psi(self.ctx, ptr(out)))
        return out

    def density(self):
        out = np.zeros(self.prob.n_cells * self.prob.nq)
        self._check(self.lib.ocpu_density(self.ctx, ptr(out)))
        return out
