"""ctypes binding of ``include/invdft_force.h`` (libinvdft_b200.so).

There is no CPU fallback: if the shared library is missing or cannot be
loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libinvdft_b200.so"

STATUS = {0: "OK", 1: "MAXITER", 2: "NONFINITE", 3: "BREAKDOWN", 4: "OOM", 5: "BAD_ARG",
          6: "CUDA_ERROR", 7: "NOT_READY"}

EXPORTED = [
    "invdft_default_params", "invdft_force_create", "invdft_force_destroy", "invdft_last_error",
    "invdft_set_params", "invdft_set_profiling", "invdft_set_subspace", "invdft_force_eval", "invdft_dot", "invdft_get_eigen",
    "invdft_get_psi", "invdft_get_density", "invdft_get_child_quad_products", "invdft_solve_eigen",
    "invdft_force_backward",
    "invdft_set_potential", "invdft_hx", "invdft_adjoint_update_psi", "invdft_adjoint_compute_rhs",
    "invdft_adjoint_vmult", "invdft_adjoint_precondition_jacobi",
    "invdft_adjoint_precondition_jacobi_sqrt", "invdft_adjoint_distribute_x", "invdft_adjoint_solve",
    "invdft_bfgs_solve", "invdft_coldot_noalloc", "invdft_project_vxc_to_parent", "invdft_evaluate_parent_field",
    "invdft_force_backward_at", "invdft_dot_blocks", "invdft_get_index_map",
    "invdft_poisson_total_potential", "invdft_kernel_probe", "invdft_bfgs_run", "invdft_initial_guess",
]

# invdft_get_index_map selectors (include/invdft_force.h)
INDEX_MAPS = {"cell_nodes": 0, "cell_gather": 1, "cell_slots": 2, "psi_rows": 3, "psi_ptr": 4, "psi_masters": 5,
              "adj_rows": 6, "adj_ptr": 7, "adj_masters": 8, "child_rows": 9, "child_ptr": 10,
              "child_masters": 11, "child_cell_nodes": 12, "pq_child": 13}


class InvDFTError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


_P = C.POINTER
_i64p = _P(C.c_int64)
_f64p = _P(C.c_double)


class Constraints(C.Structure):
    _fields_ = [("n_rows", C.c_int64), ("rows", _i64p), ("ptr", _i64p), ("masters", _i64p),
                ("weights", _f64p)]


class ProblemDesc(C.Structure):
    _fields_ = [
        ("p", C.c_int32), ("n_cells", C.c_int64), ("n_nodes", C.c_int64), ("cell_nodes", _i64p),
        ("cell_h", _f64p), ("gll_nodes", _f64p), ("gll_weights", _f64p), ("gauss_points", _f64p),
        ("gauss_weights", _f64p), ("cons_psi", Constraints), ("cons_adj", Constraints),
        ("jxw", _f64p), ("v_base", _f64p), ("v_lda", _f64p), ("rho_target_up", _f64p), ("weight", _f64p),
        ("n_child_cells", C.c_int64), ("n_child_nodes", C.c_int64), ("child_cell_nodes", _i64p),
        ("child_jxw", _f64p), ("cons_child", Constraints), ("child_parent", _i64p),
        ("child_offset", _f64p), ("child_scale", _f64p), ("pq_child", _i64p), ("pq_xi", _f64p),
        ("n_states", C.c_int32), ("n_electrons", C.c_double), ("temperature", C.c_double),
    ]


class Params(C.Structure):
    _fields_ = [
        ("cheb_degree", C.c_int32), ("max_cheb_passes", C.c_int32), ("cheby_tol", C.c_double),
        ("initial_tol_cheb", C.c_double), ("adaptive_factor_cheb", C.c_double),
        ("adjoint_initial_tol", C.c_double), ("adaptive_factor_adjoint", C.c_double),
        ("adjoint_max_iter", C.c_int32), ("degeneracy_tol", C.c_double), ("frac_occ_tol", C.c_double),
        ("additional_states", C.c_int32), ("block_size", C.c_int32), ("inter_block_size", C.c_int32),
        ("factor_lda", C.c_double), ("lanczos_steps", C.c_int32), ("precision", C.c_int32),
        ("mixed_residual_floor", C.c_double), ("mixed_inner_tol", C.c_double), ("mixed_max_refine", C.c_int32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("passes", C.c_int32), ("max_residual", C.c_double), ("cheb_tol", C.c_double),
        ("adjoint_tol", C.c_double), ("loss", C.c_double), ("loss_unweighted", C.c_double),
        ("l1_error", C.c_double), ("int_rho_veff", C.c_double), ("fermi_energy", C.c_double),
        ("minres_iters_max", C.c_int32), ("minres_iters_sum", C.c_int64), ("n_blocks", C.c_int32),
        ("n_hx_calls", C.c_int32), ("n_hx_columns", C.c_int64), ("ms_eigen", C.c_double),
        ("ms_density", C.c_double), ("ms_adjoint", C.c_double), ("ms_transfer", C.c_double),
        ("n_cell_gemm", C.c_int32), ("ms_cell_gemm", C.c_double), ("cell_gemm_bytes", C.c_double),
        ("cell_gemm_flops", C.c_double), ("n_launches", C.c_int64), ("degree", C.c_int32),
        ("upper_bound", C.c_double), ("device_bytes", C.c_double), ("device_bytes_peak", C.c_double),
        ("passes_low", C.c_int32), ("generation", C.c_int64), ("refine_steps", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class BfgsOptions(C.Structure):
    _fields_ = [("max_iter", C.c_int32), ("tol", C.c_double), ("line_search_iters", C.c_int32),
                ("line_search_tol", C.c_double), ("history", C.c_int32), ("density_l1_target", C.c_double)]


class BfgsReport(C.Structure):
    _fields_ = [("n_iters", C.c_int32), ("n_evals", C.c_int32), ("final_loss", C.c_double),
                ("final_density_l1", C.c_double), ("reached", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class InitialGuessOptions(C.Structure):
    _fields_ = [("tau_vx", C.c_double), ("tau_fa", C.c_double), ("fermi_amaldi_bc", C.c_int32),
                ("factor_fa", C.c_double), ("hartree_rel_tol", C.c_double), ("hartree_max_iter", C.c_int32)]


_lib = None


def load() -> C.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH.name} is not built; run `python -m invdft_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    sig = {
        "invdft_default_params": (None, [_P(Params)]),
        "invdft_force_create": (C.c_int, [_P(ProblemDesc), _P(Params), _P(vp)]),
        "invdft_force_destroy": (None, [vp]),
        "invdft_last_error": (C.c_char_p, [vp]),
        "invdft_set_params": (C.c_int, [vp, _P(Params)]),
        "invdft_set_subspace": (C.c_int, [vp, _f64p]),
        "invdft_set_profiling": (C.c_int, [vp, C.c_int32]),
        "invdft_force_eval": (C.c_int, [vp, _f64p, _f64p, _f64p, _P(Stats)]),
        "invdft_dot": (C.c_int, [vp, _f64p, _f64p, C.c_int64, _f64p]),
        "invdft_get_eigen": (C.c_int, [vp, _f64p, _f64p, _f64p]),
        "invdft_get_psi": (C.c_int, [vp, _f64p]),
        "invdft_get_density": (C.c_int, [vp, _f64p]),
        "invdft_get_child_quad_products": (C.c_int, [vp, _f64p]),
        "invdft_solve_eigen": (C.c_int, [vp, _f64p, _P(Stats)]),
        "invdft_force_backward": (C.c_int, [vp, _f64p, _P(Stats)]),
        "invdft_force_backward_at": (C.c_int, [vp, C.c_int64, _f64p, _P(Stats)]),
        "invdft_dot_blocks": (C.c_int, [vp, _f64p, _f64p, C.c_int64, C.c_int32, _f64p]),
        "invdft_get_index_map": (C.c_int, [vp, C.c_int32, _P(C.c_int32), C.c_int64]),
        "invdft_kernel_probe": (C.c_int, [vp]),
        "invdft_initial_guess": (C.c_int, [vp, _f64p, _f64p, _f64p, _P(InitialGuessOptions), _f64p, _f64p, _f64p]),
        "invdft_bfgs_run": (C.c_int, [vp, _f64p, _P(BfgsOptions), _f64p, _f64p, C.c_int32, _P(BfgsReport)]),
        "invdft_poisson_total_potential": (C.c_int, [vp, _f64p, C.c_int32, _f64p, _i64p, _f64p, C.c_double,
                                                     C.c_int32, C.c_int32, _f64p, _f64p, _P(C.c_int32),
                                                     _f64p]),
        "invdft_set_potential": (C.c_int, [vp, _f64p]),
        "invdft_hx": (C.c_int, [vp, vp, vp, C.c_int32]),
        "invdft_project_vxc_to_parent": (C.c_int, [vp, _f64p, _f64p]),
        "invdft_evaluate_parent_field": (C.c_int, [vp, _f64p, C.c_int64, _i64p, _f64p, _f64p]),
        "invdft_adjoint_update_psi": (C.c_int, [vp, vp, _f64p, vp, _P(C.c_int32), _P(C.c_int32),
                                                C.c_double, _f64p, C.c_int32]),
        "invdft_adjoint_compute_rhs": (C.c_int, [vp, vp]),
        "invdft_adjoint_vmult": (C.c_int, [vp, vp, vp]),
        "invdft_adjoint_precondition_jacobi": (C.c_int, [vp, vp, vp, C.c_double]),
        "invdft_adjoint_precondition_jacobi_sqrt": (C.c_int, [vp, vp, vp, C.c_double]),
        "invdft_adjoint_distribute_x": (C.c_int, [vp, vp]),
        "invdft_adjoint_solve": (C.c_int, [vp, vp, C.c_double, C.c_int32, _P(C.c_int32)]),
        "invdft_bfgs_solve": (C.c_int, [vp, _f64p, C.c_int32, C.c_double, C.c_int32, C.c_double,
                                        C.c_int32, _f64p, _P(C.c_int32)]),
        "invdft_coldot_noalloc": (C.c_int, [vp, vp, C.c_int64, C.c_int32, vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def i64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int64)


def ptr(a: np.ndarray):
    if a.dtype == np.float64:
        return a.ctypes.data_as(_f64p)
    if a.dtype == np.int64:
        return a.ctypes.data_as(_i64p)
    if a.dtype == np.int32:
        return a.ctypes.data_as(_P(C.c_int32))
    raise TypeError(a.dtype)


def default_params(**overrides) -> Params:
    lib = load()
    p = Params()
    lib.invdft_default_params(C.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def make_desc(prob, keep: list) -> ProblemDesc:
    """Fill a ProblemDesc from a setup Problem; ``keep`` holds the arrays alive."""
    def arr(a, kind):
        a = f64(a) if kind == "f" else i64(a)
        keep.append(a)
        return ptr(a)

    def cons(c):
        return Constraints(c.n_constrained, arr(c.nodes, "i"), arr(c.ptr, "i"), arr(c.masters, "i"),
                           arr(c.weights, "f"))

    el = prob.el
    d = ProblemDesc()
    d.p = prob.p
    d.n_cells = prob.n_cells
    d.n_nodes = prob.n_nodes
    d.cell_nodes = arr(prob.cell_nodes, "i")
    d.cell_h = arr(prob.cell_h, "f")
    d.gll_nodes = arr(el.nodes, "f")
    d.gll_weights = arr(el.wgll, "f")
    d.gauss_points = arr(el.qpts, "f")
    d.gauss_weights = arr(el.wq, "f")
    d.cons_psi = cons(prob.cons_psi)
    d.cons_adj = cons(prob.cons_adj)
    d.jxw = arr(prob.jxw, "f")
    d.v_base = arr(prob.v_base, "f")
    d.v_lda = arr(prob.v_lda, "f")
    d.rho_target_up = arr(prob.rho_target_up, "f")
    d.weight = arr(prob.weight, "f")
    d.n_child_cells = prob.n_child_cells
    d.n_child_nodes = prob.n_child_nodes
    d.child_cell_nodes = arr(prob.child_cell_nodes, "i")
    d.child_jxw = arr(prob.child_jxw, "f")
    d.cons_child = cons(prob.cons_child)
    d.child_parent = arr(prob.child_parent, "i")
    d.child_offset = arr(prob.child_offset, "f")
    d.child_scale = arr(prob.child_scale, "f")
    d.pq_child = arr(prob.pq_child, "i")
    d.pq_xi = arr(prob.pq_xi, "f")
    d.n_states = prob.n_states
    d.n_electrons = float(prob.n_electrons)
    d.temperature = float(prob.temperature)
    return d


def exported_symbols(path: str | os.PathLike | None = None) -> list[str]:
    """Names of the EXPORTED entry points that the library resolves."""
    lib = C.CDLL(str(path or LIB_PATH))
    found = []
    for name in EXPORTED:
        try:
            getattr(lib, name)
            found.append(name)
        except AttributeError:
            pass
    return found
