"""Python mirror of the reference's interfaces for the force-evaluation path.

``InverseDFTSolverFunction`` mirrors include/InverseDFTSolverFunction.h:51-384
(``getForceVector``, ``dotProduct``, ``getInitialGuess``/``setInitialGuess``/
``setSolution``); ``MultiVectorAdjointLinearSolverProblem`` mirrors
include/MultiVectorAdjointLinearSolverProblem.h:15-214 (``updateInputPsi``,
``computeRhs``, ``vmult``, ``precondition_Jacobi``, ``precondition_JacobiSqrt``,
``distributeX``); ``BFGSInverseDFTSolver`` mirrors BFGSInverseDFTSolver.h:28-119.
Every call goes through the C ABI of libinvdft_b200.so; device blocks are
torch CUDA tensors of shape [n_nodes, B], float64.
Where the reference aborts (AssertThrow), these raise ``InvDFTError``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native
from .native import InvDFTError, Stats, f64, i64, ptr


def _check(lib, ctx, rc):
    if rc != 0:
        raise InvDFTError(rc, lib.invdft_last_error(ctx).decode())


class InverseDFTSolverFunction:
    """Force evaluation v_xc -> (dL/dv_xc, L) on one B200."""

    def __init__(self, problem, params: native.Params | None = None, **overrides):
        self.lib = native.load()
        self.problem = problem
        self.params = params or native.default_params(**overrides)
        keep: list = []
        desc = native.make_desc(problem, keep)
        ctx = C.c_void_p()
        rc = self.lib.invdft_force_create(C.byref(desc), C.byref(self.params), C.byref(ctx))
        if rc != 0:
            raise InvDFTError(rc, self.lib.invdft_last_error(None).decode())
        self.ctx = ctx
        self.n_child = problem.n_child_nodes
        self.N = problem.n_states
        self._pot = None
        self.last_stats: dict = {}

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.invdft_force_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, **overrides):
        for k, v in overrides.items():
            setattr(self.params, k, v)
        _check(self.lib, self.ctx, self.lib.invdft_set_params(self.ctx, C.byref(self.params)))

    def set_subspace(self, X):
        X = f64(X)
        if X.shape != (self.problem.n_nodes, self.N):
            raise ValueError("subspace shape mismatch")
        _check(self.lib, self.ctx, self.lib.invdft_set_subspace(self.ctx, ptr(X)))

    # -- reference interface -------------------------------------------------
    def get_force_vector(self, pot):
        """Returns (force, loss, stats); ``pot`` (numpy) is distributed then has its
        constrained entries zeroed in place, as the reference does."""
        if not isinstance(pot, np.ndarray) or pot.dtype != np.float64 or not pot.flags.c_contiguous:
            raise TypeError("pot must be a contiguous float64 numpy array")
        if pot.shape != (self.n_child,):
            raise ValueError("pot has the wrong length")
        force = np.zeros(self.n_child)
        loss = C.c_double()
        st = Stats()
        _check(self.lib, self.ctx, self.lib.invdft_force_eval(self.ctx, ptr(pot), ptr(force), C.byref(loss),
                                                               C.byref(st)))
        self.last_stats = st.as_dict()
        return force, float(loss.value), self.last_stats

    def getForceVector(self, pot: list, force: list, loss: list):
        """getForceVector(pot, force, loss) with per-spin lists (one spin here)."""
        if len(pot) != 1:
            raise InvDFTError(5, "one spin channel is supported")
        f, L, _ = self.get_force_vector(pot[0])
        force[:] = [f]
        loss[:] = [L]

    def dotProduct(self, a, b, blockSize: int = 1):
        """dotProduct (InverseDFTSolverFunction.cpp:1693-1705): entry i
        accumulates into out[i % blockSize]."""
        a, b = f64(a), f64(b)
        if a.size != b.size:
            raise ValueError("dotProduct of vectors of different lengths")
        out = np.zeros(int(blockSize))
        _check(self.lib, self.ctx, self.lib.invdft_dot_blocks(self.ctx, ptr(a), ptr(b), a.size, int(blockSize),
                                                               ptr(out)))
        return list(out)

    def dot_product(self, a, b) -> float:
        return self.dotProduct(a, b)[0]

    def getInitialGuess(self):
        return [self._pot.copy()] if self._pot is not None else None

    def setInitialGuess(self, pot, target_pot_values=None):
        self._pot = f64(pot[0]).copy()

    def setSolution(self, pot):
        self._pot = f64(pot[0]).copy()

    # -- results of the last evaluation ---------------------------------------
    def solve_eigen(self, pot):
        st = Stats()
        _check(self.lib, self.ctx, self.lib.invdft_solve_eigen(self.ctx, ptr(pot), C.byref(st)))
        return st.as_dict()

    def eigen(self):
        e, o, mu = np.zeros(self.N), np.zeros(self.N), C.c_double()
        _check(self.lib, self.ctx, self.lib.invdft_get_eigen(self.ctx, ptr(e), ptr(o), C.byref(mu)))
        return e, o, mu.value

    def psi(self):
        out = np.zeros((self.problem.n_nodes, self.N))
        _check(self.lib, self.ctx, self.lib.invdft_get_psi(self.ctx, ptr(out)))
        return out

    def density(self):
        out = np.zeros(self.problem.n_cells * self.problem.nq)
        _check(self.lib, self.ctx, self.lib.invdft_get_density(self.ctx, ptr(out)))
        return out

    def child_quad_products(self):
        out = np.zeros(self.problem.n_child_cells * 8)
        _check(self.lib, self.ctx, self.lib.invdft_get_child_quad_products(self.ctx, ptr(out)))
        return out

    def poisson_total_potential(self, rho_quad, Z=(), atom_cell=(), atom_xi=(), rel_tol: float = 1e-12,
                                max_iter: int = 20000, install: bool = False):
        """setPotBasePoissonNuclear (InverseDFTEngine.cpp:2459-2571) on the GPU:
        phi of -lap phi = 4 pi (rho - sum Z delta) with zero boundary values;
        returns (phi at the parent quadrature points, nodal phi, CG iterations,
        relative residual).  install=True makes it the base potential."""
        rho = f64(rho_quad)
        Zs = f64(np.asarray(Z, dtype=np.float64).reshape(-1))
        cells = i64(np.asarray(atom_cell, dtype=np.int64).reshape(-1))
        xi = f64(np.asarray(atom_xi, dtype=np.float64).reshape(-1, 3) if len(Zs) else np.zeros((0, 3)))
        phi_q = np.zeros(self.problem.n_cells * self.problem.nq)
        phi_n = np.zeros(self.problem.n_nodes)
        it = C.c_int32()
        res = C.c_double()
        _check(self.lib, self.ctx, self.lib.invdft_poisson_total_potential(
            self.ctx, ptr(rho), int(Zs.size), ptr(Zs), ptr(cells), ptr(xi), float(rel_tol), int(max_iter),
            int(bool(install)), ptr(phi_q), ptr(phi_n), C.byref(it), C.byref(res)))
        return phi_q, phi_n, it.value, res.value

    def initial_guess(self, rho_quad, sigma_quad=None, hartree_bc=None, tau_vx: float = 1e-2,
                      tau_fa: float = 1e-2, fermi_amaldi_bc: bool = False, factor_fa: float = 1.0,
                      hartree_rel_tol: float = 1e-12, hartree_max_iter: int = 20000):
        """setInitialPotL2Proj (InverseDFTEngine.cpp:1046-1498) on the GPU:
        returns (v_xc guess on the child nodes, parent nodal field, v_H at the
        parent quadrature points)."""
        o = native.InitialGuessOptions(tau_vx, tau_fa, int(bool(fermi_amaldi_bc)), factor_fa, hartree_rel_tol,
                                       hartree_max_iter)
        rho = f64(rho_quad)
        sig = None if sigma_quad is None else ptr(f64(sigma_quad))
        bc = None if hartree_bc is None else ptr(f64(hartree_bc))
        child = np.zeros(self.problem.n_child_nodes)
        parent = np.zeros(self.problem.n_nodes)
        vh = np.zeros(self.problem.n_cells * self.problem.nq)
        _check(self.lib, self.ctx, self.lib.invdft_initial_guess(self.ctx, ptr(rho), sig, bc, C.byref(o), ptr(child),
                                                                  ptr(parent), ptr(vh)))
        return child, parent, vh

    def index_map(self, name: str, n: int) -> np.ndarray:
        """An integer index map the library built on the device (int32),
        see invdft_get_index_map."""
        out = np.zeros(int(n), dtype=np.int32)
        _check(self.lib, self.ctx, self.lib.invdft_get_index_map(self.ctx, native.INDEX_MAPS[name], ptr(out), int(n)))
        return out

    def set_potential(self, pot):
        pot = f64(pot).copy()
        _check(self.lib, self.ctx, self.lib.invdft_set_potential(self.ctx, ptr(pot)))

    def project_vxc_to_parent(self, vxc_child) -> np.ndarray:
        """POST_PROCESS projection (InverseDFTEngine::projectVxcToParentMesh,
        InverseDFTEngine.cpp:3462-3545): the parent nodal field of v_xc +
        factorForLDAVxc v_LDA by a lumped-mass L2 projection."""
        v = f64(vxc_child).copy()
        out = np.zeros(self.problem.n_nodes)
        _check(self.lib, self.ctx, self.lib.invdft_project_vxc_to_parent(self.ctx, ptr(v), ptr(out)))
        return out

    def evaluate_parent_field(self, nodal, cells, xi) -> np.ndarray:
        """A parent nodal field at points given by (cell, reference coordinates
        in [0, 1]^3), as the writeToPoints branch of interpolateVxc
        (InverseDFTEngine.cpp:3275-3456) evaluates it."""
        u = f64(nodal)
        c = i64(cells)
        x = f64(xi).reshape(-1, 3)
        out = np.zeros(c.size)
        _check(self.lib, self.ctx, self.lib.invdft_evaluate_parent_field(self.ctx, ptr(u), c.size, ptr(c),
                                                                         ptr(x), ptr(out)))
        return out

    def hx(self, x):
        """Lowdin HX of a torch CUDA float64 block [n_nodes, B]."""
        import torch
        x = x.contiguous()
        y = torch.empty_like(x)
        _check(self.lib, self.ctx, self.lib.invdft_hx(self.ctx, C.c_void_p(x.data_ptr()),
                                                       C.c_void_p(y.data_ptr()), x.shape[1]))
        return y

    def bfgs_solve(self, pot, max_iter: int, tol: float = 1e-12, line_search_iters: int = 1,
                   line_search_tol: float = 1e-6, history: int = 100):
        pot = f64(pot).copy()
        losses = np.zeros(2 * max_iter + 1)
        n = C.c_int32()
        _check(self.lib, self.ctx, self.lib.invdft_bfgs_solve(self.ctx, ptr(pot), max_iter, tol,
                                                               line_search_iters, line_search_tol, history,
                                                               ptr(losses), C.byref(n)))
        return pot, losses[:n.value]


def bfgs_run(fn: "InverseDFTSolverFunction", pot, max_iter: int, density_l1_target: float = 0.0,
             tol: float = 1e-12, line_search_iters: int = 1, line_search_tol: float = 1e-6, history: int = 100):
    """L-BFGS (BFGSInverseDFTSolver::solve with the CP line search) that also
    stops once int |rho - rho*| <= density_l1_target.  Returns (v_xc, report,
    losses per evaluation, int |rho - rho*| per evaluation)."""
    pot = f64(pot).copy()
    o = native.BfgsOptions(max_iter, tol, line_search_iters, line_search_tol, history, density_l1_target)
    cap = 2 * max_iter + 1
    losses, l1 = np.zeros(cap), np.zeros(cap)
    rep = native.BfgsReport()
    _check(fn.lib, fn.ctx, fn.lib.invdft_bfgs_run(fn.ctx, ptr(pot), C.byref(o), ptr(losses), ptr(l1), cap,
                                                   C.byref(rep)))
    n = rep.n_evals
    return pot, rep.as_dict(), losses[:n], l1[:n]


class MultiVectorAdjointLinearSolverProblem:
    """The adjoint operator of one block, on torch CUDA float64 tensors."""

    def __init__(self, fn: InverseDFTSolverFunction):
        self.fn = fn
        self.lib = fn.lib
        self.B = 0

    def _c(self, rc):
        _check(self.lib, self.fn.ctx, rc)

    @staticmethod
    def _dp(t):
        import torch
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
            raise TypeError("expected a contiguous float64 CUDA tensor")
        return C.c_void_p(t.data_ptr())

    def updateInputPsi(self, psi, occupancy, u_vals, degeneracy, fermi_energy, eigenvalues, blockSize):
        B = int(blockSize)
        occ = f64(occupancy)
        eig = f64(eigenvalues)
        dptr = np.zeros(B + 1, dtype=np.int32)
        idx = []
        for i in range(B):
            idx.extend(int(j) for j in degeneracy[i])
            dptr[i + 1] = len(idx)
        didx = np.asarray(idx if idx else [0], dtype=np.int32)
        self._c(self.lib.invdft_adjoint_update_psi(self.fn.ctx, self._dp(psi), ptr(occ), self._dp(u_vals),
                                                   ptr(dptr), ptr(didx), float(fermi_energy), ptr(eig), B))
        self.B = B

    def computeRhs(self, out=None):
        import torch
        if out is None:
            out = torch.empty((self.fn.problem.n_nodes, self.B), dtype=torch.float64, device="cuda")
        self._c(self.lib.invdft_adjoint_compute_rhs(self.fn.ctx, self._dp(out)))
        return out

    def vmult(self, Ax, x, blockSize=None):
        self._c(self.lib.invdft_adjoint_vmult(self.fn.ctx, self._dp(Ax), self._dp(x)))

    def precondition_Jacobi(self, dst, src, omega=0.0):
        self._c(self.lib.invdft_adjoint_precondition_jacobi(self.fn.ctx, self._dp(dst), self._dp(src), omega))

    def precondition_JacobiSqrt(self, dst, src, omega=0.0):
        self._c(self.lib.invdft_adjoint_precondition_jacobi_sqrt(self.fn.ctx, self._dp(dst), self._dp(src),
                                                                 omega))

    def distributeX(self, x):
        self._c(self.lib.invdft_adjoint_distribute_x(self.fn.ctx, self._dp(x)))

    def solve(self, x, tol: float, max_iter: int):
        iters = np.zeros(self.B, dtype=np.int32)
        self._c(self.lib.invdft_adjoint_solve(self.fn.ctx, self._dp(x), tol, max_iter, ptr(iters)))
        return iters


class BFGSInverseDFTSolver:
    """L-BFGS with the CP line search (BFGSInverseDFTSolver.cpp:467-627), run in C++."""

    def __init__(self, max_iter: int, tol: float = 1e-12, line_search_iters: int = 1,
                 line_search_tol: float = 1e-6, history: int = 100):
        self.max_iter, self.tol = max_iter, tol
        self.ls_iters, self.ls_tol, self.history = line_search_iters, line_search_tol, history
        self.losses = None
        self._x = None

    def solve(self, fn: InverseDFTSolverFunction, lsType: str = "CP"):
        if lsType != "CP":
            raise InvDFTError(5, "only the CP line search is implemented")
        x0 = fn.getInitialGuess()
        if x0 is None:
            raise InvDFTError(7, "setInitialGuess has not been called")
        self._x, self.losses = fn.bfgs_solve(x0[0], self.max_iter, self.tol, self.ls_iters, self.ls_tol,
                                             self.history)
        return self._x

    def getSolution(self):
        return [self._x]
