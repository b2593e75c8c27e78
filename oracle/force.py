"""Oracle of ``InverseDFTSolverFunction`` (src/InverseDFTSolverFunction.cpp).

``getForceVector`` follows InverseDFTSolverFunction.cpp:657-1311 step by step:
distribute v_xc -> solveEigen (adaptive tolerance, ChFSI passes, Fermi level,
occupancies, max residual over occupied states) -> rho -> drho/loss/u ->
per block: degeneracy-aware block size, updateInputPsi, block MINRES,
distributeX, adjoint constraints, psi.p at child quad points -> projection
onto the Q1 v_xc nodes -> zero constrained entries.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .adjoint import AdjointProblem, minres_solve
from .eigen import (chfsi_pass, fermi_energy, hash_uniform, lanczos_bounds,
                    lanczos_start, partial_occupancy)
from .fe import (CellOps, child_to_parent_quad, distribute, integrate_child_shape_functions,
                 parent_to_child_quad, set_zero)


@dataclass
class ForceParams:
    """Knobs of the hot path (inverseDFTParameters / dftParameters names)."""
    cheb_degree: int = 50                  # CHEBYSHEV POLYNOMIAL DEGREE (0: from the spectrum bound)
    max_cheb_passes: int = 100             # MAX CHEBYSHEV PASSES
    cheby_tol: float = 1e-6                # CHEBYSHEV FILTER TOLERANCE
    initial_tol_cheb: float = 1e-6         # INITIAL TOL FOR CHEBYSHEV FILTERING
    adaptive_factor_cheb: float = 100.0    # ADAPTIVE FACTOR FOR CHEBYSHEV FILTERING
    adjoint_initial_tol: float = 1e-11     # INITIAL TOL FOR ADJOINT PROBLEM
    adaptive_factor_adjoint: float = 1000.0  # ADAPTIVE FACTOR FOR ADJOINT
    adjoint_max_iter: int = 5000           # MAX ITERATIONS FOR ADJOINT PROBLEM
    degeneracy_tol: float = 0.002          # TOL FOR DEGENERACY
    frac_occ_tol: float = 1e-8             # TOL FOR FRACTIONAL OCCUPANCY
    additional_states: int = 0             # Solve Additional States During Cheb Filtering
    block_size: int = 0                    # CHEBY WFC BLOCK SIZE (0: all states)
    inter_block_size: int = 10             # BLOCK SIZE OF INTERPOLATE
    factor_lda: float = 0.0                # FACTOR FOR LDA VXC
    lanczos_steps: int = 20


@dataclass
class ForceStats:
    passes: int = 0
    max_residual: float = 0.0
    cheb_tol: float = 0.0
    adjoint_tol: float = 0.0
    minres_iters: list = field(default_factory=list)
    loss: float = 0.0
    loss_unweighted: float = 0.0
    l1_error: float = 0.0
    int_rho_veff: float = 0.0
    fermi_energy: float = 0.0
    eigenvalues: np.ndarray | None = None
    occupancy: np.ndarray | None = None
    eta: list = field(default_factory=list)
    degree: int = 0


def auto_degree(upper_bound: float) -> int:
    """Filter degree when none is given: ceil(3 sqrt(b)) clamped to [24, 500].

    The damping of a state at relative distance d below the unwanted interval
    [a, b] is cosh(m acosh(1 + 2 d / (b - a))) ~ exp(2 m sqrt(d / b)), so a
    degree growing like sqrt(b) keeps the per-pass reduction roughly fixed as
    the mesh is refined (the role of DFT-FE's automatic degree choice)."""
    import math
    return int(min(500, max(24, math.ceil(3.0 * math.sqrt(max(upper_bound, 0.0))))))


def evaluate_degeneracy_map(eig, tol):
    """InverseDFTSolverFunction.cpp:37-77: groups of states closer than tol."""
    N = len(eig)
    group_of = {}
    groups = {}
    count = 0
    for i in range(N):
        if i in group_of:
            g = group_of[i]
            for j in range(N):
                if abs(eig[i] - eig[j]) < tol:
                    groups[g].add(j)
                    group_of[j] = g
        else:
            groups[count] = {i}
            group_of[i] = count
            for j in range(N):
                if abs(eig[i] - eig[j]) < tol:
                    groups[count].add(j)
                    group_of[j] = count
            count += 1
    return [sorted(groups[group_of[i]]) for i in range(N)]


class InverseDFTSolverFunction:
    """Oracle of the force evaluation for one spin channel and the Gamma point."""

    def __init__(self, prob, params: ForceParams | None = None, X0=None):
        self.prob = prob
        self.params = params or ForceParams()
        self.ops = CellOps(prob)
        self.adjoint = AdjointProblem(self.ops, prob.temperature)
        self.N = prob.n_states
        n = prob.n_nodes
        self.free = ~prob.cons_psi.is_constrained()
        if X0 is None:
            X0 = initial_subspace(n, self.N, self.free)
        self.X = np.array(X0, dtype=np.float64)          # Lowdin coefficients
        self.eig = None
        self.counter = 0
        self.tol_cheb = 1e-8
        self.loss_prev = 0.0
        self.adjoint_tol = self.params.adjoint_initial_tol

    # -- a2: solveEigen (InverseDFTSolverFunction.cpp:1315-1477)
    def solve_eigen(self, pot, stats: ForceStats):
        prm, prob = self.params, self.prob
        if self.counter > 3:
            prev = self.tol_cheb
            self.tol_cheb = min(prm.cheby_tol, self.loss_prev / prm.adaptive_factor_cheb)
            self.tol_cheb = min(self.tol_cheb, prev)
        else:
            self.tol_cheb = min(prm.cheby_tol, prm.initial_tol_cheb)
        v_xc_q = child_to_parent_quad(prob, pot)
        self.v_ks = prob.v_base + v_xc_q + prm.factor_lda * prob.v_lda
        self.ops.cell_hamiltonians(self.v_ks)
        hx = self.ops.hx
        lo, b = lanczos_bounds(hx, lanczos_start(prob.n_nodes, self.free), prm.lanczos_steps)
        degree = prm.cheb_degree if prm.cheb_degree > 0 else auto_degree(b)
        stats.degree = degree
        stats.passes = 0
        while True:
            if self.eig is None:
                a0 = lo
                a = lo + 0.1 * (b - lo)
            else:
                a0 = float(self.eig[0])
                a = float(self.eig[-1])
            self.X, self.eig, res = chfsi_pass(hx, self.X, degree, a, b, a0)
            mu = fermi_energy(self.eig, prob.n_electrons, prob.temperature)
            occ = partial_occupancy(self.eig, mu, prob.temperature)
            homo = 0
            for i in range(self.N):
                if self.eig[i] < mu + 1e-3 and homo < i:
                    homo = i
            mask = (occ > prm.frac_occ_tol) | (np.arange(self.N) <= homo + prm.additional_states)
            maxres = float(np.max(res[mask])) if mask.any() else 0.0
            stats.passes += 1
            if not (maxres > self.tol_cheb and stats.passes < prm.max_cheb_passes):
                break
        self.mu, self.occ = mu, occ
        stats.max_residual = maxres
        stats.cheb_tol = self.tol_cheb
        # nodal values of the eigenvectors (M^{-1/2}, distribute)
        psi = self.ops.inv_sqrt_mass[:, None] * self.X
        self.psi = distribute(prob.cons_psi, psi)

    def density(self):
        """rho(q) = 2 sum_i f_i psi_i(q)^2 (computeRhoFromPSI, :748-758)."""
        Q = self.ops.to_quad(self.psi)
        return (2.0 * np.sum(self.occ[None, None, :] * Q * Q, axis=2)).ravel()

    # -- a1: getForceVector (InverseDFTSolverFunction.cpp:657-1311)
    def get_force_vector(self, pot):
        prm, prob = self.params, self.prob
        stats = ForceStats()
        pot = distribute(prob.cons_child, np.array(pot, dtype=np.float64))
        self.solve_eigen(pot, stats)
        eig, mu, occ = self.eig, self.mu, self.occ
        rho = self.density()
        drho = prob.rho_target_up - 0.5 * rho
        jxw = prob.jxw
        u = drho * prob.weight
        stats.l1_error = float(np.sum(np.abs(drho * jxw)))
        stats.loss_unweighted = float(np.sum(drho * drho * jxw))
        loss = float(np.sum(drho * drho * prob.weight * jxw))
        stats.int_rho_veff = float(np.sum(self.v_ks * rho * jxw))
        S = np.zeros(prob.n_child_cells * 8)
        N = self.N
        block = prm.block_size if prm.block_size > 0 else N
        jvec = 0
        while jvec < N:
            bs = min(block, N - jvec)
            while True:
                last = jvec + bs - 1
                if last + 1 != N and abs(eig[last] - eig[last + 1]) < prm.degeneracy_tol:
                    bs -= 1
                else:
                    break
            sl = slice(jvec, jvec + bs)
            shifts = eig[sl]
            focc = occ[sl] * 1.0                                # * k-point weight
            degen = evaluate_degeneracy_map(list(shifts), prm.degeneracy_tol)
            self.adjoint.update_input_psi(self.psi[:, sl], focc, u, degen, mu, shifts)
            self.adjoint_tol = min(self.adjoint_tol, self.tol_cheb / prm.adaptive_factor_adjoint)
            x, iters, _ = minres_solve(self.adjoint, self.adjoint_tol, prm.adjoint_max_iter)
            x = self.adjoint.distribute_x(x)
            stats.minres_iters.extend(int(i) for i in iters)
            stats.eta.append(self.adjoint.eta)
            p = distribute(prob.cons_adj, x.copy())
            psi_b = self.adjoint.psi
            for s0 in range(0, bs, prm.inter_block_size):
                s1 = min(bs, s0 + prm.inter_block_size)
                pq = parent_to_child_quad(prob, psi_b[:, s0:s1])
                aq = parent_to_child_quad(prob, p[:, s0:s1])
                S += np.sum(pq * aq, axis=1)
            jvec += bs
        force = integrate_child_shape_functions(prob, S)
        force = set_zero(prob.cons_child, force)
        stats.adjoint_tol = self.adjoint_tol
        stats.loss = loss
        stats.fermi_energy = mu
        stats.eigenvalues = eig.copy()
        stats.occupancy = occ.copy()
        self.loss_prev = loss
        self.counter += 1
        self.last_rho = rho
        self.last_S = S
        return force, loss, stats

    @staticmethod
    def dot_product(a, b):
        """dotProduct with blockSize 1 (InverseDFTSolverFunction.cpp:1693-1705)."""
        return float(np.dot(a, b))

    @staticmethod
    def dot_product_blocks(a, b, block_size: int):
        """dotProduct (InverseDFTSolverFunction.cpp:1693-1705): entry i adds
        a_i b_i to out[i % blockSize], in entry order."""
        out = [0.0] * block_size
        for i, (x, y) in enumerate(zip(np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64))):
            out[i % block_size] += float(x) * float(y)
        return out


def initial_subspace(n: int, N: int, free: np.ndarray) -> np.ndarray:
    """Deterministic start block X[i, j] = hash_uniform(i * N + j, salt 11), free rows."""
    idx = np.arange(n, dtype=np.int64)[:, None] * N + np.arange(N)[None, :]
    X = hash_uniform(idx.ravel(), 11).reshape(n, N)
    X[~free] = 0.0
    return X
