"""Multi-vector adjoint problem and block MINRES (oracle).

``AdjointProblem`` restates ``MultiVectorAdjointLinearSolverProblem``
(src/MultiVectorAdjointLinearSolverProblem.cpp) operation by operation.
``minres_solve`` restates the preconditioned MINRES of Paige & Saunders that
DFT-FE's ``MultiVectorMinResSolver::solve`` runs column by column (called at
InverseDFTSolverFunction.cpp:1106-1112; DFT-FE's source is not in the reference
tree).  Each column carries its own Lanczos scalars and stops once its
preconditioned residual estimate falls below the absolute tolerance.
"""
from __future__ import annotations

import numpy as np

from .eigen import partial_occupancy_der
from .fe import distribute, distribute_slave_to_master, set_zero


class AdjointProblem:
    def __init__(self, ops, temperature: float):
        """reinit (MultiVectorAdjointLinearSolverProblem.cpp:476-538) with the psi
        constraints (InverseDFTSolverFunction.cpp:260-265 passes the homogeneous
        psi constraint matrix)."""
        self.ops = ops
        self.prob = ops.prob
        self.cons = self.prob.cons_psi
        self.T = temperature
        self.compute_diagonal_a()

    def compute_diagonal_a(self):
        """D = (1/0.5) K^-1 sqrt(M)^2 and sqrt(1/0.5) K^-1/2 sqrt(M) (:541-585)."""
        o = self.ops
        self.diagA = (1.0 / 0.5) * o.inv_stiff * o.sqrt_mass * o.sqrt_mass
        self.diagSqrtA = np.sqrt(1.0 / 0.5) * o.inv_sqrt_stiff * o.sqrt_mass

    def precondition_jacobi(self, src):
        """dst = D .* src column-wise (:588-598)."""
        return self.diagA[:, None] * src

    def precondition_jacobi_sqrt(self, src):
        """dst = sqrt(D) .* src column-wise (:601-612)."""
        return self.diagSqrtA[:, None] * src

    def update_input_psi(self, psi, occ, u_vals, degeneracy, mu, eig):
        """updateInputPsi (:818-910): distribute psi, store f, 4f, -eps, the
        degenerate pair list and inputJxW = u * JxW."""
        self.psi = distribute(self.cons, np.array(psi, dtype=np.float64))
        self.B = psi.shape[1]
        self.occ = np.asarray(occ, dtype=np.float64)
        self.occ4 = 4.0 * self.occ
        self.mu = mu
        self.eig = np.asarray(eig, dtype=np.float64)
        self.neg_eig = -self.eig
        vl = []
        for i in range(self.B):
            for j in degeneracy[i]:
                vl.append((i, j))
        self.vector_list = np.asarray(vl, dtype=np.int64).reshape(-1, 2)
        self.input_jxw = u_vals * self.prob.jxw

    def compute_mu_matrix(self, occ):
        """Mu[i*B + j] = sum_cells sum_q 2 f_i psi_i psi_j u JxW over pairs (:913-986)."""
        Q = self.ops.to_quad(self.psi)                       # [nc, nq, B]
        ij = self.vector_list
        uj = self.input_jxw.reshape(Q.shape[0], Q.shape[1])
        vals = np.einsum("cqk,cq->k", Q[:, :, ij[:, 0]] * Q[:, :, ij[:, 1]], uj)
        mu = np.zeros(self.B * self.B)
        np.add.at(mu, ij[:, 0] * self.B + ij[:, 1], 2.0 * occ[ij[:, 0]] * vals)
        self.Mu = mu
        return mu

    def r_times(self, X):
        """sum_e R_e X_e with R_e = N^T diag(u JxW) N (:989-1000 and :750-785)."""
        o = self.ops
        Q = o.to_quad(X)                                     # [nc, nq, B]
        uj = self.input_jxw.reshape(Q.shape[0], Q.shape[1])
        Y = np.matmul(o.N.T[None, :, :], Q * uj[:, :, None])
        return o.assemble(Y)

    def compute_rhs(self):
        """computeRhs (:616-812).

        rhs_i = 4 f_i M^{-1/2} C^T sum_e R_e (C M^{-1/2} M^{1/2} psi)_e
                - 2 sum_k Mu[k*B + i] (M^{1/2} psi_k),  constrained rows zero.
        """
        o = self.ops
        cons = self.cons
        t = distribute(cons, self.psi.copy())
        t = o.sqrt_mass[:, None] * t                         # psiTemp = M^{1/2} psi
        mu = self.compute_mu_matrix(self.occ)
        B = self.B
        Mu = mu.reshape(B, B)                                # Mu[k, i] at k*B+i
        rhs = -2.0 * (t @ Mu)                                # rhs[:, i] = -2 sum_k Mu[k,i] t[:, k]
        t = o.inv_sqrt_mass[:, None] * t
        t = distribute(cons, t)
        t2 = self.r_times(t)
        t2 = distribute_slave_to_master(cons, t2)
        t2 = distribute(cons, t2)
        t2 = o.inv_sqrt_mass[:, None] * t2
        t2 = distribute(cons, t2)
        rhs = rhs + t2 * self.occ4[None, :]
        return set_zero(cons, rhs)

    def vmult(self, x):
        """Ax = Ht x - eps_i x with constrained entries of x and Ax zeroed (:1346-1367).

        Returns (Ax, x) since the reference zeroes x in place."""
        Ax = self.ops.hx(x)
        x = set_zero(self.cons, x)
        Ax = set_zero(self.cons, Ax)
        return Ax + x * self.neg_eig[None, :], x

    def dot_quad_wise(self, v1, v2):
        """d_k = sum_q JxW v1_i(q) v2_j(q) over the pair list (:1145-1243)."""
        Q1 = self.ops.to_quad(v1)
        Q2 = self.ops.to_quad(v2)
        ij = self.vector_list
        jxw = self.prob.jxw.reshape(Q1.shape[0], Q1.shape[1])
        return np.einsum("cqk,cq->k", Q1[:, :, ij[:, 0]] * Q2[:, :, ij[:, 1]], jxw)

    def distribute_x(self, x):
        """distributeX (:1003-1141): back to nodal values, then remove the
        null-space component with the Fermi-level (eta) correction."""
        o = self.ops
        x = o.inv_sqrt_mass[:, None] * x
        x = distribute(self.cons, x)
        dots = self.dot_quad_wise(x, self.psi)
        mu_unit = self.compute_mu_matrix(np.ones(self.B))
        B = self.B
        dfi = -partial_occupancy_der(self.eig, self.mu, self.T)
        sum_d = float(np.sum(dfi))
        eta_rhs = float(np.sum(dfi * mu_unit[np.arange(B) * B + np.arange(B)]))
        eta = 0.0 if abs(eta_rhs) < 1e-16 else eta_rhs / sum_d
        ij = self.vector_list
        der = partial_occupancy_der(self.eig[ij[:, 0]], self.mu, self.T)
        corr = -der * mu_unit[ij[:, 0] * B + ij[:, 1]]
        corr = corr + np.where(ij[:, 0] == ij[:, 1], der * eta, 0.0)
        coef = -dots + corr
        # removeNullSpace: x[:, i] += coef_k psi[:, j]
        for k, (i, j) in enumerate(ij):
            x[:, i] += coef[k] * self.psi[:, j]
        self.eta = eta
        return x


def minres_solve(problem: AdjointProblem, tol: float, maxit: int):
    """Preconditioned block MINRES, independent per column, zero initial guess.

    Returns (x, iterations per column, final residual estimates).
    """
    b = problem.compute_rhs()
    n, B = b.shape
    x = np.zeros((n, B))
    r1 = b.copy()
    y = problem.precondition_jacobi(r1)
    beta1 = np.sqrt(np.maximum(np.einsum("ij,ij->j", r1, y), 0.0))
    oldb = np.zeros(B)
    beta = beta1.copy()
    dbar = np.zeros(B)
    epsln = np.zeros(B)
    phibar = beta1.copy()
    cs = -np.ones(B)
    sn = np.zeros(B)
    w = np.zeros((n, B))
    w2 = np.zeros((n, B))
    r2 = r1.copy()
    active = phibar >= tol
    iters = np.zeros(B, dtype=np.int64)
    eps = np.finfo(np.float64).eps
    for itn in range(1, maxit + 1):
        if not active.any():
            break
        a = active
        s = np.where(a, 1.0 / np.where(beta > 0, beta, 1.0), 0.0)
        v = y * s[None, :]
        yn, v = problem.vmult(v)
        if itn >= 2:
            yn = yn - (beta / np.where(oldb > 0, oldb, 1.0))[None, :] * r1
        alfa = np.einsum("ij,ij->j", v, yn)
        yn = yn - (alfa / np.where(beta > 0, beta, 1.0))[None, :] * r2
        r1n = r2
        r2n = yn
        yp = problem.precondition_jacobi(r2n)
        oldbn = beta
        betan = np.sqrt(np.maximum(np.einsum("ij,ij->j", r2n, yp), 0.0))
        oldeps = epsln
        delta = cs * dbar + sn * alfa
        gbar = sn * dbar - cs * alfa
        epslnn = sn * betan
        dbarn = -cs * betan
        gamma = np.maximum(np.sqrt(gbar * gbar + betan * betan), eps)
        csn = gbar / gamma
        snn = betan / gamma
        phi = csn * phibar
        phibarn = snn * phibar
        w1 = w2
        w2n = w
        wn = (v - oldeps[None, :] * w1 - delta[None, :] * w2n) / gamma[None, :]
        xn = x + phi[None, :] * wn
        # commit only the active columns
        sel = a[None, :]
        x = np.where(sel, xn, x)
        r1 = np.where(sel, r1n, r1)
        r2 = np.where(sel, r2n, r2)
        y = np.where(sel, yp, y)
        w = np.where(sel, wn, w)
        w2 = np.where(sel, w2n, w2)
        oldb = np.where(a, oldbn, oldb)
        beta = np.where(a, betan, beta)
        epsln = np.where(a, epslnn, epsln)
        dbar = np.where(a, dbarn, dbar)
        cs = np.where(a, csn, cs)
        sn = np.where(a, snn, sn)
        phibar = np.where(a, phibarn, phibar)
        iters = iters + a
        active = a & (phibar >= tol)
    return x, iters, phibar
