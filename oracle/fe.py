"""Finite-element operators of the oracle (FP64, numpy/scipy).

Restated from the mathematics of DFT-FE's spectral finite elements, which the
reference calls but does not contain:

* lumped mass  M = C^T m, m_i = sum_e h_e^3 w^GLL_i  (diagonal)
* cell Hamiltonian  H_e = 1/2 h_e K_ref + N^T diag(v_KS JxW) N
  (``KohnShamDFTBaseOperator::computeCellHamiltonianMatrix``, called at
  InverseDFTSolverFunction.cpp:1388)
* Lowdin Hamiltonian  Ht x = M^{-1/2} C^T sum_e A_e H_e A_e^T C M^{-1/2} x
  (``HXWithLowdinOrthonormalisedInput``, called at
  MultiVectorAdjointLinearSolverProblem.cpp:1353)
* constraint operations distribute / set_zero / distribute_slave_to_master
  (``dftUtils::constraintMatrixInfo``, called at
  MultiVectorAdjointLinearSolverProblem.cpp:678,784,807,1361).

Vectors are [n_nodes] or [n_nodes, B] with the vector index fastest.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from invdft_b200.problem.fe import lagrange_eval


# -- constraints -----------------------------------------------------------
def _rows(cons):
    return np.repeat(np.arange(cons.n_constrained), np.diff(cons.ptr))


def distribute(cons, x):
    """x[s] = sum_m w_sm x[m] for hanging s; x[d] = 0 for Dirichlet d."""
    rows = _rows(cons)
    val = np.zeros((cons.n_constrained,) + x.shape[1:])
    contrib = cons.weights.reshape((-1,) + (1,) * (x.ndim - 1)) * x[cons.masters]
    np.add.at(val, rows, contrib)
    x[cons.nodes] = val
    return x


def set_zero(cons, x):
    x[cons.nodes] = 0.0
    return x


def distribute_slave_to_master(cons, x):
    """x[m] += w_sm x[s] for every slave s; constrained entries become zero."""
    slave_vals = x[cons.nodes].copy()
    rows = _rows(cons)
    contrib = cons.weights.reshape((-1,) + (1,) * (x.ndim - 1)) * slave_vals[rows]
    np.add.at(x, cons.masters, contrib)
    x[cons.nodes] = 0.0
    return x


# -- parent-cell operators ---------------------------------------------------
class CellOps:
    def __init__(self, prob):
        self.prob = prob
        el = prob.el
        self.el = el
        self.nd, self.nq = prob.nd, prob.nq
        self.Kref = el.stiffness_ref()
        self.N = el.shape_at_quad()              # [nq, nd]
        self.wgll = el.gll_weights3()
        n, nc, nd = prob.n_nodes, prob.n_cells, prob.nd
        cols = np.arange(nc * nd)
        self.A = sp.csr_matrix((np.ones(nc * nd), (prob.cell_nodes.ravel(), cols)), shape=(n, nc * nd))
        cons = prob.cons_psi
        # lumped mass, condensed as a vector (distribute_slave_to_master)
        m = self.A @ (prob.cell_h[:, None] ** 3 * self.wgll[None, :]).ravel()
        m = distribute_slave_to_master(cons, m)
        self.mass = m
        self.sqrt_mass = np.sqrt(m)
        self.inv_sqrt_mass = np.where(m > 0.0, 1.0 / np.sqrt(np.where(m > 0, m, 1.0)), 0.0)
        # diagonal of the Laplace stiffness, condensed the same way
        kd = self.A @ (prob.cell_h[:, None] * np.diag(self.Kref)[None, :]).ravel()
        kd = distribute_slave_to_master(cons, kd)
        self.inv_stiff = np.where(kd > 0.0, 1.0 / np.where(kd > 0, kd, 1.0), 0.0)
        self.inv_sqrt_stiff = np.sqrt(self.inv_stiff)
        self.H = None

    def assemble(self, cell_vals):
        """sum_e A_e y_e for y [n_c, nd] or [n_c, nd, B]."""
        nc, nd = self.prob.n_cells, self.nd
        if cell_vals.ndim == 2:
            return self.A @ cell_vals.reshape(nc * nd)
        return np.asarray(self.A @ cell_vals.reshape(nc * nd, -1))

    def cell_hamiltonians(self, v_ks_quad):
        """H_e = 1/2 h_e K_ref + N^T diag(v JxW) N for every cell."""
        prob = self.prob
        nc, nq, nd = prob.n_cells, self.nq, self.nd
        vj = (v_ks_quad * prob.jxw).reshape(nc, nq)
        H = np.empty((nc, nd, nd))
        step = 512
        for s in range(0, nc, step):
            e = min(nc, s + step)
            NV = vj[s:e, :, None] * self.N[None, :, :]           # [c, nq, nd]
            H[s:e] = np.matmul(self.N.T[None, :, :], NV)
        H += 0.5 * prob.cell_h[:, None, None] * self.Kref[None, :, :]
        self.H = H
        return H

    def hx(self, x):
        """Lowdin HX: M^{-1/2} C^T sum_e H_e (C M^{-1/2} x)_e."""
        prob = self.prob
        cons = prob.cons_psi
        t = self.inv_sqrt_mass.reshape((-1,) + (1,) * (x.ndim - 1)) * x
        t = distribute(cons, t)
        X = t[prob.cell_nodes]                                  # [nc, nd, (B)]
        if X.ndim == 2:
            Y = np.einsum("eij,ej->ei", self.H, X)
        else:
            Y = np.matmul(self.H, X)
        z = self.assemble(Y)
        z = distribute_slave_to_master(cons, z)
        return self.inv_sqrt_mass.reshape((-1,) + (1,) * (x.ndim - 1)) * z

    def to_quad(self, X):
        """Values of nodal block X [n, B] at the parent quad points: [n_c, nq, B]."""
        U = X[self.prob.cell_nodes]                           # [nc, nd, B]
        return np.matmul(self.N[None, :, :], U)


# -- mesh transfers (DFT-FE TransferDataBetweenMeshesIncompatiblePartitioning)
def child_to_parent_quad(prob, v_child):
    """Q1 child field at parent quad points (InverseDFTSolverFunction.cpp:860,1360).

    The child field is distributed first (its slave values are recomputed from
    the masters, InverseDFTSolverFunction.cpp:671-676).
    """
    v = distribute(prob.cons_child, np.array(v_child, dtype=np.float64))
    xi = prob.pq_xi
    nodes = prob.child_cell_nodes[prob.pq_child]
    out = np.zeros(xi.shape[0])
    for k in range(8):
        wx = xi[:, 0] if (k & 1) else 1.0 - xi[:, 0]
        wy = xi[:, 1] if (k & 2) else 1.0 - xi[:, 1]
        wz = xi[:, 2] if (k & 4) else 1.0 - xi[:, 2]
        out += wx * wy * wz * v[nodes[:, k]]
    return out


def parent_to_child_quad(prob, X, chunk=4096):
    """Parent nodal block X [n, B] at the 2x2x2 Gauss points of every child cell.

    Child cells are nested in parent cells, so each child quadrature point is
    evaluated with the parent cell's Lagrange basis (InverseDFTSolverFunction.cpp:1175-1189).
    Returns [n_cc * 8, B].
    """
    el = prob.el
    g = prob.extras["child_quad_ref"]                       # [8, 3] in [0,1]
    ncc = prob.n_child_cells
    n1 = el.n1
    ia = np.arange(prob.nd) % n1
    ib = (np.arange(prob.nd) // n1) % n1
    ic = np.arange(prob.nd) // (n1 * n1)
    out = np.empty((ncc * 8, X.shape[1]))
    for s in range(0, ncc, chunk):
        e = min(ncc, s + chunk)
        xi = prob.child_offset[s:e, None, :] + prob.child_scale[s:e, None, None] * g[None, :, :]
        xi = xi.reshape(-1, 3)
        Lx = lagrange_eval(el.nodes, xi[:, 0])
        Ly = lagrange_eval(el.nodes, xi[:, 1])
        Lz = lagrange_eval(el.nodes, xi[:, 2])
        W = (Lx[:, ia] * Ly[:, ib] * Lz[:, ic]).reshape(e - s, 8, prob.nd)
        U = X[prob.cell_nodes[prob.child_parent[s:e]]]      # [c, nd, B]
        out[s * 8:e * 8] = np.matmul(W, U).reshape(-1, X.shape[1])
    return out


def integrate_child_shape_functions(prob, S):
    """force_I = sum_c sum_q N_I(q) JxW(q) S(q), condensed with the child hanging
    constraints (InverseDFTSolverFunction.cpp:1611-1674, then compress(add))."""
    from invdft_b200.problem.fe import GAUSS2
    g = GAUSS2[0]
    q = np.arange(8)
    gx, gy, gz = g[q % 2], g[(q // 2) % 2], g[q // 4]
    Nq = np.empty((8, 8))                               # [q, k]
    for k in range(8):
        wx = gx if (k & 1) else 1.0 - gx
        wy = gy if (k & 2) else 1.0 - gy
        wz = gz if (k & 4) else 1.0 - gz
        Nq[:, k] = wx * wy * wz
    sj = (S * prob.child_jxw).reshape(prob.n_child_cells, 8)
    local = sj @ Nq                                      # [ncc, 8]
    f = np.zeros(prob.n_child_nodes)
    np.add.at(f, prob.child_cell_nodes.ravel(), local.ravel())
    # distribute_local_to_global with constraints == assemble then condense
    return distribute_slave_to_master(prob.cons_child, f)
