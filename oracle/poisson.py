"""Oracle of the base potential solve (test infrastructure only).

``InverseDFTEngine::setPotBasePoissonNuclear`` (src/InverseDFTEngine.cpp:
2459-2571) forms the total density of the target at the parent quadrature
points and hands it to ``solvePhiTotalAllElectronNonPeriodic`` (:2573-2621),
which solves DFT-FE's all-electron, non-periodic Poisson problem for the total
electrostatic potential with CG, then interpolates the nodal solution to the
quadrature points (:2523-2541) as v_base.  DFT-FE's ``poissonSolverProblem``
is not in the reference tree; restated from the mathematics:

    -lap phi = 4 pi (rho - sum_a Z_a delta(r - R_a)),  phi = 0 on the boundary

in weak form with the order-p GLL elements of the wavefunctions:
    sum_e int grad N_i . grad N_j phi_j = 4 pi sum_e int N_i rho - 4 pi sum_a Z_a N_i(R_a),
condensed with the psi constraints (hanging nodes, zero boundary), so that
phi = C phi_free.  With the Hartree potential v_H = int rho / |r - r'| and the
nuclear -Z/|r - R| this phi is v_H + v_nuc, the reference's v_base.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from invdft_b200.problem.fe import lagrange_eval


def stiffness(prob) -> sp.csr_matrix:
    """sum_e h_e K_ref assembled (the Laplacian; the Hamiltonian uses 1/2 of it)."""
    K = prob.el.stiffness_ref()
    nd = prob.nd
    rows = np.repeat(prob.cell_nodes, nd, axis=1).ravel()
    cols = np.tile(prob.cell_nodes, (1, nd)).ravel()
    vals = (prob.cell_h[:, None, None] * K[None, :, :]).ravel()
    return sp.csr_matrix((vals, (rows, cols)), shape=(prob.n_nodes, prob.n_nodes))


def point_charge_rhs(prob, Z, atom_cell, atom_xi) -> np.ndarray:
    """-4 pi sum_a Z_a N_i(R_a), nucleus a in cell atom_cell[a] at reference
    coordinates atom_xi[a] in [0, 1]^3."""
    out = np.zeros(prob.n_nodes)
    n1 = prob.el.n1
    for z, e, xi in zip(Z, atom_cell, np.asarray(atom_xi).reshape(-1, 3)):
        lx = lagrange_eval(prob.el.nodes, xi[0])[0]
        ly = lagrange_eval(prob.el.nodes, xi[1])[0]
        lz = lagrange_eval(prob.el.nodes, xi[2])[0]
        w = np.einsum("c,b,a->cba", lz, ly, lx).ravel()      # x fastest
        np.add.at(out, prob.cell_nodes[e], -4.0 * np.pi * z * w)
    assert w.size == n1 ** 3
    return out


def total_potential(prob, rho_quad, Z=(), atom_cell=(), atom_xi=(), boundary=None):
    """phi (nodal, constraints distributed) and its values at the parent
    quadrature points, by a direct sparse solve of the condensed system.
    ``boundary`` [n_nodes] gives values on the Dirichlet rows of the psi
    constraints (zero when None); hanging rows interpolate them."""
    N = prob.el.shape_at_quad()                              # [nq, nd]
    fw = (4.0 * np.pi * np.asarray(rho_quad) * prob.jxw).reshape(prob.n_cells, prob.nq)
    cell_rhs = fw @ N                                        # [nc, nd]
    b = np.zeros(prob.n_nodes)
    np.add.at(b, prob.cell_nodes.ravel(), cell_rhs.ravel())
    if len(Z):
        b += point_charge_rhs(prob, Z, atom_cell, atom_xi)
    C = prob.cons_psi.matrix()
    free = ~prob.cons_psi.is_constrained()
    Cf = C[:, free]
    K = stiffness(prob)
    g = np.zeros(prob.n_nodes)
    if boundary is not None:
        cons = prob.cons_psi
        dirichlet = cons.nodes[np.diff(cons.ptr) == 0]
        g[dirichlet] = np.asarray(boundary)[dirichlet]
        rows = np.repeat(np.arange(cons.n_constrained), np.diff(cons.ptr))
        vals = np.zeros(cons.n_constrained)
        np.add.at(vals, rows, cons.weights * g[cons.masters])
        hanging = np.diff(cons.ptr) > 0
        g[cons.nodes[hanging]] = vals[hanging]
        b = b - K @ g
    A = (Cf.T @ K @ Cf).tocsc()
    phi_f = spla.spsolve(A, Cf.T @ b)
    phi = Cf @ phi_f + g
    phi_q = np.einsum("qi,ci->cq", N, phi[prob.cell_nodes]).ravel()
    return phi, phi_q


def locate_atoms(prob, positions):
    """(cell, reference coordinates) of each position in the parent mesh."""
    cells, xis = [], []
    for R in np.asarray(positions, dtype=np.float64).reshape(-1, 3):
        lo, h = prob.cell_lo, prob.cell_h
        inside = np.all((R[None, :] >= lo - 1e-12) & (R[None, :] <= lo + h[:, None] + 1e-12), axis=1)
        e = int(np.nonzero(inside)[0][0])
        cells.append(e)
        xis.append(np.clip((R - lo[e]) / h[e], 0.0, 1.0))
    return np.asarray(cells, dtype=np.int64), np.asarray(xis)
