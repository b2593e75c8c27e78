"""Oracle of the initial v_xc guess (test infrastructure only).

``InverseDFTEngine::setInitialPotL2Proj`` (src/InverseDFTEngine.cpp:1046-1498):
exchange (LDA, or LB94 given |grad rho|^2) and PW92 correlation of the total
target density at the parent quadrature points, blended as
v = (1 - p) v_x + p (v_x + v_c), p = rho / (rho + tau_vx) (:1255-1270), with
the optional Fermi-Amaldi far field v = q v - (1 - q) factor_fa / N_e v_H,
q = rho / (rho + tau_fa) (:1272-1289); projected onto the parent nodes and
distributed (:1311-1320), evaluated at the child Gauss points (:1415-1419),
scaled by 1 - factorForLDAVxc (:1421-1427), projected onto the child nodes
(:1429-1433) and zeroed on the child constraints (:1434).  libxc's XC_LDA_X,
XC_LDA_C_PW and XC_GGA_X_LB are not vendored; their published forms are
restated below.  DFT-FE's l2ProjectionQuadToNodal is restated as the
lumped-mass L2 projection, as in oracle/postprocess.py.
"""
from __future__ import annotations

import math

import numpy as np

from .fe import CellOps, distribute, distribute_slave_to_master, integrate_child_shape_functions, \
    parent_to_child_quad, set_zero
from .poisson import total_potential


def lda_exchange(rho):
    """Slater exchange potential of the total density: -(3 rho / pi)^(1/3)."""
    return -np.cbrt(3.0 * np.maximum(rho, 1e-30) / math.pi)


def lb94_exchange(rho, sigma, beta=0.05):
    """van Leeuwen-Baerends 1994 per spin channel of an unpolarised density:
    v_LDA - beta rho_s^(1/3) x^2 / (1 + 3 beta x asinh(x)), x = |grad rho_s| / rho_s^(4/3)."""
    rs = 0.5 * np.maximum(rho, 1e-30)
    gs = 0.5 * np.sqrt(np.maximum(sigma, 0.0))
    x = gs / rs ** (4.0 / 3.0)
    return lda_exchange(rho) - beta * np.cbrt(rs) * x * x / (1.0 + 3.0 * beta * x * np.arcsinh(x))


def pw92_correlation(rho):
    """Perdew-Wang 1992 correlation potential, spin-unpolarised:
    e_c = -2A (1 + a1 rs) ln(1 + 1 / (2A (b1 rs^1/2 + b2 rs + b3 rs^3/2 + b4 rs^2))),
    v_c = e_c - (rs / 3) de_c/drs."""
    A, a1, b1, b2, b3, b4 = 0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294
    rs = np.cbrt(3.0 / (4.0 * math.pi * np.maximum(rho, 1e-30)))
    sr = np.sqrt(rs)
    g0 = -2.0 * A * (1.0 + a1 * rs)
    g1 = 2.0 * A * (b1 * sr + b2 * rs + b3 * rs * sr + b4 * rs * rs)
    g1p = A * (b1 / sr + 2.0 * b2 + 3.0 * b3 * sr + 4.0 * b4 * rs)
    ln = np.log1p(1.0 / g1)
    ec = g0 * ln
    dec = -2.0 * A * a1 * ln - g0 * g1p / (g1 * g1 + g1)
    return ec - rs / 3.0 * dec


def initial_guess(prob, rho_quad, sigma_quad=None, hartree_bc=None, tau_vx=1e-2, tau_fa=1e-2,
                  fermi_amaldi_bc=False, factor_fa=1.0, factor_lda=0.0):
    """Returns (child nodal guess, parent nodal field, v_H at the parent quadrature points)."""
    rho = np.asarray(rho_quad, dtype=np.float64)
    vx = lda_exchange(rho) if sigma_quad is None else lb94_exchange(rho, sigma_quad)
    vc = pw92_correlation(rho)
    p = rho / (rho + tau_vx)
    v = (1.0 - p) * vx + p * (vx + vc)
    vh = np.zeros_like(rho)
    if fermi_amaldi_bc:
        _, vh = total_potential(prob, rho, boundary=hartree_bc)
        q = rho / (rho + tau_fa)
        v = q * v + (1.0 - q) * (-factor_fa / prob.n_electrons) * vh
    ops = CellOps(prob)
    r = ops.assemble((v * prob.jxw).reshape(prob.n_cells, prob.nq) @ ops.N)
    r = distribute_slave_to_master(prob.cons_psi, r)
    m = ops.mass
    parent = distribute(prob.cons_psi, np.where(m > 0.0, r / np.where(m > 0.0, m, 1.0), 0.0))
    cq = parent_to_child_quad(prob, parent[:, None])[:, 0] * (1.0 - factor_lda)
    rc = integrate_child_shape_functions(prob, cq)
    mc = integrate_child_shape_functions(prob, np.ones_like(cq))
    child = set_zero(prob.cons_child, np.where(mc > 0.0, rc / np.where(mc > 0.0, mc, 1.0), 0.0))
    return child, parent, vh


def hartree_boundary_values(prob, net_charge: float = 0.0) -> np.ndarray:
    """Boundary values of computeHartreePotOnParentQuad (InverseDFTEngine.cpp:
    1840-1895): sum over atoms of (Z_a + net_charge / n_atoms) / |x - R_a| at
    every node (only the Dirichlet rows are used)."""
    x = prob.node_xyz
    out = np.zeros(prob.n_nodes)
    for Z, R in zip(prob.cfg.Z, prob.cfg.pos):
        out += (Z + net_charge / len(prob.cfg.Z)) / np.maximum(np.linalg.norm(x - np.asarray(R), axis=1), 1e-12)
    return out
