"""POST_PROCESS step of the reference, restated in numpy -- TEST INFRASTRUCTURE ONLY.

``InverseDFTEngine::projectVxcToParentMesh`` (InverseDFTEngine.cpp:3462-3545)
interpolates the child v_xc to the parent quadrature points, adds
factorForLDAVxc * v_LDA (:3509-3518) and calls DFT-FE's
``l2ProjectionQuadToNodal`` with the psi constraints (:3524-3534), then
distributes them (:3536-3538).  DFT-FE's routine is not in the reference tree;
it is restated here as the L2 projection with the GLL-lumped mass of the psi
space: u = (C^T r) / (C^T m) on free nodes, r_i = sum_e sum_q N_i(q) f(q) JxW(q),
then the constraints distributed.  ``evaluate`` is the Lagrange interpolation of
a parent nodal field at points (the writeToPoints branch, :3275-3456).
"""
from __future__ import annotations

import numpy as np

from invdft_b200.problem.fe import lagrange_eval

from .fe import CellOps, child_to_parent_quad, distribute, distribute_slave_to_master


def project_vxc_to_parent(prob, vxc_child, factor_lda: float) -> np.ndarray:
    ops = CellOps(prob)
    f = child_to_parent_quad(prob, vxc_child) + factor_lda * prob.v_lda
    fw = (f * prob.jxw).reshape(prob.n_cells, prob.nq)
    r = ops.assemble(fw @ ops.N)
    r = distribute_slave_to_master(prob.cons_psi, r)
    m = ops.mass
    u = np.where(m > 0.0, r / np.where(m > 0.0, m, 1.0), 0.0)
    return distribute(prob.cons_psi, u)


def evaluate(prob, u, cells, xi) -> np.ndarray:
    nodes = prob.el.nodes
    xi = np.asarray(xi, dtype=np.float64).reshape(-1, 3)
    lx, ly, lz = (lagrange_eval(nodes, xi[:, d]) for d in range(3))      # [npts, n1] each
    n1 = nodes.size
    basis = (lz[:, :, None, None] * ly[:, None, :, None] * lx[:, None, None, :]).reshape(-1, n1 ** 3)
    return np.sum(basis * np.asarray(u)[prob.cell_nodes[np.asarray(cells)]], axis=1)
