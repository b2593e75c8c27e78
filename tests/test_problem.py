"""Invariants of the synthetic problem generator (CPU)."""
import numpy as np
import pytest

from conftest import problem


def _small_tree():
    from invdft_b200.problem.octree import Octree
    t = Octree(-4.0, 8.0, level0=1)

    def pred(tr):
        c, h = tr.cell_center(), tr.cell_size()
        return (np.linalg.norm(c - 0.3, axis=1) < 2.0 * h) & (h > 0.6)

    t.refine_while(pred)
    t.balance()
    return t


def test_octree_is_two_to_one_balanced():
    t = _small_tree()
    h = t.cell_size()
    c = t.cell_center()
    from invdft_b200.problem.octree import _OFFS26
    for off in _OFFS26:
        # the same-size neighbour region's centre lies in a touching leaf
        # whenever that leaf is coarser; finer ones are checked from their side
        nb = t.locate(c + off[None, :] * h[:, None])
        ok = nb >= 0
        lv, ln = t.level[ok], t.level[nb[ok]]
        assert np.all(lv - ln <= 1)


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_hanging_constraints_reproduce_polynomials(p):
    from invdft_b200.problem.space import FESpace
    from oracle.fe import distribute
    S = FESpace(_small_tree(), p)
    C = S.constraints(None)
    assert C.n_constrained > 0
    x = S.node_xyz
    v = x[:, 0] ** p * x[:, 1] + 0.3 * x[:, 2] ** p - x[:, 0] * x[:, 1] + 1.0
    vd = distribute(C, v.copy())
    assert np.max(np.abs(vd - v)) < 1e-11 * np.max(np.abs(v))
    # closed: no master is constrained, weights of a hanging node sum to one
    cons = C.is_constrained()
    assert not np.any(cons[C.masters])
    sums = np.add.reduceat(C.weights, C.ptr[:-1][np.diff(C.ptr) > 0])
    assert np.allclose(sums, 1.0, atol=1e-12)


def test_problem_arrays_are_consistent():
    P = problem("tiny_h2")
    assert P.cell_nodes.shape == (P.n_cells, P.nd)
    assert P.cell_nodes.min() >= 0 and P.cell_nodes.max() < P.n_nodes
    assert np.all(np.diff(P.child_parent) >= 0)
    assert np.all((P.child_offset >= -1e-12) & (P.child_offset + P.child_scale[:, None] <= 1 + 1e-12))
    assert np.all((P.pq_xi >= 0) & (P.pq_xi <= 1))
    # total child and parent volumes agree
    assert abs(P.child_jxw.sum() - P.jxw.sum()) < 1e-9 * P.jxw.sum()
    # target density integrates to the electron count (Gauss vs lumped normalisation)
    assert abs(2 * np.sum(P.rho_target_up * P.jxw) - P.n_electrons) < 1e-2 * P.n_electrons
    # boundary nodes are Dirichlet in the psi constraints
    cons = P.cons_psi.is_constrained()
    assert np.all(cons[P.extras["space"].on_boundary])


def test_named_workload_sizes():
    from invdft_b200.problem.system import _parent_tree, config
    n0 = _parent_tree(config("c0_lih")).n_cells * 64
    assert 1.2e5 < n0 < 3.5e5          # ~2e5 DoF at p=4
    n1 = _parent_tree(config("c1_c2h4")).n_cells * 125
    assert 1.0e6 < n1 < 2.0e6          # ~1.5e6 DoF at p=5
