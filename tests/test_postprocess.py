"""POST_PROCESS step (projection of v_xc to the parent mesh, values at points):
known answers for the oracle and the host helpers, on the CPU."""
import numpy as np
import pytest

from conftest import problem


def test_constant_field_projects_exactly():
    """A constant v_xc (and no LDA part) projects to that constant on every
    free node (the lumped GLL mass integrates each basis function exactly) and
    on every hanging node whose weights sum to one; boundary nodes are zero,
    and hanging nodes next to the boundary, whose zero-boundary masters the
    constraint closure removed, interpolate those zeros."""
    from oracle.postprocess import project_vxc_to_parent
    P = problem("small_lih")
    u = project_vxc_to_parent(P, np.full(P.n_child_nodes, -0.37), factor_lda=0.0)
    cons = P.cons_psi
    free = np.ones(P.n_nodes, dtype=bool)
    free[cons.nodes] = False
    assert np.max(np.abs(u[free] + 0.37)) < 1e-12
    nm = np.diff(cons.ptr)
    wsum = np.add.reduceat(cons.weights, cons.ptr[:-1][nm > 0]) if np.any(nm > 0) else np.zeros(0)
    hang = cons.nodes[nm > 0]
    full = np.abs(wsum - 1.0) < 1e-12
    assert full.sum() > 0
    assert np.max(np.abs(u[hang[full]] + 0.37)) < 1e-12
    assert np.all(u[cons.nodes[nm == 0]] == 0.0)


def test_point_evaluation_reproduces_linear_field():
    """The nodal interpolant of a linear function is exact in every cell, so
    evaluating it anywhere returns the function."""
    from invdft_b200.postprocess import locate_points
    from oracle.postprocess import evaluate
    P = problem("small_lih")
    u = P.node_xyz @ np.array([0.3, -1.1, 0.7]) + 0.25
    rng = np.random.default_rng(7)
    lo = P.cell_lo.min(axis=0)
    hi = (P.cell_lo + P.cell_h[:, None]).max(axis=0)
    pts = lo + (hi - lo) * rng.random((500, 3))
    cells, xi = locate_points(P, pts)
    assert np.all((xi >= 0.0) & (xi <= 1.0))
    assert np.max(np.abs(P.cell_lo[cells] + xi * P.cell_h[cells][:, None] - pts)) < 1e-12
    v = evaluate(P, u, cells, xi)
    assert np.max(np.abs(v - (pts @ np.array([0.3, -1.1, 0.7]) + 0.25))) < 1e-11


def test_grid_points_follow_reference_order_and_checks():
    from invdft_b200.postprocess import grid_points
    pts = grid_points((0.0, -1.0, 2.0), (1.0, 1.0, 2.0), (3, 2, 1))
    assert pts.shape == (6, 3)
    # index = ix*(ny*nz) + iy*nz + iz
    assert np.allclose(pts[0], [0.0, -1.0, 2.0]) and np.allclose(pts[1], [0.0, 1.0, 2.0])
    assert np.allclose(pts[2], [0.5, -1.0, 2.0]) and np.allclose(pts[5], [1.0, 1.0, 2.0])
    with pytest.raises(ValueError):
        grid_points((0.0, 0.0, 0.0), (0.0, 1.0, 1.0), (2, 2, 2))
    with pytest.raises(ValueError):
        grid_points((1.0, 0.0, 0.0), (0.0, 1.0, 1.0), (2, 2, 2))


def test_points_file_format(tmp_path):
    from invdft_b200.postprocess import write_points
    pts = np.array([[0.0, 1.0, 2.0], [3.5, -1.25, 0.125]])
    write_points(tmp_path / "v.txt", pts, np.array([-0.5, 0.75]))
    rows = np.loadtxt(tmp_path / "v.txt")
    assert rows.shape == (2, 5)
    assert np.array_equal(rows[:, 0], [0, 1]) and np.array_equal(rows[:, 1:4], pts)
    assert np.array_equal(rows[:, 4], [-0.5, 0.75])


def test_locate_rejects_outside_points():
    from invdft_b200.postprocess import locate_points
    P = problem("tiny_h2")
    hi = (P.cell_lo + P.cell_h[:, None]).max(axis=0)
    with pytest.raises(ValueError):
        locate_points(P, hi[None, :] + 1.0)


def test_postprocess_golden_fixture():
    """The oracle's projection and point values reproduce their committed
    output (tests/golden/make_golden.py), including the reference's point order."""
    import os
    from invdft_b200.postprocess import grid_points, locate_points
    from oracle.postprocess import evaluate, project_vxc_to_parent
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "small_lih_postprocess.npz"))
    P = problem("small_lih")
    u = project_vxc_to_parent(P, g["vxc"], float(g["factor_lda"]))
    assert np.max(np.abs(u - g["parent_nodal"])) < 1e-12 * np.max(np.abs(g["parent_nodal"]))
    lo = P.cell_lo.min(axis=0)
    hi = (P.cell_lo + P.cell_h[:, None]).max(axis=0)
    pts = grid_points(lo + 0.25, hi - 0.25, (9, 7, 5))
    assert np.array_equal(pts, g["points"])
    cells, xi = locate_points(P, pts)
    assert np.max(np.abs(evaluate(P, u, cells, xi) - g["values"])) < 1e-12 * np.max(np.abs(g["values"]))
