"""GPU parity of the POST_PROCESS step through the C ABI: the projection of
v_xc to the parent mesh and the parent field at points, against the oracle."""
import numpy as np
import pytest

from conftest import native_params, problem, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["small_lih", "tiny_h2_p5"])
def test_projection_and_points_match_oracle(name):
    from invdft_b200.postprocess import grid_points, locate_points
    from invdft_b200.solver import InverseDFTSolverFunction
    from oracle.postprocess import evaluate, project_vxc_to_parent
    if name == "small_lih":
        P = problem(name)
    else:
        from invdft_b200.problem.system import build_problem
        P = build_problem(name, target_solver="atoms")
    fn = InverseDFTSolverFunction(P, native_params())
    rng = np.random.default_rng(11)
    vxc = P.vxc_init + 0.05 * np.sin(P.child_node_xyz[:, 0]) * rng.random(P.n_child_nodes)
    u_g = fn.project_vxc_to_parent(vxc)
    u_o = project_vxc_to_parent(P, vxc, fn.params.factor_lda)
    assert rel(u_g, u_o) < 1e-12
    lo = P.cell_lo.min(axis=0)
    hi = (P.cell_lo + P.cell_h[:, None]).max(axis=0)
    pts = grid_points(lo + 0.1, hi - 0.1, (7, 6, 5))
    cells, xi = locate_points(P, pts)
    v_g = fn.evaluate_parent_field(u_g, cells, xi)
    assert rel(v_g, evaluate(P, u_g, cells, xi)) < 1e-12
    # the projection leaves the force path's state alone: this context's first
    # force evaluation equals a fresh context's, bit for bit
    f1, L1, _ = fn.get_force_vector(P.vxc_init.copy())
    fresh = InverseDFTSolverFunction(P, native_params())
    f2, L2, _ = fresh.get_force_vector(P.vxc_init.copy())
    assert L1 == L2 and np.array_equal(f1, f2)
    fn.close()
    fresh.close()
