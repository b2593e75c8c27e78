"""Generate the golden fixtures of tests/golden from the FP64 oracle.

The reference has no golden vectors for this path (no tests, and its demo's
final v_xc outputs are not shipped), so these fixtures pin the oracle's own
output on a small synthetic system; the oracle itself is pinned by the
known-answer tests of tests/test_oracle.py.  Run: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from invdft_b200.problem.system import build_problem  # noqa: E402
from oracle import ForceParams, InverseDFTSolverFunction  # noqa: E402


PARAMS = dict(cheb_degree=30, cheby_tol=1e-10, initial_tol_cheb=1e-10, adjoint_initial_tol=1e-10,
              adaptive_factor_adjoint=1.0, adjoint_max_iter=2000, max_cheb_passes=60)


def force_fixture(name):
    """getForceVector at the initial guess: force, loss, eigenvalues."""
    P = build_problem(name)
    fn = InverseDFTSolverFunction(P, ForceParams(**PARAMS))
    pot = P.vxc_init.copy()
    f, L, st = fn.get_force_vector(pot.copy())
    np.savez_compressed(os.path.join(HERE, f"{name}_force.npz"), pot=pot, force=f, loss=L,
                        eigenvalues=st.eigenvalues, params=np.array(PARAMS, dtype=object),
                        minres_iters=np.array(st.minres_iters), passes=st.passes)
    print(f"wrote {name}_force.npz", L, st.passes, st.minres_iters)


def postprocess_fixture(name, factor_lda=1.0):
    """POST_PROCESS: a seeded v_xc projected to the parent nodes and its values
    on the reference's point grid (index = ix*(ny*nz) + iy*nz + iz)."""
    from invdft_b200.postprocess import grid_points, locate_points
    from oracle.postprocess import evaluate, project_vxc_to_parent
    P = build_problem(name)
    rng = np.random.default_rng(17)
    vxc = P.vxc_init + 0.05 * np.sin(P.child_node_xyz[:, 1]) * rng.random(P.n_child_nodes)
    u = project_vxc_to_parent(P, vxc, factor_lda)
    lo = P.cell_lo.min(axis=0)
    hi = (P.cell_lo + P.cell_h[:, None]).max(axis=0)
    pts = grid_points(lo + 0.25, hi - 0.25, (9, 7, 5))
    cells, xi = locate_points(P, pts)
    vals = evaluate(P, u, cells, xi)
    np.savez_compressed(os.path.join(HERE, f"{name}_postprocess.npz"), vxc=vxc, factor_lda=factor_lda,
                        parent_nodal=u, points=pts, values=vals)
    print(f"wrote {name}_postprocess.npz", float(np.abs(u).max()), float(np.abs(vals).max()))


def main():
    force_fixture("tiny_h2")
    force_fixture("small_lih")
    postprocess_fixture("small_lih")


if __name__ == "__main__":
    main()
