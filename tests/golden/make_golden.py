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


def main():
    P = build_problem("tiny_h2")
    params = dict(cheb_degree=30, cheby_tol=1e-10, initial_tol_cheb=1e-10, adjoint_initial_tol=1e-10,
                  adaptive_factor_adjoint=1.0, adjoint_max_iter=2000, max_cheb_passes=60)
    fn = InverseDFTSolverFunction(P, ForceParams(**params))
    pot = P.vxc_init.copy()
    f, L, st = fn.get_force_vector(pot.copy())
    np.savez_compressed(os.path.join(HERE, "tiny_h2_force.npz"), pot=pot, force=f, loss=L,
                        eigenvalues=st.eigenvalues, params=np.array(params, dtype=object),
                        minres_iters=np.array(st.minres_iters), passes=st.passes)
    print("wrote tiny_h2_force.npz", L, st.passes, st.minres_iters)


if __name__ == "__main__":
    main()
