"""The C++/OpenMP restatement of the oracle (oracle/cpu) against the numpy oracle (CPU).

The C++ port serves as the fast checker on the large meshes and as the timed
CPU baseline of the benchmark, so it is itself pinned to the numpy oracle here:
the Lowdin HX on odd and even orders (the even ones take its even-odd path),
and whole getForceVector calls (eigenvalue pass counts, MINRES iteration
counts, loss and force) including the warm-started second call.
"""
import numpy as np
import pytest

from conftest import oracle_params, problem, rel

KNOBS = dict(cheb_degree=30, cheby_tol=1e-10, initial_tol_cheb=1e-10, adjoint_initial_tol=1e-10,
             adaptive_factor_adjoint=1.0, adjoint_max_iter=2000, max_cheb_passes=60, lanczos_steps=20)


@pytest.mark.parametrize("name,target", [("tiny_h2", None), ("small_lih", None), ("tiny_h2_p5", "atoms"),
                                         ("tiny_h2_p4", "atoms")])
def test_cpu_hx_matches_numpy_oracle(name, target):
    from invdft_b200.problem.system import build_problem
    from oracle import InverseDFTSolverFunction as Oracle
    from oracle.cpu import CpuForce
    from oracle.fe import child_to_parent_quad
    P = problem(name) if target is None else build_problem(name, target_solver=target)
    orc = Oracle(P, oracle_params())
    cpu = CpuForce(P, **KNOBS)
    pot = P.vxc_init.copy()
    cpu.set_potential(pot)
    orc.ops.cell_hamiltonians(P.v_base + child_to_parent_quad(P, pot))
    rng = np.random.default_rng(7)
    for B in (1, 3, 9):
        x = rng.standard_normal((P.n_nodes, B))
        x[~orc.free] = 0.0
        assert rel(cpu.hx(x), orc.ops.hx(x)) < 1e-13, B


@pytest.mark.parametrize("name", ["tiny_h2", "small_lih"])
def test_cpu_force_matches_numpy_oracle(name):
    from oracle import InverseDFTSolverFunction as Oracle
    from oracle.cpu import CpuForce
    P = problem(name)
    orc = Oracle(P, oracle_params())
    cpu = CpuForce(P, **KNOBS)
    for k in range(2):
        pot = P.vxc_init + 0.01 * k * np.sin(P.child_node_xyz[:, 0])
        f_c, L_c, st = cpu.get_force_vector(pot.copy())
        f_o, L_o, ost = orc.get_force_vector(pot.copy())
        assert st["passes"] == ost.passes
        assert st["minres_iters_max"] == max(ost.minres_iters)
        assert abs(L_c - L_o) <= 1e-10 * abs(L_o)
        assert rel(f_c, f_o) < 1e-9
        e, _, mu = cpu.eigen()
        assert np.max(np.abs(e - ost.eigenvalues)) < 1e-10
        assert np.all(f_c[P.cons_child.nodes] == 0.0)


def test_cpu_state_hand_over_repeats_the_next_evaluation():
    """Given the numpy oracle's state after one evaluation (eigenvectors, Ritz
    values, counter, loss and tolerances), the C++ port's next evaluation is
    the oracle's next one: same passes, MINRES counts, loss and force."""
    from oracle import InverseDFTSolverFunction as Oracle
    from oracle.cpu import CpuForce
    P = problem("small_lih")
    orc = Oracle(P, oracle_params())
    _, L0, s0 = orc.get_force_vector(P.vxc_init.copy())
    cpu = CpuForce(P, **KNOBS)
    cpu.set_state(orc.psi, orc.eig, orc.counter, L0, orc.tol_cheb, orc.adjoint_tol)
    pot = P.vxc_init + 0.01 * np.sin(P.child_node_xyz[:, 0])
    f_o, L_o, ost = orc.get_force_vector(pot.copy())
    f_c, L_c, st = cpu.get_force_vector(pot.copy())
    assert st["passes"] == ost.passes
    assert st["minres_iters_max"] == max(ost.minres_iters)
    assert abs(L_c - L_o) <= 1e-10 * abs(L_o)
    assert rel(f_c, f_o) < 1e-9


def test_cpu_defaults_are_the_library_defaults():
    """The checker and the library start from the same reference defaults."""
    from invdft_b200 import native
    from oracle.cpu import params
    a, b = params(), native.default_params()
    for name, _ in a._fields_:
        assert getattr(a, name) == getattr(b, name), name
