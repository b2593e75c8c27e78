"""Row f2: the initial v_xc guess (InverseDFTEngine::setInitialPotL2Proj,
InverseDFTEngine.cpp:1046-1498) on the GPU against the numpy oracle, with LDA
and LB94 exchange, with and without the Fermi-Amaldi far field."""
import numpy as np
import pytest

from conftest import native_params, problem, rel

pytestmark = pytest.mark.gpu


def _sigma_atoms(P):
    """|grad rho|^2 of the superposed Gaussian clouds at the quadrature points."""
    from invdft_b200.problem.system import atom_beta
    g = np.zeros((P.quad_xyz.shape[0], 3))
    for Z, R in zip(P.cfg.Z, P.cfg.pos):
        b = atom_beta(Z)
        d = P.quad_xyz - np.asarray(R)
        g += (-2.0 * b * Z * (b / np.pi) ** 1.5 * np.exp(-b * np.sum(d * d, axis=1)))[:, None] * d
    return np.sum(g * g, axis=1)


@pytest.mark.parametrize("exchange,fa", [("lda", False), ("lda", True), ("lb94", True)])
def test_initial_guess_matches_oracle(exchange, fa):
    from invdft_b200.solver import InverseDFTSolverFunction
    from oracle.initial_guess import hartree_boundary_values, initial_guess
    P = problem("small_lih")
    rho = 2.0 * P.rho_target_up
    sigma = _sigma_atoms(P) if exchange == "lb94" else None
    bc = hartree_boundary_values(P)
    fn = InverseDFTSolverFunction(P, native_params(factor_lda=0.25))
    child, parent, vh = fn.initial_guess(rho, sigma, bc, fermi_amaldi_bc=fa, hartree_rel_tol=1e-14)
    o_child, o_parent, o_vh = initial_guess(P, rho, sigma, bc, fermi_amaldi_bc=fa, factor_lda=0.25)
    assert rel(parent, o_parent) < 1e-10
    assert rel(child, o_child) < 1e-10
    assert np.all(child[P.cons_child.nodes] == 0.0)
    if fa:
        assert rel(vh, o_vh) < 1e-9
    fn.close()


def test_hartree_known_answer_of_gaussian_atoms():
    """v_H of the Gaussian clouds is sum Z erf(sqrt(beta) r)/r; with the
    reference's monopole boundary values the FE solution follows it to 3 %."""
    from invdft_b200.problem.system import rho_atoms, v_hartree_atoms
    from invdft_b200.solver import InverseDFTSolverFunction
    from oracle.initial_guess import hartree_boundary_values
    P = problem("small_lih")
    fn = InverseDFTSolverFunction(P, native_params())
    _, _, vh = fn.initial_guess(rho_atoms(P.cfg, P.quad_xyz), None, hartree_boundary_values(P),
                                fermi_amaldi_bc=True, hartree_rel_tol=1e-13)
    assert rel(vh, v_hartree_atoms(P.cfg, P.quad_xyz)) < 3e-2
    fn.close()
