"""Known-answer pins of the FP64 oracle (CPU).

The reference ships no golden vectors for this path, so the oracle is pinned
against mathematics: a central finite difference of the loss, the hydrogen
spectrum, MINRES residuals and operator symmetry; and against committed
fixtures of its own earlier output (tests/golden/) to catch regressions.
"""
import os

import numpy as np
import pytest

from conftest import oracle_params, problem, rel

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _fd_setup(name="tiny_h2"):
    from oracle import InverseDFTSolverFunction
    P = problem(name)
    prm = oracle_params(cheb_degree=30, cheby_tol=1e-11, initial_tol_cheb=1e-11, adjoint_initial_tol=1e-11,
                        adjoint_max_iter=3000, max_cheb_passes=80)
    return P, InverseDFTSolverFunction(P, prm)


def _directions(P, k):
    rng = np.random.default_rng(0)
    free = ~P.cons_child.is_constrained()
    c = P.child_node_xyz
    out = []
    for _ in range(k):
        d = np.exp(-np.sum((c - rng.uniform(-1, 1, 3)) ** 2, axis=1) / 2.0) * rng.choice([-1.0, 1.0])
        d[~free] = 0.0
        out.append(d)
    return out


def test_adjoint_gradient_is_exact_with_consistent_projection(monkeypatch):
    """With the null-space component removed in the Lowdin inner product and psi.p
    integrated on the parent quadrature, the adjoint gradient equals the central
    finite difference of L to 1e-6: the oracle's HX, eigensolver, density, rhs,
    MINRES and transfers are exact."""
    import oracle.adjoint as oa
    import oracle.force as of
    from oracle.fe import distribute, distribute_slave_to_master
    P, fn = _fd_setup()
    v = P.vxc_init.copy()
    cap = []
    orig_p2c = of.parent_to_child_quad

    def grab(prob, X, chunk=4096):
        cap.append(X.copy())
        return orig_p2c(prob, X, chunk)

    def dx_exact(self, x):
        X = fn_exact.X[:, :x.shape[1]]
        for i in range(x.shape[1]):
            x[:, i] -= X[:, i] * (X[:, i] @ x[:, i])
        self.eta = 0.0
        return distribute(self.cons, self.ops.inv_sqrt_mass[:, None] * x)

    from oracle import InverseDFTSolverFunction
    fn_exact = InverseDFTSolverFunction(P, fn.params)
    monkeypatch.setattr(of, "parent_to_child_quad", grab)
    monkeypatch.setattr(oa.AdjointProblem, "distribute_x", dx_exact)
    fn_exact.get_force_vector(v.copy())
    monkeypatch.undo()
    psi, p = cap[0], cap[1]
    S = np.sum(fn_exact.ops.to_quad(psi).reshape(-1, psi.shape[1]) * fn_exact.ops.to_quad(p).reshape(-1, p.shape[1]),
               axis=1) * P.jxw
    g = np.zeros(P.n_child_nodes)
    xi, nodes = P.pq_xi, P.child_cell_nodes[P.pq_child]
    for k in range(8):
        w = ((xi[:, 0] if k & 1 else 1 - xi[:, 0]) * (xi[:, 1] if k & 2 else 1 - xi[:, 1])
             * (xi[:, 2] if k & 4 else 1 - xi[:, 2]))
        np.add.at(g, nodes[:, k], w * S)
    g = distribute_slave_to_master(P.cons_child, g)
    h = 1e-4
    for d in _directions(P, 2):
        _, Lp, _ = fn.get_force_vector(v + h * d)
        _, Lm, _ = fn.get_force_vector(v - h * d)
        fd = (Lp - Lm) / (2 * h)
        assert abs(g @ d / fd - 1.0) < 1e-6


def test_reference_force_matches_finite_differences_to_discretisation_error():
    """The reference's own formula (Gauss-quadrature projection in distributeX,
    child-quadrature integration) agrees with FD up to its discretisation error."""
    P, fn = _fd_setup()
    v = P.vxc_init.copy()
    f, L, _ = fn.get_force_vector(v.copy())
    h = 1e-4
    for d in _directions(P, 2):
        _, Lp, _ = fn.get_force_vector(v + h * d)
        _, Lm, _ = fn.get_force_vector(v - h * d)
        fd = (Lp - Lm) / (2 * h)
        assert abs(f @ d / fd - 1.0) < 2e-2


def test_hydrogen_spectrum():
    """Bare -1/r potential, zero v_xc: 1s at -1/2 and the n=2 shell near -1/8."""
    from invdft_b200.problem.system import SystemConfig, build_problem
    from oracle import ForceParams, InverseDFTSolverFunction
    from oracle.force import ForceStats
    cfg = SystemConfig("h_atom", [1], [[0.0, 0.0, 0.0]], 1, 5, 3, 12.0, 0.375, 3.0, 0.6, 0, 1,
                       vxc_domain=0.5, child_level_cap=4)
    P = build_problem(cfg, target_solver="atoms")
    P.v_base = -1.0 / np.maximum(np.linalg.norm(P.quad_xyz, axis=1), 1e-12)
    fn = InverseDFTSolverFunction(P, ForceParams(cheb_degree=0, cheby_tol=1e-7, initial_tol_cheb=1e-7,
                                                 max_cheb_passes=60))
    fn.solve_eigen(np.zeros(P.n_child_nodes), ForceStats())
    assert abs(fn.eig[0] + 0.5) < 5e-3
    assert np.all(np.abs(fn.eig[1:5] + 0.125) < 1e-2)


def test_minres_residual_and_symmetry():
    from oracle.adjoint import minres_solve
    P, fn = _fd_setup()
    fn.get_force_vector(P.vxc_init.copy())
    A = fn.adjoint
    b = A.compute_rhs()
    x, it, ph = minres_solve(A, 1e-11, 2000)
    Ax, _ = A.vmult(x.copy())
    bmax = np.max(np.linalg.norm(b, axis=0))
    # MINRES stops on the D-preconditioned residual (1e-11 absolute); D ~ 0.04..1.2 here
    assert np.max(np.linalg.norm(Ax - b, axis=0)) < 1e-8 * bmax
    rng = np.random.default_rng(1)
    u = rng.standard_normal((P.n_nodes, 1))
    w = rng.standard_normal((P.n_nodes, 1))
    u[~fn.free] = 0
    w[~fn.free] = 0
    assert abs((u.T @ fn.ops.hx(w))[0, 0] - (w.T @ fn.ops.hx(u))[0, 0]) < 1e-10 * abs((u.T @ fn.ops.hx(w))[0, 0])


def test_rhs_is_orthogonal_to_its_own_state():
    """The -2 Mu psi term removes the psi_i component of 4 f_i M^-1/2 R psi_i."""
    P, fn = _fd_setup()
    fn.get_force_vector(P.vxc_init.copy())
    b = fn.adjoint.compute_rhs()
    X = fn.X
    for j in range(b.shape[1]):
        nb = np.linalg.norm(b[:, j])
        if nb > 0:
            assert abs(X[:, j] @ b[:, j]) < 1e-8 * nb


def test_degeneracy_map_groups():
    from oracle.force import evaluate_degeneracy_map
    m = evaluate_degeneracy_map([-1.0, -0.5, -0.4995, -0.499, 0.2], 0.002)
    assert m[0] == [0] and m[4] == [4]
    assert m[1] == m[2] == m[3] == [1, 2, 3]


def test_fermi_level_fills_electrons():
    from oracle.eigen import fermi_energy, partial_occupancy
    e = np.array([-1.0, -0.3, -0.1, 0.05, 0.2])
    mu = fermi_energy(e, 4, 500.0)
    assert abs(2 * partial_occupancy(e, mu, 500.0).sum() - 4) < 1e-9
    assert -0.3 < mu < -0.1


@pytest.mark.parametrize("name", ["tiny_h2", "small_lih"])
def test_golden_fixture(name):
    """The oracle reproduces its committed output (tests/golden/make_golden.py):
    tiny_h2, and small_lih with hanging nodes on its refined mesh."""
    from oracle import ForceParams, InverseDFTSolverFunction
    g = np.load(os.path.join(GOLDEN, f"{name}_force.npz"), allow_pickle=True)
    P = problem(name)
    fn = InverseDFTSolverFunction(P, ForceParams(**{k: g["params"][()][k] for k in g["params"][()]}))
    f, L, st = fn.get_force_vector(g["pot"].copy())
    assert np.max(np.abs(st.eigenvalues - g["eigenvalues"])) < 1e-10
    assert abs(L - float(g["loss"])) < 1e-10 * abs(float(g["loss"]))
    assert rel(f, g["force"]) < 1e-9


def test_poisson_oracle_known_answer():
    """The base-potential oracle (setPotBasePoissonNuclear restated) on neutral
    Gaussian atoms approaches the closed form -sum Z erfc(sqrt(beta) r)/r away
    from the point nuclei."""
    from invdft_b200.problem.system import rho_atoms, v_base_atoms
    from oracle.poisson import locate_atoms, total_potential
    P = problem("small_lih")
    cells, xi = locate_atoms(P, P.cfg.pos)
    phi, phi_q = total_potential(P, rho_atoms(P.cfg, P.quad_xyz), P.cfg.Z, cells, xi)
    r = np.min([np.linalg.norm(P.quad_xyz - np.asarray(a), axis=1) for a in P.cfg.pos], axis=0)
    far = r > 2.0
    assert np.max(np.abs(phi_q[far] - v_base_atoms(P.cfg, P.quad_xyz)[far])) < 2e-2
    assert np.all(phi[P.cons_psi.nodes[np.diff(P.cons_psi.ptr) == 0]] == 0.0)
