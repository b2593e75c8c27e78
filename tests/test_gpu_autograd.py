"""Differentiation form: torch.autograd over the C ABI (GPU).

The forward half (eigensolve -> rho -> L) and the adjoint backward (block
MINRES + projection) are exposed as a torch.autograd.Function.  Its gradient
must equal the force vector of getForceVector (and the oracle's, 1e-10), and
agree with central finite differences of L along smoothed random directions
up to the reference formula's discretisation error (see test_oracle).
"""
import numpy as np
import pytest

from conftest import native_params, oracle_params, problem, rel

pytestmark = pytest.mark.gpu


def smoothed_directions(P, k, seed=0, sigma=1.0):
    """White noise on the v_xc nodes smoothed with a Gaussian of width sigma (bohr)."""
    rng = np.random.default_rng(seed)
    x = P.child_node_xyz
    d2 = np.sum((x[:, None, :] - x[None, :, :]) ** 2, axis=2)
    G = np.exp(-d2 / (2 * sigma * sigma))
    free = ~P.cons_child.is_constrained()
    out = []
    for _ in range(k):
        d = G @ rng.standard_normal(P.n_child_nodes)
        d[~free] = 0.0
        out.append(d / np.linalg.norm(d))
    return out


def _fn(P, **kw):
    from invdft_b200.solver import InverseDFTSolverFunction
    base = dict(cheby_tol=1e-11, initial_tol_cheb=1e-11, max_cheb_passes=80)
    base.update(kw)
    return InverseDFTSolverFunction(P, native_params(**base))


def test_autograd_gradient_is_the_force_vector():
    import torch
    from invdft_b200.autograd import inverse_ks_loss
    from oracle import InverseDFTSolverFunction as Oracle
    P = problem("tiny_h2")
    fn = _fn(P)
    v = torch.tensor(P.vxc_init, dtype=torch.float64, requires_grad=True)
    L = inverse_ks_loss(v, fn)
    L.backward()
    g = v.grad.numpy()
    orc = Oracle(P, oracle_params(cheby_tol=1e-11, initial_tol_cheb=1e-11, max_cheb_passes=80))
    f_o, L_o, _ = orc.get_force_vector(P.vxc_init.copy())
    assert abs(L.item() - L_o) <= 1e-10 * abs(L_o)
    assert rel(g, f_o) < 1e-10
    assert fn.last_backward_stats["device_bytes_peak"] > 0


def test_autograd_matches_finite_differences():
    """p=4 mesh: the reference formula's discretisation error is small enough
    for a 2 % bound (p=2 tiny meshes reach ~5 % on smooth global directions)."""
    import torch
    from invdft_b200.autograd import inverse_ks_loss
    from invdft_b200.problem.system import build_problem
    P = build_problem("tiny_h2_p4", target_solver="atoms")
    fn = _fn(P)
    v0 = torch.tensor(P.vxc_init, dtype=torch.float64, requires_grad=True)
    L = inverse_ks_loss(v0, fn)
    L.backward()
    g = v0.grad.numpy().copy()
    h = 1e-4
    for d in smoothed_directions(P, 8):
        Lp = inverse_ks_loss(torch.tensor(P.vxc_init + h * d), fn).item()
        Lm = inverse_ks_loss(torch.tensor(P.vxc_init - h * d), fn).item()
        fd = (Lp - Lm) / (2 * h)
        # reference-formula discretisation error, scale-aware for directions
        # along which the derivative nearly cancels (|d| = 1)
        assert abs(g @ d - fd) <= 2e-2 * abs(fd) + 1e-3 * np.linalg.norm(g)


def test_backward_refuses_a_stale_forward():
    import torch
    from invdft_b200.autograd import inverse_ks_loss
    P = problem("tiny_h2")
    fn = _fn(P)
    v = torch.tensor(P.vxc_init, dtype=torch.float64, requires_grad=True)
    L1 = inverse_ks_loss(v, fn)
    inverse_ks_loss(torch.tensor(P.vxc_init * 1.01), fn)   # another forward on the same context
    with pytest.raises(RuntimeError):
        L1.backward()


def test_library_refuses_backward_after_state_changes():
    """The C ABI itself refuses (NOT_READY) a backward whose forward is no
    longer the context's state: after a getForceVector at another v_xc, and
    after set_potential, whichever Python object holds the forward."""
    import ctypes as C
    from invdft_b200.native import Stats, ptr
    P = problem("tiny_h2")
    fn = _fn(P)
    lib = fn.lib
    st = Stats()
    pot = P.vxc_init.copy()
    assert lib.invdft_solve_eigen(fn.ctx, ptr(pot), C.byref(st)) == 0
    gen = int(st.generation)
    force = np.zeros(P.n_child_nodes)
    assert lib.invdft_force_backward_at(fn.ctx, gen, ptr(force), C.byref(Stats())) == 0
    fn.get_force_vector(P.vxc_init * 1.01)                 # a later forward half
    assert lib.invdft_force_backward_at(fn.ctx, gen, ptr(force), C.byref(Stats())) == 7
    assert lib.invdft_solve_eigen(fn.ctx, ptr(P.vxc_init.copy()), C.byref(st)) == 0
    fn.set_potential(P.vxc_init * 0.99)                     # the Hamiltonian changed
    assert lib.invdft_force_backward(fn.ctx, ptr(force), C.byref(Stats())) == 7
    assert lib.invdft_force_backward_at(fn.ctx, int(st.generation), ptr(force), C.byref(Stats())) == 7
