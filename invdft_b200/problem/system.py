"""Synthetic inverse-DFT problems: the inputs of ``InverseDFTSolverFunction::reinit``.

The reference receives from ``InverseDFTEngine::run`` (InverseDFTEngine.cpp:3555-3705):
the target density rho* at the parent quadrature points, the loss weights
w = 1/(rho*^a1 + tau) + rho*^a2 (:3663-3675), the base potential
v_base = nuclear + Hartree (:2459-2571), the child (v_xc) mesh with its
hanging-node constraints (:207-380), the psi constraints (hanging + zero
boundary) and the adjoint constraints (hanging + rho* < tol, :1502-1573).
None of the reference's own inputs (DFT-FE ground states, Gaussian density
matrices) exist here, so this module manufactures them:

* neutral atoms with Gaussian electron clouds, whose nuclear + Hartree
  potential is -Z erfc(sqrt(beta) r)/r in closed form;
* v_xc* = LDA(rho0) + a seeded sum of Gaussians, held as a Q1 field on the
  child mesh so that the exact answer lies in the discrete space;
* rho* from a forward Kohn-Sham solve with v_base + v_xc* (a callback; the
  dense solver here is for small problems);
* the initial guess is the Fermi-Amaldi potential -v_H[rho0]/N_e.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
from scipy import special

from .fe import Element1D, GAUSS2, lagrange_eval
from .octree import Octree
from .space import Constraints, FESpace

C_KB = 3.166811429e-06  # Boltzmann constant in Ha/K (DFT-FE's C_kb)


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
@dataclass
class SystemConfig:
    name: str
    Z: list
    pos: list
    n_electrons: int
    n_states: int
    p: int
    half_width: float
    h_min: float
    h_max: float
    slope: float
    n_gauss: int
    seed: int
    temperature: float = 500.0
    vxc_domain: float = 6.0          # VXC MESH DOMAIN SIZE
    gauss_ball: float = 3.0
    gauss_sigma: float = 1.0
    gauss_amp: float = 0.05
    rho_tol_constraints: float = 1e-6
    alpha1: float = 0.0
    alpha2: float = 0.0
    tau: float = 1e-2
    unit_weights: bool = False
    child_level_cap: int = 99         # limit on child refinement (tests)
    padding: float | None = None      # cube half-width = extent + padding
    child_extra_levels: int = 0       # refine the child mesh below the parent's minimum size


def _ethylene():
    cc, ch, ang = 2.53, 2.05, math.radians(117.0)
    c1 = np.array([-cc / 2, 0, 0.0])
    c2 = np.array([cc / 2, 0, 0.0])
    h = []
    for c, s in ((c1, -1.0), (c2, 1.0)):
        for t in (+1.0, -1.0):
            d = np.array([s * math.cos(ang / 2), t * math.sin(ang / 2), 0.0])
            h.append(c + ch * d)
    return [6, 6, 1, 1, 1, 1], [c1, c2] + h


def _water():
    r, ang = 1.81, math.radians(104.5)
    o = np.zeros(3)
    h1 = r * np.array([math.sin(ang / 2), 0.0, math.cos(ang / 2)])
    h2 = r * np.array([-math.sin(ang / 2), 0.0, math.cos(ang / 2)])
    return [8, 1, 1], [o, h1, h2]


def _octane():
    cc, chb = 2.91, 2.06
    tet = math.radians(109.47)
    half = (math.pi - tet) / 2.0
    Z, P = [], []
    cs = []
    for n in range(8):
        x = n * cc * math.cos(half)
        y = (0.5 if n % 2 else -0.5) * cc * math.sin(half)
        cs.append(np.array([x, y, 0.0]))
    for n, c in enumerate(cs):
        Z.append(6)
        P.append(c)
    for n, c in enumerate(cs):
        out = np.array([0.0, 1.0 if n % 2 else -1.0, 0.0])
        zdir = np.array([0.0, 0.0, 1.0])
        nh = 3 if n in (0, 7) else 2
        dirs = [out * math.cos(tet / 2) + zdir * math.sin(tet / 2),
                out * math.cos(tet / 2) - zdir * math.sin(tet / 2)]
        if nh == 3:
            ax = np.array([-1.0 if n == 0 else 1.0, 0.0, 0.0])
            dirs.append(ax)
        for d in dirs[:nh]:
            d = d / np.linalg.norm(d)
            Z.append(1)
            P.append(c + chb * d)
    ctr = np.mean(cs, axis=0)
    return Z, [p - ctr for p in P]


def config(name: str, **overrides) -> SystemConfig:
    """Named workloads: c0..c4 and small test systems (fields overridable)."""
    import dataclasses
    return dataclasses.replace(_config(name), **overrides) if overrides else _config(name)


def _config(name: str) -> SystemConfig:
    if name == "c0_lih":
        return SystemConfig("c0_lih", [3, 1], [[0, 0, 0], [0, 0, 3.0]], 4, 6, 4,
                            15.0, 0.25, 4.0, 0.5, 6, 1000)
    if name in ("c1_c2h4", "c2_c2h4"):
        Z, P = _ethylene()
        return SystemConfig(name, Z, [list(p) for p in P], 16, 16, 5, 20.0, 0.32, 2.5,
                            0.35, 10, 1001 if name == "c1_c2h4" else 1002)
    if name == "c3_h2o":
        Z, P = _water()
        return SystemConfig("c3_h2o", Z, [list(p) for p in P], 10, 9, 4, 15.0, 0.2, 2.0,
                            0.3, 6, 1003, unit_weights=True)
    if name == "c4_c8h18":
        Z, P = _octane()
        return SystemConfig("c4_c8h18", Z, [list(p) for p in P], 66, 50, 5, 0.0, 0.32, 2.6,
                            0.35, 12, 1004, padding=15.0)
    if name == "tiny_h2":
        return SystemConfig("tiny_h2", [1, 1], [[-0.7, 0, 0], [0.7, 0, 0]], 2, 4, 2,
                            6.0, 0.75, 3.0, 0.6, 4, 7, vxc_domain=0.5, child_level_cap=6,
                            child_extra_levels=1)
    if name == "small_lih":
        return SystemConfig("small_lih", [3, 1], [[0, 0, 0], [0, 0, 3.0]], 4, 6, 2,
                            8.0, 0.5, 4.0, 0.7, 6, 1000, vxc_domain=1.0, child_level_cap=6)
    if name in ("tiny_h2_p4", "tiny_h2_p5"):
        return SystemConfig(name, [1, 1], [[-0.7, 0, 0], [0.7, 0, 0]], 2, 4, int(name[-1]),
                            6.0, 0.75, 3.0, 0.6, 4, 7, vxc_domain=1.0, child_level_cap=6,
                            child_extra_levels=1)
    if name == "small_lih_p4":
        return SystemConfig("small_lih_p4", [3, 1], [[0, 0, 0], [0, 0, 3.0]], 4, 6, 4,
                            10.0, 0.625, 2.5, 0.5, 6, 1000, vxc_domain=3.0)
    raise KeyError(name)


# ---------------------------------------------------------------------------
# analytic potentials
# ---------------------------------------------------------------------------
def atom_beta(Z: int) -> float:
    """Exponent of the Gaussian electron cloud of a neutral atom."""
    return 0.5 * math.sqrt(Z)


def rho_atoms(cfg: SystemConfig, x: np.ndarray) -> np.ndarray:
    r = np.zeros(x.shape[0])
    for Z, P in zip(cfg.Z, cfg.pos):
        b = atom_beta(Z)
        d2 = np.sum((x - np.asarray(P)) ** 2, axis=1)
        r += Z * (b / math.pi) ** 1.5 * np.exp(-b * d2)
    return r


def _erf_over_r(b: float, r: np.ndarray) -> np.ndarray:
    s = math.sqrt(b)
    small = r < 1e-8
    out = np.empty_like(r)
    out[~small] = special.erf(s * r[~small]) / r[~small]
    out[small] = 2.0 * s / math.sqrt(math.pi)
    return out


def v_hartree_atoms(cfg: SystemConfig, x: np.ndarray) -> np.ndarray:
    v = np.zeros(x.shape[0])
    for Z, P in zip(cfg.Z, cfg.pos):
        r = np.linalg.norm(x - np.asarray(P), axis=1)
        v += Z * _erf_over_r(atom_beta(Z), r)
    return v


def v_base_atoms(cfg: SystemConfig, x: np.ndarray) -> np.ndarray:
    """Nuclear + Hartree of neutral Gaussian atoms: sum -Z erfc(sqrt(b) r)/r."""
    v = np.zeros(x.shape[0])
    for Z, P in zip(cfg.Z, cfg.pos):
        r = np.maximum(np.linalg.norm(x - np.asarray(P), axis=1), 1e-12)
        v += -Z * special.erfc(math.sqrt(atom_beta(Z)) * r) / r
    return v


def v_lda(rho: np.ndarray) -> np.ndarray:
    """Spin-unpolarised LDA: Slater exchange + Perdew-Wang 1992 correlation."""
    rho = np.maximum(rho, 1e-30)
    vx = -((3.0 / math.pi) * rho) ** (1.0 / 3.0)
    rs = (3.0 / (4.0 * math.pi * rho)) ** (1.0 / 3.0)
    A, a1, b1, b2, b3, b4 = 0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294
    sr = np.sqrt(rs)
    Q0 = -2.0 * A * (1.0 + a1 * rs)
    Q1 = 2.0 * A * (b1 * sr + b2 * rs + b3 * rs * sr + b4 * rs * rs)
    Q1p = A * (b1 / sr + 2.0 * b2 + 3.0 * b3 * sr + 4.0 * b4 * rs)
    lg = np.log1p(1.0 / Q1)
    ec = Q0 * lg
    dec = -2.0 * A * a1 * lg - Q0 * Q1p / (Q1 * Q1 + Q1)
    vc = ec - rs / 3.0 * dec
    return vx + vc


# ---------------------------------------------------------------------------
# problem container
# ---------------------------------------------------------------------------
@dataclass
class Problem:
    cfg: SystemConfig
    # parent space
    p: int
    n1: int
    nd: int
    n_cells: int
    n_nodes: int
    cell_nodes: np.ndarray      # [n_c, nd] int64
    cell_h: np.ndarray          # [n_c]
    cell_lo: np.ndarray         # [n_c, 3]
    node_xyz: np.ndarray        # [n_nodes, 3]
    cons_psi: Constraints       # hanging + zero boundary
    cons_adj: Constraints       # hanging + rho* < tol
    el: Element1D
    # quadrature on parent cells: [n_c * n_q], x fastest within a cell
    nq: int
    quad_xyz: np.ndarray
    jxw: np.ndarray
    v_base: np.ndarray          # nuclear + Hartree at parent quad
    v_lda: np.ndarray           # LDA(rho*) at parent quad (scaled by factorForLDAVxc)
    rho_target_up: np.ndarray   # rho*/2 at parent quad (spin-up of an unpolarised target)
    weight: np.ndarray          # loss weights at parent quad
    rho_target_nodal: np.ndarray
    # child (Q1 v_xc) space
    n_child_cells: int
    n_child_nodes: int
    child_cell_nodes: np.ndarray  # [n_cc, 8]
    child_cell_h: np.ndarray
    child_cell_lo: np.ndarray
    child_node_xyz: np.ndarray
    cons_child: Constraints       # hanging only
    child_parent: np.ndarray      # [n_cc] parent cell of each child cell
    child_offset: np.ndarray      # [n_cc, 3] child lo in parent reference coords
    child_scale: np.ndarray       # [n_cc] child size / parent size
    child_jxw: np.ndarray         # [n_cc * 8]
    pq_child: np.ndarray          # [n_c*n_q] child cell containing each parent quad pt
    pq_xi: np.ndarray             # [n_c*n_q, 3] its coordinates in that child cell
    # physics
    n_electrons: int
    n_states: int
    temperature: float
    vxc_exact: np.ndarray         # v_xc* on child nodes
    vxc_init: np.ndarray          # initial guess on child nodes
    extras: dict = field(default_factory=dict)

    def summary(self) -> dict:
        return dict(name=self.cfg.name, p=self.p, n_cells=self.n_cells, n_dofs=self.n_nodes,
                    n_constrained_psi=self.cons_psi.n_constrained,
                    n_constrained_adjoint=self.cons_adj.n_constrained,
                    n_child_cells=self.n_child_cells, n_child_nodes=self.n_child_nodes,
                    n_child_hanging=self.cons_child.n_constrained,
                    n_states=self.n_states, n_electrons=self.n_electrons)


def _parent_tree(cfg: SystemConfig) -> Octree:
    pos = np.asarray(cfg.pos, dtype=np.float64)
    if cfg.padding is not None:
        half = float(np.max(np.abs(pos)) + cfg.padding)
        # round to a size whose dyadic levels hit h_min
        lev = math.ceil(math.log2(2 * half / cfg.h_min))
        size = cfg.h_min * 2 ** lev
        lo = -size / 2
    else:
        size = 2 * cfg.half_width
        lo = -cfg.half_width
    tree = Octree(lo, size, level0=1)

    def pred(t: Octree):
        h = t.cell_size()
        clo = t.cell_lo()
        d = np.full(t.n_cells, np.inf)
        for P in pos:
            q = np.clip(P[None, :], clo, clo + h[:, None])
            d = np.minimum(d, np.linalg.norm(q - P[None, :], axis=1))
        target = np.minimum(cfg.h_max, cfg.h_min + cfg.slope * d)
        return h > target * (1 + 1e-9)

    tree.refine_while(pred)
    tree.balance()
    return tree


def _child_tree(cfg: SystemConfig, parent: Octree) -> Octree:
    """Copy of the parent mesh refined inside the atoms' box +- vxc_domain.

    Rule of TriangulationManagerVxc.cpp:143-181: refine cells whose centre lies
    in the box until their size reaches the minimum cell size.
    """
    pos = np.asarray(cfg.pos, dtype=np.float64)
    lo = pos.min(axis=0) - cfg.vxc_domain
    hi = pos.max(axis=0) + cfg.vxc_domain
    t = parent.copy()
    hmin = float(parent.cell_size().min()) / 2 ** cfg.child_extra_levels
    cap = cfg.child_level_cap

    def pred(tr: Octree):
        c = tr.cell_center()
        inside = np.all((c >= lo) & (c <= hi), axis=1)
        return inside & (tr.cell_size() > hmin + 1e-4) & (tr.level < cap)

    t.refine_while(pred)
    t.balance()
    return t


def build_problem(cfg: SystemConfig | str, target_solver=None, vxc_target=None) -> Problem:
    """Build every input of the force evaluation for ``cfg``.

    ``target_solver(problem, v_ks_quad) -> (psi_nodal [n_nodes, N], eig [N],
    occ [N])`` produces the forward ground state used for rho*; by default a
    dense eigensolve (small problems only).  ``target_solver="atoms"`` takes
    rho* = the superposition of the atomic clouds instead (no forward solve;
    the target is then not exactly reachable, which parity checks do not need).
    """
    if isinstance(cfg, str):
        cfg = config(cfg)
    rng = np.random.default_rng(cfg.seed)
    ptree = _parent_tree(cfg)
    S = FESpace(ptree, cfg.p)
    el = S.el
    nq = el.n1 ** 3
    ref_q = el.quad_points3()
    wq = el.quad_weights()
    quad_xyz = (S.cell_lo[:, None, :] + S.cell_h[:, None, None] * ref_q[None, :, :]).reshape(-1, 3)
    jxw = (S.cell_h[:, None] ** 3 * wq[None, :]).ravel()
    cons_psi = S.constraints(S.on_boundary)

    # child mesh
    ctree = _child_tree(cfg, ptree)
    CS = FESpace(ctree, 1)
    cons_child = CS.constraints(None)
    child_parent = ctree.ancestor_in(ptree)
    child_offset = (CS.cell_lo - S.cell_lo[child_parent]) / S.cell_h[child_parent][:, None]
    child_scale = CS.cell_h / S.cell_h[child_parent]
    g2 = GAUSS2[0]
    q8 = np.stack([g2[np.arange(8) % 2], g2[(np.arange(8) // 2) % 2], g2[np.arange(8) // 4]], axis=1)
    child_jxw = (CS.cell_h[:, None] ** 3 * np.full(8, 0.125)[None, :]).ravel()
    pq_child = ctree.locate(quad_xyz)
    if np.any(pq_child < 0):
        raise RuntimeError("parent quadrature point outside the child mesh")
    pq_xi = (quad_xyz - CS.cell_lo[pq_child]) / CS.cell_h[pq_child][:, None]
    pq_xi = np.clip(pq_xi, 0.0, 1.0)

    # potentials
    pos = np.asarray(cfg.pos, dtype=np.float64)
    v_base = v_base_atoms(cfg, quad_xyz)
    xc = CS.node_xyz
    rho0_child = rho_atoms(cfg, xc)
    centre = 0.5 * (pos.min(axis=0) + pos.max(axis=0))
    vxc_exact = v_lda(rho0_child)
    gauss = []
    for _ in range(cfg.n_gauss):
        amp = rng.uniform(-cfg.gauss_amp, cfg.gauss_amp)
        while True:
            c = rng.uniform(-cfg.gauss_ball, cfg.gauss_ball, size=3)
            if np.linalg.norm(c) <= cfg.gauss_ball:
                break
        gauss.append((amp, centre + c))
        vxc_exact += amp * np.exp(-np.sum((xc - centre - c) ** 2, axis=1) / (2 * cfg.gauss_sigma ** 2))
    if vxc_target is not None:
        vxc_exact = np.asarray(vxc_target, dtype=np.float64)
    vxc_init = -v_hartree_atoms(cfg, xc) / cfg.n_electrons

    prob = Problem(
        cfg=cfg, p=cfg.p, n1=el.n1, nd=S.nd, n_cells=ptree.n_cells, n_nodes=S.n_nodes,
        cell_nodes=S.cell_nodes, cell_h=S.cell_h, cell_lo=S.cell_lo, node_xyz=S.node_xyz,
        cons_psi=cons_psi, cons_adj=cons_psi, el=el, nq=nq, quad_xyz=quad_xyz, jxw=jxw,
        v_base=v_base, v_lda=np.zeros_like(v_base), rho_target_up=np.zeros_like(v_base),
        weight=np.ones_like(v_base), rho_target_nodal=np.zeros(S.n_nodes),
        n_child_cells=ctree.n_cells, n_child_nodes=CS.n_nodes, child_cell_nodes=CS.cell_nodes,
        child_cell_h=CS.cell_h, child_cell_lo=CS.cell_lo, child_node_xyz=CS.node_xyz,
        cons_child=cons_child, child_parent=child_parent, child_offset=child_offset,
        child_scale=child_scale, child_jxw=child_jxw, pq_child=pq_child, pq_xi=pq_xi,
        n_electrons=cfg.n_electrons, n_states=cfg.n_states, temperature=cfg.temperature,
        vxc_exact=vxc_exact, vxc_init=vxc_init,
        extras=dict(gaussians=gauss, child_quad_ref=q8, space=S, child_space=CS,
                    parent_tree=ptree, child_tree=ctree))

    # forward solve for the target density
    if isinstance(target_solver, str) and target_solver == "atoms":
        set_target_density(prob, rho_atoms(cfg, quad_xyz), rho_atoms(cfg, S.node_xyz))
        return prob
    v_ks = v_base + interpolate_child_to_parent_quad(prob, vxc_exact)
    if target_solver is None:
        target_solver = dense_ground_state
    psi, eig, occ = target_solver(prob, v_ks)
    set_target(prob, psi, occ)
    prob.extras["target_eigenvalues"] = np.asarray(eig)
    prob.extras["target_occupancy"] = np.asarray(occ)
    return prob


def set_target(prob: Problem, psi_nodal: np.ndarray, occ: np.ndarray):
    """rho*, loss weights and adjoint constraints from a forward ground state."""
    rho_q = density_at_quad(prob, psi_nodal, occ)
    rho_n = 2.0 * np.sum(np.asarray(occ)[None, :] * psi_nodal ** 2, axis=1)
    set_target_density(prob, rho_q, rho_n)


def set_target_density(prob: Problem, rho_q: np.ndarray, rho_n: np.ndarray):
    """Install a total target density given at the quad points and the nodes."""
    cfg = prob.cfg
    prob.rho_target_up = 0.5 * rho_q
    prob.rho_target_nodal = rho_n
    if cfg.unit_weights:
        prob.weight = np.ones_like(rho_q)
    else:
        r = rho_q  # spinFactor * rho_up
        prob.weight = 1.0 / (r ** cfg.alpha1 + cfg.tau) + r ** cfg.alpha2
    S = prob.extras["space"]
    low = prob.rho_target_nodal < cfg.rho_tol_constraints
    prob.cons_adj = S.constraints(low)
    prob.v_lda = v_lda(rho_q)


# ---------------------------------------------------------------------------
# small host helpers shared by setup (not the hot path)
# ---------------------------------------------------------------------------
def interpolate_child_to_parent_quad(prob: Problem, v_child: np.ndarray) -> np.ndarray:
    """Q1 child field (hanging nodes distributed first) at the parent quad points."""
    v = distribute(prob.cons_child, np.asarray(v_child, dtype=np.float64).copy())
    xi = prob.pq_xi
    nodes = prob.child_cell_nodes[prob.pq_child]  # [nQ, 8]
    out = np.zeros(xi.shape[0])
    for k in range(8):
        wx = xi[:, 0] if (k & 1) else 1.0 - xi[:, 0]
        wy = xi[:, 1] if (k & 2) else 1.0 - xi[:, 1]
        wz = xi[:, 2] if (k & 4) else 1.0 - xi[:, 2]
        out += wx * wy * wz * v[nodes[:, k]]
    return out


def distribute(cons: Constraints, x: np.ndarray) -> np.ndarray:
    """x[slave] = sum w x[master]; Dirichlet entries set to zero (in place)."""
    cnt = np.diff(cons.ptr)
    rows = np.repeat(np.arange(cons.n_constrained), cnt)
    if x.ndim == 1:
        val = np.zeros(cons.n_constrained)
        np.add.at(val, rows, cons.weights * x[cons.masters])
    else:
        val = np.zeros((cons.n_constrained,) + x.shape[1:])
        np.add.at(val, rows, cons.weights[:, None] * x[cons.masters])
    x[cons.nodes] = val
    return x


def density_at_quad(prob: Problem, psi_nodal: np.ndarray, occ: np.ndarray) -> np.ndarray:
    """rho(q) = 2 sum_i f_i psi_i(q)^2 (spin-unpolarised total density)."""
    N = prob.el.shape_at_quad()  # [nq, nd]
    out = np.empty(prob.n_cells * prob.nq)
    occ = np.asarray(occ)
    step = 2048
    for s in range(0, prob.n_cells, step):
        e = min(prob.n_cells, s + step)
        U = psi_nodal[prob.cell_nodes[s:e]]              # [c, nd, Ns]
        Q = np.einsum("qi,cin->cqn", N, U, optimize=True)
        out[s * prob.nq:e * prob.nq] = (2.0 * np.sum(occ[None, None, :] * Q * Q, axis=2)).ravel()
    return out


def fermi_occupancy(eig, mu, T):
    kT = C_KB * T
    x = (np.asarray(eig) - mu) / kT
    return np.where(x >= 0, np.exp(-np.abs(x)) / (1 + np.exp(-np.abs(x))), 1.0 / (1 + np.exp(-np.abs(x))))


def fermi_level(eig, n_electrons, T):
    eig = np.asarray(eig)
    lo, hi = eig.min() - 1.0, eig.max() + 1.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        n = 2.0 * np.sum(fermi_occupancy(eig, mid, T))
        if n > n_electrons:
            hi = mid
        else:
            lo = mid
    return 0.5 * (lo + hi)


def dense_ground_state(prob: Problem, v_ks: np.ndarray):
    """Lowest states of the Lowdin-orthonormalised Hamiltonian by dense eigh."""
    import scipy.linalg as sla
    import scipy.sparse as sp
    el = prob.el
    Kref = el.stiffness_ref()
    Nq = el.shape_at_quad()
    n = prob.n_nodes
    rows, cols, vals = [], [], []
    mass = np.zeros(n)
    wg = el.gll_weights3()
    for e in range(prob.n_cells):
        h = prob.cell_h[e]
        vq = v_ks[e * prob.nq:(e + 1) * prob.nq] * prob.jxw[e * prob.nq:(e + 1) * prob.nq]
        He = 0.5 * h * Kref + Nq.T @ (vq[:, None] * Nq)
        idx = prob.cell_nodes[e]
        rows.append(np.repeat(idx, prob.nd))
        cols.append(np.tile(idx, prob.nd))
        vals.append(He.ravel())
        np.add.at(mass, idx, h ** 3 * wg)
    H = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    C = prob.cons_psi.matrix()
    free = ~prob.cons_psi.is_constrained()
    Cf = C[:, free]
    Hc = (Cf.T @ H @ Cf).toarray()
    Mc = Cf.T @ mass
    if Hc.shape[0] > 12000:
        raise ValueError("dense forward solve is for small problems; pass target_solver")
    s = 1.0 / np.sqrt(Mc)
    Ht = s[:, None] * Hc * s[None, :]
    Ht = 0.5 * (Ht + Ht.T)
    w, V = sla.eigh(Ht, subset_by_index=[0, prob.n_states - 1])
    X = np.zeros((n, prob.n_states))
    X[free] = s[:, None] * V
    X = distribute(prob.cons_psi, X)
    mu = fermi_level(w, prob.n_electrons, prob.temperature)
    occ = fermi_occupancy(w, mu, prob.temperature)
    return X, w, occ
