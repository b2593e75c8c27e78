"""Continuous Lagrange spaces on an octree mesh, with hanging-node constraints.

Global vectors hold one entry per geometric node, constrained nodes included,
exactly like the deal.II vectors of the reference: a constrained entry is
either a *hanging* node whose value is a weighted sum of master values
(``constraintMatrixInfo::distribute``) or a homogeneous *Dirichlet* node whose
value is zero.  The constraint lists are closed: no master is itself
constrained, as after ``dealii::AffineConstraints::close()``.

The reference sets these constraints up with
``DoFTools::make_hanging_node_constraints`` plus zero boundary values for the
wavefunctions, plus ``rho_target < tol`` nodes for the adjoint
(InverseDFTEngine.cpp:1502-1573), plus hanging nodes only for the v_xc mesh
(InverseDFTEngine.cpp:284-297).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

from .fe import Element1D, lagrange_eval
from .octree import Octree

_VERTEX_LIMIT = np.int64(1) << np.int64(40)


@dataclass
class Constraints:
    """Closed constraint set in CSR form, rows sorted by node id.

    ``masters[ptr[r]:ptr[r+1]]`` with ``weights`` define node ``nodes[r]``;
    an empty row is a homogeneous Dirichlet node.
    """
    n_nodes: int
    nodes: np.ndarray
    ptr: np.ndarray
    masters: np.ndarray
    weights: np.ndarray

    @property
    def n_constrained(self) -> int:
        return int(self.nodes.size)

    def is_constrained(self) -> np.ndarray:
        m = np.zeros(self.n_nodes, dtype=bool)
        m[self.nodes] = True
        return m

    def matrix(self) -> sp.csr_matrix:
        """C with x_full = C x for x holding only unconstrained values."""
        n = self.n_nodes
        free = ~self.is_constrained()
        rows = [np.nonzero(free)[0]]
        cols = [np.nonzero(free)[0]]
        vals = [np.ones(int(free.sum()))]
        cnt = np.diff(self.ptr)
        rows.append(np.repeat(self.nodes, cnt))
        cols.append(self.masters)
        vals.append(self.weights)
        return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                             shape=(n, n))


class FESpace:
    """Order-p continuous space on the leaves of ``tree``."""

    def __init__(self, tree: Octree, p: int):
        self.tree = tree
        self.p = p
        self.el = Element1D(p)
        self.n1 = p + 1
        self.nd = self.n1 ** 3
        self._build_nodes()
        self._build_hanging()

    # ------------------------------------------------------------------
    def _axis_keys(self, lev, idx, Lf):
        """Canonical 1D keys and coordinates of the n1 GLL positions of cells."""
        p, n1 = self.p, self.n1
        t = self.tree
        h = t.size / (2.0 ** lev)
        keys = np.empty((lev.size, n1), dtype=np.int64)
        coord = np.empty((lev.size, n1))
        unit = t.size / float(1 << Lf)
        for a in range(n1):
            if a == 0 or a == p or (p % 2 == 0 and 2 * a == p):
                if a == 0:
                    pos = idx << (Lf - lev)
                elif a == p:
                    pos = (idx + 1) << (Lf - lev)
                else:
                    pos = (2 * idx + 1) << (Lf - lev - 1)
                keys[:, a] = pos
                coord[:, a] = t.lo + pos.astype(np.float64) * unit
            else:
                keys[:, a] = _VERTEX_LIMIT + ((lev << 20) + idx) * n1 + a
                coord[:, a] = t.lo + h * (idx.astype(np.float64) + self.el.nodes[a])
        return keys, coord

    def _build_nodes(self):
        t, n1 = self.tree, self.n1
        Lf = t.max_level + 1
        self._Lf = Lf
        kx, cx = self._axis_keys(t.level, t.i, Lf)
        ky, cy = self._axis_keys(t.level, t.j, Lf)
        kz, cz = self._axis_keys(t.level, t.k, Lf)
        nc = t.n_cells
        ia = np.arange(self.nd) % n1
        ib = (np.arange(self.nd) // n1) % n1
        ic = np.arange(self.nd) // (n1 * n1)
        K = np.stack([kx[:, ia], ky[:, ib], kz[:, ic]], axis=2).reshape(-1, 3)
        X = np.stack([cx[:, ia], cy[:, ib], cz[:, ic]], axis=2).reshape(-1, 3)
        uniq, first, inv = np.unique(K, axis=0, return_index=True, return_inverse=True)
        inv = inv.ravel()
        # number nodes by first appearance in (Morton) cell order
        order = np.argsort(first, kind="stable")
        rank = np.empty_like(order)
        rank[order] = np.arange(order.size)
        self.cell_nodes = rank[inv].reshape(nc, self.nd).astype(np.int64)
        self.n_nodes = int(uniq.shape[0])
        self.node_xyz = X[first[order]]
        ukeys = uniq[order]
        full = np.int64(1) << np.int64(Lf)
        on_b = np.zeros(self.n_nodes, dtype=bool)
        for d in range(3):
            kd = ukeys[:, d]
            on_b |= (kd == 0) | (kd == full)
        self.on_boundary = on_b
        self.cell_lo = t.cell_lo()
        self.cell_h = t.cell_size()

    def _build_hanging(self):
        t, p, n1 = self.tree, self.p, self.n1
        # candidate nodes: those on a face of their owning cell
        a = np.arange(self.nd)
        ia, ib, ic = a % n1, (a // n1) % n1, a // (n1 * n1)
        on_face = (ia == 0) | (ia == p) | (ib == 0) | (ib == p) | (ic == 0) | (ic == p)
        cand = np.unique(self.cell_nodes[:, on_face].ravel())
        x = self.node_xyz[cand]
        eps = 1e-3 * float(self.cell_h.min())
        n = self.n_nodes
        # a node hangs on a cell only if that cell is coarser than every cell
        # owning the node (a coarse node lying on a fine face is a master)
        owner_lev = np.full(n, np.iinfo(np.int64).max, dtype=np.int64)
        np.minimum.at(owner_lev, self.cell_nodes.ravel(),
                      np.repeat(t.level, self.nd))
        cand_lev = owner_lev[cand]
        member = np.sort((np.arange(t.n_cells, dtype=np.int64)[:, None] * n
                          + self.cell_nodes).ravel())
        hang_node, hang_cell = [], []
        for sx in (-1, 1):
            for sy in (-1, 1):
                for sz in (-1, 1):
                    c = t.locate(x + eps * np.array([sx, sy, sz], dtype=np.float64))
                    ok = c >= 0
                    code = c[ok] * n + cand[ok]
                    pos = np.minimum(np.searchsorted(member, code), member.size - 1)
                    notnode = (member[pos] != code) & (t.level[c[ok]] < cand_lev[ok])
                    hang_node.append(cand[ok][notnode])
                    hang_cell.append(c[ok][notnode])
        hn = np.concatenate(hang_node)
        hc = np.concatenate(hang_cell)
        if hn.size == 0:
            self.hang_nodes = np.zeros(0, np.int64)
            self._hang_T = sp.identity(n, format="csr")
            return
        # one constraining cell per hanging node: the lowest cell index
        order = np.lexsort((hc, hn))
        hn, hc = hn[order], hc[order]
        keep = np.ones(hn.size, dtype=bool)
        keep[1:] = hn[1:] != hn[:-1]
        hn, hc = hn[keep], hc[keep]
        xi = (self.node_xyz[hn] - self.cell_lo[hc]) / self.cell_h[hc][:, None]
        xi = np.clip(xi, 0.0, 1.0)
        nodes1 = self.el.nodes
        Lx = lagrange_eval(nodes1, xi[:, 0])
        Ly = lagrange_eval(nodes1, xi[:, 1])
        Lz = lagrange_eval(nodes1, xi[:, 2])
        W = (Lx[:, ia] * Ly[:, ib] * Lz[:, ic])  # (n_hang, nd)
        rows = np.repeat(hn, self.nd)
        cols = self.cell_nodes[hc].ravel()
        vals = W.ravel()
        nz = vals != 0.0
        free = np.ones(n, dtype=bool)
        free[hn] = False
        fi = np.nonzero(free)[0]
        T = sp.csr_matrix((np.concatenate([np.ones(fi.size), vals[nz]]),
                           (np.concatenate([fi, rows[nz]]), np.concatenate([fi, cols[nz]]))),
                          shape=(n, n))
        # close chains: masters of masters
        for _ in range(32):
            T2 = (T @ T).tocsr()
            T2.eliminate_zeros()
            if (T2 != T).nnz == 0:
                break
            T = T2
        else:
            raise RuntimeError("hanging-node chains did not close")
        self.hang_nodes = hn
        self._hang_T = T

    # ------------------------------------------------------------------
    def constraints(self, dirichlet: np.ndarray | None = None) -> Constraints:
        """Closed constraints: hanging nodes plus zero values on ``dirichlet``.

        Dirichlet nodes that are hanging keep their hanging constraint (the
        reference adds a Dirichlet line only to unconstrained nodes,
        InverseDFTEngine.cpp:1566-1573); masters that are Dirichlet drop out.
        """
        n = self.n_nodes
        hang = np.zeros(n, dtype=bool)
        hang[self.hang_nodes] = True
        dmask = np.zeros(n, dtype=bool) if dirichlet is None else np.asarray(dirichlet, bool).copy()
        dmask &= ~hang
        T = self._hang_T.tocsc(copy=True)
        # zero the columns of Dirichlet masters
        keepcol = sp.diags((~dmask).astype(np.float64))
        T = (T @ keepcol).tocsr()
        T.eliminate_zeros()
        cons = np.nonzero(hang | dmask)[0]
        ptr = [0]
        ms, ws = [], []
        Tc = T[cons]
        Tc.sort_indices()
        for r, node in enumerate(cons):
            if dmask[node]:
                ptr.append(ptr[-1])
                continue
            s, e = Tc.indptr[r], Tc.indptr[r + 1]
            ms.append(Tc.indices[s:e])
            ws.append(Tc.data[s:e])
            ptr.append(ptr[-1] + (e - s))
        masters = np.concatenate(ms).astype(np.int64) if ms else np.zeros(0, np.int64)
        weights = np.concatenate(ws) if ws else np.zeros(0)
        return Constraints(n, cons.astype(np.int64), np.asarray(ptr, np.int64), masters, weights)
