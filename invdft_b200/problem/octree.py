"""Adaptive octree hexahedral meshes with 2:1 balance (setup only).

The reference builds its meshes with deal.II/p4est through DFT-FE's
``triangulationManager``; the v_xc mesh is a copy of that mesh refined inside the
atoms' bounding box (TriangulationManagerVxc.cpp:113-221).  Those libraries are
not available here, so this module produces meshes of the same kind: axis-aligned
cubic cells on an octree, refined by a size rule, balanced so that cells sharing
a face, an edge or a vertex differ by at most one level (which is what makes the
hanging-node constraints of space.py well defined).

Cells are stored as (level, i, j, k) with integer anchors on the level's grid.
Leaves are kept in Morton (Z-curve) order, which keeps the descendants of any
cell contiguous and gives spatially local node numbering.
"""
from __future__ import annotations

import numpy as np

_SHIFT_L = 60
_SHIFT_I = 40
_SHIFT_J = 20
MAX_LEVEL = 19


def encode(level, i, j, k) -> np.ndarray:
    level = np.asarray(level, dtype=np.int64)
    return (level << _SHIFT_L) | (np.asarray(i, np.int64) << _SHIFT_I) | (
        np.asarray(j, np.int64) << _SHIFT_J) | np.asarray(k, np.int64)


def _morton(i, j, k, bits: int) -> np.ndarray:
    out = np.zeros(np.shape(i), dtype=np.uint64)
    i = np.asarray(i, np.uint64)
    j = np.asarray(j, np.uint64)
    k = np.asarray(k, np.uint64)
    for b in range(bits):
        one = np.uint64(1)
        sb = np.uint64(b)
        out |= ((i >> sb) & one) << np.uint64(3 * b)
        out |= ((j >> sb) & one) << np.uint64(3 * b + 1)
        out |= ((k >> sb) & one) << np.uint64(3 * b + 2)
    return out


_OFFS26 = np.array([(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1)
                    for dx in (-1, 0, 1) if (dx, dy, dz) != (0, 0, 0)], dtype=np.int64)


class Octree:
    """Leaves of an octree over the cube [lo, lo+size]^3."""

    def __init__(self, lo: float, size: float, level0: int = 0):
        self.lo = float(lo)
        self.size = float(size)
        n = 1 << level0
        g = np.arange(n, dtype=np.int64)
        k, j, i = np.meshgrid(g, g, g, indexing="ij")
        self.level = np.full(n ** 3, level0, dtype=np.int64)
        self.i = i.ravel().copy()
        self.j = j.ravel().copy()
        self.k = k.ravel().copy()
        self._reindex()

    # ------------------------------------------------------------------
    def copy(self) -> "Octree":
        t = Octree.__new__(Octree)
        t.lo, t.size = self.lo, self.size
        t.level, t.i, t.j, t.k = (self.level.copy(), self.i.copy(),
                                  self.j.copy(), self.k.copy())
        t._reindex()
        return t

    @property
    def n_cells(self) -> int:
        return int(self.level.size)

    @property
    def max_level(self) -> int:
        return int(self.level.max())

    def cell_size(self) -> np.ndarray:
        return self.size / (2.0 ** self.level)

    def cell_lo(self) -> np.ndarray:
        h = self.cell_size()
        return self.lo + np.stack([self.i, self.j, self.k], axis=1) * h[:, None]

    def cell_center(self) -> np.ndarray:
        return self.cell_lo() + 0.5 * self.cell_size()[:, None]

    def _reindex(self):
        lmax = int(self.level.max()) if self.level.size else 0
        bits = lmax + 1
        s = lmax - self.level
        code = _morton(self.i << s, self.j << s, self.k << s, bits)
        order = np.lexsort((self.level, code))
        self.level, self.i, self.j, self.k = (self.level[order], self.i[order],
                                              self.j[order], self.k[order])
        self.keys = encode(self.level, self.i, self.j, self.k)
        self._sort = np.argsort(self.keys, kind="stable")
        self._sorted_keys = self.keys[self._sort]

    def find(self, keys: np.ndarray) -> np.ndarray:
        """Leaf index of each key, or -1."""
        pos = np.searchsorted(self._sorted_keys, keys)
        pos = np.minimum(pos, self._sorted_keys.size - 1)
        hit = self._sorted_keys[pos] == keys
        return np.where(hit, self._sort[pos], -1)

    def locate(self, pts: np.ndarray) -> np.ndarray:
        """Leaf index containing each point (-1 outside the domain).

        Points on a face between leaves go to the leaf on the + side.
        """
        pts = np.asarray(pts, dtype=np.float64).reshape(-1, 3)
        out = np.full(pts.shape[0], -1, dtype=np.int64)
        rel = (pts - self.lo) / self.size
        inside = np.all((rel >= 0.0) & (rel <= 1.0), axis=1)
        todo = np.nonzero(inside)[0]
        for lev in range(0, self.max_level + 1):
            if todo.size == 0:
                break
            n = 1 << lev
            ijk = np.floor(rel[todo] * n).astype(np.int64)
            np.clip(ijk, 0, n - 1, out=ijk)
            idx = self.find(encode(lev, ijk[:, 0], ijk[:, 1], ijk[:, 2]))
            hit = idx >= 0
            out[todo[hit]] = idx[hit]
            todo = todo[~hit]
        return out

    # ------------------------------------------------------------------
    def split(self, mask: np.ndarray):
        mask = np.asarray(mask, dtype=bool)
        if not mask.any():
            return
        keep = ~mask
        L, I, J, K = self.level[mask], self.i[mask], self.j[mask], self.k[mask]
        ch = []
        for dz in (0, 1):
            for dy in (0, 1):
                for dx in (0, 1):
                    ch.append((L + 1, 2 * I + dx, 2 * J + dy, 2 * K + dz))
        self.level = np.concatenate([self.level[keep]] + [c[0] for c in ch])
        self.i = np.concatenate([self.i[keep]] + [c[1] for c in ch])
        self.j = np.concatenate([self.j[keep]] + [c[2] for c in ch])
        self.k = np.concatenate([self.k[keep]] + [c[3] for c in ch])
        if self.level.max() > MAX_LEVEL:
            raise ValueError("octree deeper than supported")
        self._reindex()

    def refine_while(self, predicate, max_iter: int = 64):
        """Split leaves while ``predicate(tree) -> bool mask`` selects any."""
        for _ in range(max_iter):
            m = predicate(self)
            if not np.any(m):
                return
            self.split(m)
        raise RuntimeError("refinement did not terminate")

    def balance(self):
        """Enforce 2:1 balance across faces, edges and vertices."""
        for _ in range(64):
            h = self.cell_size()
            centers = self.cell_center()
            mark = np.zeros(self.n_cells, dtype=bool)
            for off in _OFFS26:
                q = centers + off[None, :] * h[:, None]
                nb = self.locate(q)
                ok = nb >= 0
                too_coarse = ok.copy()
                too_coarse[ok] = self.level[nb[ok]] < self.level[ok] - 1
                mark[nb[too_coarse]] = True
            if not mark.any():
                return
            self.split(mark)
        raise RuntimeError("balance did not terminate")

    def ancestor_in(self, other: "Octree") -> np.ndarray:
        """For each leaf of ``self`` the leaf of ``other`` that contains it.

        ``self`` must be a refinement of ``other``.
        """
        out = other.locate(self.cell_center())
        if np.any(out < 0) or np.any(other.level[out] > self.level):
            raise ValueError("mesh is not a refinement of the given mesh")
        return out
