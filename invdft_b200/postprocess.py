"""Host side of the POST_PROCESS step that follows the inverse solve.

The reference's ``InverseDFTEngine::interpolateVxc`` (InverseDFTEngine.cpp:
3241-3456) projects the converged v_xc onto the parent mesh and, when asked,
evaluates it on a regular grid of points that it writes as rows
``index x y z value``.  The projection and the evaluation run on the GPU
(``InverseDFTSolverFunction.project_vxc_to_parent`` / ``evaluate_parent_field``);
this module builds the point grid in the reference's order, locates points in
the parent cells and writes the file.
"""
from __future__ import annotations

import os

import numpy as np


def grid_points(start, end, counts) -> np.ndarray:
    """The reference's target points (InverseDFTEngine.cpp:3281-3372): per axis
    ``n`` equispaced coordinates from start to end (one coordinate when n = 1),
    point ``index = ix*(ny*nz) + iy*nz + iz``.  Raises ValueError where the
    reference aborts (end too close to start, or end before start)."""
    axes = []
    for a, b, n in zip(start, end, counts):
        n = int(n)
        if n < 1:
            raise ValueError("point count must be positive")
        if n != 1 and abs(a - b) < 1e-6:
            raise ValueError("coordinates are too close to interpolate")
        if n != 1 and b - a <= 0.0:
            raise ValueError("the step is negative")
        c = np.empty(n)
        c[0] = a
        if n > 1:
            c[-1] = b
            d = (b - a) / (n - 1)
            for i in range(1, n - 1):
                c[i] = c[i - 1] + d
        axes.append(c)
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    return np.column_stack([X.ravel(), Y.ravel(), Z.ravel()])


def locate_points(problem, pts: np.ndarray):
    """Parent cell and reference coordinates in [0, 1]^3 of each point.

    Cells of equal size form a regular lattice, so each refinement level is
    searched by its integer cell coordinates; a point on a face between cells
    goes to the cell whose lower corner it does not exceed.  Raises ValueError
    for points outside the mesh."""
    pts = np.asarray(pts, dtype=np.float64).reshape(-1, 3)
    lo_all = problem.cell_lo
    h_all = problem.cell_h
    origin = lo_all.min(axis=0)
    top = (lo_all + h_all[:, None]).max(axis=0)
    if np.any(pts < origin - 1e-9) or np.any(pts > top + 1e-9):
        raise ValueError("point outside the mesh")
    cells = np.full(pts.shape[0], -1, dtype=np.int64)
    for h in np.unique(h_all):
        sel = np.nonzero(h_all == h)[0]
        ijk = np.rint((lo_all[sel] - origin) / h).astype(np.int64)
        n = np.rint((top - origin) / h).astype(np.int64) + 1
        keys = (ijk[:, 0] * n[1] + ijk[:, 1]) * n[2] + ijk[:, 2]
        order = np.argsort(keys)
        skeys = keys[order]
        todo = np.nonzero(cells < 0)[0]
        if todo.size == 0:
            break
        q = np.floor((pts[todo] - origin) / h).astype(np.int64)
        q = np.minimum(np.maximum(q, 0), n - 2)
        qk = (q[:, 0] * n[1] + q[:, 1]) * n[2] + q[:, 2]
        pos = np.searchsorted(skeys, qk)
        pos = np.minimum(pos, skeys.size - 1)
        hit = skeys[pos] == qk
        cells[todo[hit]] = sel[order[pos[hit]]]
    if np.any(cells < 0):
        raise ValueError("point not covered by any cell")
    xi = (pts - lo_all[cells]) / h_all[cells][:, None]
    return cells, np.clip(xi, 0.0, 1.0)


def write_points(path: str | os.PathLike, pts: np.ndarray, values: np.ndarray) -> None:
    """Rows ``index x y z value`` (InverseDFTEngine.cpp:3441-3455)."""
    pts = np.asarray(pts, dtype=np.float64).reshape(-1, 3)
    values = np.asarray(values, dtype=np.float64).ravel()
    if values.size != pts.shape[0]:
        raise ValueError("points and values disagree in size")
    idx = np.arange(values.size, dtype=np.float64)
    np.savetxt(path, np.column_stack([idx, pts, values]), fmt=["%d", "%.17g", "%.17g", "%.17g", "%.17g"])
