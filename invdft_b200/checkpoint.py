"""v_xc checkpoints in the reference's text format.

Writer: one row per child (Q1) node, ``iNode x y z v`` (writeVxcDataToFile ->
writeChildMeshDataToFile, InverseDFTSolverFunction.cpp:596-655; one spin).
Readers: ``read_vxc`` takes row i as node i, checks the row's coordinates
against node i within ``tol`` and stores its value at node i, whatever its
``iNode`` column says (readVxcDataFromFile, InverseDFTEngine.cpp:2915-2980,
places by row position and uses the column only for its MPI ownership test;
here a column outside [0, n) is rejected); ``search=True`` matches rows to
nodes by coordinates instead (readVxcDataFromFileWithSearch, :2984-3143).  A
mismatch raises ValueError where the reference aborts.
"""
from __future__ import annotations

import os

import numpy as np


def write_vxc(path: str | os.PathLike, node_xyz: np.ndarray, pot: np.ndarray) -> None:
    node_xyz = np.asarray(node_xyz, dtype=np.float64)
    pot = np.asarray(pot, dtype=np.float64)
    if node_xyz.shape != (pot.size, 3):
        raise ValueError("node coordinates and potential disagree in size")
    idx = np.arange(pot.size, dtype=np.float64)
    np.savetxt(path, np.column_stack([idx, node_xyz, pot]), fmt=["%d", "%.17g", "%.17g", "%.17g", "%.17g"])


def read_vxc(path: str | os.PathLike, node_xyz: np.ndarray, tol: float = 1e-3,
             search: bool = False) -> np.ndarray:
    node_xyz = np.asarray(node_xyz, dtype=np.float64)
    data = np.loadtxt(path, ndmin=2)
    if data.shape[1] < 5:
        raise ValueError("expected rows 'iNode x y z v'")
    out = np.zeros(node_xyz.shape[0])
    if not search:
        if data.shape[0] < node_xyz.shape[0]:
            raise ValueError("file has fewer rows than the mesh has nodes")
        rows = data[: node_xyz.shape[0]]
        ids = rows[:, 0].astype(np.int64)
        if np.any(ids < 0) or np.any(ids >= node_xyz.shape[0]):
            raise ValueError("node index out of range")
        dist = np.linalg.norm(rows[:, 1:4] - node_xyz, axis=1)
        bad = np.nonzero(dist > tol)[0]
        if bad.size:
            raise ValueError(f"v_xc nodal coordinates differ from the mesh at row {int(bad[0])} "
                             f"(distance {dist[bad[0]]:.3e} > {tol})")
        out[:] = rows[:, 4]
        return out
    from scipy.spatial import cKDTree
    dist, ids = cKDTree(node_xyz).query(data[:, 1:4])
    bad = np.nonzero(dist > tol)[0]
    if bad.size:
        raise ValueError(f"no mesh node within {tol} of file row {int(bad[0])}")
    out[ids] = data[:, 4]
    return out
