"""Triangle mesh with boundary extraction (reference: flatworld/mesh.py:11-149).

The reference counts undirected edges in a Python dict and keeps the edges seen
once, in first-seen order and orientation (mesh.py:53-71); boundary nodes are
the sorted unique endpoints (mesh.py:42-47).  This version does the same with
numpy sorts, so 20k-node meshes build in milliseconds.  Edge lengths are
float32 ``norm(a - b)`` per element edge in (0,1), (1,2), (2,0) order
(mesh.py:90-112); ``charLength`` is their minimum and ``charAverageLength`` their
float32 mean, both bit-identical to the reference's loop.
"""

from __future__ import annotations

import numpy as np


def boundary_edges(conn: np.ndarray) -> np.ndarray:
    """Edges used by exactly one triangle, in first-seen order and orientation."""
    conn = np.asarray(conn)
    e = np.stack([conn[:, [0, 1]], conn[:, [1, 2]], conn[:, [2, 0]]], axis=1).reshape(-1, 2)
    lo = np.minimum(e[:, 0], e[:, 1]).astype(np.int64)
    hi = np.maximum(e[:, 0], e[:, 1]).astype(np.int64)
    key = lo * (int(hi.max(initial=0)) + 1) + hi
    _, first, counts = np.unique(key, return_index=True, return_counts=True)
    once = np.sort(first[counts == 1])
    return e[once]


def edge_lengths(conn: np.ndarray, coords: np.ndarray) -> np.ndarray:
    """float32 length of every element edge, (0,1), (1,2), (2,0) per element."""
    c = np.asarray(coords, dtype=np.float32)
    conn = np.asarray(conn)
    a = c[conn[:, [0, 1, 2]]]
    b = c[conn[:, [1, 2, 0]]]
    d = (a - b).reshape(-1, 2)
    return np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]).astype(np.float32)


class Mesh:
    def __init__(self, d, conns, coords, is_rigid=False):
        if d != 2:
            raise NotImplementedError("flatworld_b200 implements the 2D FEM step (d=2) only")
        self.d = d
        self.connectivity = conns
        self.coords = coords
        self.numNodes = self.coords.shape[0]
        self.numElements = conns.shape[0]
        self.is_rigid = is_rigid
        if is_rigid:
            self.numNodePerEl = 2
            self.massWeights = 1 / 2
            self.numBoundElements = self.numElements
            self.boundaryElements = self.connectivity
            self.numBoundNodes = self.numNodes
            self.boundaryNodes = np.arange(self.numNodes)
        else:
            self.numNodePerEl = 3
            self.massWeights = 1 / 3
            if np.asarray(conns).shape[1] != 3:
                raise ValueError("2D FEM meshes must be P1 triangles (3 nodes per element)")
            self.boundaryElements = boundary_edges(conns)
            self.numBoundElements = self.boundaryElements.shape[0]
            self.boundaryNodes = np.unique(self.boundaryElements)
            self.numBoundNodes = self.boundaryNodes.shape[0]
        self.charLength = self.calCharacteristicLength()
        self.charAverageLength = self.calPenaltyLength()
        self.charLengthSquare = 0.5 * (self.charLength * self.charLength)

    def _collect_edge_lengths(self):
        if self.numElements == 0 or self.is_rigid:
            return np.array([], dtype=np.float32)
        return edge_lengths(self.connectivity, self.coords)

    def calCharacteristicLength(self):
        el = self._collect_edge_lengths()
        return 0.0 if el.size == 0 else float(np.min(el))

    def calPenaltyLength(self):
        el = self._collect_edge_lengths()
        return 0.0 if el.size == 0 else float(np.mean(el))

    def getBoundaryEdges_(self, conns):
        return boundary_edges(conns)

    def getCenterPoint(self):
        coord = np.zeros((self.d,), dtype=np.float32)
        for i in range(self.numNodes):
            coord += self.coords[i]
        return coord / self.numNodes

    def computeBoundaryNodeNormals(self):
        """Averaged boundary-edge normals (used by FEM-FEM contact only)."""
        normals = np.zeros((self.numNodes, self.d), dtype=np.float32)
        for n1, n2 in self.boundaryElements:
            edge = self.coords[n2] - self.coords[n1]
            nrm = np.array([-edge[1], edge[0]], dtype=np.float32)
            ln = np.linalg.norm(nrm)
            if ln > 1e-10:
                nrm = nrm / ln
            normals[n1] += nrm
            normals[n2] += nrm
        ln = np.linalg.norm(normals, axis=1)
        ok = ln > 1e-10
        normals[ok] = normals[ok] / ln[ok, None]
        return normals


def structured_rectangle(nx: int, ny: int, lx: float, ly: float, origin=(0.0, 0.0),
                         jitter: float = 0.0, seed: int | None = None):
    """(nx x ny) quads over [origin, origin + (lx, ly)], each split into two
    triangles with the pattern of test2D/test_2Dfem_elastic10000.py:17-32
    (node id = i*(ny+1) + j, i along x).  ``jitter`` moves interior nodes by
    U(-jitter*h, +jitter*h) per axis (h = cell size along that axis).

    Returns (conn int32 [2*nx*ny, 3], coords float32 [(nx+1)*(ny+1), 2]).
    """
    hx, hy = lx / nx, ly / ny
    ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="ij")
    coords = np.stack([ii * hx, jj * hy], axis=-1).reshape(-1, 2).astype(np.float64)
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        interior = ((ii > 0) & (ii < nx) & (jj > 0) & (jj < ny)).reshape(-1)
        k = int(interior.sum())
        coords[interior, 0] += rng.uniform(-jitter * hx, jitter * hx, size=k)
        coords[interior, 1] += rng.uniform(-jitter * hy, jitter * hy, size=k)
    coords += np.asarray(origin, dtype=np.float64)
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    i = i.reshape(-1)
    j = j.reshape(-1)
    a = i * (ny + 1) + j
    b = i * (ny + 1) + j + 1
    c = (i + 1) * (ny + 1) + j
    dd = (i + 1) * (ny + 1) + j + 1
    conn = np.empty((2 * nx * ny, 3), dtype=np.int32)
    conn[0::2] = np.stack([a, b, c], axis=1)
    conn[1::2] = np.stack([b, dd, c], axis=1)
    return conn, coords.astype(np.float32)
