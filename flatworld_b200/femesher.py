"""Mesh generators of the reference's FEMesher (flatworld/femesher.py:115-149).

``read_msh`` needs meshio, which this image does not have, and reading mesh
files is outside the FEM step; the generators are kept because the reference's
contact tests build their bodies with them.
"""

import numpy as np

from .mesh import Mesh


class FEMesher:
    def __init__(self, d=2):
        self.d = d

    def read_msh(self, filename):
        raise NotImplementedError("mesh file IO (meshio) is not part of flatworld_b200")

    def createTriangle(self, pt1, pt2, pt3):
        return Mesh(2, np.array([[0, 1, 2]], dtype=np.int32), np.array([pt1, pt2, pt3], dtype=np.float32))

    def createRectangle(self, lb, up):
        lx, ly = lb
        ux, uy = up
        verts = [[lx, ly], [ux, ly], [ux, uy], [lx, uy]]
        conn = np.array([[0, 1, 2], [0, 2, 3]], dtype=np.int32)
        return Mesh(2, conn, np.array(verts, dtype=np.float32))

    def createCircle(self, origin, radius):
        """16-segment triangle fan around ``origin`` (femesher.py:132-149)."""
        x, y = origin
        segments = 16
        verts = []
        for i in range(segments):
            theta = 2.0 * np.pi * i / segments
            verts.append([x + radius * np.cos(theta), y + radius * np.sin(theta)])
        center = len(verts)
        verts.append([x, y])
        conn = np.array([[i, (i + 1) % segments, center] for i in range(segments)], dtype=np.int32)
        return Mesh(2, conn, np.array(verts, dtype=np.float32))
