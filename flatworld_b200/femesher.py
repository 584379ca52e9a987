"""Mesh generators and readers of the reference's FEMesher
(flatworld/femesher.py:4-149).

The reference reads Gmsh ``.msh`` and VTK ``.vtu`` files through meshio
(femesher.py:19-109), which this image does not have; the readers here parse
the two formats themselves and hand back what the reference builds from
meshio's result: ``Mesh(2, triangles, points[:, :2])`` -- the points in file
order, node tags mapped to those indices, the triangle blocks concatenated in
file order.  Tetrahedral meshes (3D) are refused: the FEM step here is 2D.
Supported: Gmsh ASCII 2.2 and 4.1; VTU UnstructuredGrid with ASCII or
inline base64 (uncompressed) data arrays.
"""

import numpy as np

from .mesh import Mesh


class FEMesher:
    def __init__(self, d=2):
        self.d = d

    def read(self, filename, readGroup=False):
        """femesher.py:8-14: dispatch on the file extension."""
        lower = filename.lower()
        if lower.endswith(".msh"):
            return self.read_msh(filename, readGroup)
        if lower.endswith(".vtu"):
            return self.read_vtu(filename, readGroup)
        raise RuntimeError(f"Unsupported mesh format for reading: {filename}")

    def read_msh(self, filename, readGroup=False):
        """Gmsh ASCII 2.2 / 4.1 triangles (femesher.py:16-56)."""
        with open(filename) as f:
            tokens = f.read().split("\n")
        sections, k = {}, 0
        while k < len(tokens):
            line = tokens[k].strip()
            if line.startswith("$") and not line.startswith("$End"):
                name = line[1:]
                body = []
                k += 1
                while k < len(tokens) and tokens[k].strip() != "$End" + name:
                    body.append(tokens[k])
                    k += 1
                sections[name] = body
            k += 1
        if "MeshFormat" not in sections:
            raise RuntimeError(f"{filename}: no $MeshFormat section")
        fmt = sections["MeshFormat"][0].split()
        version, binary = fmt[0], int(fmt[1])
        if binary:
            raise RuntimeError(f"{filename}: binary Gmsh files are not supported (ASCII 2.2 / 4.1 are)")
        if version.startswith("2"):
            tags, pts, tris, tets = _msh2(sections)
        elif version.startswith("4"):
            tags, pts, tris, tets = _msh4(sections)
        else:
            raise RuntimeError(f"{filename}: Gmsh format {version} is not supported")
        return _to_mesh(filename, tags, pts, tris, tets)

    def read_vtu(self, filename, readGroup=False):
        """VTK UnstructuredGrid triangles (femesher.py:58-109)."""
        import xml.etree.ElementTree as ET

        root = ET.parse(filename).getroot()
        if root.get("compressor"):
            raise RuntimeError(f"{filename}: compressed VTU files are not supported")
        header = np.uint64 if root.get("header_type", "UInt32") == "UInt64" else np.uint32
        piece = root.find("UnstructuredGrid/Piece")
        if piece is None:
            raise RuntimeError(f"{filename}: no UnstructuredGrid piece")
        pts = _vtu_array(piece.find("Points/DataArray"), header, filename).reshape(-1, 3)
        cells = {a.get("Name"): a for a in piece.findall("Cells/DataArray")}
        conn = _vtu_array(cells["connectivity"], header, filename).astype(np.int64)
        offs = _vtu_array(cells["offsets"], header, filename).astype(np.int64)
        types = _vtu_array(cells["types"], header, filename).astype(np.int64)
        starts = np.concatenate([[0], offs[:-1]])
        tris = [conn[a:b] for a, b, t in zip(starts, offs, types) if t == 5]   # VTK_TRIANGLE
        tets = [conn[a:b] for a, b, t in zip(starts, offs, types) if t == 10]  # VTK_TETRA
        return _to_mesh(filename, np.arange(len(pts)), pts, tris, tets)

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


_MSH_TRIANGLE, _MSH_TETRA = 2, 4  # Gmsh element type codes


def _msh2(sec):
    lines = [l.split() for l in sec.get("Nodes", []) if l.strip()]
    n = int(lines[0][0])
    tags = np.array([int(r[0]) for r in lines[1:n + 1]], np.int64)
    pts = np.array([[float(v) for v in r[1:4]] for r in lines[1:n + 1]], np.float64)
    tris, tets = [], []
    els = [l.split() for l in sec.get("Elements", []) if l.strip()]
    for r in els[1:int(els[0][0]) + 1]:
        etype, ntags = int(r[1]), int(r[2])
        nodes = [int(v) for v in r[3 + ntags:]]
        if etype == _MSH_TRIANGLE:
            tris.append(nodes)
        elif etype == _MSH_TETRA:
            tets.append(nodes)
    return tags, pts, tris, tets


def _msh4(sec):
    rows = [l.split() for l in sec.get("Nodes", []) if l.strip()]
    n_blocks = int(rows[0][0])
    k, tags, pts = 1, [], []
    for _ in range(n_blocks):
        nb = int(rows[k][3])
        k += 1
        tags += [int(rows[k + i][0]) for i in range(nb)]
        pts += [[float(v) for v in rows[k + nb + i][:3]] for i in range(nb)]
        k += 2 * nb
    rows = [l.split() for l in sec.get("Elements", []) if l.strip()]
    n_blocks = int(rows[0][0])
    k, tris, tets = 1, [], []
    for _ in range(n_blocks):
        etype, nb = int(rows[k][2]), int(rows[k][3])
        k += 1
        for i in range(nb):
            nodes = [int(v) for v in rows[k + i][1:]]
            if etype == _MSH_TRIANGLE:
                tris.append(nodes)
            elif etype == _MSH_TETRA:
                tets.append(nodes)
        k += nb
    return np.array(tags, np.int64), np.array(pts, np.float64), tris, tets


def _vtu_array(el, header, filename):
    import base64

    dtypes = {"Float32": np.float32, "Float64": np.float64, "Int8": np.int8, "UInt8": np.uint8, "Int16": np.int16,
              "UInt16": np.uint16, "Int32": np.int32, "UInt32": np.uint32, "Int64": np.int64, "UInt64": np.uint64}
    dt = dtypes[el.get("type")]
    fmt = el.get("format", "ascii")
    if fmt == "ascii":
        return np.array(el.text.split(), dtype=dt)
    if fmt == "binary":
        raw = base64.b64decode("".join(el.text.split()))
        nbytes = int(np.frombuffer(raw[:np.dtype(header).itemsize], header)[0])
        return np.frombuffer(raw[np.dtype(header).itemsize:np.dtype(header).itemsize + nbytes], dt)
    raise RuntimeError(f"{filename}: VTU data format '{fmt}' is not supported (ascii, inline binary are)")


def _to_mesh(filename, tags, pts, tris, tets):
    """femesher.py:40-56: tetrahedra first, else triangles."""
    if tets:
        raise NotImplementedError(f"{filename}: tetrahedral (3D) meshes are outside flatworld_b200's 2D FEM step")
    if not tris:
        raise RuntimeError(f"No supported cells (triangle/tetra) found in {filename}")
    index = {int(t): i for i, t in enumerate(tags)}
    conn = np.array([[index[int(v)] for v in t[:3]] for t in tris], dtype=np.int32)
    return Mesh(2, conn, np.asarray(pts, dtype=np.float32)[:, :2])
