"""FEMesher.read (reference: flatworld/femesher.py:8-109, which goes through
meshio): Gmsh ASCII 2.2 / 4.1 and VTU (ascii, inline base64) triangle meshes
read back to the mesh they were written from -- points in file order, node
tags mapped to those indices, triangles in file order, z dropped."""

import base64

import numpy as np
import pytest

import flatworld_b200 as fw


def source_mesh():
    conn, coords = fw.structured_rectangle(3, 2, 0.3, 0.2, origin=(0.1, 0.05))
    return conn.astype(np.int64), coords.astype(np.float32)


def write_msh2(path, conn, coords, tag0=11):
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$Nodes", str(len(coords))]
    lines += [f"{tag0 + i} {float(x)!r} {float(y)!r} 0" for i, (x, y) in enumerate(coords)]
    lines += ["$EndNodes", "$Elements", str(len(conn) + 1), "1 15 2 0 1 11"]  # a point element first
    lines += [f"{k + 2} 2 2 0 1 {' '.join(str(tag0 + v) for v in t)}" for k, t in enumerate(conn)]
    lines += ["$EndElements"]
    path.write_text("\n".join(lines) + "\n")


def write_msh4(path, conn, coords, tag0=5):
    n, m = len(coords), len(conn)
    half = n // 2
    lines = ["$MeshFormat", "4.1 0 8", "$EndMeshFormat", "$Nodes", f"2 {n} {tag0} {tag0 + n - 1}"]
    for lo, hi in ((0, half), (half, n)):  # two node blocks
        lines.append(f"2 1 0 {hi - lo}")
        lines += [str(tag0 + i) for i in range(lo, hi)]
        lines += [f"{float(coords[i, 0])!r} {float(coords[i, 1])!r} 0" for i in range(lo, hi)]
    lines += ["$EndNodes", "$Elements", f"2 {m + 1} 1 {m + 1}", "0 1 15 1", f"1 {tag0}", f"2 1 2 {m}"]
    lines += [f"{k + 2} {' '.join(str(tag0 + v) for v in t)}" for k, t in enumerate(conn)]
    lines += ["$EndElements"]
    path.write_text("\n".join(lines) + "\n")


def write_vtu(path, conn, coords, binary=False):
    pts = np.zeros((len(coords), 3), np.float32)
    pts[:, :2] = coords
    offs = np.arange(1, len(conn) + 1, dtype=np.int64) * 3
    types = np.full(len(conn), 5, np.uint8)

    def arr(a, name, vtype, comps=None):
        attrs = f'type="{vtype}" Name="{name}"' + (f' NumberOfComponents="{comps}"' if comps else "")
        if binary:
            raw = a.tobytes()
            data = base64.b64encode(np.uint32(len(raw)).tobytes() + raw).decode()
            return f'<DataArray {attrs} format="binary">{data}</DataArray>'
        return f'<DataArray {attrs} format="ascii">{" ".join(repr(v) for v in a.reshape(-1).tolist())}</DataArray>'

    path.write_text(
        '<?xml version="1.0"?><VTKFile type="UnstructuredGrid" version="1.0" header_type="UInt32">'
        f'<UnstructuredGrid><Piece NumberOfPoints="{len(pts)}" NumberOfCells="{len(conn)}">'
        f'<Points>{arr(pts, "Points", "Float32", 3)}</Points>'
        f'<Cells>{arr(conn.astype(np.int64), "connectivity", "Int64")}{arr(offs, "offsets", "Int64")}'
        f'{arr(types, "types", "UInt8")}</Cells></Piece></UnstructuredGrid></VTKFile>')


@pytest.mark.parametrize("kind", ["msh2", "msh4", "vtu-ascii", "vtu-binary"])
def test_read_round_trip(tmp_path, kind):
    conn, coords = source_mesh()
    path = tmp_path / ("m.msh" if kind.startswith("msh") else "m.vtu")
    {"msh2": lambda: write_msh2(path, conn, coords), "msh4": lambda: write_msh4(path, conn, coords),
     "vtu-ascii": lambda: write_vtu(path, conn, coords), "vtu-binary": lambda: write_vtu(path, conn, coords, True)}[kind]()
    m = fw.FEMesher(2).read(str(path))
    assert m.d == 2 and m.connectivity.dtype == np.int32
    assert np.array_equal(m.connectivity, conn)
    assert np.array_equal(m.coords, coords)
    ref = fw.Mesh(2, conn.astype(np.int32), coords)
    assert np.array_equal(m.boundaryNodes, ref.boundaryNodes) and m.charLength == ref.charLength


def test_read_refusals(tmp_path):
    p = tmp_path / "m.obj"
    p.write_text("")
    with pytest.raises(RuntimeError):
        fw.FEMesher(2).read(str(p))
    tet = tmp_path / "t.msh"
    tet.write_text("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n4\n1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1\n$EndNodes\n"
                   "$Elements\n1\n1 4 2 0 1 1 2 3 4\n$EndElements\n")
    with pytest.raises(NotImplementedError):
        fw.FEMesher(2).read(str(tet))
