"""Mesh and result files (jax-fem_b200/utils.py), on the CPU.

- save_sol writes what the reference's save_sol (utils.py:13-57) writes: the
  mesh, the solution as FP32 point field ``sol``, FP32 cell and point fields;
  read back bit for bit (binary and ASCII VTU);
- the reader takes zlib-compressed inline arrays (meshio's default) and the
  dolfinx ASCII form of the reference's FEniCSx fixtures (VTK type 72);
- Gmsh 2.2 / 4.1 ASCII and Abaqus meshes give the same hexahedral Mesh,
  unused nodes and non-hexahedral elements dropped;
- TET4, TET10, HEX20 and HEX27 meshes and solutions round-trip through VTU
  with their VTK cell types; their Gmsh (edge and face nodes renumbered)
  and Abaqus cells come back in VTK order, checked by geometry: every
  edge / face / centre node sits where the cell's corners put it;
- QUAD4, QUAD8, TRI3 and TRI6 meshes round-trip through VTU (z = 0 written,
  (N, 2) points read back), Gmsh and Abaqus CPS / CPE cells; a 3D file's
  boundary triangles do not shadow its tetrahedra."""
import base64
import os
import struct
import zlib

import numpy as np
import pytest

from __graft_entry__ import load_package


@pytest.fixture(scope="module")
def io():
    pkg = load_package()
    import importlib
    return pkg, importlib.import_module("jax_fem_b200.utils")


def _fe(pkg):
    m = pkg.box_mesh(3, 2, 2, 1.5, 1.0, 1.0)
    return pkg.fe.FiniteElement(pkg.Mesh(m.points, m.cells_dict["hexahedron"]), 3, 3)


@pytest.mark.parametrize("fmt", ["binary", "ascii"])
def test_save_sol_round_trip(io, tmp_path, fmt):
    pkg, ut = io
    fe = _fe(pkg)
    rng = np.random.default_rng(0)
    sol = rng.normal(size=(len(fe.points), 3))
    rho = rng.uniform(size=len(fe.cells))
    T = rng.normal(size=len(fe.points))
    path = str(tmp_path / "out" / "u.vtu")
    if fmt == "binary":
        ut.save_sol(fe, sol, path, cell_infos=[("rho", rho)], point_infos=[("T", T)])
    else:
        ut.write_vtu(path, fe.points, fe.cells, {"sol": sol.astype(np.float32), "T": T.astype(np.float32)},
                     {"rho": rho.astype(np.float32)}, fmt="ascii")
    pts, cells, pd, cd = ut.read_vtu(path)
    np.testing.assert_array_equal(pts, fe.points)
    np.testing.assert_array_equal(cells, fe.cells)
    np.testing.assert_array_equal(pd["sol"], sol.astype(np.float32))
    np.testing.assert_array_equal(pd["T"], T.astype(np.float32))
    np.testing.assert_array_equal(cd["rho"], rho.astype(np.float32))
    assert pd["sol"].dtype == np.float32 and pd["sol"].shape == (len(fe.points), 3)
    with pytest.raises(ValueError):
        ut.save_sol(fe, sol, path, cell_infos=[("bad", np.zeros(len(fe.cells) + 1))])
    m = ut.read_mesh(path)
    np.testing.assert_array_equal(m.cells, fe.cells)


def _zlib_inline(arr, blocksize=64):
    raw = np.ascontiguousarray(arr).tobytes()
    blocks = [raw[i:i + blocksize] for i in range(0, len(raw), blocksize)]
    comp = [zlib.compress(b) for b in blocks]
    last = len(blocks[-1]) if len(blocks[-1]) < blocksize else blocksize
    hdr = struct.pack("<%dI" % (3 + len(comp)), len(comp), blocksize, last, *[len(c) for c in comp])
    return base64.b64encode(hdr).decode() + base64.b64encode(b"".join(comp)).decode()


def test_read_compressed_vtu(io, tmp_path):
    """Inline zlib blocks with UInt32 headers, header and data encoded apart."""
    pkg, ut = io
    fe = _fe(pkg)
    sol = np.random.default_rng(1).normal(size=(len(fe.points), 3)).astype(np.float32)
    conn, offs = fe.cells.astype(np.int64).reshape(-1), np.arange(1, len(fe.cells) + 1, dtype=np.int64) * 8
    types = np.full(len(fe.cells), 12, dtype=np.uint8)
    def arr(a, t, extra=""):
        return f'<DataArray type="{t}" {extra} format="binary">{_zlib_inline(a)}</DataArray>'

    text = ('<?xml version="1.0"?><VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian" '
            'compressor="vtkZLibDataCompressor"><UnstructuredGrid>'
            f'<Piece NumberOfPoints="{len(fe.points)}" NumberOfCells="{len(fe.cells)}">'
            '<Points>' + arr(fe.points, "Float64", 'NumberOfComponents="3"') + '</Points><Cells>'
            + arr(conn, "Int64", 'Name="connectivity"') + arr(offs, "Int64", 'Name="offsets"')
            + arr(types, "UInt8", 'Name="types"') + '</Cells><PointData>'
            + arr(sol, "Float32", 'Name="sol" NumberOfComponents="3"')
            + '</PointData></Piece></UnstructuredGrid></VTKFile>')
    path = tmp_path / "c.vtu"
    path.write_text(text)
    pts, cells, pd, cd = ut.read_vtu(str(path))
    np.testing.assert_array_equal(pts, fe.points)
    np.testing.assert_array_equal(cells, fe.cells)
    np.testing.assert_array_equal(pd["sol"], sol)
    assert cd == {}


def test_read_dolfinx_ascii_vtu(io, tmp_path):
    """The ASCII form dolfinx writes (version 2.2, no header type, Lagrange
    hexahedra, type 72), as in the reference's FEniCSx fixtures."""
    pkg, ut = io
    pts = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    sol = np.arange(8, dtype=float) * 0.5
    text = ('<?xml version="1.0"?>\n<VTKFile type="UnstructuredGrid" version="2.2">\n<UnstructuredGrid>\n'
            '<Piece NumberOfPoints="8" NumberOfCells="1">\n<Points>\n'
            '<DataArray type="Float64" NumberOfComponents="3" format="ascii">'
            + " ".join(str(v) for v in pts.reshape(-1)) + '</DataArray>\n</Points>\n<Cells>\n'
            '<DataArray type="Int64" Name="connectivity" format="ascii">0 1 2 3 4 5 6 7</DataArray>\n'
            '<DataArray type="Int64" Name="offsets" format="ascii">8</DataArray>\n'
            '<DataArray type="Int8" Name="types" format="ascii">72</DataArray>\n</Cells>\n<PointData>\n'
            '<DataArray type="Float64" Name="sol" format="ascii">' + " ".join(str(v) for v in sol)
            + '</DataArray>\n</PointData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n')
    path = tmp_path / "d.vtu"
    path.write_text(text)
    p, c, pd, _ = ut.read_vtu(str(path))
    np.testing.assert_array_equal(p, pts)
    np.testing.assert_array_equal(c, np.arange(8)[None])
    np.testing.assert_array_equal(pd["sol"], sol)


# Two hexahedra side by side in x; node 99 is unused; element 3 is a boundary quad.
_NODES = {1: (0, 0, 0), 2: (1, 0, 0), 3: (1, 1, 0), 4: (0, 1, 0), 5: (0, 0, 1), 6: (1, 0, 1), 7: (1, 1, 1),
          8: (0, 1, 1), 9: (2, 0, 0), 10: (2, 1, 0), 11: (2, 0, 1), 12: (2, 1, 1), 99: (5, 5, 5)}
_HEXES = [[1, 2, 3, 4, 5, 6, 7, 8], [2, 9, 10, 3, 6, 11, 12, 7]]


def _expected(pkg):
    used = sorted({t for h in _HEXES for t in h}, key=list(_NODES).index)
    index = {t: i for i, t in enumerate(used)}
    return (np.array([_NODES[t] for t in used], float),
            np.array([[index[t] for t in h] for h in _HEXES], np.int32))


def test_read_gmsh_and_abaqus(io, tmp_path):
    pkg, ut = io
    pts, cells = _expected(pkg)
    nodes22 = "\n".join(f"{t} {x} {y} {z}" for t, (x, y, z) in _NODES.items())
    msh22 = (f"$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n{len(_NODES)}\n{nodes22}\n$EndNodes\n"
             f"$Elements\n3\n1 5 2 1 1 {' '.join(map(str, _HEXES[0]))}\n2 5 2 1 1 {' '.join(map(str, _HEXES[1]))}\n"
             f"3 3 2 2 2 1 2 6 5\n$EndElements\n")
    ids = list(_NODES)
    msh41 = ("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n$Nodes\n2 13 1 99\n"
             f"3 1 0 12\n" + "\n".join(map(str, ids[:12])) + "\n"
             + "\n".join(" ".join(map(str, _NODES[t])) for t in ids[:12]) + "\n"
             f"0 2 0 1\n99\n5 5 5\n$EndNodes\n$Elements\n2 3 1 3\n"
             f"2 1 3 1\n3 1 2 6 5\n3 1 5 2\n1 {' '.join(map(str, _HEXES[0]))}\n2 {' '.join(map(str, _HEXES[1]))}\n"
             "$EndElements\n")
    inp = ("*HEADING\n** two hexahedra\n*NODE\n" + "\n".join(f"{t}, {x}, {y}, {z}" for t, (x, y, z) in _NODES.items())
           + "\n*ELEMENT, TYPE=S4R\n3, 1, 2, 6, 5\n*ELEMENT, TYPE=C3D8, ELSET=body\n"
           + f"1, {', '.join(map(str, _HEXES[0]))}\n2, {', '.join(map(str, _HEXES[1][:5]))},\n"
           + f"{', '.join(map(str, _HEXES[1][5:]))}\n*END STEP\n")
    for name, text in (("a.msh", msh22), ("b.msh", msh41), ("c.inp", inp)):
        path = tmp_path / name
        path.write_text(text)
        m = ut.read_mesh(str(path))
        np.testing.assert_array_equal(m.points, pts, err_msg=name)
        np.testing.assert_array_equal(m.cells, cells, err_msg=name)
    with pytest.raises(NotImplementedError):
        ut.read_mesh(str(tmp_path / "x.stl"))


@pytest.mark.parametrize("ele", ["TET4", "TET10", "HEX20", "HEX27"])
def test_element_types_round_trip(io, tmp_path, ele):
    pkg, ut = io
    from helpers import element_box
    m = element_box(pkg, ele, (2, 1, 2))
    fe = pkg.fe.FiniteElement(m, 1, 3, ele_type=ele)
    sol = np.random.default_rng(2).normal(size=len(m.points))
    path = str(tmp_path / f"{ele}.vtu")
    ut.save_sol(fe, sol, path)
    pts, cells, pd, _, got = ut.read_vtu(path, with_type=True)
    assert got == ele
    np.testing.assert_array_equal(cells, m.cells)
    np.testing.assert_array_equal(pd["sol"].reshape(-1), sol.astype(np.float32))
    mm = ut.read_mesh(path)
    assert mm.ele_type == ele and mm.cells.shape == m.cells.shape
    with pytest.raises(ValueError):
        ut.read_mesh(path, ele_type="HEX8")


def _isoparametric_ok(pkg, mesh):
    """Every node of every cell sits at the linear map of its reference
    position from the cell's corners (straight-sided cells)."""
    import importlib
    B = importlib.import_module("jax_fem_b200.basis")
    lin = "TET4" if mesh.ele_type.startswith("TET") else "HEX8"
    vn = B.shape_fn(lin, B.node_coords(mesh.ele_type))[0]
    X = mesh.points[mesh.cells]
    return np.allclose(np.einsum("ka,cai->cki", vn, X[:, :vn.shape[1]]), X, atol=1e-12)


# Gmsh node numbering of quadratic cells (edge corner pairs, hexahedron face
# corner sets), used here to write the cells in Gmsh order.
_GMSH_TET_EDGES = [(0, 1), (1, 2), (2, 0), (3, 0), (3, 2), (3, 1)]
_GMSH_HEX_EDGES = [(0, 1), (0, 3), (0, 4), (1, 2), (1, 5), (2, 3), (2, 6), (3, 7), (4, 5), (4, 7), (5, 6), (6, 7)]
_GMSH_HEX_FACES = [(0, 1, 2, 3), (0, 1, 4, 5), (0, 3, 4, 7), (1, 2, 5, 6), (2, 3, 6, 7), (4, 5, 6, 7)]


def _gmsh_cell(corner_xyz, ele, add_node):
    """Node numbers of one cell in Gmsh order, new nodes created by add_node(xyz)."""
    ids = [add_node(x) for x in corner_xyz]
    if ele in ("TET10", "HEX20", "HEX27"):
        edges = _GMSH_TET_EDGES if ele == "TET10" else _GMSH_HEX_EDGES
        ids += [add_node(0.5 * (corner_xyz[a] + corner_xyz[b])) for a, b in edges]
    if ele == "HEX27":
        ids += [add_node(corner_xyz[list(f)].mean(axis=0)) for f in _GMSH_HEX_FACES]
        ids.append(add_node(corner_xyz.mean(axis=0)))
    return ids


@pytest.mark.parametrize("ele,gtype", [("TET4", 4), ("TET10", 11), ("HEX20", 17), ("HEX27", 12)])
def test_gmsh_quadratic_cells_come_back_in_vtk_order(io, tmp_path, ele, gtype):
    pkg, ut = io
    rng = np.random.default_rng(4)
    if ele.startswith("TET"):
        corners = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float)
    else:
        corners = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1],
                            [0, 1, 1]], float)
    corners = corners @ np.array([[1.0, 0.2, 0.1], [0.0, 1.1, 0.3], [0.1, 0.0, 0.9]]) + rng.normal(size=3)
    nodes = {}

    def add(x):
        nodes[100 + 3 * len(nodes)] = x  # sparse Gmsh node tags
        return 100 + 3 * (len(nodes) - 1)

    cell = _gmsh_cell(corners, ele, add)
    node_lines = "\n".join(f"{t} {float(x[0])!r} {float(x[1])!r} {float(x[2])!r}" for t, x in nodes.items())
    msh22 = (f"$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n{len(nodes)}\n{node_lines}\n$EndNodes\n"
             f"$Elements\n2\n1 15 2 0 1 {cell[0]}\n2 {gtype} 2 0 1 {' '.join(map(str, cell))}\n$EndElements\n")
    tags = list(nodes)
    msh41 = ("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n"
             f"$Nodes\n1 {len(tags)} {min(tags)} {max(tags)}\n3 1 0 {len(tags)}\n"
             + "\n".join(map(str, tags)) + "\n" + "\n".join(" ".join(repr(float(v)) for v in nodes[t]) for t in tags)
             + f"\n$EndNodes\n$Elements\n1 1 1 1\n3 1 {gtype} 1\n1 {' '.join(map(str, cell))}\n$EndElements\n")
    for name, text in (("a.msh", msh22), ("b.msh", msh41)):
        (tmp_path / name).write_text(text)
        m = ut.read_mesh(str(tmp_path / name))
        assert m.ele_type == ele and m.cells.shape == (1, len(cell))
        assert _isoparametric_ok(pkg, m), name


def test_abaqus_tet10_and_hex20(io, tmp_path):
    pkg, ut = io
    from helpers import element_box
    for ele, typ in (("TET10", "C3D10"), ("HEX20", "C3D20R")):
        m = element_box(pkg, ele, (1, 1, 1))
        lines = ["*HEADING", "*NODE"] + [f"{i + 1}, {float(x)!r}, {float(y)!r}, {float(z)!r}"
                                         for i, (x, y, z) in enumerate(m.points)]
        lines.append(f"*ELEMENT, TYPE={typ}, ELSET=body")
        for k, c in enumerate(m.cells):
            vals = [str(k + 1)] + [str(int(v) + 1) for v in c]
            lines += [", ".join(vals[:8]) + ",", ", ".join(vals[8:16]) + ("," if len(vals) > 16 else "")]
            if len(vals) > 16:
                lines.append(", ".join(vals[16:]))
        (tmp_path / f"{ele}.inp").write_text("\n".join(lines) + "\n")
        got = ut.read_mesh(str(tmp_path / f"{ele}.inp"))
        assert got.ele_type == ele
        np.testing.assert_array_equal(got.points[got.cells], m.points[m.cells])
        assert _isoparametric_ok(pkg, got)


def test_small_helpers(io, tmp_path, capsys):
    """modify_vtu_file, read_abaqus_and_write_vtk, json_parse, walltime and
    check_mesh_TET4 (the reference's utils.py:60-200, generate_mesh.py:58-80)."""
    import importlib
    import json
    pkg, ut = io
    gm = importlib.import_module("jax_fem_b200.generate_mesh")
    src = tmp_path / "in.vtu"
    src.write_text('<?xml version="1.0"?>\n<VTKFile type="UnstructuredGrid" version="2.2">\n</VTKFile>\n')
    ut.modify_vtu_file(str(src), str(tmp_path / "out" / "o.vtu"))
    assert 'version="1.0"' in (tmp_path / "out" / "o.vtu").read_text()
    from helpers import element_box
    m = element_box(pkg, "TET10", (1, 1, 1))
    lines = ["*NODE"] + [f"{i + 1}, {float(x)!r}, {float(y)!r}, {float(z)!r}" for i, (x, y, z) in enumerate(m.points)]
    lines.append("*ELEMENT, TYPE=C3D10")
    lines += [", ".join(str(v) for v in [k + 1] + [int(c) + 1 for c in cell]) for k, cell in enumerate(m.cells)]
    (tmp_path / "a.inp").write_text("\n".join(lines) + "\n")
    ut.read_abaqus_and_write_vtk(str(tmp_path / "a.inp"), str(tmp_path / "a.vtu"))
    got = ut.read_mesh(str(tmp_path / "a.vtu"))
    assert got.ele_type == "TET10" and np.array_equal(got.points[got.cells], m.points[m.cells])
    (tmp_path / "c.json").write_text(json.dumps({"E": 70e3, "nu": 0.3}))
    assert ut.json_parse(str(tmp_path / "c.json")) == {"E": 70e3, "nu": 0.3}
    assert '"nu": 0.3' in capsys.readouterr().out
    timed = ut.walltime(str(tmp_path / "t"), "run")(lambda a: a + 1)
    assert timed(1) == 2 and any(f.startswith("run_") for f in os.listdir(tmp_path / "t"))
    assert ut.timeit(lambda: 3)() == 3
    m4 = element_box(pkg, "TET4", (2, 1, 1))
    q = gm.check_mesh_TET4(m4.points, m4.cells)
    assert q.shape == (len(m4.cells),) and (q > 0).all()
    flipped = m4.cells[:, [0, 2, 1, 3]]
    assert (gm.check_mesh_TET4(m4.points, flipped) < 0).all()


@pytest.mark.parametrize("ele", ["QUAD4", "QUAD8", "TRI3", "TRI6"])
def test_planar_types_round_trip(io, tmp_path, ele):
    """2D meshes: VTU round trip (points written with z = 0, read back as
    (N, 2)), Gmsh cells (node order = VTK's for these types) and Abaqus
    CPS / CPE cells."""
    pkg, ut = io
    from helpers import planar_box
    m = planar_box(pkg, ele, (2, 3), amp=0.1, seed=1)
    fe = pkg.fe.FiniteElement(m, 2, 2, ele_type=ele)
    sol = np.random.default_rng(3).normal(size=(len(m.points), 2))
    path = str(tmp_path / f"{ele}.vtu")
    ut.save_sol(fe, sol, path)
    pts, cells, pd, _, got = ut.read_vtu(path, with_type=True)
    assert got == ele and pts.shape == (len(m.points), 3) and not pts[:, 2].any()
    np.testing.assert_array_equal(cells, m.cells)
    np.testing.assert_array_equal(pd["sol"], sol.astype(np.float32))
    mm = ut.read_mesh(path)
    assert mm.ele_type == ele and mm.points.shape == m.points.shape
    np.testing.assert_array_equal(mm.points, m.points)
    # Gmsh 2.2 with line elements beside the cells, Abaqus with 2D node lines
    gtype = {"TRI3": 2, "QUAD4": 3, "TRI6": 9, "QUAD8": 16}[ele]
    node_lines = "\n".join(f"{i + 1} {float(x)!r} {float(y)!r} 0" for i, (x, y) in enumerate(m.points))
    els = [f"1 1 2 0 1 {m.cells[0, 0] + 1} {m.cells[0, 1] + 1}"]
    els += [f"{k + 2} {gtype} 2 0 1 " + " ".join(str(int(v) + 1) for v in c) for k, c in enumerate(m.cells)]
    (tmp_path / "p.msh").write_text(f"$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n{len(m.points)}\n{node_lines}\n"
                                    f"$EndNodes\n$Elements\n{len(els)}\n" + "\n".join(els) + "\n$EndElements\n")
    typ = {"TRI3": "CPS3", "QUAD4": "CPE4R", "TRI6": "CPS6M", "QUAD8": "CPE8"}[ele]
    lines = ["*NODE"] + [f"{i + 1}, {float(x)!r}, {float(y)!r}" for i, (x, y) in enumerate(m.points)]
    lines += [f"*ELEMENT, TYPE={typ}"] + [", ".join([str(k + 1)] + [str(int(v) + 1) for v in c])
                                           for k, c in enumerate(m.cells)]
    (tmp_path / "p.inp").write_text("\n".join(lines) + "\n")
    for name in ("p.msh", "p.inp"):
        g = ut.read_mesh(str(tmp_path / name))
        assert g.ele_type == ele and g.points.shape[1] == 2, name
        np.testing.assert_array_equal(g.points[g.cells], m.points[m.cells])


def test_boundary_cells_do_not_shadow_volume_cells(io, tmp_path):
    """A 3D Gmsh mesh with its boundary triangles gives the tetrahedra unless
    TRI3 is asked for; 2D cells off the z = 0 plane are refused."""
    pkg, ut = io
    nodes = "1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1"
    text = ("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n4\n" + nodes + "\n$EndNodes\n"
            "$Elements\n3\n1 2 2 0 1 1 2 3\n2 4 2 0 1 1 2 3 4\n3 2 2 0 1 2 3 4\n$EndElements\n")
    (tmp_path / "t.msh").write_text(text)
    assert ut.read_mesh(str(tmp_path / "t.msh")).ele_type == "TET4"
    with pytest.raises(ValueError, match="off the z = 0 plane"):
        ut.read_mesh(str(tmp_path / "t.msh"), ele_type="TRI3")
    (tmp_path / "u.msh").write_text(text.replace("3 2 2 0 1 2 3 4\n", "").replace("$Elements\n3", "$Elements\n2"))
    tri = ut.read_mesh(str(tmp_path / "u.msh"), ele_type="TRI3")
    assert tri.ele_type == "TRI3" and tri.points.shape == (3, 2)
