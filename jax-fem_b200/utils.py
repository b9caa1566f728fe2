"""Mesh and result files without meshio: VTU output and mesh input.

Mirrors ``save_sol`` (utils.py:13-57 in the reference), which writes the
solution and optional point/cell fields of a finite element to a VTK XML
UnstructuredGrid (.vtu) through meshio, and gives the reading side the
reference gets from ``meshio.read``: VTU files (ASCII, base64 binary, zlib
compressed; what dolfinx and meshio write), Gmsh ``.msh`` (ASCII, formats 2.2
and 4.1) and Abaqus ``.inp`` meshes, returning the cells of one element
type (TET4, TET10, HEX8, HEX20, HEX27; the 2D TRI3, QUAD4, TRI6, QUAD8 with
(N, 2) points) as a ``Mesh``.

File formats followed: the VTK XML file format (UnstructuredGrid, inline
DataArrays, ``header_type`` UInt32/UInt64, ``vtkZLibDataCompressor`` block
layout; cell types 10, 24, 12, 25, 29, 5, 9, 22, 23 and the order-1 Lagrange
cells 71, 72, 69, 70), the Gmsh MSH 2.2 / 4.1 ASCII formats (element types
4, 11, 5, 17, 12, 2, 3, 9, 16) and the Abaqus input format (``*NODE``,
``*ELEMENT, TYPE=C3D4 / C3D10 / C3D8 / C3D20`` and their R/I/M/H variants,
the 2D CPS / CPE / CAX 3, 4, 6, 8).  ``Mesh`` uses the VTK (= meshio) node
order; Abaqus lists the same order, Gmsh numbers the edge (and face) nodes of
its quadratic cells differently and is permuted on reading (Gmsh node
ordering: edges in the order of their corner pairs listed below).
"""
import base64
import os
import re
import struct
import xml.etree.ElementTree as ET
import zlib

import numpy as np

from . import basis
from .generate_mesh import Mesh

# VTK cell type of each element type, and the types read back: the order-1
# Lagrange cells of dolfinx (71 tetrahedron, 72 hexahedron, 69 triangle,
# 70 quadrilateral) list the same nodes in the same order as 10, 12, 5, 9.
_VTK_CELL = {"TET4": 10, "TET10": 24, "HEX8": 12, "HEX20": 25, "HEX27": 29,
             "TRI3": 5, "QUAD4": 9, "TRI6": 22, "QUAD8": 23}
_VTK_READ = {10: "TET4", 24: "TET10", 12: "HEX8", 25: "HEX20", 29: "HEX27", 71: "TET4", 72: "HEX8",
             5: "TRI3", 9: "QUAD4", 22: "TRI6", 23: "QUAD8", 69: "TRI3", 70: "QUAD4"}
_VTK_TYPES = {"Float32": np.float32, "Float64": np.float64, "Int8": np.int8, "UInt8": np.uint8,
              "Int16": np.int16, "UInt16": np.uint16, "Int32": np.int32, "UInt32": np.uint32,
              "Int64": np.int64, "UInt64": np.uint64}
_VTK_NAMES = {np.dtype(v): k for k, v in _VTK_TYPES.items()}


# ---- VTU output ---------------------------------------------------------------

def _data_array(arr, name=None, ncomp=None, fmt="binary"):
    arr = np.ascontiguousarray(arr)
    attrs = {"type": _VTK_NAMES[arr.dtype], "format": fmt}
    if name is not None:
        attrs["Name"] = name
    if ncomp is not None:
        attrs["NumberOfComponents"] = str(ncomp)
    el = ET.Element("DataArray", attrs)
    if fmt == "ascii":
        el.text = " ".join(repr(v) if arr.dtype.kind == "f" else str(v) for v in arr.reshape(-1).tolist())
    else:  # inline base64: UInt64 byte count, then the little-endian values
        raw = arr.astype(arr.dtype.newbyteorder("<"), copy=False).tobytes()
        el.text = base64.b64encode(struct.pack("<Q", len(raw)) + raw).decode("ascii")
    return el


def write_vtu(path, points, cells, point_data=None, cell_data=None, fmt="binary", ele_type=None):
    """Write a mesh of one element type with point and cell fields as a .vtu file.

    points (N, 3) or (N, 2) (written with z = 0); cells (C, nen) in VTK node
    order (the element type follows from nen and the points' dimension
    unless given); point_data / cell_data: dicts name -> array with N (or C)
    rows.  ``fmt`` is "binary" (inline base64, UInt64 headers) or "ascii"."""
    points = np.asarray(points, dtype=np.float64)
    dim = points.shape[1]
    if dim == 2:
        points = np.hstack([points, np.zeros((len(points), 1))])
    cells = np.asarray(cells, dtype=np.int64)
    if ele_type is None:
        by_nen = {n: e for e, n in basis.NODES_PER_CELL.items() if basis.ELEMENT_DIM[e] == dim}
        if cells.shape[1] not in by_nen:
            raise NotImplementedError(f"cells of {cells.shape[1]} nodes: no {dim}D element type has that many")
        ele_type = by_nen[cells.shape[1]]
    vtk_type = _VTK_CELL[basis.check_ele_type(ele_type)]
    root = ET.Element("VTKFile", {"type": "UnstructuredGrid", "version": "1.0", "byte_order": "LittleEndian",
                                  "header_type": "UInt64"})
    piece = ET.SubElement(ET.SubElement(root, "UnstructuredGrid"), "Piece",
                          {"NumberOfPoints": str(len(points)), "NumberOfCells": str(len(cells))})
    ET.SubElement(piece, "Points").append(_data_array(points, ncomp=3, fmt=fmt))
    ce = ET.SubElement(piece, "Cells")
    ce.append(_data_array(cells.reshape(-1), "connectivity", fmt=fmt))
    ce.append(_data_array(np.arange(1, len(cells) + 1, dtype=np.int64) * cells.shape[1], "offsets", fmt=fmt))
    ce.append(_data_array(np.full(len(cells), vtk_type, dtype=np.uint8), "types", fmt=fmt))
    for tag, fields, rows in (("PointData", point_data, len(points)), ("CellData", cell_data, len(cells))):
        if not fields:
            continue
        sec = ET.SubElement(piece, tag)
        for name, data in fields.items():
            data = np.asarray(data)
            if data.shape[0] != rows:
                raise ValueError(f"{tag} '{name}' has {data.shape[0]} rows, expected {rows}")
            ncomp = int(np.prod(data.shape[1:])) if data.ndim > 1 else None
            sec.append(_data_array(data.reshape(rows, -1) if ncomp else data, name, ncomp, fmt=fmt))
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    ET.ElementTree(root).write(path, xml_declaration=True, encoding="utf-8")


def save_sol(fe, sol, sol_file, cell_infos=None, point_infos=None):
    """Save a solution and extra point/cell fields of a finite element (or a
    ``Problem``'s first one) to ``sol_file`` (.vtu), as the reference's
    save_sol (utils.py:13-57): the solution as point field ``sol``, every
    field in FP32, cell fields of shape (num_cells,)."""
    fe = fe.fes[0] if hasattr(fe, "fes") else fe
    basis.check_ele_type(fe.ele_type)
    sol = _host(sol)
    num_cells = len(fe.cells)
    point_data = {"sol": np.asarray(sol, dtype=np.float32).reshape(len(fe.points), -1)}
    cell_data = {}
    for name, data in cell_infos or []:
        data = _host(data)
        if data.shape != (num_cells,):
            raise ValueError(f"cell data wrong shape, get {data.shape}, while num_cells = {num_cells}")
        cell_data[name] = np.asarray(data, dtype=np.float32)
    for name, data in point_infos or []:
        data = _host(data)
        if len(data) != len(point_data["sol"]):
            raise ValueError("point data wrong shape!")
        point_data[name] = np.asarray(data, dtype=np.float32)
    write_vtu(sol_file, fe.points, fe.cells, point_data, cell_data, ele_type=fe.ele_type)


def _host(a):
    if hasattr(a, "detach"):  # torch tensor (any device)
        a = a.detach().cpu().numpy()
    return np.asarray(a)


# ---- VTU input ----------------------------------------------------------------

def _b64_prefix(text, nbytes):
    """Decode just enough leading base64 characters for nbytes bytes."""
    nchar = 4 * ((nbytes + 2) // 3)
    return base64.b64decode(text[:nchar])[:nbytes]


def _decode_binary(text, dtype, header, compressor):
    text = "".join(text.split())
    hs = np.dtype(header).itemsize
    if compressor is None:
        n = int(np.frombuffer(_b64_prefix(text, hs), dtype=header)[0])
        raw = base64.b64decode(text)
        if len(raw) == hs + n:  # header and data encoded as one stream
            data = raw[hs:]
        else:  # header and data encoded separately
            k = 4 * ((hs + 2) // 3)
            data = base64.b64decode(text[k:])[:n]
        return np.frombuffer(data, dtype=np.dtype(dtype).newbyteorder("<"))
    if compressor != "vtkZLibDataCompressor":
        raise NotImplementedError(f"VTU compressor {compressor}")
    nblocks = int(np.frombuffer(_b64_prefix(text, hs), dtype=header)[0])
    hbytes = (3 + nblocks) * hs
    hdr = np.frombuffer(_b64_prefix(text, hbytes), dtype=header).astype(np.int64)
    csizes = hdr[3:3 + nblocks]
    k = 4 * ((hbytes + 2) // 3)
    comp = base64.b64decode(text[k:])
    out, pos = [], 0
    for c in csizes:
        out.append(zlib.decompress(comp[pos:pos + c]))
        pos += c
    return np.frombuffer(b"".join(out), dtype=np.dtype(dtype).newbyteorder("<"))


def _read_array(el, header, compressor):
    dtype = _VTK_TYPES[el.get("type")]
    fmt = el.get("format", "ascii")
    if fmt == "ascii":
        data = np.array((el.text or "").split(), dtype=np.float64 if np.dtype(dtype).kind == "f" else np.int64)
        data = data.astype(dtype)
    elif fmt == "binary":
        data = _decode_binary(el.text or "", dtype, header, compressor)
    else:
        raise NotImplementedError(f"VTU DataArray format '{fmt}' (appended data is not supported)")
    nc = el.get("NumberOfComponents")
    return data.reshape(-1, int(nc)) if nc is not None and int(nc) > 1 else data


def read_vtu(path, with_type=False):
    """Read a .vtu file: returns (points (N,3) float64, cells (C,nen) int32,
    point_data dict, cell_data dict), and the element type when
    ``with_type``.  All cells must be of one supported type (VTK 10, 24, 12,
    25, 29, 5, 9, 22, 23, or 71 / 72 / 69 / 70 of order 1); others raise
    NotImplementedError."""
    root = ET.parse(path).getroot()
    if root.get("type") != "UnstructuredGrid":
        raise NotImplementedError("only VTK UnstructuredGrid files are read")
    if root.get("byte_order", "LittleEndian") != "LittleEndian":
        raise NotImplementedError("big-endian VTU files are not read")
    header = np.uint64 if root.get("header_type") == "UInt64" else np.uint32
    compressor = root.get("compressor")
    piece = root.find("UnstructuredGrid/Piece")
    points = _read_array(piece.find("Points/DataArray"), header, compressor).reshape(-1, 3).astype(np.float64)
    cd = {el.get("Name"): _read_array(el, header, compressor) for el in piece.find("Cells")}
    conn, offs, types = cd["connectivity"].astype(np.int64), cd["offsets"].astype(np.int64), cd["types"]
    sizes = np.diff(np.concatenate([[0], offs]))
    eles = {_VTK_READ.get(int(t)) for t in np.unique(types)}
    ele = eles.pop() if len(eles) == 1 else None
    if ele is None or not np.all(sizes == basis.NODES_PER_CELL[ele]):
        raise NotImplementedError("the cells must be of one type: TET4, TET10, HEX8, HEX20, HEX27, TRI3, "
                                  "QUAD4, TRI6 or QUAD8 (VTK 10, 24, 12, 25, 29, 5, 9, 22, 23; "
                                  "71/72/69/70 of order 1)")
    cells = conn.reshape(-1, basis.NODES_PER_CELL[ele]).astype(np.int32)
    fields = []
    for tag in ("PointData", "CellData"):
        sec = piece.find(tag)
        fields.append({} if sec is None else {el.get("Name"): _read_array(el, header, compressor) for el in sec})
    if with_type:
        return points, cells, fields[0], fields[1], ele
    return points, cells, fields[0], fields[1]


# ---- Gmsh and Abaqus meshes -------------------------------------------------------

# Gmsh element type -> element; Gmsh's corner pairs of the edge nodes of the
# quadratic tetrahedron and hexahedron, and the corner sets of the
# hexahedron's face nodes (Gmsh node ordering).  Gmsh's 2D cells list their
# nodes in VTK order (corners, then edges (0,1), (1,2), ... in turn).
_GMSH_TYPES = {4: "TET4", 11: "TET10", 5: "HEX8", 17: "HEX20", 12: "HEX27",
               2: "TRI3", 3: "QUAD4", 9: "TRI6", 16: "QUAD8"}
_GMSH_TET_EDGES = [(0, 1), (1, 2), (2, 0), (3, 0), (3, 2), (3, 1)]
_GMSH_HEX_EDGES = [(0, 1), (0, 3), (0, 4), (1, 2), (1, 5), (2, 3), (2, 6), (3, 7), (4, 5), (4, 7), (5, 6), (6, 7)]
_GMSH_HEX_FACES = [(0, 1, 2, 3), (0, 1, 4, 5), (0, 3, 4, 7), (1, 2, 5, 6), (2, 3, 6, 7), (4, 5, 6, 7)]


def _gmsh_to_vtk(ele):
    """perm with vtk_cell = gmsh_cell[perm]."""
    if basis.ELEMENT_DIM[ele] == 2:
        return np.arange(basis.NODES_PER_CELL[ele])
    tet = ele.startswith("TET")
    nc = 4 if tet else 8
    perm = list(range(nc))
    if ele in ("TET10", "HEX20", "HEX27"):
        g_edges = [frozenset(e) for e in (_GMSH_TET_EDGES if tet else _GMSH_HEX_EDGES)]
        v_edges = basis.TET_EDGES if tet else basis.HEX_EDGES
        perm += [nc + g_edges.index(frozenset(int(c) for c in e)) for e in v_edges]
    if ele == "HEX27":
        g_faces = [frozenset(f) for f in _GMSH_HEX_FACES]
        perm += [20 + g_faces.index(frozenset(int(c) for c in f)) for f in basis.HEX_FACE_CORNERS]
        perm.append(26)
    return np.array(perm)


def _pick(found, ele_type, path, what):
    """The cells of the requested element type, or of the single one of the
    highest dimension found (a 3D mesh's boundary triangles and quadrangles
    are not cells of it)."""
    if ele_type is not None:
        if ele_type not in found:
            raise ValueError(f"{path}: no {ele_type} {what}")
        return ele_type
    top = max((basis.ELEMENT_DIM[e] for e in found), default=3)
    cand = sorted(e for e in found if basis.ELEMENT_DIM[e] == top)
    if len(cand) != 1:
        raise ValueError(f"{path}: {'no' if not cand else 'several'} {top}D element types "
                         f"({cand}); pass ele_type")
    return cand[0]


def _planar(points, ele, path):
    """Points of a 2D element type as (N, 2): z dropped, which must be 0."""
    if basis.ELEMENT_DIM[ele] == 3 or points.shape[1] == 2:
        return points
    if len(points) and np.abs(points[:, 2]).max() > 0.0:
        raise ValueError(f"{path}: {ele} cells off the z = 0 plane")
    return np.ascontiguousarray(points[:, :2])


def _compact(points, node_ids, cells_ids, ele, path=""):
    """Mesh from node ids and cells of ids: the points the cells use, in the
    order of the node table (unused nodes, e.g. geometry points, dropped)."""
    nen = basis.NODES_PER_CELL[ele]
    index = {int(t): i for i, t in enumerate(node_ids)}
    cells = np.array([[index[int(t)] for t in c] for c in cells_ids], dtype=np.int64).reshape(-1, nen)
    used, inv = np.unique(cells.reshape(-1), return_inverse=True)
    return Mesh(_planar(points[used], ele, path), inv.reshape(-1, nen).astype(np.int32), ele)


def read_gmsh(path, ele_type=None):
    """Mesh from a Gmsh ASCII .msh file (format 2.2 or 4.1): the cells of
    one element type (``ele_type``, or the only one of the highest
    dimension in the file), in VTK node order; nodes not used by them
    dropped; 2D cells get (N, 2) points."""
    with open(path) as f:
        lines = [ln.strip() for ln in f]
    sec = {}
    i = 0
    while i < len(lines):
        if lines[i].startswith("$") and not lines[i].startswith("$End"):
            name = lines[i][1:]
            j = lines.index("$End" + name, i)
            sec[name] = lines[i + 1:j]
            i = j
        i += 1
    version = float(sec["MeshFormat"][0].split()[0])
    if int(sec["MeshFormat"][0].split()[1]) != 0:
        raise NotImplementedError("binary .msh files are not read")
    ids, xyz, found = [], [], {}
    if version >= 4.0:
        nodes = sec["Nodes"]
        nblocks = int(nodes[0].split()[0])
        p = 1
        for _ in range(nblocks):
            n = int(nodes[p].split()[3])
            ids += [int(t) for t in nodes[p + 1:p + 1 + n]]
            xyz += [[float(v) for v in ln.split()[:3]] for ln in nodes[p + 1 + n:p + 1 + 2 * n]]
            p += 1 + 2 * n
        els = sec["Elements"]
        nblocks = int(els[0].split()[0])
        p = 1
        for _ in range(nblocks):
            _, _, etype, n = (int(v) for v in els[p].split())
            if etype in _GMSH_TYPES:
                nen = basis.NODES_PER_CELL[_GMSH_TYPES[etype]]
                found.setdefault(_GMSH_TYPES[etype], []).extend(
                    [int(v) for v in ln.split()[1:1 + nen]] for ln in els[p + 1:p + 1 + n])
            p += 1 + n
    else:
        nodes = sec["Nodes"]
        for ln in nodes[1:1 + int(nodes[0])]:
            v = ln.split()
            ids.append(int(v[0]))
            xyz.append([float(t) for t in v[1:4]])
        els = sec["Elements"]
        for ln in els[1:1 + int(els[0])]:
            v = [int(t) for t in ln.split()]
            if v[1] in _GMSH_TYPES:
                nen = basis.NODES_PER_CELL[_GMSH_TYPES[v[1]]]
                found.setdefault(_GMSH_TYPES[v[1]], []).append(v[3 + v[2]:3 + v[2] + nen])
    ele = _pick(found, ele_type, path, "cells (Gmsh element types 4, 11, 5, 17, 12, 2, 3, 9, 16)")
    cells = np.array(found[ele], dtype=np.int64)[:, _gmsh_to_vtk(ele)]
    return _compact(np.array(xyz, dtype=np.float64), ids, cells, ele, path)


_ABAQUS_TYPES = {"C3D4": "TET4", "C3D4H": "TET4", "C3D10": "TET10", "C3D10H": "TET10", "C3D10M": "TET10",
                 "C3D10MH": "TET10", "C3D8": "HEX8", "C3D8R": "HEX8", "C3D8I": "HEX8", "C3D8H": "HEX8",
                 "C3D20": "HEX20", "C3D20R": "HEX20", "C3D20H": "HEX20", "C3D20RH": "HEX20"}
# plane stress / plane strain / axisymmetric continuum cells
for _fam in ("CPS", "CPE", "CAX"):
    _ABAQUS_TYPES.update({_fam + "3": "TRI3", _fam + "4": "QUAD4", _fam + "4R": "QUAD4", _fam + "4I": "QUAD4",
                          _fam + "6": "TRI6", _fam + "6M": "TRI6", _fam + "8": "QUAD8", _fam + "8R": "QUAD8"})


def read_abaqus(path, ele_type=None):
    """Mesh from an Abaqus .inp file: the *NODE table and the *ELEMENT
    blocks of one element type (C3D4, C3D10, C3D8, C3D20 and their R/I/M/H
    variants; the 2D CPS/CPE/CAX 3, 4, 6, 8; ``ele_type`` or the only one
    of the highest dimension in the file).  Abaqus lists the nodes of these
    cells in VTK order; 2D cells get (N, 2) points."""
    ids, xyz, found = [], [], {}
    mode, pending = None, []
    with open(path) as f:
        for raw in f:
            ln = raw.strip()
            if not ln or ln.startswith("**"):
                continue
            if ln.startswith("*"):
                kw = ln.upper()
                if kw.startswith("*NODE") and not kw.startswith("*NODE OUTPUT") and not kw.startswith("*NODE PRINT"):
                    mode = "node"
                elif kw.startswith("*ELEMENT") and not kw.startswith("*ELEMENT OUTPUT"):
                    m = re.search(r"TYPE\s*=\s*([A-Z0-9]+)", kw)
                    mode = _ABAQUS_TYPES.get(m.group(1)) if m else None
                else:
                    mode = None
                pending = []
                continue
            vals = [v for v in ln.split(",") if v.strip()]
            if mode == "node":
                ids.append(int(vals[0]))
                xyz.append([float(v) for v in vals[1:4]] + [0.0] * (3 - len(vals[1:4])))
            elif mode is not None:  # a row may continue on the next line after a trailing comma
                pending += [int(v) for v in vals]
                nen = basis.NODES_PER_CELL[mode]
                if len(pending) >= nen + 1:
                    found.setdefault(mode, []).append(pending[1:nen + 1])
                    pending = []
    ele = _pick(found, ele_type, path, "elements (C3D4, C3D10, C3D8, C3D20, CPS/CPE/CAX 3, 4, 6, 8)")
    return _compact(np.array(xyz, dtype=np.float64), ids, found[ele], ele, path)


def read_mesh(path, ele_type=None):
    """``Mesh`` of the cells of one element type in a .vtu, .msh or .inp
    file (by extension); 2D cells get (N, 2) points."""
    ext = os.path.splitext(path)[1].lower()
    if ext == ".vtu":
        points, cells, _, _, ele = read_vtu(path, with_type=True)
        if ele_type is not None and ele_type != ele:
            raise ValueError(f"{path}: holds {ele} cells, not {ele_type}")
        return Mesh(_planar(points, ele, path), cells, ele)
    if ext == ".msh":
        return read_gmsh(path, ele_type)
    if ext == ".inp":
        return read_abaqus(path, ele_type)
    raise NotImplementedError(f"mesh file type '{ext}' (read .vtu, .msh or .inp)")


# ---- the reference's small helpers (utils.py:60-180) ---------------------------------

def modify_vtu_file(input_file_path, output_file_path):
    """Copy a VTU file, declaring VTK XML version 1.0 where it says 2.2 (the
    form dolfinx writes; utils.py:60-80)."""
    with open(input_file_path) as f:
        text = f.read()
    text = text.replace('<VTKFile type="UnstructuredGrid" version="2.2">',
                        '<VTKFile type="UnstructuredGrid" version="1.0">')
    d = os.path.dirname(os.path.abspath(output_file_path))
    os.makedirs(d, exist_ok=True)
    with open(output_file_path, "w") as f:
        f.write(text)


def read_abaqus_and_write_vtk(abaqus_file, vtk_file):
    """Convert an Abaqus .inp mesh to a .vtu file for viewing (utils.py:83-94)."""
    mesh = read_abaqus(abaqus_file)
    write_vtu(vtk_file, mesh.points, mesh.cells, ele_type=mesh.ele_type)


def json_parse(json_filepath):
    """Read a JSON configuration file, print it indented and return it (utils.py:97-114)."""
    import json
    with open(json_filepath) as f:
        args = json.load(f)
    print(json.dumps(args, indent=4))
    return args


def timeit(func):
    """Decorator that logs how long each call of ``func`` took (utils.py:141-163)."""
    import functools
    import logging
    import time

    @functools.wraps(func)
    def wrapper(*args, **kwargs):
        t0 = time.perf_counter()
        out = func(*args, **kwargs)
        logging.getLogger("jax_fem_b200").debug(f"Function {func.__name__} took {time.perf_counter() - t0:.4f} seconds")
        return out

    return wrapper


def walltime(txt_dir=None, filename=None):
    """Decorator factory that logs a call's wall time and, with ``txt_dir``,
    writes it to ``{txt_dir}/{filename or 'walltime'}_{platform}.txt``
    (utils.py:166-200); the platform is "cuda" when a device is present."""
    import functools
    import logging
    import time

    def decorate(func):
        @functools.wraps(func)
        def wrapper(*args, **kwargs):
            t0 = time.time()
            out = func(*args, **kwargs)
            elapsed = time.time() - t0
            import torch
            platform = "cuda" if torch.cuda.is_available() else "cpu"
            logging.getLogger("jax_fem_b200").info(
                f"Time elapsed {elapsed} of function {func.__name__} on platform {platform}")
            if txt_dir is not None:
                os.makedirs(txt_dir, exist_ok=True)
                with open(os.path.join(txt_dir, f"{filename or 'walltime'}_{platform}.txt"), "w") as f:
                    f.write(f"{elapsed}\n")
            return out

        return wrapper

    return decorate
