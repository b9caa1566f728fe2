"""Mesh and result files without meshio: VTU output and hexahedral mesh input.

Mirrors ``save_sol`` (utils.py:13-57 in the reference), which writes the
solution and optional point/cell fields of a finite element to a VTK XML
UnstructuredGrid (.vtu) through meshio, and gives the reading side the
reference gets from ``meshio.read``: VTU files (ASCII, base64 binary, zlib
compressed; what dolfinx and meshio write), Gmsh ``.msh`` (ASCII, formats 2.2
and 4.1) and Abaqus ``.inp`` meshes, returning the hexahedra as a ``Mesh``.

File formats followed: the VTK XML file format (UnstructuredGrid, inline
DataArrays, ``header_type`` UInt32/UInt64, ``vtkZLibDataCompressor`` block
layout), the Gmsh MSH 2.2 / 4.1 ASCII formats (8-node hexahedron = type 5)
and the Abaqus input format (``*NODE``, ``*ELEMENT, TYPE=C3D8``/``C3D8R``/
``C3D8I``).  The 8-node hexahedron node order is the same in VTK, Gmsh and
Abaqus, and it is the order ``Mesh`` uses.
"""
import base64
import os
import re
import struct
import xml.etree.ElementTree as ET
import zlib

import numpy as np

from .generate_mesh import Mesh, get_meshio_cell_type

_VTK_HEXAHEDRON = 12
_VTK_LAGRANGE_HEXAHEDRON = 72  # order 1: the same 8 nodes in the same order
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


def write_vtu(path, points, cells, point_data=None, cell_data=None, fmt="binary"):
    """Write a hexahedral mesh with point and cell fields as a .vtu file.

    points (N, 3); cells (C, 8) in VTK hexahedron order; point_data /
    cell_data: dicts name -> array with N (or C) rows.  ``fmt`` is "binary"
    (inline base64, UInt64 headers) or "ascii"."""
    points = np.asarray(points, dtype=np.float64)
    if points.shape[1] == 2:
        points = np.hstack([points, np.zeros((len(points), 1))])
    cells = np.asarray(cells, dtype=np.int64)
    root = ET.Element("VTKFile", {"type": "UnstructuredGrid", "version": "1.0", "byte_order": "LittleEndian",
                                  "header_type": "UInt64"})
    piece = ET.SubElement(ET.SubElement(root, "UnstructuredGrid"), "Piece",
                          {"NumberOfPoints": str(len(points)), "NumberOfCells": str(len(cells))})
    ET.SubElement(piece, "Points").append(_data_array(points, ncomp=3, fmt=fmt))
    ce = ET.SubElement(piece, "Cells")
    ce.append(_data_array(cells.reshape(-1), "connectivity", fmt=fmt))
    ce.append(_data_array(np.arange(1, len(cells) + 1, dtype=np.int64) * cells.shape[1], "offsets", fmt=fmt))
    ce.append(_data_array(np.full(len(cells), _VTK_HEXAHEDRON, dtype=np.uint8), "types", fmt=fmt))
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
    get_meshio_cell_type(fe.ele_type)  # HEX8 only
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
    write_vtu(sol_file, fe.points, fe.cells, point_data, cell_data)


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


def read_vtu(path):
    """Read a .vtu file: returns (points (N,3) float64, cells (C,8) int32,
    point_data dict, cell_data dict).  Only hexahedra (VTK types 12, and 72
    of order 1) are returned; other cells raise NotImplementedError."""
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
    if not np.all(np.isin(types, (_VTK_HEXAHEDRON, _VTK_LAGRANGE_HEXAHEDRON))) or not np.all(sizes == 8):
        raise NotImplementedError("only 8-node hexahedral cells are read")
    cells = conn.reshape(-1, 8).astype(np.int32)
    fields = []
    for tag in ("PointData", "CellData"):
        sec = piece.find(tag)
        fields.append({} if sec is None else {el.get("Name"): _read_array(el, header, compressor) for el in sec})
    return points, cells, fields[0], fields[1]


# ---- Gmsh and Abaqus meshes -------------------------------------------------------

def _compact(points, node_ids, cells_ids):
    """Mesh from node ids and cells of ids: points ordered by first use in
    the hexahedra (unused nodes, e.g. geometry points, are dropped)."""
    index = {int(t): i for i, t in enumerate(node_ids)}
    cells = np.array([[index[int(t)] for t in c] for c in cells_ids], dtype=np.int64).reshape(-1, 8)
    used, inv = np.unique(cells.reshape(-1), return_inverse=True)
    return Mesh(points[used], inv.reshape(-1, 8).astype(np.int32))


def read_gmsh(path):
    """Hexahedral mesh from a Gmsh ASCII .msh file (format 2.2 or 4.1):
    the 8-node hexahedra (element type 5); nodes not used by them dropped."""
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
    ids, xyz, hexes = [], [], []
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
            if etype == 5:
                hexes += [[int(v) for v in ln.split()[1:9]] for ln in els[p + 1:p + 1 + n]]
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
            if v[1] == 5:
                hexes.append(v[3 + v[2]:3 + v[2] + 8])
    if not hexes:
        raise ValueError(f"{path}: no 8-node hexahedra (Gmsh element type 5)")
    return _compact(np.array(xyz, dtype=np.float64), ids, hexes)


def read_abaqus(path):
    """Hexahedral mesh from an Abaqus .inp file: the *NODE table and the
    *ELEMENT blocks of TYPE=C3D8, C3D8R or C3D8I."""
    ids, xyz, hexes = [], [], []
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
                    mode = "hex" if m and m.group(1) in ("C3D8", "C3D8R", "C3D8I") else None
                else:
                    mode = None
                pending = []
                continue
            vals = [v for v in ln.split(",") if v.strip()]
            if mode == "node":
                ids.append(int(vals[0]))
                xyz.append([float(v) for v in vals[1:4]] + [0.0] * (3 - len(vals[1:4])))
            elif mode == "hex":  # a row may continue on the next line after a trailing comma
                pending += [int(v) for v in vals]
                if len(pending) >= 9:
                    hexes.append(pending[1:9])
                    pending = []
    if not hexes:
        raise ValueError(f"{path}: no C3D8 elements")
    return _compact(np.array(xyz, dtype=np.float64), ids, hexes)


def read_mesh(path):
    """``Mesh`` of the hexahedra in a .vtu, .msh or .inp file (by extension)."""
    ext = os.path.splitext(path)[1].lower()
    if ext == ".vtu":
        points, cells, _, _ = read_vtu(path)
        return Mesh(points, cells)
    if ext == ".msh":
        return read_gmsh(path)
    if ext == ".inp":
        return read_abaqus(path)
    raise NotImplementedError(f"mesh file type '{ext}' (read .vtu, .msh or .inp)")
