"""Mesh container and structured box generators.

Mirrors ``Mesh`` (generate_mesh.py:13-27 in the reference) and ``box_mesh``
(generate_mesh.py:151-189): node (i, j, k) of an (Nx+1, Ny+1, Nz+1) grid has
index (i*(Ny+1) + j)*(Nz+1) + k and cells list their nodes in VTK HEX8 order,
so meshes, solutions and per-cell data line up with the reference's.

``rectangle_mesh`` (generate_mesh.py:120-148) is the 2D counterpart: node
(i, j) of an (Nx+1, Ny+1) grid has index i*(Ny+1) + j.

``box_mesh_gmsh`` (generate_mesh.py:192-260) meshes the same box with gmsh,
which is not available here; this version builds the structured mesh of
the requested element type directly: HEX8 as ``box_mesh``, TET4 by
splitting every hexahedron into the six tetrahedra around its (0,0,0)-(1,1,1)
diagonal (a conforming split, every tetrahedron positively oriented), and
the quadratic types by adding one node per edge (TET10, HEX20, HEX27), per
face and per cell (HEX27), in VTK node order.  Corner nodes keep the
numbering of ``box_mesh``; added nodes follow them.
"""
import numpy as np

from .basis import (ELEMENT_DIM, HEX_EDGES, HEX_FACE_CORNERS, MESHIO_CELL_TYPE, NODES_PER_CELL, QUAD_EDGES,
                    TET_EDGES, TRI_EDGES, check_ele_type)

# element type of (dim, nodes per cell)
_ELE_OF_NEN = {(ELEMENT_DIM[e], n): e for e, n in NODES_PER_CELL.items()}


class Mesh:
    """points (num_nodes, dim) float64 and cells (num_cells, nen) int32.

    ``ele_type`` defaults to the element type of the points' dimension
    with ``nen`` nodes."""

    def __init__(self, points, cells, ele_type=None):
        self.points = np.ascontiguousarray(np.asarray(points, dtype=np.float64))
        self.cells = np.ascontiguousarray(np.asarray(cells, dtype=np.int32))
        key = (self.points.shape[1] if self.points.ndim == 2 else 0,
               self.cells.shape[1] if self.cells.ndim == 2 else 0)
        if ele_type is None and key not in _ELE_OF_NEN:
            raise NotImplementedError("cells must be (num_cells, nen) with nen in 4, 8, 10, 20, 27 for 3D points "
                                      "(TET4, HEX8, TET10, HEX20, HEX27) or 3, 4, 6, 8 for 2D points "
                                      "(TRI3, QUAD4, TRI6, QUAD8)")
        self.ele_type = _ELE_OF_NEN[key] if ele_type is None else check_ele_type(ele_type)
        if NODES_PER_CELL[self.ele_type] != self.cells.shape[1]:
            raise ValueError(f"{self.ele_type} cells have {NODES_PER_CELL[self.ele_type]} nodes, "
                             f"got {self.cells.shape[1]}")


class _BoxMesh:
    """What ``box_mesh`` returns: meshio-like ``points`` and ``cells_dict``."""

    def __init__(self, points, cells):
        self.points = points
        self.cells_dict = {"hexahedron": cells}


def rectangle_mesh(Nx, Ny, domain_x, domain_y, ele_type="QUAD4"):
    """Structured mesh of [0,Lx]x[0,Ly] with Nx*Ny squares
    (generate_mesh.py:120-148): node (i, j) of the (Nx+1, Ny+1) grid has
    index i*(Ny+1) + j, QUAD4 cells list (i,j) (i+1,j) (i+1,j+1) (i,j+1).
    Other 2D types (an extension): TRI3 splits every square along its
    (i,j)-(i+1,j+1) diagonal into two counter-clockwise triangles; QUAD8
    and TRI6 add one node per edge, numbered after the grid's."""
    check_ele_type(ele_type)
    if ELEMENT_DIM[ele_type] != 2:
        raise ValueError(f"rectangle_mesh makes 2D cells, not {ele_type}")
    ix, iy = np.meshgrid(np.arange(Nx + 1), np.arange(Ny + 1), indexing="ij")
    points = np.stack([np.linspace(0, domain_x, Nx + 1)[ix], np.linspace(0, domain_y, Ny + 1)[iy]],
                      axis=-1).reshape(-1, 2)
    i, j = np.meshgrid(np.arange(Nx), np.arange(Ny), indexing="ij")
    base = (i * (Ny + 1) + j).reshape(-1)
    quads = (base[:, None] + np.array([0, Ny + 1, Ny + 2, 1])[None, :]).astype(np.int32)
    if ele_type.startswith("TRI"):
        cells = quads[:, [[0, 1, 2], [0, 2, 3]]].reshape(-1, 3)
        edges = TRI_EDGES
    else:
        cells = quads
        edges = QUAD_EDGES
    if ele_type in ("QUAD8", "TRI6"):
        points, mid = _add_entity_nodes(points, cells, cells[:, edges])
        cells = np.hstack([cells, mid])
    out = _BoxMesh(np.ascontiguousarray(points), np.ascontiguousarray(cells, dtype=np.int32))
    out.cells_dict = {get_meshio_cell_type(ele_type): out.cells_dict.pop("hexahedron")}
    return out


def box_mesh(Nx, Ny, Nz, domain_x, domain_y, domain_z):
    """Structured HEX8 mesh of [0,Lx]x[0,Ly]x[0,Lz] with Nx*Ny*Nz cells."""
    ix, iy, iz = np.meshgrid(np.arange(Nx + 1), np.arange(Ny + 1), np.arange(Nz + 1), indexing="ij")
    points = np.stack([np.linspace(0, domain_x, Nx + 1)[ix],
                       np.linspace(0, domain_y, Ny + 1)[iy],
                       np.linspace(0, domain_z, Nz + 1)[iz]], axis=-1).reshape(-1, 3)
    sy, sx = Nz + 1, (Ny + 1) * (Nz + 1)  # index strides of j and i
    i, j, k = np.meshgrid(np.arange(Nx), np.arange(Ny), np.arange(Nz), indexing="ij")
    base = (i * sx + j * sy + k).reshape(-1)
    # VTK order: (0,0,0) (1,0,0) (1,1,0) (0,1,0) then the same at k+1
    offs = np.array([0, sx, sx + sy, sy, 1, sx + 1, sx + sy + 1, sy + 1])
    cells = (base[:, None] + offs[None, :]).astype(np.int32)
    return _BoxMesh(points, cells)


def check_mesh_TET4(points, cells):  # noqa: N802 - the reference's name
    """Orientation measure of TET4 cells (generate_mesh.py:58-80): the triple
    product (p1 - p0) x (p2 - p0) . (p3 - p0), positive for the node order
    the element tables assume."""
    X = np.asarray(points, dtype=np.float64)[np.asarray(cells)[:, :4]]
    return np.einsum("ci,ci->c", np.cross(X[:, 1] - X[:, 0], X[:, 2] - X[:, 0]), X[:, 3] - X[:, 0])


def get_meshio_cell_type(ele_type):
    """meshio cell type of an element type (generate_mesh.py:83-117)."""
    return MESHIO_CELL_TYPE[check_ele_type(ele_type)]


# Six tetrahedra of a hexahedron around its corner-0 -> corner-6 diagonal:
# one per order of the axes along the path (0,0,0) -> (1,1,1).  VTK corner of
# each (x, y, z) bit triple.
_CORNER_OF_BITS = {(0, 0, 0): 0, (1, 0, 0): 1, (1, 1, 0): 2, (0, 1, 0): 3,
                   (0, 0, 1): 4, (1, 0, 1): 5, (1, 1, 1): 6, (0, 1, 1): 7}


def _kuhn_tets():
    tets = []
    for order in ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)):
        b = [0, 0, 0]
        path = [_CORNER_OF_BITS[tuple(b)]]
        for ax in order:
            b[ax] = 1
            path.append(_CORNER_OF_BITS[tuple(b)])
        tets.append(path)
    return np.array(tets)


def _add_entity_nodes(points, cells, groups):
    """One new node per distinct corner set (rows of ``groups``: (C, k, m)
    corner numbers per cell), at the mean of its corners; returns points and
    the (C, k) new node numbers."""
    C, k, m = groups.shape
    keys = np.sort(groups.reshape(-1, m), axis=1)
    uniq, inv = np.unique(keys, axis=0, return_inverse=True)
    new = points[uniq].mean(axis=1)
    return np.vstack([points, new]), (len(points) + inv.reshape(C, k)).astype(np.int32)


def box_mesh_gmsh(Nx, Ny, Nz, domain_x, domain_y, domain_z, data_dir=None, ele_type="HEX8"):
    """Structured mesh of [0,Lx]x[0,Ly]x[0,Lz] with Nx*Ny*Nz hexahedral
    blocks in the given element type (see the module docstring); returns a
    meshio-like object with ``points`` and ``cells_dict[cell_type]``.
    ``data_dir`` is accepted for the reference's signature; nothing is
    written."""
    check_ele_type(ele_type)
    if ELEMENT_DIM[ele_type] != 3:
        raise ValueError(f"box_mesh_gmsh makes 3D cells; use rectangle_mesh for {ele_type}")
    hexmesh = box_mesh(Nx, Ny, Nz, domain_x, domain_y, domain_z)
    points, hexes = hexmesh.points, hexmesh.cells_dict["hexahedron"]
    if ele_type.startswith("TET"):
        tets = hexes[:, _kuhn_tets()].reshape(-1, 4)
        X = points[tets]
        vol = np.einsum("ci,ci->c", np.cross(X[:, 1] - X[:, 0], X[:, 2] - X[:, 0]), X[:, 3] - X[:, 0])
        flip = vol < 0
        tets[flip] = tets[flip][:, [0, 2, 1, 3]]
        cells = tets
        if ele_type == "TET10":
            points, mid = _add_entity_nodes(points, tets, tets[:, TET_EDGES])
            cells = np.hstack([tets, mid])
    else:
        cells = hexes
        if ele_type in ("HEX20", "HEX27"):
            points, mid = _add_entity_nodes(points, hexes, hexes[:, HEX_EDGES])
            cells = np.hstack([hexes, mid])
        if ele_type == "HEX27":
            points, fc = _add_entity_nodes(points, hexes, hexes[:, HEX_FACE_CORNERS])
            centre = (len(points) + np.arange(len(hexes), dtype=np.int32))[:, None]
            points = np.vstack([points, points[hexes].mean(axis=1)])
            cells = np.hstack([cells, fc, centre])
    out = _BoxMesh(np.ascontiguousarray(points), np.ascontiguousarray(cells, dtype=np.int32))
    out.cells_dict = {get_meshio_cell_type(ele_type): out.cells_dict.pop("hexahedron")}
    return out
