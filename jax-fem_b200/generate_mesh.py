"""Mesh container and structured HEX8 box generator.

Mirrors ``Mesh`` (generate_mesh.py:13-27 in the reference) and ``box_mesh``
(generate_mesh.py:151-189): node (i, j, k) of an (Nx+1, Ny+1, Nz+1) grid has
index (i*(Ny+1) + j)*(Nz+1) + k and cells list their nodes in VTK HEX8 order,
so meshes, solutions and per-cell data line up with the reference's.
"""
import numpy as np


class Mesh:
    """points (num_nodes, dim) float64 and cells (num_cells, 8) int32."""

    def __init__(self, points, cells, ele_type="HEX8"):
        self.points = np.ascontiguousarray(np.asarray(points, dtype=np.float64))
        self.cells = np.ascontiguousarray(np.asarray(cells, dtype=np.int32))
        self.ele_type = ele_type
        if self.cells.ndim != 2 or self.cells.shape[1] != 8:
            raise NotImplementedError("only HEX8 meshes (cells of 8 nodes) are supported")


class _BoxMesh:
    """What ``box_mesh`` returns: meshio-like ``points`` and ``cells_dict``."""

    def __init__(self, points, cells):
        self.points = points
        self.cells_dict = {"hexahedron": cells}


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


def get_meshio_cell_type(ele_type):
    if ele_type != "HEX8":
        raise NotImplementedError(f"element {ele_type} is not supported (HEX8 only)")
    return "hexahedron"
