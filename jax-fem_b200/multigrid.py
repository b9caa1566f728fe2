"""Geometric multigrid preconditioner for box-lattice meshes.

Stands in for the reference's optional AMGX path (solver.py:136-259) on the
meshes ``box_mesh`` builds (generate_mesh.py:151-189): tensor lattices with
node (i, j, k) = (i*ny + j)*nz + k, whose cells couple each node to lattice
neighbours only (a 27-point stencil): HEX8 boxes, and the TET4 boxes of
``box_mesh_gmsh`` (six tetrahedra per lattice cell, the same nodes).  Other
meshes raise ``NotImplementedError`` when ``precond='gmg'`` is asked for.

The hierarchy coarsens 2:1 per direction (a last odd interval stays one fine
cell wide) down to a few nodes per direction.  Prolongation is trilinear
interpolation in the lattice coordinates, restriction its transpose, and
coarse operators are Galerkin products P^T A P formed on the device
(``fem_mg_setup_*``).  A V-cycle smooths with Chebyshev-Jacobi polynomials
(``fem_mg_vcycle_*``) and solves a small coarsest level exactly (a dense
inverse formed by setup), and ``fem_mg_pcg_solve`` runs CG in FP64 with one
V-cycle per iteration.  The V-cycle is in FP64 or, for the mixed-precision
path, in FP32 on a rounded copy of the hierarchy, whose finest level smooths
with an FP16 copy of its values.
"""
import ctypes

import numpy as np
import torch

from . import _native as nat


def lattice_of(points, cells=None):
    """Nodes per direction (nx, ny, nz) and the coordinate of each lattice
    line if the points form a box lattice numbered as box_mesh numbers it
    (and, when ``cells`` are given, the cells are box_mesh's HEX8 cells),
    else None."""
    pts = np.asarray(points, dtype=np.float64)
    axes = [np.unique(pts[:, d]) for d in range(3)]
    n = tuple(len(a) for a in axes)
    if n[0] * n[1] * n[2] != len(pts) or min(n) < 2:
        return None
    I, J, K = np.meshgrid(np.arange(n[0]), np.arange(n[1]), np.arange(n[2]), indexing="ij")
    expect = np.stack([axes[0][I], axes[1][J], axes[2][K]], axis=-1).reshape(-1, 3)
    if not np.array_equal(expect, pts):
        return None
    if cells is not None and not np.array_equal(np.asarray(cells, dtype=np.int64), lattice_cells(n)):
        return None
    return n, axes


def lattice_cells(n):
    """HEX8 cells of a lattice with n = (nx, ny, nz) nodes, in box_mesh's
    cell and vertex order (VTK hexahedron)."""
    nx, ny, nz = n
    i, j, k = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), np.arange(nz - 1), indexing="ij")
    idx = lambda a, b, c: (a * ny + b) * nz + c  # noqa: E731
    v = [idx(i, j, k), idx(i + 1, j, k), idx(i + 1, j + 1, k), idx(i, j + 1, k),
         idx(i, j, k + 1), idx(i + 1, j, k + 1), idx(i + 1, j + 1, k + 1), idx(i, j + 1, k + 1)]
    return np.stack([a.reshape(-1) for a in v], axis=1).astype(np.int64)


def coarsen_1d(coords):
    """One direction's coarsening: (coarse coordinates, cpos, ilo, whi)."""
    c = len(coords) - 1  # fine cells
    cc = (c + 1) // 2
    cpos = np.minimum(2 * np.arange(cc + 1), c).astype(np.int32)
    i = np.arange(c + 1)
    ilo = np.minimum(i // 2, cc - 1).astype(np.int32)
    x0, x1 = coords[cpos[ilo]], coords[cpos[ilo + 1]]
    whi = (coords - x0) / (x1 - x0)
    return coords[cpos], cpos, ilo, whi


def stencil_of(n, row_ptr, col_idx):
    """(N, 27) block index of neighbour (dx, dy, dz) at (dx+1)*9 + (dy+1)*3 +
    (dz+1), -1 where absent."""
    N = n[0] * n[1] * n[2]
    rows = np.repeat(np.arange(N), np.diff(row_ptr))
    cols = np.asarray(col_idx, dtype=np.int64)

    def ijk(a):
        return a // (n[1] * n[2]), (a // n[2]) % n[1], a % n[2]

    ri, rj, rk = ijk(rows)
    ci, cj, ck = ijk(cols)
    d = np.stack([ci - ri, cj - rj, ck - rk])
    if np.abs(d).max() > 1:
        raise ValueError("pattern is not a 27-point lattice stencil")
    o = (d[0] + 1) * 9 + (d[1] + 1) * 3 + (d[2] + 1)
    st = np.full((N, 27), -1, dtype=np.int32)
    st[rows, o] = np.arange(len(cols), dtype=np.int32)
    return st


def _pattern(cells, N):
    lib = nat.lib()
    cells = np.ascontiguousarray(cells, dtype=np.int32)
    C = len(cells)
    rp = np.zeros(N + 1, dtype=np.int32)
    nnzb = nat.I64(0)
    nat.check(lib.fem_bsr_pattern(cells.ctypes.data, C, N, rp.ctypes.data, nnzb, None, 0, None, None), "pattern")
    col = np.zeros(nnzb.value, dtype=np.int32)
    sc = np.zeros((C, 64), dtype=np.int32)
    dg = np.zeros(N, dtype=np.int32)
    nat.check(lib.fem_bsr_pattern(cells.ctypes.data, C, N, rp.ctypes.data, nnzb, col.ctypes.data, col.size,
                                  sc.ctypes.data, dg.ctypes.data), "pattern")
    return rp, col


def _half_fine_enabled():
    import os
    return os.environ.get("FEM_MG_HALF", "1") != "0"


class Multigrid:
    """Lattice hierarchy of one mesh (``DeviceMesh``) with device buffers for
    one precision.  ``setup(A)`` forms the coarse operators of the FP64
    operator A; ``solve`` runs the V-cycle-preconditioned CG."""

    def __init__(self, dv, mesh_points, mesh_cells=None, fp32=False, max_levels=10, dense_coarse=True, nu_fine=0):
        lat = lattice_of(mesh_points, mesh_cells)
        if lat is None:
            raise NotImplementedError("precond 'gmg' needs a box-lattice mesh numbered as box_mesh numbers it")
        n, axes = lat
        try:  # the fine operator must couple lattice neighbours only
            stencil_of(n, dv.row_ptr.cpu().numpy(), dv.col_idx.cpu().numpy())
        except ValueError as e:
            raise NotImplementedError(f"precond 'gmg': the mesh's cells couple nodes beyond lattice "
                                      f"neighbours ({e})") from e
        self.vec, self.fp32 = dv.vec, fp32
        dev, dt = dv.device, (torch.float32 if fp32 else torch.float64)
        self._keep = []
        self.levels = (nat.FemMGLevel * max_levels)()
        self.nlevels = 0
        self.level_nodes = []
        self.mats = []  # per level (row_ptr, col_idx, values or None for level 0 in FP64), for inspection
        self._lmax = torch.zeros(max_levels, dtype=torch.int64, device=dev)  # FP64 bits, written by setup
        fine_rp, fine_ci = dv.row_ptr.cpu().numpy(), dv.col_idx.cpu().numpy()
        transfer = None  # (cpos, ilo, whi) from the finer level to this one
        while True:
            l = self.nlevels
            N = n[0] * n[1] * n[2]
            if l == 0:
                rp_d, ci_d = dv.row_ptr, dv.col_idx
                st = stencil_of(n, fine_rp, fine_ci)
                nnzb = dv.nnzb
            else:
                rp, ci = _pattern(lattice_cells(n), N)
                rp_d, ci_d = torch.from_numpy(rp).to(dev), torch.from_numpy(ci).to(dev)
                st = stencil_of(n, rp, ci)
                nnzb = len(ci)
            st_d = torch.from_numpy(st).to(dev)
            nd = N * self.vec
            L = self.levels[l]
            L.nodes[0], L.nodes[1], L.nodes[2] = n
            L.n_brows = N
            L.row_ptr, L.col_idx, L.stencil = rp_d.data_ptr(), ci_d.data_ptr(), st_d.data_ptr()
            bufs = {k: torch.zeros(max(nd, 2), dtype=dt, device=dev) for k in ("dinv", "x", "b", "r", "d0", "d1")}
            for k, t in bufs.items():
                setattr(L, k, t.data_ptr())
            vals = None
            if l > 0 or fp32:
                vals = torch.zeros(nnzb * self.vec * self.vec, dtype=dt, device=dev)
                L.vals = vals.data_ptr()
            if transfer is not None:
                L.cpos, L.ilo, L.whi = (t.data_ptr() for t in transfer)
            L.lmax = self._lmax.data_ptr() + 8 * l
            self._keep += [rp_d, ci_d, st_d, vals, *bufs.values(), *(transfer or ())]
            self.level_nodes.append(n)
            self.mats.append((rp_d, ci_d, vals))
            self.nlevels += 1
            if self.nlevels >= max_levels or min(a - 1 for a in n) < 4 or N <= 64:
                break
            parts = [coarsen_1d(a) for a in axes]
            axes = [q[0] for q in parts]
            n = tuple(len(a) for a in axes)
            transfer = (torch.from_numpy(np.concatenate([q[1] for q in parts]).astype(np.int32)).to(dev),
                        torch.from_numpy(np.concatenate([q[2] for q in parts]).astype(np.int32)).to(dev),
                        torch.from_numpy(np.concatenate([q[3] for q in parts]).astype(np.float64)).to(dev))
        # smoothing steps on the finest level (0: the V-cycle's nu)
        self.levels[0].nu = int(nu_fine)
        # An FP32 hierarchy smooths its finest level with an FP16 copy of the
        # values (scaled by a power of two, written by every setup): the
        # V-cycle's two finest-level products then read half the bytes.  The
        # CG operator keeps the FP32 values.  FEM_MG_HALF=0 turns it off.
        self.half_fine = bool(fp32) and _half_fine_enabled()
        if self.half_fine:
            self._vals16 = torch.empty(dv.nnzb * self.vec * self.vec, dtype=torch.float16, device=dev)
            self._scale16 = torch.zeros(2, dtype=torch.float64, device=dev)
            self.levels[0].vals_lo = self._vals16.data_ptr()
            self.levels[0].lo_scale = self._scale16.data_ptr()
        # a coarsest level of at most FEM_MG_DENSE_MAX unknowns is solved
        # exactly with a dense inverse (formed by setup) instead of smoothed
        last = self.levels[self.nlevels - 1]
        self._cinv = None
        if dense_coarse and last.n_brows * self.vec <= nat.FEM_MG_DENSE_MAX:
            nc = last.n_brows * self.vec
            self._cinv = torch.zeros(nc * nc, dtype=torch.float64, device=dev)
            last.cinv = self._cinv.data_ptr()
        self._work = None
        self._fine_ref = None
        # coarse-operator reuse bookkeeping (solver.mg_solve)
        self.setup_for, self.solves_on_coarse, self.first_rate, self.last_rate = None, 0, None, None
        nb = nat.lib().fem_mg_setup_scratch_bytes(self.vec, self.levels[0].n_brows, int(fp32))
        self._scratch = torch.empty(max(int(nb), 16), dtype=torch.uint8, device=dev)

    def setup(self, A, fine_only=False):
        """Coarse operators and smoother bounds for the operator A (a
        ``BSRMatrix`` on this mesh's pattern): FP64, or FP32 for an FP32
        hierarchy (then its finest level is A itself).  With ``fine_only``
        only the finest level takes A's values (and its Jacobi scaling and
        bound); the coarse levels keep the operators of the last full setup."""
        lib = nat.lib()
        if A.vals.dtype != torch.float64 and not (self.fp32 and A.vals.dtype == torch.float32):
            raise TypeError("the multigrid hierarchy is formed from the FP64 operator (or FP32 for an FP32 hierarchy)")
        if fine_only and self.setup_for is None:
            raise RuntimeError("fine_only needs an earlier full setup")
        nl = 1 if fine_only else self.nlevels
        if self.fp32:
            fine64 = None
            if A.vals.dtype == torch.float32:
                self.levels[0].vals = A.vals.data_ptr()
                self._fine32 = A.vals
            else:
                self.levels[0].vals = self.mats[0][2].data_ptr()
                fine64 = nat.ptr(A.vals)
            nat.check(lib.fem_mg_setup_f32(self.vec, nl, ctypes.byref(self.levels), fine64,
                                           nat.ptr(self._scratch), self._scratch.numel(), nat.stream_ptr()),
                      "mg_setup_f32")
        else:
            self.levels[0].vals = A.vals.data_ptr()
            if self._fine_ref is not A.vals:
                self._keep.append(A.vals)
                self._fine_ref = A.vals
            nat.check(lib.fem_mg_setup_f64(self.vec, nl, ctypes.byref(self.levels), nat.ptr(self._scratch),
                                           self._scratch.numel(), nat.stream_ptr()), "mg_setup_f64")
        if not fine_only:
            self.solves_on_coarse = 0
        self.setup_for = A

    def lmax(self):
        """Per-level Gershgorin bounds of the Jacobi-scaled operators (reads the device)."""
        return self._lmax[: self.nlevels].view(torch.float64).tolist()

    def vcycle(self, rhs, z, nu=2, coarse_steps=8, ratio=25.0):
        fn = nat.lib().fem_mg_vcycle_f32 if self.fp32 else nat.lib().fem_mg_vcycle_f64
        nat.check(fn(self.vec, self.nlevels, ctypes.byref(self.levels), nu, coarse_steps, float(ratio),
                     nat.ptr(rhs), nat.ptr(z), nat.stream_ptr()), "mg_vcycle")

    def solve(self, A, b, x, rtol, atol=0.0, maxiter=1000, nu=2, coarse_steps=8, ratio=25.0, check_every=4):
        """CG on A x = b with one V-cycle per iteration; x holds the initial
        guess.  CG is FP64; A is FP64, or FP32 (the products accumulate in
        FP64).  Returns (iterations, true relative residual)."""
        lib = nat.lib()
        n_brows = A.n_brows
        nb = lib.fem_mg_pcg_workspace_bytes(self.vec, n_brows)
        if self._work is None or self._work.numel() < nb:
            self._work = torch.empty(int(nb), dtype=torch.uint8, device=b.device)
        it = ctypes.c_int(0)
        rel = ctypes.c_double(0.0)
        if A.vals.dtype == torch.float32 and not self.fp32:
            raise TypeError("an FP32 operator needs the FP32 hierarchy")
        fn = lib.fem_mg_pcg_solve_mixed if A.vals.dtype == torch.float32 else lib.fem_mg_pcg_solve
        nat.check(fn(self.vec, n_brows, nat.ptr(A.row_ptr), nat.ptr(A.col_idx), nat.ptr(A.vals),
                                       nat.ptr(b), nat.ptr(x), float(rtol), float(atol), int(maxiter),
                                       int(check_every), self.nlevels, ctypes.byref(self.levels), int(self.fp32),
                                       int(nu), int(coarse_steps), float(ratio), nat.ptr(self._work), int(nb),
                                       ctypes.byref(it), ctypes.byref(rel), nat.stream_ptr()), "mg_pcg_solve")
        return it.value, rel.value
