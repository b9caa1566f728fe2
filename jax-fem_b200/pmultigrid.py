"""p-multigrid preconditioner for the quadratic element types on box lattices.

Extends ``precond='gmg'`` (the reference's optional AMGX path,
solver.py:136-259) to TET10, HEX20 and HEX27 meshes whose corner nodes form
a box lattice (as ``box_mesh_gmsh`` builds them): the coarse space is the
linear element on the corner nodes (TET4 for TET10, HEX8 for HEX20 and
HEX27), on which the lattice hierarchy of ``multigrid.py`` runs.

- Prolongation P (all nodes <- corner nodes) evaluates the linear element's
  shape functions at each node's reference position: edge nodes take the
  mean of their two corners, face and centre nodes of their four and eight.
  It is stored as a block-CSR matrix (weight times the identity), P and P^T
  applied by the library's block-CSR product.
- The coarse operator is a rediscretisation: the linear element's tangent of
  the same law, assembled by the library at the corner values of the state
  the fine tangent was assembled at (per-cell means of the internal
  variables), with the fine Dirichlet dofs of the corner nodes eliminated.
- Smoothing on the fine level: Chebyshev polynomials in the 3x3
  block-Jacobi-scaled operator on [lmax/ratio, lmax], lmax from a power
  iteration; pre- and post-smoothing use the same polynomial, so the
  preconditioner is symmetric and the outer iteration is CG (FP64).
- Dirichlet dofs are projected out of the coarse residual and of the
  correction, which keeps the eliminated system's prescribed rows fixed.
"""
import math

import numpy as np
import torch

from . import _native as nat
from . import basis
from .multigrid import Multigrid, lattice_of
from .problem import BSRMatrix

_COARSE_ELEMENT = {"TET10": "TET4", "HEX20": "HEX8", "HEX27": "HEX8"}


class _Rect:
    """A rectangular block-CSR operator (rows x cols nodes) for y = M x."""

    def __init__(self, vec, row_ptr, col_idx, weights, device):
        self.vec = vec
        self.n_brows = len(row_ptr) - 1
        self.row_ptr = torch.from_numpy(np.ascontiguousarray(row_ptr, dtype=np.int32)).to(device)
        self.col_idx = torch.from_numpy(np.ascontiguousarray(col_idx, dtype=np.int32)).to(device)
        eye = np.eye(vec)
        vals = (np.asarray(weights, dtype=np.float64)[:, None, None] * eye[None]).reshape(-1)
        self.vals = torch.from_numpy(vals).to(device)

    def apply(self, x, y):
        nat.check(nat.lib().fem_bsr_spmv_f64(self.vec, self.n_brows, nat.ptr(self.row_ptr), nat.ptr(self.col_idx),
                                             nat.ptr(self.vals), nat.ptr(x), nat.ptr(y), nat.stream_ptr()),
                  "pmg transfer")
        return y


def _csr(rows, cols, w, n_rows):
    order = np.lexsort((cols, rows))
    rows, cols, w = rows[order], cols[order], w[order]
    rp = np.zeros(n_rows + 1, dtype=np.int64)
    np.add.at(rp, rows + 1, 1)
    return np.cumsum(rp), cols, w


def coarse_space(ele_type, points, cells):
    """(corner node ids, coarse cells, (rows, cols, weights) of P) for a mesh
    of a quadratic element type."""
    lin = _COARSE_ELEMENT[ele_type]
    nc = basis.NODES_PER_CELL[lin]
    corners = np.unique(cells[:, :nc])
    remap = np.full(len(points), -1, dtype=np.int64)
    remap[corners] = np.arange(len(corners))
    coarse_cells = remap[cells[:, :nc]].astype(np.int32)
    # weights of each local node from the cell's corners: the linear shape
    # functions at the node's reference coordinates
    W = basis.shape_fn(lin, basis.node_coords(ele_type))[0]  # (nen, nc)
    first = np.full(len(points), -1, dtype=np.int64)  # one cell (and local index) per node
    flat = cells.reshape(-1)
    pos = np.arange(flat.size)
    first[flat[::-1]] = pos[::-1]
    c, a = first // cells.shape[1], first % cells.shape[1]
    rows = np.repeat(np.arange(len(points)), nc)
    cols = coarse_cells[c].reshape(-1)
    w = W[a].reshape(-1)
    keep = np.abs(w) > 1e-14
    return corners, coarse_cells, (rows[keep], cols[keep], w[keep])


class PMultigrid:
    """Two-level p-multigrid (fine quadratic level, coarse linear lattice with
    its own hierarchy) with the interface ``solver.mg_solve`` uses."""

    def __init__(self, problem, fp32=False, max_levels=10, nu_fine=0):
        from .generate_mesh import Mesh
        from .problem import Problem
        fe = problem.fes[0]
        if fe.ele_type not in _COARSE_ELEMENT or problem.cell_path:
            raise NotImplementedError("p-multigrid is for TET10, HEX20 and HEX27 on the registered-law path")
        points, cells = fe.points, np.asarray(fe.cells, dtype=np.int64)
        corners, ccells, (rows, cols, w) = coarse_space(fe.ele_type, points, cells)
        lin = _COARSE_ELEMENT[fe.ele_type]
        cpts = points[corners]
        if lattice_of(cpts) is None:
            raise NotImplementedError("precond 'gmg' on quadratic cells needs the corner nodes to form a box "
                                      "lattice numbered as box_mesh numbers it")
        self.problem = problem
        self.vec = vec = problem.vec
        dev = problem.dev().device
        self.device = dev
        Nf, Nc = len(points), len(corners)
        self.P = _Rect(vec, *_csr(rows, cols, w, Nf), dev)
        self.PT = _Rect(vec, *_csr(cols, rows, w, Nc), dev)
        law = problem.law
        coarse_mesh = Mesh(cpts, ccells, lin)

        class Coarse(Problem):
            def get_tensor_map(self):
                return law

        self.coarse = Coarse(coarse_mesh, vec=vec, dim=3, ele_type=lin)
        self.corner_dofs = torch.from_numpy((corners[:, None] * vec + np.arange(vec)[None]).reshape(-1)).to(dev)
        self.coarse.dirichlet_device = self._coarse_bc
        self.mg = Multigrid(self.coarse.dev(), cpts, ccells if lin == "HEX8" else None, fp32=fp32,
                            max_levels=max_levels, nu_fine=nu_fine)
        self.fp32 = fp32
        self.Ac = self.coarse.dev().new_matrix(torch.float64)
        self.dinv = None
        self.lmax = None
        self.first_rate = self.last_rate = None
        self.solves_on_coarse = 0
        self.setup_for = None

    def _coarse_bc(self):
        mask, vals = self.problem.dirichlet_device()
        return mask[self.corner_dofs].contiguous(), vals[self.corner_dofs].contiguous()

    def _coarse_ivars(self):
        out = []
        Qc = self.coarse.fes[0].num_quads
        for t in self.problem.law_ivars():
            if t is None:
                continue
            m = t.mean(dim=1, keepdim=True)
            out.append(m.expand(m.shape[0], Qc, *m.shape[2:]).contiguous())
        return out

    # ---- setup -------------------------------------------------------------------
    def setup(self, A, fine_only=False):
        if A.vals.dtype != torch.float64:
            raise TypeError("p-multigrid works on the FP64 fine operator")
        vec, n = self.vec, A.n_brows * self.vec
        blocks = A.vals.view(-1, vec, vec)[A.diag.long()]
        inv = torch.linalg.inv(blocks)
        # persistent buffers: the captured CG iteration reads them by address
        if self.dinv is None or self.dinv.shape != inv.shape:
            self.dinv = inv.contiguous()
        else:
            self.dinv.copy_(inv)
        if self.fp32 and A.vals.is_cuda:
            # the mixed path smooths the fine level in FP32: FP32 copies of the
            # operator values and of the block-Jacobi inverse (the CG operator
            # product stays FP64)
            if getattr(self, "_A32", None) is None or self._A32.vals.numel() != A.vals.numel():
                self._A32 = BSRMatrix(A.vec, A.row_ptr, A.col_idx, A.diag, A.vals.float())
                self._dinv32 = self.dinv.float()
            else:
                self._A32.vals.copy_(A.vals)
                self._dinv32.copy_(self.dinv)
        else:
            self._A32 = None
        if not fine_only or self.lmax is None:
            # largest eigenvalue of D^-1 A by power iteration (x 1.1), at full
            # setups; solves on kept coarse operators keep it too.  It stays
            # on the device (the Chebyshev coefficients are formed there).
            g = torch.Generator(device=A.vals.device).manual_seed(0)
            x = torch.rand(n, dtype=torch.float64, device=A.vals.device, generator=g)
            y = torch.empty_like(x)
            lam = torch.ones((), dtype=torch.float64, device=A.vals.device)
            for _ in range(12):
                x /= x.norm()
                A.matvec(x, y)
                z = self._jacobi(y)
                lam = x.dot(z)
                x = z
            if getattr(self, "_lmax_t", None) is None or self._lmax_t.device != lam.device:
                self._lmax_t = torch.empty((), dtype=torch.float64, device=lam.device)
            self._lmax_t.copy_(1.1 * lam)
            self.lmax = self._lmax_t
        if not fine_only:
            state = getattr(self.problem, "_tangent_state", None)
            if state is None:
                raise RuntimeError("p-multigrid needs the state the fine tangent was assembled at")
            uc = state[self.corner_dofs].contiguous()
            self.coarse.assemble(uc, vals=self.Ac.vals, ivars=self._coarse_ivars())
            self.mg.setup(self.Ac)
            self.solves_on_coarse = 0
        self.setup_for = A

    def _jacobi(self, r):
        v = self.vec
        dinv = self.dinv if r.dtype == torch.float64 else self._dinv32
        return torch.bmm(dinv, r.view(-1, v, 1)).view(-1)

    # ---- preconditioner ------------------------------------------------------------
    def _chebyshev(self, A, b, z, nu, ratio, tmp, zero_start=False):
        """nu Chebyshev steps for A z = b from z (in place; z = 0 when
        zero_start), on [lmax/ratio, lmax].  sigma = theta/delta depends on
        the ratio only; 1/theta and 1/delta are device scalars."""
        sigma = (1.0 + 1.0 / ratio) / (1.0 - 1.0 / ratio)
        inv_theta = 2.0 / (self.lmax * (1.0 + 1.0 / ratio))
        inv_delta = 2.0 / (self.lmax * (1.0 - 1.0 / ratio))
        rho = 1.0 / sigma
        if zero_start:
            r = b.clone()
        else:
            A.matvec(z, tmp)
            r = b - tmp
        d = self._jacobi(r) * inv_theta
        for k in range(nu):
            z += d
            if k == nu - 1:
                break
            A.matvec(d, tmp)
            r -= tmp
            rho_new = 1.0 / (2.0 * sigma - rho)
            d = rho_new * rho * d + (2.0 * rho_new) * inv_delta * self._jacobi(r)
            rho = rho_new
        return z

    def apply(self, A, r, z, free, nu, coarse_steps, ratio, tmp):
        if getattr(self, "_A32", None) is not None:
            return self._apply32(r, z, free, nu, coarse_steps, ratio)
        z.zero_()
        self._chebyshev(A, r, z, nu, ratio, tmp, zero_start=True)
        A.matvec(z, tmp)
        r1 = (r - tmp) * free
        rc = self._rc
        self.PT.apply(r1, rc)
        rc *= self._free_c
        if self.fp32:
            zc32 = torch.zeros_like(rc, dtype=torch.float32)
            self.mg.vcycle(rc.float(), zc32, nu=nu, coarse_steps=coarse_steps, ratio=ratio)
            zc = zc32.double()
        else:
            zc = torch.zeros_like(rc)
            self.mg.vcycle(rc, zc, nu=nu, coarse_steps=coarse_steps, ratio=ratio)
        zc *= self._free_c
        self.P.apply(zc, tmp)
        z += tmp * free
        self._chebyshev(A, r, z, nu, ratio, tmp)
        z *= free
        return z

    def _apply32(self, r, z, free, nu, coarse_steps, ratio):
        """The same V-cycle with the fine-level smoothing and residual in FP32
        (FP32 operator copy and block-Jacobi inverse; transfers in FP64, the
        coarse lattice V-cycle in FP32); z (FP64) = the result."""
        A32 = self._A32
        r32 = r.float()
        f32 = free.float()
        z32 = torch.zeros_like(r32)
        t32 = torch.empty_like(r32)
        self._chebyshev(A32, r32, z32, nu, ratio, t32, zero_start=True)
        A32.matvec(z32, t32)
        r1 = ((r32 - t32) * f32).double()
        rc = self._rc
        self.PT.apply(r1, rc)
        rc *= self._free_c
        zc32 = torch.zeros_like(rc, dtype=torch.float32)
        self.mg.vcycle(rc.float(), zc32, nu=nu, coarse_steps=coarse_steps, ratio=ratio)
        zc = zc32.double() * self._free_c
        tmp = torch.empty_like(r)
        self.P.apply(zc, tmp)
        z32 += tmp.float() * f32
        self._chebyshev(A32, r32, z32, nu, ratio, t32)
        torch.mul(z32, f32, out=t32)
        z.copy_(t32)
        return z

    # ---- outer CG ----------------------------------------------------------------
    def _buffers(self, b):
        """Persistent CG state (the captured iteration reads it by address)."""
        n, dev = b.numel(), b.device
        if getattr(self, "_cg", None) is None or self._cg["x"].numel() != n or self._cg["x"].device != dev:
            e = lambda: torch.empty(n, dtype=torch.float64, device=dev)  # noqa: E731
            s = lambda: torch.empty((), dtype=torch.float64, device=dev)  # noqa: E731
            self._cg = {"x": e(), "r": e(), "p": e(), "q": e(), "z": e(), "tmp": e(), "free": e(), "rz": s(),
                        "pq_min": s()}
            self._graph = None
        return self._cg

    def _iteration(self, A, nu, coarse_steps, ratio):
        """One CG iteration on the persistent state, scalars on the device:
        q = A p, x += alpha p, r -= alpha q, then the preconditioned residual
        z and the next direction."""
        c = self._cg
        A.matvec(c["p"], c["q"])
        pq = c["p"].dot(c["q"])
        torch.minimum(c["pq_min"], pq, out=c["pq_min"])
        alpha = c["rz"] / pq
        c["x"].add_(alpha * c["p"])
        c["r"].sub_(alpha * c["q"])
        self.apply(A, c["r"], c["z"], c["free"], nu, coarse_steps, ratio, c["tmp"])
        rz_new = c["r"].dot(c["z"])
        c["p"].mul_(rz_new / c["rz"]).add_(c["z"])
        c["rz"].copy_(rz_new)

    def solve(self, A, b, x, rtol, atol=0.0, maxiter=1000, nu=2, coarse_steps=8, ratio=25.0, check_every=4):
        """Preconditioned CG on A x = b (x: initial guess, in place).  The
        scalars stay on the device and the residual is read every
        ``check_every`` iterations.  On the GPU the iteration (operator
        product, updates and the whole preconditioner: fine-level Chebyshev
        smoothing, transfers and the coarse lattice V-cycle) is captured once
        as a CUDA graph and replayed; the iteration that triggers a capture
        runs eagerly.  Returns (iterations, relative residual)."""
        mask, _ = self.problem.dirichlet_device()
        c = self._buffers(b)
        c["free"].copy_(~mask.bool())
        fc = c["free"][self.corner_dofs]
        if getattr(self, "_free_c", None) is None or self._free_c.shape != fc.shape:
            self._free_c = fc.contiguous()
        else:
            self._free_c.copy_(fc)
        if getattr(self, "_rc", None) is None or self._rc.numel() != self.PT.n_brows * self.vec:
            self._rc = torch.empty(self.PT.n_brows * self.vec, dtype=torch.float64, device=b.device)
        c["x"].copy_(x)
        A.matvec(c["x"], c["tmp"])
        torch.sub(b, c["tmp"], out=c["r"])
        bn = float(b.norm())
        target = max(rtol * bn, atol)
        rn = float(c["r"].norm())
        if rn <= target:
            return 0, rn / bn if bn > 0 else rn
        self.apply(A, c["r"], c["z"], c["free"], nu, coarse_steps, ratio, c["tmp"])
        c["p"].copy_(c["z"])
        c["rz"].copy_(c["r"].dot(c["z"]))
        c["pq_min"].fill_(math.inf)
        key = (A.vals.data_ptr(), A.n_brows, nu, coarse_steps, float(ratio))
        use_graph = b.is_cuda and _graphs_enabled()
        for it in range(1, maxiter + 1):
            if use_graph and self._graph is not None and self._graph_key == key:
                self._graph.replay()
            else:
                self._iteration(A, nu, coarse_steps, ratio)
                if use_graph:
                    self._capture(A, nu, coarse_steps, ratio, key)
            if it % check_every == 0 or it == maxiter:
                rn = float(c["r"].norm())
                pqm = float(c["pq_min"])
                if not (pqm > 0.0) or not math.isfinite(rn):
                    raise nat.FEMNativeError(nat.FEM_ERR_BREAKDOWN, f"p-multigrid CG breakdown (min p.Ap = {pqm})")
                if rn <= target:
                    x.copy_(c["x"])
                    return it, rn / bn if bn > 0 else rn
        raise nat.FEMNativeError(nat.FEM_ERR_NOT_CONVERGED,
                                 f"p-multigrid CG: {maxiter} iterations, relres {rn / bn if bn > 0 else rn:.3e}")

    def _capture(self, A, nu, coarse_steps, ratio, key):
        """Record one CG iteration as a CUDA graph (recording runs nothing)."""
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._iteration(A, nu, coarse_steps, ratio)
        self._graph, self._graph_key = g, key


def _graphs_enabled():
    import os
    return os.environ.get("FEM_PMG_GRAPHS", "1") != "0"
