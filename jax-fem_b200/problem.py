"""``Problem``: the reference's plugin API over the B200 kernels.

Same class name, constructor fields and hooks as the reference
(problem.py:15-128, 184-187, 462-556): subclass it, override
``get_tensor_map`` (returning a registered law, see ``laws``),
optionally ``get_mass_map`` / ``get_surface_maps`` (u-independent loads),
``custom_init`` and ``set_params``, and pass ``dirichlet_bc_info`` /
``location_fns`` exactly as for the reference.

What changes underneath: per-cell kernels, assembly, Dirichlet elimination
and solves run in libjaxfem_b200 on the current CUDA device; solutions,
residuals and internal variables are torch CUDA tensors (float64).
"""
from dataclasses import dataclass
from typing import Any

import numpy as np
import torch

from . import _native as nat
from .fe import FiniteElement
from .generate_mesh import Mesh
from .laws import J2Plasticity, NeoHookean, SIMPElastic, as_law


class BSRMatrix:
    """Block-CSR matrix on the device (vec x vec blocks, sorted columns)."""

    def __init__(self, vec, row_ptr, col_idx, diag, vals):
        self.vec, self.row_ptr, self.col_idx, self.diag, self.vals = vec, row_ptr, col_idx, diag, vals
        self.n_brows = row_ptr.numel() - 1
        self.shape = (self.n_brows * vec, self.n_brows * vec)

    @property
    def dtype(self):
        return self.vals.dtype

    def matvec(self, x, out=None):
        x = x.to(self.vals.dtype).contiguous()
        out = torch.empty_like(x) if out is None else out
        fn = nat.lib().fem_bsr_spmv_f64 if self.vals.dtype == torch.float64 else nat.lib().fem_bsr_spmv_f32
        nat.check(fn(self.vec, self.n_brows, nat.ptr(self.row_ptr), nat.ptr(self.col_idx),
                     nat.ptr(self.vals), nat.ptr(x), nat.ptr(out), nat.stream_ptr()), "bsr_spmv")
        return out

    def __matmul__(self, x):
        return self.matvec(x)

    def to_scipy(self):
        """Host copy as scipy CSR (tests / debugging)."""
        import scipy.sparse as sp
        v = self.vec
        rp = self.row_ptr.cpu().numpy()
        ci = self.col_idx.cpu().numpy()
        vals = self.vals.double().cpu().numpy().reshape(-1, v, v)
        return sp.bsr_matrix((vals, ci, rp), shape=self.shape).tocsr()


class DeviceMesh:
    """Mesh arrays, block-CSR pattern and cell->block scatter map on the device."""

    def __init__(self, mesh, vec, device):
        cells = np.ascontiguousarray(mesh.cells, dtype=np.int32)
        C, N = cells.shape[0], mesh.points.shape[0]
        nen = cells.shape[1]
        lib = nat.lib()
        row_ptr = np.zeros(N + 1, dtype=np.int32)
        nnzb = nat.I64(0)
        nat.check(lib.fem_bsr_pattern_nen(cells.ctypes.data, C, nen, N, row_ptr.ctypes.data, nnzb, None, 0,
                                          None, None), "bsr_pattern(count)")
        col = np.zeros(max(1, nnzb.value), dtype=np.int32)
        scatter = np.zeros((max(1, C), nen * nen), dtype=np.int32)
        diag = np.zeros(max(1, N), dtype=np.int32)
        nat.check(lib.fem_bsr_pattern_nen(cells.ctypes.data, C, nen, N, row_ptr.ctypes.data, nnzb,
                                          col.ctypes.data, col.size, scatter.ctypes.data, diag.ctypes.data),
                  "bsr_pattern(fill)")
        tmap = np.zeros(max(1, nnzb.value), dtype=np.int32)
        nat.check(lib.fem_bsr_transpose_map(row_ptr.ctypes.data, col.ctypes.data, N, tmap.ctypes.data),
                  "bsr_transpose_map")
        self.vec, self.num_cells, self.num_nodes, self.nnzb, self.nen = vec, C, N, int(nnzb.value), nen
        self.ndofs = N * vec
        self.device = device
        self.points = torch.from_numpy(np.ascontiguousarray(mesh.points, dtype=np.float64)).to(device)
        self.cells = torch.from_numpy(cells).to(device)
        self.row_ptr = torch.from_numpy(row_ptr).to(device)
        self.col_idx = torch.from_numpy(col[: self.nnzb]).to(device)
        self.scatter = torch.from_numpy(scatter[:C]).to(device).contiguous()
        self.diag = torch.from_numpy(diag[:N]).to(device)
        self.transpose = torch.from_numpy(tmap[: self.nnzb]).to(device)

    def new_matrix(self, dtype):
        vals = torch.zeros(self.nnzb * self.vec * self.vec, dtype=dtype, device=self.device)
        return BSRMatrix(self.vec, self.row_ptr, self.col_idx, self.diag, vals)


class CellKernelLaw:
    """What ``problem.law`` is on the cell-kernel path: no registered kernel
    (law_id None: treated as nonlinear by the Newton forcing)."""
    law_id = None
    vec = None

    def params(self):
        return []


def _to_dev(x, device, dtype=torch.float64):
    if isinstance(x, torch.Tensor):
        return x.detach().to(device=device, dtype=dtype).contiguous()
    return torch.as_tensor(np.asarray(x), dtype=dtype, device=device).contiguous()


@dataclass
class Problem:
    """Fields on meshes of one or several element types (3D, or 2D on the
    cell-kernel path); see the module docstring.  Fields as the reference's."""
    mesh: Mesh
    vec: int
    dim: int
    ele_type: str = "HEX8"
    quadrature_rule: Any = None
    quadrature_order: int = None
    dirichlet_bc_info: list = None
    location_fns: list = None
    additional_info: tuple = ()

    def __post_init__(self):
        # one variable, or one per entry of a mesh list (problem.py:56-84)
        if isinstance(self.mesh, list):
            n = len(self.mesh)
            meshes = list(self.mesh)
            vecs = list(self.vec) if isinstance(self.vec, list) else [self.vec] * n
            etypes = list(self.ele_type) if isinstance(self.ele_type, list) else [self.ele_type] * n
            bcs = list(self.dirichlet_bc_info) if self.dirichlet_bc_info is not None else [None] * n
        else:
            n, meshes, vecs, etypes, bcs = 1, [self.mesh], [self.vec], [self.ele_type], [self.dirichlet_bc_info]
        pick = lambda v, i: v[i] if isinstance(v, list) else v  # noqa: E731
        meshes = [m if isinstance(m, Mesh) else Mesh(m.points, m.cells, e) for m, e in zip(meshes, etypes)]
        self.fes = [FiniteElement(mesh=meshes[i], vec=vecs[i], dim=self.dim, ele_type=etypes[i],
                                  quadrature_rule=pick(self.quadrature_rule, i),
                                  quadrature_order=pick(self.quadrature_order, i),
                                  dirichlet_bc_info=bcs[i]) for i in range(n)]
        self.num_vars = n
        if n == 1:
            self.mesh, self.vec, self.ele_type, self.dirichlet_bc_info = meshes[0], vecs[0], etypes[0], bcs[0]
        else:
            self.mesh, self.vec, self.ele_type, self.dirichlet_bc_info = meshes, vecs, etypes, bcs
        self.cells_list = [fe.cells for fe in self.fes]
        if any(fe.num_cells != self.fes[0].num_cells for fe in self.fes):
            raise ValueError("all variables must have the same number of cells")
        self.num_cells = self.fes[0].num_cells
        self.boundary_inds_list = self.fes[0].get_boundary_conditions_inds(self.location_fns)
        self.offset = [0]
        for fe in self.fes[:-1]:
            self.offset.append(self.offset[-1] + fe.num_total_dofs)
        self.num_total_dofs_all_vars = self.offset[-1] + self.fes[-1].num_total_dofs
        self.num_nodes_cumsum = np.cumsum([0] + [fe.num_nodes for fe in self.fes])
        self.internal_vars = ()
        self.internal_vars_surfaces = [() for _ in range(len(self.boundary_inds_list))]
        self._dev = None
        self._cells = None
        self._cell_path = None
        self._elem = None
        self._bc_cache = None
        self._fext = None
        self._law = None
        self.custom_init(*self.additional_info)
        if hasattr(self, "get_surface_maps"):
            assert len(self.boundary_inds_list) == len(self.get_surface_maps())
        elif hasattr(self, "get_universal_kernels_surface"):
            assert len(self.boundary_inds_list) == len(self.get_universal_kernels_surface())
        else:
            assert len(self.boundary_inds_list) == 0, "Missing definitions for surface integral"

    # ---- hooks (problem.py:184-187, 493-556) ---------------------------------
    def custom_init(self, *args):
        pass

    def set_params(self, params):
        raise NotImplementedError("Child class must implement this function!")

    # ---- helpers ---------------------------------------------------------------
    @property
    def cell_path(self):
        """True when the weak form is user code run by the cell-kernel path
        (cellpath.py): a universal kernel, several variables, a tensor map
        that is not a registered law, no tensor map, mass / surface maps
        that depend on u, or a 2D problem (the registered-law CUDA kernels
        are 3D).  False: the registered-law kernels."""
        if self._cell_path is None:
            cp = (self.num_vars > 1 or self.dim == 2 or hasattr(self, "get_universal_kernel")
                  or hasattr(self, "get_universal_kernels_surface") or not hasattr(self, "get_tensor_map"))
            if not cp:
                try:
                    as_law(self.get_tensor_map(), self.vec, self.dim)
                except NotImplementedError:
                    cp = True
            fe = self.fes[0]
            if not cp and hasattr(self, "get_mass_map"):
                cp = fe.depends_on_u(self.get_mass_map())
            if not cp and hasattr(self, "get_surface_maps"):
                cp = any(fe.depends_on_u(m) for m in self.get_surface_maps())
            self._cell_path = cp
        return self._cell_path

    @property
    def law(self):
        if self._law is None:
            if self.cell_path:
                self._law = CellKernelLaw()
            else:
                self._law = as_law(self.get_tensor_map(), self.vec, self.dim)
        return self._law

    def device(self):
        return torch.device("cuda", torch.cuda.current_device())

    def dev(self):
        """Device mesh + pattern, built on first use (the scalar CSR system of
        all dofs on the cell-kernel path)."""
        if self._dev is None:
            if not torch.cuda.is_available():
                raise nat.FEMNativeError(nat.FEM_ERR_CUDA, "no CUDA device: this path has no CPU fallback")
            nat.load()
            if self.cell_path:
                from .cellpath import CellPath
                self._cells = CellPath(self, self.device())
                self._dev = self._cells.sys
            else:
                self._dev = DeviceMesh(self.mesh, self.vec, self.device())
        return self._dev

    @property
    def hex8_kernel(self):
        """True when cells go through the HEX8 kernel (HEX8 with its default
        2x2x2 rule); other element types and rules use the general one."""
        fe = self.fes[0]
        return fe.ele_type == "HEX8" and fe.num_quads == 8 and fe.quadrature_order == 2

    def element_tables(self):
        """(reference shape gradients (nq, nen, 3), weights (nq,)) on the device."""
        if self._elem is None:
            fe = self.fes[0]
            d = self.dev().device
            self._elem = (torch.from_numpy(np.ascontiguousarray(fe.shape_grads_ref, dtype=np.float64)).to(d),
                          torch.from_numpy(np.ascontiguousarray(fe.quad_weights, dtype=np.float64)).to(d))
        return self._elem

    def unflatten_fn_sol_list(self, dofs):
        """Flat dofs -> [(num_nodes_i, vec_i), ...] (views)."""
        dofs = dofs.reshape(-1)
        return [dofs[off:off + fe.num_total_dofs].reshape(-1, fe.vec) for off, fe in zip(self.offset, self.fes)]

    def unflatten_fn_dof(self, cell_sol_flat):
        """A cell's flat dofs -> [(num_nodes_i, vec_i), ...] per variable (for kernels)."""
        out, k = [], 0
        for fe in self.fes:
            out.append(cell_sol_flat[k:k + fe.num_nodes * fe.vec].reshape(fe.num_nodes, fe.vec))
            k += fe.num_nodes * fe.vec
        return out

    def _dirichlet_compact(self):
        """Constrained global dofs (sorted) and their values; where conditions
        overlap the later one wins, as in FiniteElement.dirichlet_arrays.  The
        selection is kept while the conditions' nodes and components stay the
        same (load stepping changes values only)."""
        struct, vals, off = [], [], 0
        for fe in self.fes:
            for nodes, v, val in zip(fe.node_inds_list, fe.vec_inds_list, fe.vals_list):
                struct.append((off, fe.vec, nodes, v))
                vals.append(np.broadcast_to(np.asarray(val, dtype=np.float64), np.shape(nodes)))
            off += fe.num_total_dofs
        if not struct:
            return np.zeros(0, dtype=np.int64), np.zeros(0, dtype=np.float64)
        x = np.concatenate(vals)
        cache = self.__dict__.get("_bc_compact")
        if cache is not None and len(cache[0]) == len(struct) and all(
                a[0] == b[0] and a[1] == b[1] and np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])
                for a, b in zip(cache[0], struct)):
            return cache[1], x[cache[2]]
        d = np.concatenate([o + np.asarray(nodes, dtype=np.int64) * vec + v for o, vec, nodes, v in struct])
        u, last = np.unique(d[::-1], return_index=True)  # first in reverse = last in order
        sel = len(d) - 1 - last
        self._bc_compact = ([(o, vec, np.array(nodes), np.array(v)) for o, vec, nodes, v in struct], u, sel)
        return u, x[sel]

    def dirichlet_device(self):
        """(mask uint8, values f64) over all dofs on the device, refreshed after
        BC updates.  A refresh copies only the constrained dofs' values and
        scatters them on the device; the mask (and the index copy) is reused
        while the constrained dofs stay the same (load stepping)."""
        key = tuple(fe.bc_version for fe in self.fes)
        if self._bc_cache is None or self._bc_cache[0] != key:
            d = self.dev().device
            n = self.num_total_dofs_all_vars
            dofs, vals = self._dirichlet_compact()
            prev = self._bc_cache
            if prev is not None and np.array_equal(prev[3], dofs):
                mask, idx = prev[1], prev[4]
            else:
                idx = torch.from_numpy(dofs).to(d)
                mask = torch.zeros(n, dtype=torch.uint8, device=d)
                mask[idx] = 1
            ubc = torch.zeros(n, dtype=torch.float64, device=d)
            ubc[idx] = torch.from_numpy(np.ascontiguousarray(vals)).to(d)
            self._bc_cache = (key, mask, ubc, dofs, idx)
        return self._bc_cache[1], self._bc_cache[2]

    def surface_load_vectors(self):
        """Per-surface load vectors int surface_map . v ds (device f64)."""
        if not hasattr(self, "_surface_loads"):
            loads = []
            if hasattr(self, "get_surface_maps"):
                for binds, smap in zip(self.boundary_inds_list, self.get_surface_maps()):
                    loads.append(self.fes[0].surface_load(smap, binds))
            d = self.dev().device
            self._surface_loads = [torch.from_numpy(np.ascontiguousarray(f)).to(d) for f in loads]
        return self._surface_loads

    def external_load(self):
        """f_ext = int mass_map . v dx + sum_surfaces int surface_map . v ds (device f64);
        zero on the cell-kernel path, whose kernels hold these terms."""
        if self._fext is None:
            d = self.dev().device
            f = torch.zeros(self.num_total_dofs_all_vars, dtype=torch.float64, device=d)
            if self.cell_path:
                self._fext = f
                return f
            if hasattr(self, "get_mass_map"):
                f += torch.from_numpy(self.fes[0].body_load(self.get_mass_map())).to(d)
            for fs in self.surface_load_vectors():
                f += fs
            self._fext = f
        return self._fext

    def law_ivars(self, ivars=None):
        """Device tensors (iv0, iv1, iv2) of the law's internal variables,
        per (cell, quadrature point)."""
        ivars = self.internal_vars if ivars is None else ivars
        law = self.law
        d = self.dev().device
        C, Q = self.num_cells, self.fes[0].num_quads
        if isinstance(law, SIMPElastic):
            if len(ivars) < 1:
                raise ValueError("SIMPElastic needs internal_vars = [theta] (set_params)")
            th = _to_dev(ivars[0], d)
            if th.numel() == C:
                th = th.reshape(C, 1).expand(C, Q).contiguous()
            return (th.reshape(C, Q), None, None)
        if isinstance(law, NeoHookean):
            if len(ivars) == 0:
                return (None, None, None)
            sc = _to_dev(ivars[0], d)
            if sc.numel() == C:
                sc = sc.reshape(C, 1).expand(C, Q).contiguous()
            return (sc.reshape(C, Q), None, None)
        if isinstance(law, J2Plasticity):
            if len(ivars) < 2:
                raise ValueError("J2Plasticity needs internal_vars = [sigma_old, eps_old(, alpha_old)]")
            so = _to_dev(ivars[0], d).reshape(C, Q, 9)
            eo = _to_dev(ivars[1], d).reshape(C, Q, 9)
            ao = _to_dev(ivars[2], d).reshape(C, Q) if len(ivars) > 2 else torch.zeros(
                C, Q, dtype=torch.float64, device=d)
            return (so, eo, ao)
        return (None, None, None)

    # ---- assembly (problem.py:439-491) -----------------------------------------
    def assemble(self, dofs, res=None, vals=None, lift=None, dvec=None, bc=True, fp32=False,
                 ivars=None):
        """One fused pass of the cell kernel: residual, tangent, Dirichlet lift."""
        dv = self.dev()
        if self.cell_path:
            self._cells.assemble(dofs, res=res, vals=vals, lift=lift, dvec=dvec, bc=bc, fp32=fp32, ivars=ivars)
            return
        law = self.law
        mask, _ = self.dirichlet_device() if bc else (None, None)
        iv = self.law_ivars(ivars)
        pr, n = nat.params_array(law.params())
        tail = (dv.num_cells, dv.num_nodes, nat.ptr(dv.cells), nat.ptr(dv.points), nat.ptr(dofs), nat.ptr(iv[0]),
                nat.ptr(iv[1]), nat.ptr(iv[2]), nat.ptr(dv.scatter), nat.ptr(dv.diag), nat.ptr(dv.transpose),
                dv.nnzb, nat.ptr(mask) if bc else None, nat.ptr(dvec), nat.ptr(res), nat.ptr(lift),
                nat.ptr(vals), nat.stream_ptr())
        if self.hex8_kernel:
            fn = nat.lib().fem_assemble_f32 if fp32 else nat.lib().fem_assemble_f64
            nat.check(fn(law.law_id, pr, n, self.vec, *tail), "assemble")
        else:
            gref, wq = self.element_tables()
            fn = nat.lib().fem_assemble_elem_f32 if fp32 else nat.lib().fem_assemble_elem_f64
            nat.check(fn(law.law_id, pr, n, self.vec, dv.nen, wq.numel(), nat.ptr(gref), nat.ptr(wq), *tail),
                      "assemble_elem")
        if vals is not None and self.fes[0].ele_type in ("TET10", "HEX20", "HEX27"):
            # the state of this tangent, for p-multigrid's re-assembled coarse operator (pmultigrid.py)
            if getattr(self, "_tangent_state", None) is None or self._tangent_state.numel() != dofs.numel():
                self._tangent_state = torch.empty_like(dofs)
            self._tangent_state.copy_(dofs)

    def _flat_dofs(self, sol_list):
        d = self.dev().device
        if isinstance(sol_list, (list, tuple)):
            return torch.cat([_to_dev(s, d).reshape(-1) for s in sol_list[: self.num_vars]])
        return _to_dev(sol_list, d).reshape(-1)

    def compute_residual(self, sol_list):
        """Residual list (without Dirichlet rows applied), as the reference's."""
        dofs = self._flat_dofs(sol_list)
        res = torch.empty_like(dofs)
        self.assemble(dofs, res=res, bc=False)
        return self.unflatten_fn_sol_list(res + self.external_load())

    def newton_update(self, sol_list):
        """Residual list; also assembles the BC-eliminated tangent into ``self.A``."""
        dofs = self._flat_dofs(sol_list)
        res = torch.empty_like(dofs)
        if getattr(self, "A", None) is None or self.A.vals.dtype != torch.float64:
            self.A = self.dev().new_matrix(torch.float64)
        self.assemble(dofs, res=res, vals=self.A.vals)
        return self.unflatten_fn_sol_list(res + self.external_load())

    # ---- J2 state commit (test_plasticity.py:67-78) -----------------------------
    def update_j2_state(self, sol):
        """Commit the return map at the converged ``sol``: internal_vars <- new state."""
        if self.cell_path:  # the torch radial return at every quadrature point
            law = self.get_tensor_map() if hasattr(self, "get_tensor_map") else None
            if not isinstance(law, J2Plasticity):
                raise TypeError("update_j2_state needs a J2Plasticity law")
            self.dev()
            self.internal_vars = self._cells.j2_commit(self._flat_dofs(sol), law, self.internal_vars)
            return self.internal_vars
        law = self.law
        if not isinstance(law, J2Plasticity):
            raise TypeError("update_j2_state needs a J2Plasticity law")
        dv = self.dev()
        so, eo, ao = self.law_ivars()
        sn, en, an = torch.empty_like(so), torch.empty_like(eo), torch.empty_like(ao)
        dofs = self._flat_dofs(sol)
        pr, n = nat.params_array(law.params())
        state = (nat.ptr(dv.cells), nat.ptr(dv.points), nat.ptr(dofs), nat.ptr(so), nat.ptr(eo), nat.ptr(ao),
                 nat.ptr(sn), nat.ptr(en), nat.ptr(an), nat.stream_ptr())
        if self.hex8_kernel:
            nat.check(nat.lib().fem_j2_commit(pr, n, dv.num_cells, *state), "j2_commit")
        else:
            gref, wq = self.element_tables()
            nat.check(nat.lib().fem_j2_commit_elem(pr, n, dv.nen, wq.numel(), nat.ptr(gref), dv.num_cells, *state),
                      "j2_commit_elem")
        C, Q = self.num_cells, self.fes[0].num_quads
        self.internal_vars = [sn.reshape(C, Q, 3, 3), en.reshape(C, Q, 3, 3), an]
        return self.internal_vars

    def JxW(self):
        if not hasattr(self, "_jxw"):
            self._jxw = torch.from_numpy(self.fes[0].JxW()).to(self.dev().device)
        return self._jxw


def compliance(problem, sol, surface_index=0):
    """C = int t . u ds with t = -surface_map on one surface set
    (compute_compliance of the reference's topology-optimisation example).
    Differentiable in ``sol`` (a torch expression)."""
    f = problem.surface_load_vectors()[surface_index]
    u = sol[0] if isinstance(sol, (list, tuple)) else sol
    return -(f * u.reshape(-1)).sum()
