"""The cell-kernel path: weak forms written as user code.

Covers what the registered laws do not: ``get_universal_kernel`` and
``get_universal_kernels_surface`` (problem.py:260-340 in the reference),
multi-variable problems (problem.py:56-128), tensor maps that are not
registered laws, and mass / surface maps that depend on u
(problem.py:189-259).  The user's functions are torch code.  The host
evaluates the cell residual and its Jacobian on the device -- forward mode
(``torch.func.jacfwd``) over batches of cells (``torch.func.vmap``), the
counterpart of the reference's value_and_jacfwd under jax.vmap
(problem.py:262-266, 359-396) -- and the library's ``fem_scatter_cells_*``
adds them into the residual and a scalar CSR tangent (a block-CSR matrix
with 1x1 blocks over all dofs) with Dirichlet elimination and the lift.
Newton, the Krylov solvers and the outer loops are those of the law path.

Kernel signatures are the reference's, with torch tensors:

- universal kernel (per cell): ``(cell_sol_flat (nd,), x (nq, dim),
  cell_shape_grads (nq, sum nen, dim), cell_JxW (num_vars, nq),
  cell_v_grads_JxW (nq, sum nen, 1, dim), *cell_internal_vars) -> (nd,)``;
- surface universal kernel (per selected face): ``(cell_sol_flat,
  x (nfq, dim), face_shape_vals (nfq, sum nen), face_shape_grads
  (nfq, sum nen, dim), face_nanson_scale (num_vars, nfq),
  *cell_internal_vars_surface) -> (nd,)``;
- ``tensor_map(u_grad (vec, dim), *ivars)``, ``mass_map(u (vec,), x (dim,),
  *ivars)``, ``surface_map(u, x, *ivars_surface)`` per quadrature point,
  on the first variable (problem.py:189-259).

dim is 3, or 2 for the 2D element types (QUAD4, QUAD8, TRI3, TRI6), which
always run here.  A registered law on a 2D problem is its plane-strain
form (``laws.plane_strain``).

Inside torch kernels the element tables are ``fe.shape_vals_t`` and
``fe.face_shape_vals_t`` (torch copies of ``shape_vals`` and
``face_shape_vals`` on the problem's device); ``problem.unflatten_fn_dof``
splits a cell's flat dofs into the per-variable (nen_i, vec_i) blocks.
"""
import numpy as np
import torch
from torch.func import jacfwd, vmap

from . import _native as nat

# cells per batch: the batch's Jacobians take about this many doubles (the
# forward-mode intermediates a few times more); larger batches launch fewer
# kernels per cell
_BATCH_ENTRIES = 1 << 25


class CellSystem:
    """The scalar CSR pattern of a cell-kernel problem on the device (the
    counterpart of ``DeviceMesh`` with vec = 1 over all dofs)."""

    def __init__(self, cell_dofs, ndofs, device):
        cells = np.ascontiguousarray(cell_dofs, dtype=np.int32)
        C, nd = cells.shape
        lib = nat.lib()
        row_ptr = np.zeros(ndofs + 1, dtype=np.int32)
        nnz = nat.I64(0)
        nat.check(lib.fem_bsr_pattern_nen(cells.ctypes.data, C, nd, ndofs, row_ptr.ctypes.data, nnz, None, 0,
                                          None, None), "cell pattern(count)")
        col = np.zeros(max(1, nnz.value), dtype=np.int32)
        scatter = np.zeros((max(1, C), nd * nd), dtype=np.int32)
        diag = np.zeros(max(1, ndofs), dtype=np.int32)
        nat.check(lib.fem_bsr_pattern_nen(cells.ctypes.data, C, nd, ndofs, row_ptr.ctypes.data, nnz,
                                          col.ctypes.data, col.size, scatter.ctypes.data, diag.ctypes.data),
                  "cell pattern(fill)")
        tmap = np.zeros(max(1, nnz.value), dtype=np.int32)
        nat.check(lib.fem_bsr_transpose_map(row_ptr.ctypes.data, col.ctypes.data, ndofs, tmap.ctypes.data),
                  "cell transpose map")
        self.vec, self.num_cells, self.num_nodes, self.nnzb, self.nd = 1, C, ndofs, int(nnz.value), nd
        self.ndofs = ndofs
        self.device = device
        self.row_ptr = torch.from_numpy(row_ptr).to(device)
        self.col_idx = torch.from_numpy(col[: self.nnzb]).to(device)
        self.diag = torch.from_numpy(diag[:ndofs]).to(device)
        self.transpose = torch.from_numpy(tmap[: self.nnzb]).to(device).long()
        self.cell_dofs = torch.from_numpy(cells).to(device)
        self.cell_dofs_long = self.cell_dofs.long()
        self.scatter = torch.from_numpy(scatter[:C]).to(device).contiguous()

    def new_matrix(self, dtype):
        from .problem import BSRMatrix
        vals = torch.zeros(self.nnzb, dtype=dtype, device=self.device)
        return BSRMatrix(1, self.row_ptr, self.col_idx, self.diag, vals)


def _geometry(fe, points=None):
    """Physical shape gradients (C,Q,nen,dim) and JxW (C,Q) (fe.py:112-141)."""
    X = (fe.points if points is None else points)[fe.cells]
    J = np.einsum("cai,qaj->cqij", X, fe.shape_grads_ref)
    g = np.einsum("qaj,cqjk->cqak", fe.shape_grads_ref, np.linalg.inv(J))
    return g, np.linalg.det(J) * fe.quad_weights[None]


class CellPath:
    """Cell kernels, geometry and assembly of a cell-kernel problem."""

    def __init__(self, problem, device):
        p = self.p = problem
        fes = p.fes
        C = p.num_cells
        if len({fe.num_quads for fe in fes}) != 1:
            raise NotImplementedError("all variables must use the same number of quadrature points "
                                      "(set quadrature_order per variable)")
        self.device = device
        parts = []
        for fe, off in zip(fes, p.offset):  # find_ind, problem.py:86-97
            d = fe.vec * fe.cells[:, :, None].astype(np.int64) + np.arange(fe.vec)[None, None, :] + off
            parts.append(d.reshape(C, -1))
        cell_dofs = np.hstack(parts)
        self.sys = CellSystem(cell_dofs, p.num_total_dofs_all_vars, device)
        self.nd = self.sys.nd
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=device)  # noqa: E731
        # initialize_geometric_quantities (problem.py:130-190)
        grads, jxws = zip(*[_geometry(fe) for fe in fes])
        self.shape_grads = t(np.concatenate(grads, axis=2))                      # (C,Q,sum nen,dim)
        self.JxW = t(np.stack(jxws, axis=1))                                      # (C,V,Q)
        self.v_grads_JxW = t(np.concatenate([g[:, :, :, None, :] * w[:, :, None, None, None]
                                              for g, w in zip(grads, jxws)], axis=2))  # (C,Q,sum nen,1,dim)
        self.x = t(np.einsum("qa,cai->cqi", fes[0].shape_vals, fes[0].points[fes[0].cells]))
        for fe in fes:
            fe.shape_vals_t = t(fe.shape_vals)
            fe.face_shape_vals_t = t(fe.face_shape_vals)
        self.faces = []
        for binds in p.boundary_inds_list:
            binds = np.asarray(binds, dtype=np.int64).reshape(-1, 2)
            sg, ns, sv = [], [], []
            for fe in fes:
                g, scale = fe.get_face_shape_grads(binds)
                sg.append(g)
                ns.append(scale)
                sv.append(fe.face_shape_vals[binds[:, 1]])
            X0 = fes[0].points[fes[0].cells[binds[:, 0]]]
            xs = np.einsum("fqa,fai->fqi", fes[0].face_shape_vals[binds[:, 1]], X0)
            self.faces.append({"cells": torch.as_tensor(binds[:, 0], dtype=torch.int32, device=device),
                               "shape_vals": t(np.concatenate(sv, axis=2)),
                               "shape_grads": t(np.concatenate(sg, axis=2)),
                               "nanson": t(np.stack(ns, axis=1)), "x": t(xs)})
        self._fns = None

    # ---- kernels (problem.py:189-340) -------------------------------------------
    def _kernels(self):
        if self._fns is not None:
            return self._fns
        p = self.p
        fe0 = p.fes[0]
        n0, v0, nd = fe0.num_nodes, fe0.vec, self.nd
        sv0 = fe0.shape_vals_t
        tm = p.get_tensor_map() if hasattr(p, "get_tensor_map") else None
        from .laws import Laplace, Law, plane_strain
        if isinstance(tm, Law):  # a registered law: its torch form
            if tm.vec is not None and v0 != p.dim:
                raise NotImplementedError(f"{type(tm).__name__} needs vec={p.dim} on a {p.dim}D problem, got {v0}")
            law, tm = tm, tm.torch_map()
            if p.dim == 2 and not isinstance(law, Laplace):
                tm = plane_strain(tm)
        mm = p.get_mass_map() if hasattr(p, "get_mass_map") else None
        uk = p.get_universal_kernel() if hasattr(p, "get_universal_kernel") else None
        pad = nd - n0 * v0

        def first_var(v):
            return torch.nn.functional.pad(v.reshape(-1), (0, pad)) if pad else v.reshape(-1)

        def cell_kernel(sol, x, sg, jxw, vg, *iv):
            val = torch.zeros(nd, dtype=sol.dtype, device=sol.device)
            if tm is not None or mm is not None:
                u = sol[: n0 * v0].reshape(n0, v0)
            if tm is not None:  # laplace kernel
                ug = torch.einsum("ai,qaj->qij", u, sg[:, :n0, :])
                P = vmap(tm)(ug, *iv)
                val = val + first_var(torch.einsum("qij,qaj->ai", P, vg[:, :n0, 0, :]))
            if mm is not None:  # mass kernel
                uq = torch.einsum("ai,qa->qi", u, sv0)
                m = vmap(mm)(uq, x, *iv)
                val = val + first_var(torch.einsum("qi,qa,q->ai", m, sv0, jxw[0]))
            if uk is not None:
                val = val + uk(sol, x, sg, jxw, vg, *iv)
            return val

        face_kernels = []
        smaps = p.get_surface_maps() if hasattr(p, "get_surface_maps") else None
        uks = p.get_universal_kernels_surface() if hasattr(p, "get_universal_kernels_surface") else None
        for ind in range(len(self.faces)):
            sm = smaps[ind] if smaps is not None else None
            us = uks[ind] if uks is not None else None

            def face_kernel(sol, x, fsv, fsg, nanson, *iv, sm=sm, us=us):
                val = torch.zeros(nd, dtype=sol.dtype, device=sol.device)
                if sm is not None:  # surface kernel
                    u = sol[: n0 * v0].reshape(n0, v0)
                    uq = torch.einsum("ai,qa->qi", u, fsv[:, :n0])
                    tq = vmap(sm)(uq, x, *iv)
                    val = val + first_var(torch.einsum("qi,qa,q->ai", tq, fsv[:, :n0], nanson[0]))
                if us is not None:
                    val = val + us(sol, x, fsv, fsg, nanson, *iv)
                return val

            face_kernels.append(face_kernel)

        def with_jac(k):
            def both(sol, *args):
                r = k(sol, *args)
                return r, r
            return vmap(jacfwd(both, argnums=0, has_aux=True))

        self._fns = (cell_kernel, vmap(cell_kernel), with_jac(cell_kernel),
                     [(vmap(f), with_jac(f)) for f in face_kernels])
        return self._fns

    def _ivars(self, ivars, n):
        out = []
        for v in ivars:
            v = v if isinstance(v, torch.Tensor) else torch.as_tensor(np.asarray(v))
            v = v.to(device=self.device, dtype=torch.float64)
            if v.shape[0] != n:
                raise ValueError(f"internal variables need a leading axis of {n}, got {tuple(v.shape)}")
            out.append(v)
        return out

    # ---- assembly ---------------------------------------------------------------
    def assemble(self, dofs, res=None, vals=None, lift=None, dvec=None, bc=True, fp32=False, ivars=None,
                 ivars_surfaces=None):
        p = self.p
        sys_ = self.sys
        C, nd = sys_.num_cells, self.nd
        mask = p.dirichlet_device()[0] if bc else None
        want_jac = vals is not None or lift is not None
        for t in (res, lift):
            if t is not None:
                t.zero_()
        if vals is not None:
            vals.zero_()
        _, k_val, k_jac, faces = self._kernels()
        iv = self._ivars(p.internal_vars if ivars is None else ivars, C)
        scat = nat.lib().fem_scatter_cells_f32 if fp32 else nat.lib().fem_scatter_cells_f64
        dofs = dofs.reshape(-1)
        batch = max(1, min(C, _BATCH_ENTRIES // (nd * nd)))

        def run(items, sol, args, kv, kj, item_cell):
            if want_jac:
                jac, r = kj(sol, *args)
                jac = jac.contiguous()
            else:
                r, jac = kv(sol, *args), None
            r = r.contiguous()
            nat.check(scat(nd, items, nat.ptr(item_cell), nat.ptr(sys_.cell_dofs), nat.ptr(sys_.scatter),
                           nat.ptr(r), nat.ptr(jac), nat.ptr(mask), nat.ptr(dvec), nat.ptr(res),
                           nat.ptr(lift), nat.ptr(vals), nat.stream_ptr()), "scatter_cells")

        for c0 in range(0, C, batch):
            c1 = min(C, c0 + batch)
            sol = dofs[sys_.cell_dofs_long[c0:c1]]
            args = (self.x[c0:c1], self.shape_grads[c0:c1], self.JxW[c0:c1], self.v_grads_JxW[c0:c1],
                    *[v[c0:c1] for v in iv])
            cells = torch.arange(c0, c1, dtype=torch.int32, device=self.device)
            run(c1 - c0, sol, args, k_val, k_jac, cells)
        ivs_all = p.internal_vars_surfaces if ivars_surfaces is None else ivars_surfaces
        for ind, (face, (fv, fj)) in enumerate(zip(self.faces, faces)):
            F = int(face["cells"].numel())
            if F == 0:
                continue
            ivs = self._ivars(ivs_all[ind] if ind < len(ivs_all) else (), F)
            sol = dofs[sys_.cell_dofs_long[face["cells"].long()]]
            args = (face["x"], face["shape_vals"], face["shape_grads"], face["nanson"], *ivs)
            run(F, sol, args, fv, fj, face["cells"])
        if vals is not None and mask is not None:
            fn = nat.lib().fem_bsr_bc_diag_f32 if fp32 else nat.lib().fem_bsr_bc_diag_f64
            nat.check(fn(1, sys_.num_nodes, nat.ptr(mask), nat.ptr(sys_.diag), nat.ptr(vals), nat.stream_ptr()),
                      "bc_diag")

    # ---- J2 state commit (test_plasticity.py:67-78) ------------------------------------
    def j2_commit(self, dofs, law, ivars):
        """The state a converged increment commits, at every quadrature point:
        [sigma (C,Q,3,3), eps (C,Q,3,3), alpha (C,Q)] from the radial return
        of ``law`` (J2Plasticity) at the first variable's gradient (2D
        gradients embedded as plane strain)."""
        fe0 = self.p.fes[0]
        n0, v0, d = fe0.num_nodes, fe0.vec, self.p.dim
        C, Q = self.sys.num_cells, fe0.num_quads
        iv = self._ivars(ivars, C)
        if len(iv) < 2:
            raise ValueError("J2Plasticity needs internal_vars = [sigma_old, eps_old(, alpha_old)]")
        u = dofs.reshape(-1)[self.sys.cell_dofs_long[:, : n0 * v0]].reshape(C, n0, v0)
        ug = torch.einsum("cai,cqaj->cqij", u, self.shape_grads[:, :, :n0, :])
        ug = torch.nn.functional.pad(ug, (0, 3 - d, 0, 3 - v0))
        so, eo = iv[0].reshape(C, Q, 3, 3), iv[1].reshape(C, Q, 3, 3)
        ao = iv[2].reshape(C, Q) if len(iv) > 2 else torch.zeros(C, Q, dtype=torch.float64, device=self.device)
        sn, en, an = vmap(vmap(law.torch_state()))(ug, so, eo, ao)
        return [sn, en, an]

    # ---- adjoint (solver.py:1340-1378) ---------------------------------------------
    def param_vjp(self, dofs, ivars, lam):
        """-(dR/d ivars)^T lambda for every internal variable of the cells (the
        reference's jax.vjp of the residual w.r.t. internal_vars); returns a
        list shaped like ``ivars``."""
        C = self.sys.num_cells
        cell_kernel = self._kernels()[0]
        iv = self._ivars(ivars, C)
        dofs = dofs.reshape(-1)
        lam = lam.reshape(-1)
        grads = [torch.zeros_like(v) for v in iv]
        batch = max(1, min(C, _BATCH_ENTRIES // (self.nd * self.nd)))

        def one(sol, lam_c, x, sg, jxw, vg, *ivc):
            _, pull = torch.func.vjp(lambda *w: cell_kernel(sol, x, sg, jxw, vg, *w), *ivc)
            return pull(lam_c)

        vone = vmap(one)
        for c0 in range(0, C, batch):
            c1 = min(C, c0 + batch)
            idx = self.sys.cell_dofs_long[c0:c1]
            g = vone(dofs[idx], lam[idx], self.x[c0:c1], self.shape_grads[c0:c1], self.JxW[c0:c1],
                     self.v_grads_JxW[c0:c1], *[v[c0:c1] for v in iv])
            for k, gk in enumerate(g):
                grads[k][c0:c1] = -gk
        return grads
