"""The 2D element types QUAD4, QUAD8, TRI3 and TRI6 (basis.py:19-114 in the
reference) on the CPU: tables, meshes, the oracle's convergence study, and
the cell-kernel path's torch kernels, which are what 2D problems run on.

- The product's tables (basis.py: mesh node order) equal the oracle's
  (basix numbering, moved with the reference's re_order, dual bases by
  inverting the dof functionals) at every quadrature order, faces (edges)
  included;
- shape functions: partition of unity, exact reproduction of linear
  fields, the Kronecker property at the dofs (QUAD8: vertex values and
  edge means, basix's serendipity dofs);
- the quadrature rules integrate the monomials of their order exactly,
  the edge rules give each edge's length and outward normal;
- ``rectangle_mesh`` numbers nodes and cells as the reference's
  (generate_mesh.py:120-148), the other types are conforming and
  positively oriented, and ``Mesh`` infers 2D types from the points;
- the oracle's Poisson convergence study in 2D gives L2 / H1-seminorm rates
  2 / 1 (QUAD4, TRI3), 3 / 2 (TRI6) and 2 / 1.5 (QUAD8, whose edge dofs are
  means while Dirichlet data are midside values, as for HEX20);
- Newton with the product's torch kernels (summed into a global system by
  the test, where the GPU runs ``fem_scatter_cells``) reaches the oracle's
  solution (1e-10) for a nonlinear reaction-diffusion problem with a flux
  on QUAD8 and a plane-strain Neo-Hookean body with a traction on TRI6;
- registered laws in 2D are plane strain: SIMP on QUAD4 and J2 with
  hardening on TRI3 give the oracle's cell residuals and complex-step
  Jacobians, and the J2 commit on the cell-kernel path gives the oracle's
  return map at every quadrature point."""
import importlib
import math

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from helpers import face_fn, planar_box
from oracle import fem_oracle as fo

TYPES2D = ["QUAD4", "QUAD8", "TRI3", "TRI6"]


@pytest.fixture(scope="module")
def B(pkg):
    return importlib.import_module("jax_fem_b200.basis")


@pytest.mark.parametrize("ele", TYPES2D)
def test_planar_tables_match_oracle(B, ele):
    for order in [None, 0, 1, 2] + ([3, 4] if ele.startswith("QUAD") else []):
        got = B.get_shape_vals_and_grads(ele, order) + B.get_face_shape_vals_and_grads(ele, order)
        ref = fo.element_tables(ele, order) + fo.element_face_tables(ele, order)
        for a, b in zip(got, ref):
            np.testing.assert_allclose(np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64),
                                       rtol=0, atol=1e-12)


@pytest.mark.parametrize("ele", TYPES2D)
def test_planar_shape_functions(B, ele):
    xi = np.random.default_rng(0).uniform(0, 1, size=(64, 2))
    if ele.startswith("TRI"):
        xi = xi[xi.sum(axis=1) <= 1.0]
    v, g = B.shape_fn(ele, xi)
    X = B.node_coords(ele)
    assert v.shape == (len(xi), B.NODES_PER_CELL[ele]) and g.shape == v.shape + (2,)
    np.testing.assert_allclose(v.sum(axis=1), 1.0, rtol=0, atol=1e-13)
    np.testing.assert_allclose(g.sum(axis=1), 0.0, rtol=0, atol=1e-12)
    np.testing.assert_allclose(v @ X, xi, rtol=0, atol=1e-13)
    np.testing.assert_allclose(np.einsum("nad,ae->ned", g, X), np.broadcast_to(np.eye(2), (len(xi), 2, 2)),
                               rtol=0, atol=1e-12)
    if ele == "QUAD8":  # vertex values, then the mean over each edge
        np.testing.assert_allclose(B.shape_fn(ele, X[:4])[0], np.eye(8)[:4], rtol=0, atol=1e-13)
        t, w = B.gauss_legendre_01(3)
        for e, (i, j) in enumerate(B.QUAD_EDGES):
            pts = X[i][None] + t[:, None] * (X[j] - X[i])[None]
            np.testing.assert_allclose(w @ B.shape_fn(ele, pts)[0], np.eye(8)[4 + e], rtol=0, atol=1e-13)
    else:
        np.testing.assert_allclose(B.shape_fn(ele, X)[0], np.eye(len(X)), rtol=0, atol=1e-13)
    with pytest.raises(ValueError, match="coordinates"):
        B.shape_fn(ele, np.zeros((1, 3)))


def test_planar_quadrature_and_edges(B):
    for order in range(6):
        pts, w = B.volume_quadrature("QUAD4", order)
        for a in range(order + 1):
            for b in range(order + 1):
                assert abs(w @ (pts[:, 0] ** a * pts[:, 1] ** b) - 1.0 / ((a + 1) * (b + 1))) < 1e-14
    for order in range(3):
        pts, w = B.volume_quadrature("TRI6", order)
        for a in range(max(order, 1) + 1):
            for b in range(max(order, 1) + 1 - a):
                exact = math.factorial(a) * math.factorial(b) / math.factorial(a + b + 2)
                assert abs(w @ (pts[:, 0] ** a * pts[:, 1] ** b) - exact) < 1e-15
    for ele in ("QUAD8", "TRI6"):
        finds, fpts, fw, normals = B.face_rule(ele)
        X = B.node_coords(ele)
        centre = X[:4 if ele == "QUAD8" else 3].mean(axis=0)
        for f, (i, j) in enumerate(finds):
            edge = X[j] - X[i]
            assert abs(fw[f].sum() - np.linalg.norm(edge)) < 1e-15
            assert abs(normals[f] @ edge) < 1e-15 and abs(np.linalg.norm(normals[f]) - 1.0) < 1e-15
            assert normals[f] @ (0.5 * (X[i] + X[j]) - centre) > 0
            # points on the edge
            s = (fpts[f] - X[i]) @ edge / (edge @ edge)
            np.testing.assert_allclose(X[i][None] + s[:, None] * edge[None], fpts[f], rtol=0, atol=1e-15)


def test_rectangle_mesh_and_inference(pkg):
    m = pkg.rectangle_mesh(3, 2, 1.5, 1.0)
    pts, cells = m.points, m.cells_dict["quad"]
    assert pts.shape == (12, 2) and cells.shape == (6, 4)
    for i in range(4):
        for j in range(3):
            np.testing.assert_allclose(pts[i * 3 + j], [0.5 * i, 0.5 * j])
    for i in range(3):
        for j in range(2):
            n = i * 3 + j
            assert cells[i * 2 + j].tolist() == [n, n + 3, n + 4, n + 1]
    n_edges = 3 * 3 + 4 * 2
    for ele, nn in (("QUAD4", 12), ("TRI3", 12), ("QUAD8", 12 + n_edges), ("TRI6", 12 + n_edges + 6)):
        mesh = planar_box(pkg, ele, (3, 2), L=(1.5, 1.0))
        assert mesh.ele_type == ele and len(mesh.points) == nn
        nc = 4 if ele.startswith("QUAD") else 3
        Xc = mesh.points[mesh.cells[:, :nc]]
        area = 0.5 * np.sum(Xc[:, :, 0] * np.roll(Xc[:, :, 1], -1, axis=1)
                            - np.roll(Xc[:, :, 0], -1, axis=1) * Xc[:, :, 1], axis=1)
        assert np.all(area > 0) and abs(area.sum() - 1.5) < 1e-14
        if nc < mesh.cells.shape[1]:
            E = pkg.basis.QUAD_EDGES if nc == 4 else pkg.basis.TRI_EDGES
            np.testing.assert_allclose(mesh.points[mesh.cells[:, nc:]], Xc[:, E].mean(axis=2), rtol=0, atol=1e-15)
    assert pkg.Mesh(np.zeros((4, 2)), [[0, 1, 2, 3]]).ele_type == "QUAD4"
    assert pkg.Mesh(np.zeros((4, 3)), [[0, 1, 2, 3]]).ele_type == "TET4"
    assert pkg.Mesh(np.zeros((6, 2)), [[0, 1, 2, 3, 4, 5]]).ele_type == "TRI6"
    with pytest.raises(NotImplementedError):
        pkg.Mesh(np.zeros((3, 3)), [[0, 1, 2]])
    with pytest.raises(ValueError, match="2D element"):
        pkg.fe.FiniteElement(pkg.Mesh(np.zeros((4, 2)), [[0, 1, 2, 3]]), 1, 3, ele_type="QUAD4")
    with pytest.raises(ValueError):
        pkg.rectangle_mesh(2, 2, 1.0, 1.0, ele_type="HEX8")
    with pytest.raises(ValueError):
        pkg.box_mesh_gmsh(2, 2, 2, 1.0, 1.0, 1.0, None, "QUAD4")


def _u2(p):
    return 1e2 * ((p[..., 0] - 0.5) ** 3 + 2.0 * np.sin(2.0 * p[..., 1]) * np.exp(p[..., 0]))


def _grad2(p):
    x, y = p[..., 0], p[..., 1]
    return 1e2 * np.stack([3.0 * (x - 0.5) ** 2 + 2.0 * np.sin(2.0 * y) * np.exp(x),
                           4.0 * np.cos(2.0 * y) * np.exp(x)], axis=-1)


def _lap2(p):
    x, y = p[..., 0], p[..., 1]
    return 1e2 * (6.0 * (x - 0.5) - 6.0 * np.sin(2.0 * y) * np.exp(x))


@pytest.mark.parametrize("ele,rates", [("QUAD4", (2, 1)), ("TRI3", (2, 1)), ("TRI6", (3, 2)), ("QUAD8", (2, 1.5))])
def test_planar_oracle_convergence_rates(pkg, ele, rates):
    """The reference's convergence-rate study (applications/convergence_rate)
    restated on the unit square: -lap u = -f with f = lap u_true as the mass
    map and u = u_true on the boundary, N = 4 and 8."""
    errs = []
    for N in (4, 8):
        m = planar_box(pkg, ele, (N, N))
        bnd = lambda p: np.isclose(p[0], 0) | np.isclose(p[0], 1) | np.isclose(p[1], 0) | np.isclose(p[1], 1)  # noqa
        kp = fo.KernelProblem([dict(points=m.points, cells=m.cells, vec=1, ele_type=ele,
                                    dirichlet=[[bnd], [0], [_u2]])],
                              tensor_map=lambda g: g, mass_map=lambda u, x: np.array([_lap2(x)]))
        u = kp.newton()
        vals, gref, w = fo.element_tables(ele)
        X = m.points[m.cells]
        J = np.einsum("cai,qaj->cqij", X, gref)
        jxw = np.linalg.det(J) * w[None]
        g = np.einsum("qaj,cqjk->cqak", gref, np.linalg.inv(J))
        cu = u[m.cells]
        xq = np.einsum("qa,cai->cqi", vals, X)
        l2 = np.sqrt(np.sum((np.einsum("qa,ca->cq", vals, cu) - _u2(xq)) ** 2 * jxw))
        h1 = np.sqrt(np.sum(((np.einsum("ca,cqaj->cqj", cu, g) - _grad2(xq)) ** 2).sum(-1) * jxw))
        errs.append((l2, h1))
    l2_rate, h1_rate = np.log2(np.array(errs[0]) / np.array(errs[1]))
    assert abs(l2_rate - rates[0]) < 0.1 and abs(h1_rate - rates[1]) < 0.1, (l2_rate, h1_rate)


# ---- the cell-kernel path in 2D ------------------------------------------------------

def _cell_path(pkg, prob):
    import torch
    cp = importlib.import_module("jax_fem_b200.cellpath")
    assert prob.cell_path
    return cp.CellPath(prob, torch.device("cpu"))


def _cpu_system(path, dofs, ivars=()):
    """Global residual and tangent from the product's torch kernels; the
    test sums the cell and face contributions (on the GPU the library's
    fem_scatter_cells does)."""
    import torch
    n = path.sys.ndofs
    nd = path.nd
    idx = path.sys.cell_dofs_long
    _, _, k_jac, faces = path._kernels()
    d = torch.tensor(dofs)
    parts = [(idx.numpy(), *k_jac(d[idx], path.x, path.shape_grads, path.JxW, path.v_grads_JxW,
                                  *[torch.as_tensor(v) for v in ivars]))]
    for face, (_, fj) in zip(path.faces, faces):
        fidx = idx[face["cells"].long()]
        parts.append((fidx.numpy(), *fj(d[fidx], face["x"], face["shape_vals"], face["shape_grads"],
                                        face["nanson"])))
    R = np.zeros(n)
    rows, cols, vals = [], [], []
    for ix, jac, r in parts:
        np.add.at(R, ix.reshape(-1), r.numpy().reshape(-1))
        rows.append(np.repeat(ix, nd, axis=1).reshape(-1))
        cols.append(np.tile(ix, (1, nd)).reshape(-1))
        vals.append(jac.numpy().reshape(-1))
    K = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    return R, K


def _cpu_newton(prob, path, tol=1e-12, max_iter=30):
    mask, bvals = prob.fes[0].dirichlet_arrays()
    free = mask == 0
    dofs = np.where(free, 0.0, bvals)
    for _ in range(max_iter):
        R, K = _cpu_system(path, dofs)
        if np.linalg.norm(R[free]) < tol:
            return dofs
        dofs[free] -= spla.spsolve(K[free][:, free].tocsc(), R[free])
    raise AssertionError("Newton did not converge")


def _plane_strain_np(stress3):
    def tm(ug, *iv):
        g = np.zeros((3, 3), dtype=ug.dtype)
        g[:2, :2] = ug
        return stress3(g, *iv)[:2, :2]
    return tm


def test_planar_newton_matches_oracle(pkg):
    import torch
    # nonlinear reaction-diffusion with a flux on QUAD8 (curved cells)
    mesh = planar_box(pkg, "QUAD8", (4, 3), L=(2.0, 1.0), amp=0.1, seed=1)
    bc = [[face_fn(0, 0.0), face_fn(0, 2.0)], [0, 0], [lambda p: 0.0, lambda p: 1.0]]
    top = face_fn(1, 1.0)

    class Reaction(pkg.Problem):
        def get_tensor_map(self):
            return lambda g: g

        def get_mass_map(self):
            return lambda u, x: 4.0 * u ** 3 - 3.0 * x[..., 1:2]

        def get_surface_maps(self):
            return [lambda u, x: -(1.0 + x[..., 0:1]) + 0.0 * u]

    prob = Reaction(mesh, vec=1, dim=2, ele_type="QUAD8", dirichlet_bc_info=bc, location_fns=[top])
    path = _cell_path(pkg, prob)
    assert len(path.faces) == 1 and path.faces[0]["cells"].numel() == 4
    got = _cpu_newton(prob, path)
    kp = fo.KernelProblem([dict(points=mesh.points, cells=mesh.cells, vec=1, ele_type="QUAD8", dirichlet=bc)],
                          tensor_map=lambda g: g, mass_map=lambda u, x: 4.0 * u ** 3 - 3.0 * x[1:2],
                          location_fns=[top], surface_maps=[lambda u, x: -(1.0 + x[0:1]) + 0.0 * u])
    ref = kp.newton(rel_tol=1e-13, tol=1e-13)
    assert np.abs(ref).max() > 0.5
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-10 * np.abs(ref).max())

    # plane-strain Neo-Hookean (a registered law) with a traction on TRI6
    mesh = planar_box(pkg, "TRI6", (4, 2), L=(2.0, 1.0), amp=0.1, seed=2)
    bc = [[face_fn(0, 0.0)] * 2, [0, 1], [lambda p: 0.0] * 2]
    right = face_fn(0, 2.0)

    class Body(pkg.Problem):
        def get_tensor_map(self):
            return pkg.NeoHookean(10.0, 0.3)

        def get_surface_maps(self):
            return [lambda u, x: torch.stack([0.4 + 0.0 * x[0], -0.2 * x[1]])]

    prob = Body(mesh, vec=2, dim=2, ele_type="TRI6", dirichlet_bc_info=bc, location_fns=[right])
    got = _cpu_newton(prob, _cell_path(pkg, prob))
    kp = fo.KernelProblem([dict(points=mesh.points, cells=mesh.cells, vec=2, ele_type="TRI6", dirichlet=bc)],
                          tensor_map=_plane_strain_np(lambda g: fo.stress_neo_hookean(g, 10.0, 0.3)),
                          location_fns=[right], surface_maps=[lambda u, x: np.array([0.4, -0.2 * x[1]])])
    ref = kp.newton(rel_tol=1e-13, tol=1e-13)
    assert np.abs(ref).max() > 0.05
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-10 * np.abs(ref).max())


def test_planar_registered_laws_and_j2_commit(pkg):
    import torch
    rng = np.random.default_rng(5)
    # SIMP with theta per point on QUAD4
    mesh = planar_box(pkg, "QUAD4", (3, 2), amp=0.15, seed=3)
    C = len(mesh.cells)
    theta = rng.uniform(0.2, 1.0, size=(C, 4))
    law = pkg.SIMPElastic(70e3, 70.0, 0.3, 3.0)
    prob = type("P", (pkg.Problem,), {"get_tensor_map": lambda self: law})(mesh, vec=2, dim=2, ele_type="QUAD4")
    path = _cell_path(pkg, prob)
    dofs = rng.normal(0, 1e-3, size=prob.num_total_dofs_all_vars)
    idx = path.sys.cell_dofs_long
    jac, r = path._kernels()[2](torch.tensor(dofs)[idx], path.x, path.shape_grads, path.JxW, path.v_grads_JxW,
                                torch.tensor(theta))
    np_simp = _plane_strain_np(lambda g, th: fo.stress_simp(g, th, 70e3, 70.0, 0.3, 3.0))
    kp = fo.KernelProblem([dict(points=mesh.points, cells=mesh.cells, vec=2, ele_type="QUAD4")],
                          tensor_map=np_simp, internal_vars=[theta])
    for c, (oidx, k) in enumerate(kp._items()):
        ref = k(dofs[oidx])
        np.testing.assert_allclose(r[c].numpy(), ref, rtol=0, atol=1e-12 * np.abs(ref).max())
        up = dofs[oidx].astype(np.complex128)
        up[3] += 1e-30j
        col = np.imag(k(up)) / 1e-30
        np.testing.assert_allclose(jac[c][:, 3].numpy(), col, rtol=0, atol=1e-10 * np.abs(col).max())

    # J2 with hardening from a yielding prior state on TRI3 (one point per cell)
    mesh = planar_box(pkg, "TRI3", (3, 2), amp=0.15, seed=4)
    C = len(mesh.cells)
    so = rng.normal(0, 150.0, size=(C, 1, 3, 3))
    so = 0.5 * (so + np.swapaxes(so, -1, -2))
    eo = rng.normal(0, 2e-3, size=(C, 1, 3, 3))
    eo = 0.5 * (eo + np.swapaxes(eo, -1, -2))
    eo[..., 2, :] = eo[..., :, 2] = 0.0  # plane strain history
    ao = rng.uniform(0, 0.01, size=(C, 1))
    law = pkg.J2Plasticity(70e3, 0.3, 250.0, 700.0)
    prob = type("P", (pkg.Problem,), {"get_tensor_map": lambda self: law})(mesh, vec=2, dim=2, ele_type="TRI3")
    path = _cell_path(pkg, prob)
    dofs = rng.normal(0, 6e-4, size=prob.num_total_dofs_all_vars)
    ivs = [torch.tensor(so), torch.tensor(eo), torch.tensor(ao)]
    idx = path.sys.cell_dofs_long
    jac, r = path._kernels()[2](torch.tensor(dofs)[idx], path.x, path.shape_grads, path.JxW, path.v_grads_JxW,
                                *ivs)
    np_j2 = _plane_strain_np(lambda g, s_, e_, a_: fo.j2_return_map(g, s_, e_, a_, 70e3, 0.3, 250.0, 700.0)[0])
    kp = fo.KernelProblem([dict(points=mesh.points, cells=mesh.cells, vec=2, ele_type="TRI3")],
                          tensor_map=np_j2, internal_vars=[so, eo, ao])
    for c, (oidx, k) in enumerate(kp._items()):
        ref = k(dofs[oidx])
        np.testing.assert_allclose(r[c].numpy(), ref, rtol=0, atol=1e-11 * np.abs(ref).max())
        up = dofs[oidx].astype(np.complex128)
        up[2] += 1e-30j
        col = np.imag(k(up)) / 1e-30
        np.testing.assert_allclose(jac[c][:, 2].numpy(), col, rtol=0, atol=1e-9 * max(1.0, np.abs(col).max()))
    # the commit: sigma, eps and alpha of the oracle's return map at the points
    sn, en, an = path.j2_commit(torch.tensor(dofs), law, ivs)
    ug = np.zeros((C, 1, 3, 3))
    ug[:, :, :2, :2] = np.einsum("cai,cqaj->cqij", dofs.reshape(-1, 2)[mesh.cells], path.shape_grads.numpy())
    s_ref, a_ref = fo.j2_return_map(ug, so, eo, ao, 70e3, 0.3, 250.0, 700.0)
    assert (a_ref > ao).any() and (a_ref == ao).any()  # yielding and elastic points both present
    np.testing.assert_allclose(sn.numpy(), s_ref, rtol=0, atol=1e-9 * np.abs(s_ref).max())
    np.testing.assert_allclose(en.numpy(), 0.5 * (ug + np.swapaxes(ug, -1, -2)), rtol=0, atol=1e-18)
    np.testing.assert_allclose(an.numpy(), a_ref, rtol=0, atol=1e-15)
    # vec must match the dimension for the elastic laws
    bad = type("P", (pkg.Problem,), {"get_tensor_map": lambda self: pkg.LinearElastic(1.0, 0.3)})(
        mesh, vec=3, dim=2, ele_type="TRI3")
    with pytest.raises(NotImplementedError, match="vec=2"):
        _cell_path(pkg, bad)._kernels()


def test_planar_param_vjp_through_expanded_density(pkg):
    """The adjoint's parameter pull-back on a 2D SIMP plate whose per-point
    densities are a per-cell density expanded over the quadrature points
    (``set_params`` of the reference's 2D topology-optimisation example):
    CellPath.param_vjp, summed over each cell's points by autograd through
    the expand, equals -(dR/d theta_c)^T lambda from complex-step
    derivatives of the oracle's cell residuals (1e-12)."""
    import torch
    mesh = planar_box(pkg, "QUAD4", (3, 2), L=(2.0, 1.0), amp=0.1, seed=8)
    C, Q = len(mesh.cells), 4
    law = pkg.SIMPElastic(70e3, 70.0, 0.3, 3.0)
    prob = type("P", (pkg.Problem,), {"get_tensor_map": lambda self: law})(mesh, vec=2, dim=2, ele_type="QUAD4")
    path = _cell_path(pkg, prob)
    rng = np.random.default_rng(10)
    th0 = rng.uniform(0.3, 1.0, size=C)
    dofs = rng.normal(0, 1e-3, size=prob.num_total_dofs_all_vars)
    lam = rng.normal(size=prob.num_total_dofs_all_vars)
    th = torch.tensor(th0, requires_grad=True)
    (gq,) = path.param_vjp(torch.tensor(dofs), [th[:, None].expand(C, Q)], torch.tensor(lam))
    assert gq.shape == (C, Q)
    th[:, None].expand(C, Q).backward(gq)
    np_simp = _plane_strain_np(lambda g, t: fo.stress_simp(g, t, 70e3, 70.0, 0.3, 3.0))
    ref = np.zeros(C)
    for c in range(C):
        t = np.repeat(th0.astype(np.complex128)[:, None], Q, axis=1)
        t[c] += 1e-30j
        kp = fo.KernelProblem([dict(points=mesh.points, cells=mesh.cells, vec=2, ele_type="QUAD4")],
                              tensor_map=np_simp, internal_vars=[t])
        idx = kp.cell_dofs[c]
        ref[c] = -np.imag(kp.cell_kernel(c, dofs[idx].astype(np.complex128), kp.internal_vars)) @ lam[idx] / 1e-30
    np.testing.assert_allclose(th.grad.numpy(), ref, rtol=0, atol=1e-12 * np.abs(ref).max())
