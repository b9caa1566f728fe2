"""The cell-kernel path on the CPU: the oracle's multi-variable kernel
machinery (fem_oracle.KernelProblem) against its law-path problem, and the
host side of multi-variable ``Problem`` objects (no device calls).

- A universal kernel that restates linear elasticity, plus a body force,
  gives the law path's residual and tangent (1e-12);
- a tensor map given as a callable with an internal variable gives the same
  residual and tangent through KernelProblem and OracleProblem (1e-12);
- ``Problem([mesh_u, mesh_T], vec=[3, 1], ...)`` lays out dofs with the
  reference's offsets (problem.py:77-84), splits flat dofs per variable and
  per cell, and picks the cell-kernel path for universal kernels, several
  variables, unregistered tensor maps and u-dependent maps."""
import numpy as np
import pytest

import kernels as K
from helpers import element_box, face_fn, perturbed_box, thermo_meshes, thermo_problem
from oracle import fem_oracle as fo


def test_universal_linear_kernel_matches_law_problem(pkg):
    mesh = perturbed_box(pkg, (2, 3, 2), seed=1)
    bc = [[face_fn(0, 0.0)] * 3, [0, 1, 2], [lambda p: 0.0] * 3]
    body = lambda u, x: np.array([x[1], -1.0, 0.5 * x[0]])  # noqa: E731
    law = fo.OracleProblem(mesh.points, mesh.cells, 3, fo.Law("linear", E=70e3, nu=0.3), dirichlet_bc_info=bc,
                           mass_map=body)
    kp = fo.KernelProblem([dict(points=mesh.points, cells=mesh.cells, vec=3, dirichlet=bc)], mass_map=body,
                          universal_kernel=K.linear_elastic_universal(np, 70e3, 0.3))
    u = np.random.default_rng(0).normal(0, 1e-3, size=kp.ndofs)
    R, Kk = kp.residual_and_tangent(u)
    R_law = law.residual(u)
    law.newton_update(u)
    K_law = law.assemble_global()
    np.testing.assert_allclose(R, R_law, rtol=0, atol=1e-12 * np.abs(R_law).max())
    assert np.abs((Kk - K_law).toarray()).max() <= 1e-12 * np.abs(K_law.data).max()


def test_callable_tensor_map_with_internal_variable(pkg):
    mesh = element_box(pkg, "TET10", (1, 2, 1), amp=0.1)
    C = len(mesh.cells)
    s = np.random.default_rng(1).uniform(0.5, 1.5, size=(C, 4))
    tm = K.svk_tensor_map(np, 10.0, 0.3)
    kp = fo.KernelProblem([dict(points=mesh.points, cells=mesh.cells, vec=3, ele_type="TET10")], tensor_map=tm,
                          internal_vars=[s])
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, lambda ug, iv: np.array(
        [[tm(ug[c, q], iv[0][c, q]) for q in range(ug.shape[1])] for c in range(ug.shape[0])]),
        internal_vars=[s], ele_type="TET10")
    u = np.random.default_rng(2).normal(0, 0.02, size=kp.ndofs)
    R, Kk = kp.residual_and_tangent(u)
    cell_u = u.reshape(-1, 3)[op.cells]
    r_ref, jac = op.cell_residual_and_jacobian(cell_u, op.internal_vars)
    R_ref = np.zeros(kp.ndofs)
    np.add.at(R_ref, op.cell_dofs.reshape(-1), r_ref.reshape(-1))
    np.testing.assert_allclose(R, R_ref, rtol=0, atol=1e-12 * np.abs(R_ref).max())
    K_ref = op.assemble_global(jac)
    assert np.abs((Kk - K_ref).toarray()).max() <= 1e-12 * np.abs(K_ref.data).max()


def test_multivariable_problem_layout(pkg):
    import torch
    m10, m4 = thermo_meshes(pkg)
    bc_u = [[face_fn(0, 0.0)] * 3, [0, 1, 2], [lambda p: 0.0] * 3]
    bc_T = [[face_fn(0, 0.0)], [0], [lambda p: 0.0]]

    class Thermo(pkg.Problem):
        def get_universal_kernel(self):
            return lambda *a: None

    p = Thermo([m10, m4], vec=[3, 1], dim=3, ele_type=["TET10", "TET4"], quadrature_order=[2, 2],
               dirichlet_bc_info=[bc_u, bc_T])
    assert p.num_vars == 2 and p.cell_path
    n_u, n_T = len(m10.points) * 3, len(m4.points)
    assert p.offset == [0, n_u] and p.num_total_dofs_all_vars == n_u + n_T
    assert list(p.num_nodes_cumsum) == [0, 10, 14]
    flat = torch.arange(n_u + n_T, dtype=torch.float64)
    su, sT = p.unflatten_fn_sol_list(flat)
    assert su.shape == (len(m10.points), 3) and sT.shape == (len(m4.points), 1) and sT[0, 0] == n_u
    cu, cT = p.unflatten_fn_dof(torch.arange(34.0))
    assert cu.shape == (10, 3) and cT.shape == (4, 1) and cT[0, 0] == 30
    masks = [fe.dirichlet_arrays()[0] for fe in p.fes]
    assert masks[0].sum() == 3 * np.isclose(m10.points[:, 0], 0).sum()
    assert masks[1].sum() == np.isclose(m4.points[:, 0], 0).sum()
    # the compact form the device refresh copies: both variables' constrained
    # dofs at their global offsets, with the full arrays' values
    arrays = [fe.dirichlet_arrays() for fe in p.fes]
    full_mask = np.concatenate([a[0] for a in arrays])
    full_vals = np.concatenate([a[1] for a in arrays])
    dofs, vals = p._dirichlet_compact()
    np.testing.assert_array_equal(dofs, np.flatnonzero(full_mask))
    np.testing.assert_array_equal(vals, full_vals[dofs])
    assert dofs.max() >= n_u  # the temperature variable's dofs come after the displacements


def test_cell_path_selection(pkg):
    mesh = perturbed_box(pkg, (1, 1, 1))

    def make(**hooks):
        cls = type("P", (pkg.Problem,), {k: (lambda v: lambda self: v)(v) for k, v in hooks.items()})
        return cls(mesh, vec=3, dim=3)

    assert not make(get_tensor_map=pkg.NeoHookean(10.0, 0.3)).cell_path
    assert not make(get_tensor_map=lambda x: x).cell_path  # recognised: the Laplace law
    assert make(get_tensor_map=K.svk_tensor_map(np, 10.0, 0.3)).cell_path  # not a registered law
    assert make(get_tensor_map=pkg.LinearElastic(1.0, 0.3), get_mass_map=lambda u, x: u ** 3).cell_path
    assert not make(get_tensor_map=pkg.LinearElastic(1.0, 0.3), get_mass_map=lambda u, x: 0 * x + 1.0).cell_path
    assert make(get_universal_kernel=lambda: None).cell_path
    with pytest.raises(ValueError):
        m4 = element_box(pkg, "TET4", (1, 1, 1))
        pkg.Problem([mesh, m4], vec=[3, 1], dim=3, ele_type=["HEX8", "TET4"])


def test_torch_kernels_match_oracle_on_cpu(pkg):
    """The cell-kernel path's torch evaluation (vmap of jacfwd) on CPU
    tensors gives the oracle's per-cell residuals and complex-step
    Jacobians (1e-12); the scatter itself is a GPU kernel (test_gpu_cellpath)."""
    import importlib

    import torch
    cp = importlib.import_module("jax_fem_b200.cellpath")
    m10, m4 = thermo_meshes(pkg)
    p, oracle, _, _ = thermo_problem(pkg, m10, m4)
    C = p.num_cells
    c_scale = np.random.default_rng(3).uniform(0.5, 2.0, size=C)
    p.internal_vars = [torch.tensor(c_scale)]
    oracle.internal_vars = [c_scale]
    path = cp.CellPath(p, torch.device("cpu"))
    assert path.nd == 34 and len(path.faces) == 1 and path.faces[0]["cells"].numel() == 2  # one square, 2 triangles
    dofs = np.random.default_rng(4).normal(0, 0.1, size=p.num_total_dofs_all_vars)
    _, _, k_jac, faces = path._kernels()
    idx = path.sys.cell_dofs_long
    sol = torch.tensor(dofs)[idx]
    jac, r = k_jac(sol, path.x, path.shape_grads, path.JxW, path.v_grads_JxW, torch.tensor(c_scale))
    items = oracle._items()
    for c in range(C):
        oidx, k = items[c]
        assert np.array_equal(oidx, idx[c].numpy())
        base = dofs[oidx].astype(np.complex128)
        np.testing.assert_allclose(r[c].numpy(), k(dofs[oidx]), rtol=0, atol=1e-12)
        for d in (0, 7, 31, 33):
            up = base.copy()
            up[d] += 1e-30j
            np.testing.assert_allclose(jac[c][:, d].numpy(), np.imag(k(up)) / 1e-30, rtol=0, atol=1e-10)
    face = path.faces[0]
    fv, fj = faces[0]
    fsol = torch.tensor(dofs)[idx[face["cells"].long()]]
    jf, rf = fj(fsol, face["x"], face["shape_vals"], face["shape_grads"], face["nanson"])
    for f in range(face["cells"].numel()):
        oidx, k = items[C + f]
        np.testing.assert_allclose(rf[f].numpy(), k(dofs[oidx]), rtol=0, atol=1e-12)
        up = dofs[oidx].astype(np.complex128)
        up[33] += 1e-30j
        np.testing.assert_allclose(jf[f][:, 33].numpy(), np.imag(k(up)) / 1e-30, rtol=0, atol=1e-10)


def test_param_vjp_matches_complex_step_on_cpu(pkg):
    """CellPath.param_vjp (the cell-kernel path's adjoint VJP: torch VJP of
    the user kernel w.r.t. its internal variables, summed over cells) on CPU
    tensors equals -(dR/dc)^T lambda from complex-step derivatives of the
    oracle's cell residuals w.r.t. each cell's conductivity (1e-12)."""
    import importlib

    import torch
    cp = importlib.import_module("jax_fem_b200.cellpath")
    m10, m4 = thermo_meshes(pkg)
    p, oracle, _, _ = thermo_problem(pkg, m10, m4)
    C = p.num_cells
    rng = np.random.default_rng(6)
    c_scale = rng.uniform(0.5, 2.0, size=C)
    dofs = rng.normal(0, 0.1, size=p.num_total_dofs_all_vars)
    lam = rng.normal(size=p.num_total_dofs_all_vars)
    path = cp.CellPath(p, torch.device("cpu"))
    (g,) = path.param_vjp(torch.tensor(dofs), [torch.tensor(c_scale)], torch.tensor(lam))
    ref = np.zeros(C)
    idx = oracle.cell_dofs
    for c in range(C):
        cs = c_scale.astype(np.complex128)
        cs[c] += 1e-30j
        r = oracle.cell_kernel(c, dofs[idx[c]].astype(np.complex128), [cs])
        ref[c] = -np.imag(r) @ lam[idx[c]] / 1e-30
    np.testing.assert_allclose(g.numpy(), ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_ad_wrapper_rejects_differentiable_surface_variables(pkg):
    """Gradients flow through internal_vars only: a set_params that puts
    parameter-dependent tensors into internal_vars_surfaces is refused
    before any solve, instead of returning a silently partial gradient."""
    import torch
    m10, m4 = thermo_meshes(pkg)
    p, _, _, _ = thermo_problem(pkg, m10, m4)

    def set_params(params):
        p.internal_vars = [params]
        p.internal_vars_surfaces = [[params[:2] * 1.0]]

    p.set_params = set_params
    fwd = pkg.ad_wrapper(p, {}, {})
    with pytest.raises(NotImplementedError):
        fwd(torch.ones(p.num_cells, dtype=torch.float64, requires_grad=True))


def test_registered_laws_on_the_cell_path(pkg):
    """On the cell-kernel path a registered law runs as its torch form
    (Law.torch_map): Neo-Hookean with a u-dependent load and SIMP with theta
    per point, and J2 with hardening from a yielding prior state, give the
    oracle's per-cell residuals and complex-step Jacobians (CPU tensors)."""
    import importlib

    import torch
    cp = importlib.import_module("jax_fem_b200.cellpath")
    mesh = perturbed_box(pkg, (2, 2, 1), seed=3)
    C = len(mesh.cells)
    rng = np.random.default_rng(9)
    theta = rng.uniform(0.2, 1.0, size=(C, 8))
    cases = [
        (pkg.NeoHookean(10.0, 0.3), "get_mass_map", lambda u, x: 0.5 * u ** 3,
         lambda ug: fo.stress_neo_hookean(ug, 10.0, 0.3), None, 0.05),
        (pkg.SIMPElastic(70e3, 70.0, 0.3, 3.0), "get_universal_kernel", lambda *a: 0.0,
         lambda ug, th: fo.stress_simp(ug, th, 70e3, 70.0, 0.3, 3.0), theta, 2e-3),
    ]
    for law, hook, extra, np_map, iv, scale in cases:
        hooks = {"get_tensor_map": (lambda law: lambda self: law)(law),
                 hook: (lambda e: lambda self: e)(extra)}
        prob = type("P", (pkg.Problem,), hooks)(mesh, vec=3, dim=3)
        assert prob.cell_path
        ivs = [torch.tensor(iv)] if iv is not None else []
        path = cp.CellPath(prob, torch.device("cpu"))
        dofs = rng.normal(0, scale, size=prob.num_total_dofs_all_vars)
        idx = path.sys.cell_dofs_long
        jac, r = path._kernels()[2](torch.tensor(dofs)[idx], path.x, path.shape_grads, path.JxW,
                                    path.v_grads_JxW, *ivs)
        kp = fo.KernelProblem([dict(points=mesh.points, cells=mesh.cells, vec=3)], tensor_map=np_map,
                              mass_map=extra if hook == "get_mass_map" else None,
                              internal_vars=[iv] if iv is not None else [])
        for c, (oidx, k) in enumerate(kp._items()):
            ref = k(dofs[oidx])
            np.testing.assert_allclose(r[c].numpy(), ref, rtol=0, atol=1e-12 * max(1.0, np.abs(ref).max()))
            up = dofs[oidx].astype(np.complex128)
            up[5] += 1e-30j
            col = np.imag(k(up)) / 1e-30
            np.testing.assert_allclose(jac[c][:, 5].numpy(), col, rtol=0, atol=1e-10 * max(1.0, np.abs(col).max()))
    # J2 with hardening: a random prior state with most points yielding
    so = rng.normal(0, 150.0, size=(C, 8, 3, 3))
    so = 0.5 * (so + np.swapaxes(so, -1, -2))
    eo = rng.normal(0, 2e-3, size=(C, 8, 3, 3))
    eo = 0.5 * (eo + np.swapaxes(eo, -1, -2))
    ao = rng.uniform(0, 0.01, size=(C, 8))
    law = pkg.J2Plasticity(70e3, 0.3, 250.0, 700.0)
    prob = type("P", (pkg.Problem,), {"get_tensor_map": lambda self: law,
                                      "get_universal_kernel": lambda self: (lambda *a: 0.0)})(mesh, vec=3, dim=3)
    path = cp.CellPath(prob, torch.device("cpu"))
    dofs = rng.normal(0, 6e-4, size=prob.num_total_dofs_all_vars)
    idx = path.sys.cell_dofs_long
    jac, r = path._kernels()[2](torch.tensor(dofs)[idx], path.x, path.shape_grads, path.JxW, path.v_grads_JxW,
                                torch.tensor(so), torch.tensor(eo), torch.tensor(ao))
    np_j2 = lambda ug, s_, e_, a_: fo.j2_return_map(ug, s_, e_, a_, 70e3, 0.3, 250.0, 700.0)[0]  # noqa: E731
    kp = fo.KernelProblem([dict(points=mesh.points, cells=mesh.cells, vec=3)], tensor_map=np_j2,
                          internal_vars=[so, eo, ao])
    for c, (oidx, k) in enumerate(kp._items()):
        ref = k(dofs[oidx])
        np.testing.assert_allclose(r[c].numpy(), ref, rtol=0, atol=1e-11 * np.abs(ref).max())
        up = dofs[oidx].astype(np.complex128)
        up[7] += 1e-30j
        col = np.imag(k(up)) / 1e-30
        np.testing.assert_allclose(jac[c][:, 7].numpy(), col, rtol=0, atol=1e-9 * max(1.0, np.abs(col).max()))
    with pytest.raises(NotImplementedError, match="torch form"):
        pkg.laws.Law().torch_map()
