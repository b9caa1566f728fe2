"""The cell-kernel path on the GPU (cellpath.py + fem_scatter_cells_* +
fem_bsr_bc_diag_*): weak forms as torch code, Jacobians by forward-mode
differentiation, the scalar CSR system solved by the library's Krylov
solvers.  Each against an independent result:

- a universal kernel restating the Neo-Hookean law gives the registered
  NeoHookean kernel's residual and eliminated tangent (1e-10) and Newton
  solution (1e-9) on a jittered HEX8 box;
- a torch tensor map (Saint Venant-Kirchhoff with a per-point stiffness
  scale) on TET10: Newton vs the oracle's (1e-8);
- two variables (u on TET10, T on TET4; thermo-elastic coupling, a Robin
  condition on T through a surface universal kernel): Newton vs the
  oracle's KernelProblem (1e-9), mixed precision within 1e-6;
- a u-dependent mass map (nonlinear reaction) on HEX8 vs the oracle (1e-9);
- ad_wrapper through the cell-kernel path (transposed solve of a
  non-symmetric tangent, torch VJP of the kernel w.r.t. a per-cell
  conductivity) vs central differences (h = 1e-4: the problem is linear
  in (u, T) for given conductivities, smooth in them; 1e-6 relative)."""
import numpy as np
import pytest
import torch

import kernels as K
from helpers import element_box, face_fn, make_problem, perturbed_box, thermo_meshes, thermo_problem
from oracle import fem_oracle as fo

LIN_BICG = {"bicgstab": {"precond": "jacobi", "rtol": 1e-13, "atol": 0.0, "maxiter": 50000}}


@pytest.mark.gpu
def test_universal_neo_hookean_matches_law_kernel(pkg, cuda):
    mesh = perturbed_box(pkg, (3, 3, 3), seed=7)
    bc = [[face_fn(0, 0.0)] * 3 + [face_fn(0, 1.0)] * 2, [0, 1, 2, 0, 1],
          [lambda p: 0.0] * 3 + [lambda p: 0.1, lambda p: 0.05]]
    law = make_problem(pkg, mesh, pkg.NeoHookean(10.0, 0.3), bc=bc)

    class Universal(pkg.Problem):
        def get_universal_kernel(self):
            return K.neo_hookean_universal(torch, 10.0, 0.3)

    uni = Universal(mesh, vec=3, dim=3, dirichlet_bc_info=bc)
    assert uni.cell_path and not law.cell_path
    u = torch.tensor(np.random.default_rng(0).normal(0, 0.03, size=law.num_total_dofs_all_vars), device=cuda)
    ra, rb = torch.empty_like(u), torch.empty_like(u)
    A = law.dev().new_matrix(torch.float64)
    B = uni.dev().new_matrix(torch.float64)
    law.assemble(u, res=ra, vals=A.vals)
    uni.assemble(u, res=rb, vals=B.vals)
    np.testing.assert_allclose(rb.cpu().numpy(), ra.cpu().numpy(), rtol=0, atol=1e-10 * ra.abs().max().item())
    Ka, Kb = A.to_scipy(), B.to_scipy()
    assert abs(Kb - Ka).max() <= 1e-10 * abs(Ka).max()
    opts = {"newton": {"rel_tol": 1e-11, "tol": 1e-14, "linear": LIN_BICG}}
    sa = pkg.solver(law, opts)[0].cpu().numpy()
    sb = pkg.solver(uni, opts)[0].cpu().numpy()
    assert np.abs(sa - sb).max() <= 1e-9 * np.abs(sa).max()


@pytest.mark.gpu
def test_torch_tensor_map_matches_oracle(pkg, cuda):
    mesh = element_box(pkg, "TET10", (2, 1, 1), L=(2.0, 1.0, 1.0), amp=0.08, seed=2)
    C = len(mesh.cells)
    s = np.random.default_rng(3).uniform(0.5, 1.5, size=(C, 4))
    bc = [[face_fn(0, 0.0)] * 3 + [face_fn(0, 2.0)], [0, 1, 2, 2], [lambda p: 0.0] * 3 + [lambda p: -0.1]]

    class SVK(pkg.Problem):
        def get_tensor_map(self):
            return K.svk_tensor_map(torch, 10.0, 0.3)

    prob = SVK(mesh, vec=3, dim=3, ele_type="TET10", dirichlet_bc_info=bc)
    prob.internal_vars = [torch.tensor(s, device=cuda)]
    assert prob.cell_path
    sol = pkg.solver(prob, {"newton": {"rel_tol": 1e-11, "tol": 1e-14, "linear": LIN_BICG}})[0]
    tm = K.svk_tensor_map(np, 10.0, 0.3)
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, lambda ug, iv: np.array(
        [[tm(ug[c, q], iv[0][c, q]) for q in range(ug.shape[1])] for c in range(ug.shape[0])]),
        dirichlet_bc_info=bc, internal_vars=[s], ele_type="TET10")
    ref = fo.newton_solve(op, rel_tol=1e-12, tol=1e-14)
    got = sol.cpu().numpy().reshape(-1)
    assert np.abs(got - ref).max() <= 1e-8 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_multivariable_thermoelastic_matches_oracle(pkg, cuda, precision):
    m10, m4 = thermo_meshes(pkg)
    prob, oracle, _, _ = thermo_problem(pkg, m10, m4)
    c_scale = np.random.default_rng(5).uniform(0.5, 2.0, size=prob.num_cells)
    prob.internal_vars = [torch.tensor(c_scale, device=cuda)]
    oracle.internal_vars = [c_scale]
    sol_u, sol_T = pkg.solver(prob, {"newton": {"rel_tol": 1e-11, "tol": 1e-14, "precision": precision,
                                               "linear": LIN_BICG}})
    assert sol_u.shape == (len(m10.points), 3) and sol_T.shape == (len(m4.points), 1)
    ref = oracle.newton()
    got = torch.cat([sol_u.reshape(-1), sol_T.reshape(-1)]).cpu().numpy()
    tol = 1e-9 if precision == "fp64" else 1e-6
    assert np.abs(got - ref).max() <= tol * np.abs(ref).max()
    assert np.abs(ref[prob.offset[1]:]).max() > 0.1  # the temperature field is not trivial


@pytest.mark.gpu
def test_u_dependent_mass_map_matches_oracle(pkg, cuda):
    mesh = perturbed_box(pkg, (4, 3, 3), seed=9)
    bc = [[face_fn(0, 0.0), face_fn(0, 1.0)], [0, 0], [lambda p: 0.0, lambda p: 1.0]]

    class Reaction(pkg.Problem):
        def get_tensor_map(self):
            return lambda g: g

        def get_mass_map(self):
            return lambda u, x: 5.0 * u ** 3 - 2.0 * x[..., 1:2]

    prob = Reaction(mesh, vec=1, dim=3, dirichlet_bc_info=bc)
    assert prob.cell_path
    sol = pkg.solver(prob, {"newton": {"rel_tol": 1e-11, "tol": 1e-14, "linear": LIN_BICG}})[0]
    kp = fo.KernelProblem([dict(points=mesh.points, cells=mesh.cells, vec=1, dirichlet=bc)],
                          tensor_map=lambda g: g, mass_map=lambda u, x: 5.0 * u ** 3 - 2.0 * x[1:2])
    ref = kp.newton()
    got = sol.cpu().numpy().reshape(-1)
    assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max()


@pytest.mark.gpu
def test_cell_path_adjoint_matches_finite_differences(pkg, cuda):
    m10, m4 = thermo_meshes(pkg)
    prob, _, _, _ = thermo_problem(pkg, m10, m4)
    prob.set_params = lambda params: setattr(prob, "internal_vars", [params])
    opts = {"newton": {"rel_tol": 1e-12, "tol": 1e-14, "linear": LIN_BICG}}
    fwd = pkg.ad_wrapper(prob, opts, LIN_BICG)
    rng = np.random.default_rng(8)
    c0 = rng.uniform(0.5, 2.0, size=prob.num_cells)

    def objective(sols):
        u, T = sols
        return (T ** 2).sum() + 10.0 * (u ** 2).sum()

    c = torch.tensor(c0, device=cuda, requires_grad=True)
    J = objective(fwd(c))
    J.backward()
    g = c.grad.cpu().numpy()
    h = 1e-4
    for k in rng.choice(prob.num_cells, size=3, replace=False):
        vals = []
        for sgn in (1, -1):
            cc = c0.copy()
            cc[k] += sgn * h
            vals.append(objective(fwd(torch.tensor(cc, device=cuda))).item())
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(abs(g).max(), 1e-12), (k, fd, g[k])


@pytest.mark.gpu
def test_registered_law_with_u_dependent_load_matches_oracle(pkg, cuda):
    """A registered law with a u-dependent body load goes to the cell-kernel
    path as its torch form: Newton on a jittered HEX8 box vs the oracle's
    KernelProblem with the oracle's Neo-Hookean stress (1e-9)."""
    mesh = perturbed_box(pkg, (3, 2, 2), seed=11)
    bc = [[face_fn(0, 0.0)] * 3 + [face_fn(0, 1.0)], [0, 1, 2, 0], [lambda p: 0.0] * 3 + [lambda p: 0.05]]

    class NHReaction(pkg.Problem):
        def get_tensor_map(self):
            return pkg.NeoHookean(10.0, 0.3)

        def get_mass_map(self):
            return lambda u, x: 2.0 * u ** 3

    prob = NHReaction(mesh, vec=3, dim=3, dirichlet_bc_info=bc)
    assert prob.cell_path
    sol = pkg.solver(prob, {"newton": {"rel_tol": 1e-11, "tol": 1e-14, "linear": LIN_BICG}})[0]
    kp = fo.KernelProblem([dict(points=mesh.points, cells=mesh.cells, vec=3, dirichlet=bc)],
                          tensor_map=lambda ug: fo.stress_neo_hookean(ug, 10.0, 0.3),
                          mass_map=lambda u, x: 2.0 * u ** 3)
    ref = kp.newton()
    got = sol.cpu().numpy().reshape(-1)
    assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max()
