"""``precond='amg'`` (amg.py: smoothed-aggregation AMG, the counterpart of
the reference's AMGX path, solver.py:136-259) through ``solver`` on the GPU,
on meshes the geometric multigrid cannot take:

- linear elasticity and Neo-Hookean Newton on a TET10 box whose nodes are
  randomly renumbered (no lattice numbering): the solution equals the
  oracle's (1e-8), with fewer CG iterations than block-Jacobi; the
  reference's ``amgx_solver`` key solves the same linear problem.  Newton
  stops at rel.res 1e-9: the residual at u = 0 is dominated by the
  Dirichlet rows (a mismatch of 0.05), while the free rows are forces of
  order E = 70e3 times the strains, so the assembled FP64 residual has a
  round-off floor near eps * 70e3 / 0.05 ~ 2e-11 of it (a 1e-11 request
  stalled there, at 1.97e-11); each linear solve still goes to 1e-11;
- Poisson on curved TRI6 cells (a 2D problem on the cell-kernel path):
  the solution equals the oracle's (1e-9)."""
import numpy as np
import pytest
import torch

from helpers import element_box, face_fn, planar_box
from oracle import fem_oracle as fo


def _renumbered_tet10(pkg):
    m = element_box(pkg, "TET10", (4, 3, 3), amp=0.1, seed=1)
    perm = np.random.default_rng(3).permutation(len(m.points))
    inv = np.argsort(perm)
    return pkg.Mesh(m.points[perm], inv[m.cells], "TET10")


@pytest.mark.gpu
@pytest.mark.late
@pytest.mark.parametrize("kind", ["linear", "neo_hookean"])
def test_amg_newton_on_renumbered_tet10(pkg, cuda, kind):
    mesh = _renumbered_tet10(pkg)
    bc = [[face_fn(0, 0.0)] * 3 + [face_fn(0, 1.0)] * 2, [0, 1, 2, 1, 2],
          [lambda p: 0.0] * 3 + [lambda p: 0.05, lambda p: -0.04]]
    law = pkg.LinearElastic(70e3, 0.3) if kind == "linear" else pkg.NeoHookean(10.0, 0.3)
    olaw = fo.Law("linear", E=70e3, nu=0.3) if kind == "linear" else fo.Law("neo_hookean", E=10.0, nu=0.3)

    class P(pkg.Problem):
        def get_tensor_map(self):
            return law

    iters = {}
    for precond in ("amg", "block_jacobi"):
        prob = P(mesh, vec=3, dim=3, ele_type="TET10", dirichlet_bc_info=bc)
        opts = {"newton": {"rel_tol": 1e-9, "tol": 1e-14, "return_info": True,
                           "linear": {"cg": {"precond": precond, "rtol": 1e-11, "atol": 0.0, "maxiter": 20000}}}}
        sol, info = pkg.solver(prob, opts)
        assert info["rel_res"] <= 1e-9, info["res_hist"]
        iters[precond] = sum(info["krylov_iters"])
        if precond == "amg":
            got = sol[0].cpu().numpy().reshape(-1)
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, olaw, dirichlet_bc_info=bc, ele_type="TET10")
    ref = fo.newton_solve(op, rel_tol=1e-12, tol=1e-14)
    assert np.abs(got - ref).max() <= 1e-8 * np.abs(ref).max()
    assert iters["amg"] < iters["block_jacobi"], iters
    if kind == "linear":
        prob = P(mesh, vec=3, dim=3, ele_type="TET10", dirichlet_bc_info=bc)
        sol = pkg.solver(prob, {"newton": {"rel_tol": 1e-9, "tol": 1e-14, "linear": {"amgx_solver": {}}}})[0]
        assert np.abs(sol.cpu().numpy().reshape(-1) - ref).max() <= 1e-8 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.late
def test_amg_on_tri6_poisson(pkg, cuda):
    mesh = planar_box(pkg, "TRI6", (10, 8), amp=0.05, seed=4)
    bnd = lambda p: np.isclose(p[0], 0.0) | np.isclose(p[0], 1.0)  # noqa: E731

    class Poisson(pkg.Problem):
        def get_tensor_map(self):
            return lambda g: g

        def get_mass_map(self):
            return lambda u, x: 10.0 * torch.sin(3.0 * x[..., 0:1]) * x[..., 1:2] + 0.0 * u

    bc = [[bnd], [0], [lambda p: 0.0]]
    prob = Poisson(mesh, vec=1, dim=2, ele_type="TRI6", dirichlet_bc_info=bc)
    sol = pkg.solver(prob, {"newton": {"rel_tol": 1e-11, "tol": 1e-14,
                                       "linear": {"cg": {"precond": "amg", "rtol": 1e-12, "atol": 0.0}}}})[0]
    kp = fo.KernelProblem([dict(points=mesh.points, cells=mesh.cells, vec=1, ele_type="TRI6", dirichlet=bc)],
                          tensor_map=lambda g: g,
                          mass_map=lambda u, x: np.array([10.0 * np.sin(3.0 * x[0]) * x[1]]))
    ref = kp.newton(rel_tol=1e-13, tol=1e-13)
    got = sol.cpu().numpy().reshape(-1)
    assert np.abs(ref).max() > 0.01
    assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max()
