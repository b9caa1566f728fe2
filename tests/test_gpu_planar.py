"""2D problems (QUAD4, QUAD8, TRI3, TRI6) end to end on the GPU: they run on
the cell-kernel path (torch kernels, ``fem_scatter_cells_*``, the scalar
CSR system and the library's Krylov solvers), each against the oracle:

- Poisson with the manufactured solution of the convergence study on TRI6
  and QUAD4: the solution equals the oracle's (1e-9 relative);
- a plane-strain Neo-Hookean body (a registered law) with a traction on
  QUAD8 cells: Newton equals the oracle's, FP64 (1e-9) and mixed
  precision (1e-6);
- ad_wrapper on a SIMP plate (QUAD4, one density per cell, the layout of
  the reference's 2D topology-optimisation example): the gradient of
  sum u^2 equals central differences (h = 1e-4, 1e-6 of the largest
  component)."""
import numpy as np
import pytest
import torch

from helpers import face_fn, planar_box
from oracle import fem_oracle as fo

# rtol 1e-12: on the QUAD8 Neo-Hookean body the true residual of BiCGSTAB floors near
# 1.3e-13 of ||b|| in FP64 (a 1e-13 request ran out there)
LIN_BICG = {"bicgstab": {"precond": "jacobi", "rtol": 1e-12, "atol": 0.0, "maxiter": 50000}}
NEWTON = {"newton": {"rel_tol": 1e-11, "tol": 1e-14, "linear": LIN_BICG}}


def _u_true(x, y, xp=np):
    return 1e2 * ((x - 0.5) ** 3 + 2.0 * xp.sin(2.0 * y) * xp.exp(x))


def _lap_true(x, y, xp=np):
    return 1e2 * (6.0 * (x - 0.5) - 6.0 * xp.sin(2.0 * y) * xp.exp(x))


def _boundary(p):
    return np.isclose(p[0], 0) | np.isclose(p[0], 1) | np.isclose(p[1], 0) | np.isclose(p[1], 1)


@pytest.mark.gpu
@pytest.mark.late
@pytest.mark.parametrize("ele", ["TRI6", "QUAD4"])
def test_planar_poisson_matches_oracle(pkg, cuda, ele):
    mesh = planar_box(pkg, ele, (6, 5), amp=0.1, seed=1)
    bc = [[_boundary], [0], [lambda p: _u_true(p[0], p[1])]]

    class Poisson(pkg.Problem):
        def get_tensor_map(self):
            return lambda g: g

        def get_mass_map(self):
            return lambda u, x: _lap_true(x[..., 0:1], x[..., 1:2], torch) + 0.0 * u

    prob = Poisson(mesh, vec=1, dim=2, ele_type=ele, dirichlet_bc_info=bc)
    assert prob.cell_path
    sol = pkg.solver(prob, NEWTON)[0]
    assert sol.shape == (len(mesh.points), 1)
    kp = fo.KernelProblem([dict(points=mesh.points, cells=mesh.cells, vec=1, ele_type=ele, dirichlet=bc)],
                          tensor_map=lambda g: g, mass_map=lambda u, x: np.array([_lap_true(x[0], x[1])]))
    ref = kp.newton(rel_tol=1e-13, tol=1e-13)
    got = sol.cpu().numpy().reshape(-1)
    assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.late
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_planar_neo_hookean_traction_matches_oracle(pkg, cuda, precision):
    mesh = planar_box(pkg, "QUAD8", (4, 2), L=(2.0, 1.0), amp=0.1, seed=2)
    bc = [[face_fn(0, 0.0)] * 2, [0, 1], [lambda p: 0.0] * 2]
    right = face_fn(0, 2.0)

    class Body(pkg.Problem):
        def get_tensor_map(self):
            return pkg.NeoHookean(10.0, 0.3)

        def get_surface_maps(self):
            return [lambda u, x: torch.stack([0.4 + 0.0 * x[0], -0.2 * x[1]])]

    prob = Body(mesh, vec=2, dim=2, ele_type="QUAD8", dirichlet_bc_info=bc, location_fns=[right])
    opts = {"newton": dict(NEWTON["newton"], precision=precision)}
    sol = pkg.solver(prob, opts)[0]

    def stress(ug):
        g = np.zeros((3, 3), dtype=ug.dtype)
        g[:2, :2] = ug
        return fo.stress_neo_hookean(g, 10.0, 0.3)[:2, :2]

    kp = fo.KernelProblem([dict(points=mesh.points, cells=mesh.cells, vec=2, ele_type="QUAD8", dirichlet=bc)],
                          tensor_map=stress, location_fns=[right],
                          surface_maps=[lambda u, x: np.array([0.4, -0.2 * x[1]])])
    ref = kp.newton(rel_tol=1e-13, tol=1e-13)
    got = sol.cpu().numpy().reshape(-1)
    tol = 1e-9 if precision == "fp64" else 1e-6
    assert np.abs(ref).max() > 0.05
    assert np.abs(got - ref).max() <= tol * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.late
def test_planar_simp_adjoint_matches_finite_differences(pkg, cuda):
    mesh = planar_box(pkg, "QUAD4", (6, 3), L=(2.0, 1.0))
    C, Q = len(mesh.cells), 4
    bc = [[face_fn(0, 0.0)] * 2, [0, 1], [lambda p: 0.0] * 2]
    right = face_fn(0, 2.0)

    class Plate(pkg.Problem):
        def get_tensor_map(self):
            return pkg.SIMPElastic(70e3, 70.0, 0.3, 3.0)

        def get_surface_maps(self):
            return [lambda u, x: torch.stack([0.0 * x[0], -1.0 + 0.0 * x[1]])]

        def set_params(self, params):
            self.internal_vars = [params[:, None].expand(C, Q)]

    prob = Plate(mesh, vec=2, dim=2, ele_type="QUAD4", dirichlet_bc_info=bc, location_fns=[right])
    fwd = pkg.ad_wrapper(prob, NEWTON, LIN_BICG)
    rng = np.random.default_rng(6)
    th0 = rng.uniform(0.3, 1.0, size=C)

    def objective(sols):
        return (sols[0] ** 2).sum()

    th = torch.tensor(th0, device=cuda, requires_grad=True)
    objective(fwd(th)).backward()
    g = th.grad.cpu().numpy()
    h = 1e-4
    for k in rng.choice(C, size=3, replace=False):
        vals = []
        for sgn in (1, -1):
            t = th0.copy()
            t[k] += sgn * h
            vals.append(objective(fwd(torch.tensor(t, device=cuda))).item())
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * np.abs(g).max(), (k, fd, g[k])
