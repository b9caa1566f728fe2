"""The reference's five integration tests (tests/benchmarks/*/test_*.py) run
through this package's public API on the GPU, against the FEniCSx golden
data at the reference's own tolerances (decimal=5 / decimal=3), and against
the FP64 oracle at 1e-8."""
import numpy as np
import pytest
import torch

from helpers import golden
from oracle import fem_oracle as fo

TIGHT = {"newton": {"rel_tol": 1e-10, "tol": 1e-12,
                    "linear": {"cg": {"precond": "block_jacobi", "rtol": 1e-13, "atol": 0.0}}}}


def _mesh(pkg, d):
    return pkg.Mesh(d["points"], d["cells"])


def _close(p):
    return lambda x: np.isclose(x, p, atol=1e-5)


@pytest.mark.gpu
def test_linear_poisson(pkg, cuda):
    d = golden("linear_poisson")

    class LinearPoisson(pkg.Problem):
        def get_tensor_map(self):
            return lambda x: x  # recognised as the identity tensor map

    left = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    right = lambda p: np.isclose(p[0], 1.0, atol=1e-5)  # noqa: E731
    bc = [[left, right], [0, 0], [lambda p: 0.0, lambda p: 1.0]]
    prob = LinearPoisson(_mesh(pkg, d), vec=1, dim=3, dirichlet_bc_info=bc)
    sol = pkg.solver(prob)[0].cpu().numpy()
    np.testing.assert_array_almost_equal(d["sol"], sol, decimal=5)


@pytest.mark.gpu
def test_linear_elasticity_cube(pkg, cuda):
    d = golden("linear_elasticity_cube")

    class LinearElasticity(pkg.Problem):
        def get_tensor_map(self):
            def stress(u_grad):
                E, nu = 70e3, 0.3
                mu = E / (2.0 * (1.0 + nu))
                lmbda = E * nu / ((1 + nu) * (1 - 2 * nu))
                eps = 0.5 * (u_grad + u_grad.T)
                return lmbda * np.trace(eps) * np.eye(3) + 2 * mu * eps
            return stress  # recognised as linear isotropic elasticity

        def get_mass_map(self):
            return lambda u, x: -np.array([0.0, 10.0, 10.0])

        def get_surface_maps(self):
            return [lambda u, x: -np.array([10.0, 0.0, 0.0])]

    left = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    right = lambda p: np.isclose(p[0], 1.0, atol=1e-5)  # noqa: E731
    bc = [[left] * 3, [0, 1, 2], [lambda p: 1.0] * 3]
    prob = LinearElasticity(_mesh(pkg, d), vec=3, dim=3, dirichlet_bc_info=bc, location_fns=[right])
    assert isinstance(prob.law, pkg.LinearElastic)
    sol = pkg.solver(prob)[0].cpu().numpy()
    np.testing.assert_array_almost_equal(d["sol"], sol, decimal=5)
    sol2 = pkg.solver(prob, TIGHT)[0].cpu().numpy()
    op = fo.OracleProblem(d["points"], d["cells"], 3, fo.Law("linear", E=70e3, nu=0.3), dirichlet_bc_info=bc,
                          location_fns=[right], mass_map=lambda u, x: -np.array([0.0, 10.0, 10.0]),
                          surface_maps=[lambda u, x: -np.array([10.0, 0.0, 0.0])])
    ref = fo.newton_solve(op).reshape(-1, 3)
    assert np.abs(sol2 - ref).max() <= 1e-8 * np.abs(ref).max()


@pytest.mark.gpu
def test_linear_elasticity_cylinder(pkg, cuda):
    d = golden("linear_elasticity_cylinder")
    mass = lambda u, x: -np.array([1e3 * x[0], 2e3 * x[1], 3e3 * x[2]])  # noqa: E731
    surf = lambda u, x: -np.array([1e3 * x[0] ** 2 + 1e3 * x[1] ** 2, 0.0, 0.0])  # noqa: E731

    class LinearElasticity(pkg.Problem):
        def get_tensor_map(self):
            return pkg.LinearElastic(70e3, 0.3)

        def get_mass_map(self):
            return mass

        def get_surface_maps(self):
            return [surf]

    top = lambda p: np.isclose(p[2], 10.0, atol=1e-5)  # noqa: E731
    bottom = lambda p: np.isclose(p[2], 0.0, atol=1e-5)  # noqa: E731
    bc = [[bottom] * 3, [0, 1, 2], [lambda p: 0.0] * 3]
    prob = LinearElasticity(_mesh(pkg, d), vec=3, dim=3, dirichlet_bc_info=bc, location_fns=[top])
    sol = pkg.solver(prob)[0].cpu().numpy()
    np.testing.assert_array_almost_equal(d["sol"], sol, decimal=3)
    # top surface area from the face geometry (test_linear_elasticity_cylinder.py:126-132)
    binds = prob.fes[0].get_boundary_conditions_inds([top])[0]
    _, scale = prob.fes[0].get_face_shape_grads(binds)
    np.testing.assert_almost_equal(d["surface_area"], scale.sum(), decimal=4)


@pytest.mark.gpu
def test_hyperelasticity(pkg, cuda):
    d = golden("hyperelasticity")

    class HyperElasticity(pkg.Problem):
        def get_tensor_map(self):
            return pkg.NeoHookean(1e3, 0.3)

    top = lambda p: np.isclose(p[2], 10.0, atol=1e-5)  # noqa: E731
    bottom = lambda p: np.isclose(p[2], 0.0, atol=1e-5)  # noqa: E731
    z = lambda p: 0.0  # noqa: E731
    bc = [[bottom] * 3 + [top] * 3, [0, 1, 2] * 2, [z] * 5 + [lambda p: 1.0]]
    prob = HyperElasticity(_mesh(pkg, d), vec=3, dim=3, dirichlet_bc_info=bc)
    sol = pkg.solver(prob)[0].cpu().numpy()
    np.testing.assert_array_almost_equal(d["sol"], sol, decimal=5)
    # traction on the top face (test_hyper_elasticity.py:46-71, 121-127)
    fe = prob.fes[0]
    binds = fe.get_boundary_conditions_inds([top])[0]
    g, scale = fe.get_face_shape_grads(binds)
    cu = sol[fe.cells[binds[:, 0]]]
    ug = np.einsum("fai,fqaj->fqij", cu, g)
    P = fo.stress_neo_hookean(ug, 1e3, 0.3)
    tz = np.sum((P @ np.array([0.0, 0.0, 1.0]))[..., 2] * scale)
    np.testing.assert_almost_equal(d["traction"], tz, decimal=5)


@pytest.mark.gpu
def test_plasticity(pkg, cuda):
    d = golden("plasticity")
    C = len(d["cells"])

    class Plasticity(pkg.Problem):
        def custom_init(self):
            self.fe = self.fes[0]
            z = torch.zeros(C, 8, 3, 3, dtype=torch.float64)
            self.internal_vars = [z, z.clone(), torch.zeros(C, 8, dtype=torch.float64)]

        def get_tensor_map(self):
            return pkg.J2Plasticity(70e3, 0.3, 250.0, 0.0)

    top = lambda p: np.isclose(p[2], 10.0, atol=1e-5)  # noqa: E731
    bottom = lambda p: np.isclose(p[2], 0.0, atol=1e-5)  # noqa: E731
    z = lambda p: 0.0  # noqa: E731
    bc = [[bottom] * 3 + [top] * 3, [0, 1, 2] * 2, [z] * 6]
    prob = Plasticity(_mesh(pkg, d), vec=3, dim=3, dirichlet_bc_info=bc)
    jxw = torch.tensor(prob.fes[0].JxW(), device=cuda)
    avg = []
    for disp in d["disps"]:
        bc[2][-1] = (lambda v: (lambda p: v))(float(disp))
        prob.fe.update_Dirichlet_boundary_conditions(bc)
        sol = pkg.solver(prob)[0]
        sig = prob.update_j2_state(sol)[0]
        avg.append(float((sig[:, :, 2, 2] * jxw).sum() / jxw.sum()))
    np.testing.assert_array_almost_equal(d["sol"], sol.cpu().numpy(), decimal=5)
    np.testing.assert_array_almost_equal(d["avg_stresses"], np.array(avg), decimal=3)
