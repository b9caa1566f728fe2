"""MMA topology optimisation driving the solver on the GPU (jax-fem_b200/mma.py).

A 24x12x12 SIMP cantilever (clamped at x=0, unit traction on a patch of the
x=24 face), compliance minimised under a 40 % volume constraint as in the
reference's topology-optimisation example: the compliance and its gradient
come from ad_wrapper (multigrid CG forward and adjoint), the constraint is
mean(rho)/0.4 - 1.  After 12 MMA iterations the compliance has fallen below
half of the uniform design's, the volume constraint holds (within 1e-3, and
the design uses at least 95 % of the allowed volume), every density lies in
[0, 1], and every MMA subproblem ended with its relaxed-KKT residual below
1e-6."""
import numpy as np
import pytest
import torch


@pytest.mark.gpu
def test_mma_compliance_minimisation(pkg, cuda):
    import importlib
    mma = importlib.import_module("jax_fem_b200.mma")
    nx, ny, nz, vf = 24, 12, 12, 0.4
    m = pkg.box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
    mesh = pkg.Mesh(m.points, m.cells_dict["hexahedron"])

    class Cantilever(pkg.Problem):
        def get_tensor_map(self):
            return pkg.SIMPElastic(70e3, 70.0, 0.3, 3.0)

        def get_surface_maps(self):
            return [lambda u, x: np.array([0.0, 0.0, 1.0])]

        def set_params(self, params):
            C = self.num_cells
            self.internal_vars = [params.reshape(C, 1, 1).expand(C, 8, 1)]

    fixed = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    patch = lambda p: np.isclose(p[0], float(nx), atol=1e-5) & (p[2] <= 3.0 + 1e-5)  # noqa: E731
    prob = Cantilever(mesh, vec=3, dim=3, dirichlet_bc_info=[[fixed] * 3, [0, 1, 2], [lambda p: 0.0 * p[0]] * 3],
                      location_fns=[patch])
    lin = {"cg": {"precond": "gmg", "rtol": 1e-10, "atol": 0.0}}
    fwd = pkg.ad_wrapper(prob, {"newton": {"rel_tol": 1e-8, "tol": 1e-14, "linear": lin}}, lin)
    fe = prob.fes[0]
    fe.flex_inds = np.arange(len(fe.cells))
    n = len(fe.cells)

    def objective(rho):
        rho = rho.detach().requires_grad_(True)
        J = pkg.compliance(prob, fwd(rho))
        (dJ,) = torch.autograd.grad(J, rho)
        return float(J.detach()), dJ

    def constraint(rho, it):
        g = rho.mean() / vf - 1.0
        return g.reshape(1), torch.full((1, n, 1), 1.0 / (n * vf), dtype=torch.float64, device=rho.device)

    rho0 = torch.full((n, 1), vf, dtype=torch.float64, device=cuda)
    rho = mma.optimize(fe, rho0, {"maxIters": 12, "movelimit": 0.2}, objective, constraint, 1)
    hist = mma.optimize.history
    J0, J_end = hist[0]["J"], objective(rho)[0]
    print("compliance", [round(h["J"], 2) for h in hist], "final", round(J_end, 2),
          "mma step ms", round(1e3 * float(np.mean([h["mma_s"] for h in hist[1:]])), 1))
    assert J_end < 0.5 * J0
    g_end = float(rho.mean()) / vf - 1.0  # MMA's convex model of a linear constraint is conservative
    assert -0.05 <= g_end <= 1e-3
    assert float(rho.min()) >= 0.0 and float(rho.max()) <= 1.0
    assert max(h["kkt"] for h in hist) <= 1e-6
