"""The benchmark configurations at full size, checked through properties that
do not need an oracle solve of the whole problem:

- 20^3 linear elasticity (27,783 dofs): GPU solution vs the oracle's direct
  solve (1e-8 relative).
- 50^3 Neo-Hookean, 30 degree twist in 5 steps (397,953 dofs): the oracle's
  own residual of the GPU solution is <= 1e-8 of its residual at u = 0, on
  both the plain FP64 and the mixed path; the two paths agree to 1e-6.
- 60x30x30 SIMP (175,863 dofs), seeded Gaussian random density: compliance
  gradient from the adjoint vs central finite differences on 20 random cells
  (h = 1e-6: 1e-5 relative plus the round-off of C over 2h; h = 1e-4: 1e-6
  relative) and along a random smooth direction (1e-4).  The 1e-8
  comparison with the oracle's implicit VJP is in test_gpu_solver.py, at a
  size the oracle solves directly.
- 40^3 J2 with hardening, 10 increments of u_x(x=1) up to 0.02 (206,763
  dofs): after the last increment the oracle's residual, evaluated with the
  GPU's committed state of increment 9, is <= 1e-8 of its value at the
  increment's start; the committed state equals the oracle's return map;
  the direct sensitivity of the end reaction to the yield stress matches a
  central difference of two more histories (1e-5 relative).
"""
import importlib
import math

import numpy as np
import pytest
import torch

from oracle import fem_oracle as fo


def _rel_residual(op, u, u_ref):
    r = np.linalg.norm(op.apply_bc_vec(op.residual(u), u))
    r0 = np.linalg.norm(op.apply_bc_vec(op.residual(u_ref), u_ref))
    return r / r0


@pytest.mark.gpu
def test_config_linear_20(pkg, cuda):
    n = 20
    m = pkg.box_mesh(n, n, n, 1.0, 1.0, 1.0)
    mesh = pkg.Mesh(m.points, m.cells_dict["hexahedron"])
    left = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    right = lambda p: np.isclose(p[0], 1.0, atol=1e-5)  # noqa: E731
    bc = [[left] * 3 + [right], [0, 1, 2, 0], [lambda p: 0.0 * p[0]] * 3 + [lambda p: 0.01 + 0.0 * p[0]]]

    class LE(pkg.Problem):
        def get_tensor_map(self):
            return pkg.LinearElastic(70e3, 0.3)

    prob = LE(mesh, vec=3, dim=3, dirichlet_bc_info=bc)
    sol = pkg.solver(prob, {"newton": {"linear": {"cg": {"precond": "jacobi", "rtol": 1e-10, "atol": 0.0}},
                                       "tol": 1e-14}})[0].cpu().numpy().reshape(-1)
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, fo.Law("linear", E=70e3, nu=0.3), dirichlet_bc_info=bc)
    ref = fo.newton_solve(op, tol=1e-14)
    assert np.abs(sol - ref).max() <= 1e-8 * np.abs(ref).max()


@pytest.mark.gpu
def test_config_neo_hookean_50(pkg, cuda):
    import bench
    prob = bench.nh_problem(pkg, 50)
    lin = {"cg": {"precond": "block_jacobi", "rtol": "adaptive", "atol": 0.0, "maxiter": 20000}}
    sol_m, infos_m = bench.nh_solve(pkg, prob, "mixed", linear=lin)
    sol_p, _ = bench.nh_solve(pkg, prob, "fp64")
    um = sol_m.cpu().numpy().reshape(-1)
    up = sol_p.cpu().numpy().reshape(-1)
    assert np.abs(um - up).max() <= 1e-6 * np.abs(up).max()
    bc = bench.rotation_bc(math.radians(30.0))
    op = fo.OracleProblem(prob.mesh.points, prob.mesh.cells, 3, fo.Law("neo_hookean", E=10.0, nu=0.3),
                          dirichlet_bc_info=bc)
    zero = np.zeros(op.ndofs)
    for u in (um, up):
        assert _rel_residual(op, u, zero) <= 1e-8


@pytest.mark.gpu
def test_config_neo_hookean_50_headline_path(pkg, cuda):
    """The exact path bench.py times as its headline value (mixed precision,
    FP64 CG over an FP32 multigrid V-cycle, Eisenstat-Walker forcing, coarse
    operators kept for up to 4 Newton solves): the oracle's residual of its
    solution is <= 1e-8 of the residual at u = 0, and it agrees with the
    plain FP64 path (tight block-Jacobi CG) to 1e-6.  Run twice, so that the
    second solve starts with the hierarchy the first left behind."""
    import bench
    prob = bench.nh_problem(pkg, 50)
    sol_p, _ = bench.nh_solve(pkg, prob, "fp64")
    up = sol_p.cpu().numpy().reshape(-1)
    bc = bench.rotation_bc(math.radians(30.0))
    op = fo.OracleProblem(prob.mesh.points, prob.mesh.cells, 3, fo.Law("neo_hookean", E=10.0, nu=0.3),
                          dirichlet_bc_info=bc)
    zero = np.zeros(op.ndofs)
    for _ in range(2):
        sol_h, infos = bench.nh_solve(pkg, prob, bench.HEADLINE_PRECISION, linear=bench.HEADLINE_LINEAR)
        uh = sol_h.cpu().numpy().reshape(-1)
        assert all(i["rel_res"] <= 1e-8 for i in infos)
        assert np.abs(uh - up).max() <= 1e-6 * np.abs(up).max()
        assert _rel_residual(op, uh, zero) <= 1e-8


@pytest.mark.gpu
def test_config_simp_adjoint_vs_fd(pkg, cuda):
    ws = importlib.import_module("jax_fem_b200.warmstart")
    prob = ws.cantilever_problem(z0=0.0)
    g = torch.Generator().manual_seed(20261203)
    rho0 = ws.random_density(g).reshape(-1).double()
    lin = {"cg": {"precond": "block_jacobi", "rtol": 1e-11, "atol": 0.0, "maxiter": 50000}}
    opts = {"newton": {"rel_tol": 1e-10, "tol": 1e-30, "linear": lin}}
    fwd = pkg.ad_wrapper(prob, opts, lin)
    rho = rho0.to(cuda).requires_grad_(True)
    sol = fwd(rho)
    c = pkg.compliance(prob, sol)
    c.backward()
    grad = rho.grad.cpu().numpy()
    # The problem is linear, so each perturbed solve is one Newton step from
    # the base solution with a tight CG (rtol 1e-11 of the O(h) right-hand
    # side): the change in u is computed to ~1e-11 relative, and C is then
    # exact to within the round-off of C itself (~1e-16 C).  That round-off,
    # divided by 2h, is the noise term of the h = 1e-6 check; at h = 1e-4 the
    # noise is 100x smaller and the truncation error (h^2) still negligible,
    # so that check is held to 1e-6.
    fd_lin = {"cg": {"precond": "block_jacobi", "rtol": 1e-11, "atol": 0.0, "maxiter": 50000}}
    fd_opts = {"newton": {"rel_tol": 1e-3, "tol": 1e-30, "linear": fd_lin,
                          "initial_guess": sol[0].detach().clone()}}

    def comp(r):
        prob.set_params(r.to(cuda))
        return pkg.compliance(prob, pkg.solver(prob, fd_opts)).item()

    def fd_at(cell, h):
        rp, rm = rho0.clone(), rho0.clone()
        rp[cell] += h
        rm[cell] -= h
        return (comp(rp) - comp(rm)) / (2 * h)

    rng = np.random.default_rng(7)
    cval = abs(c.item())
    for cell in rng.choice(len(rho0), size=20, replace=False):
        g_ad = grad[cell]
        fd6 = fd_at(cell, 1e-6)
        assert abs(fd6 - g_ad) <= 1e-5 * abs(g_ad) + 4e-16 * cval / 1e-6, (cell, fd6, g_ad)
        fd4 = fd_at(cell, 1e-4)
        assert abs(fd4 - g_ad) <= 1e-6 * abs(g_ad), (cell, fd4, g_ad)
    h = 1e-6
    # directional derivative along a random smooth field
    gdir = torch.Generator().manual_seed(11)
    dr = ws.gaussian_random_field((ws.NX, ws.NY, ws.NZ), 4.0, gdir).reshape(-1)
    fd = (comp(rho0 + h * dr) - comp(rho0 - h * dr)) / (2 * h)
    ad = float(np.dot(grad, dr.numpy()))
    assert abs(fd - ad) <= 1e-4 * abs(ad), (fd, ad)


def _j2_history(pkg, cuda, mesh, sy, with_sens, rel_tol=1e-8, precision="fp64", linear=None):
    """10 increments of u_x(x=1) up to 0.02 on the J2 cube; returns the
    problem, the last solution, the state before the last commit, the last
    start, the bc list, the end reaction F and (with_sens) dF/dsigma_y."""
    C = len(mesh.cells)
    left = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    right = lambda p: np.isclose(p[0], 1.0, atol=1e-5)  # noqa: E731
    bc = [[left] * 3 + [right], [0, 1, 2, 0], [lambda p: 0.0 * p[0]] * 4]
    z = lambda *s: torch.zeros(*s, dtype=torch.float64, device=cuda)  # noqa: E731

    class J2(pkg.Problem):
        def get_tensor_map(self):
            return pkg.J2Plasticity(70e3, 0.3, sy, 700.0)

    prob = J2(mesh, vec=3, dim=3, dirichlet_bc_info=bc)
    prob.internal_vars = [z(C, 8, 3, 3), z(C, 8, 3, 3), z(C, 8)]
    sens = pkg.J2YieldSensitivity(prob) if with_sens else None
    opts = {"newton": {"rel_tol": rel_tol, "tol": 1e-14, "precision": precision,
                       "linear": linear or {"cg": {"precond": "block_jacobi", "rtol": 1e-10, "atol": 0.0,
                                                   "maxiter": 20000}}}}
    sol = None
    for k in range(1, 11):
        bc[2][-1] = (lambda v: (lambda p: v + 0.0 * p[0]))(0.02 * k / 10)
        prob.fes[0].update_Dirichlet_boundary_conditions(bc)
        prev_state = [t.cpu().numpy() for t in prob.internal_vars]
        start = sol.cpu().numpy().reshape(-1) if sol is not None else np.zeros(prob.num_total_dofs_all_vars)
        sol = pkg.solver(prob, {"newton": dict(opts["newton"], initial_guess=sol)})[0]
        if sens is not None:
            sens.step(sol)
        prob.update_j2_state(sol)
    mask = torch.zeros(prob.num_total_dofs_all_vars, dtype=torch.bool, device=cuda)
    mask[torch.from_numpy(np.flatnonzero(np.isclose(mesh.points[:, 0], 1.0, atol=1e-5)) * 3).to(cuda)] = True
    F = float(pkg.j2_reaction(prob, mask))
    dF = float(sens.reaction(mask)) if sens is not None else None
    return prob, sol, prev_state, start, bc, F, dF


@pytest.mark.gpu
def test_config_j2_40(pkg, cuda):
    n = 40
    m = pkg.box_mesh(n, n, n, 1.0, 1.0, 1.0)
    mesh = pkg.Mesh(m.points, m.cells_dict["hexahedron"])
    prob, sol, prev_state, start, bc, F, dF = _j2_history(pkg, cuda, mesh, 250.0, True)
    u = sol.cpu().numpy().reshape(-1)
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, fo.Law("j2", E=70e3, nu=0.3, sig0=250.0, H=700.0),
                          dirichlet_bc_info=bc, internal_vars=[prev_state[0], prev_state[1], prev_state[2]])
    assert _rel_residual(op, u, start) <= 1e-8
    fo.j2_commit(op, u)
    sig = prob.internal_vars[0].cpu().numpy()
    assert np.abs(sig - op.internal_vars[0]).max() <= 1e-8 * np.abs(op.internal_vars[0]).max()
    assert prob.internal_vars[2].max().item() > 0.0  # plastic flow happened
    # d(reaction)/d(sigma_y) vs a central difference of two more histories
    # solved to 1e-11 (h = 1e-2: truncation and solve noise both below 1e-7)
    h = 1e-2
    Fp = _j2_history(pkg, cuda, mesh, 250.0 + h, False, rel_tol=1e-11)[5]
    Fm = _j2_history(pkg, cuda, mesh, 250.0 - h, False, rel_tol=1e-11)[5]
    fd = (Fp - Fm) / (2 * h)
    print(f"J2 40^3: reaction {F:.10g}, dF/dsigma_y {dF:.10g}, central difference {fd:.10g}")
    assert abs(dF - fd) <= 1e-5 * abs(fd), (dF, fd)


@pytest.mark.gpu
def test_config_j2_40_mixed_gmg(pkg, cuda):
    """The J2 40^3 history on the mixed multigrid path bench.py times
    (mixed precision, FP64 CG over an FP32 V-cycle, adaptive forcing): after
    the last increment the oracle's residual is <= 1e-8 of its value at the
    increment's start, the committed state equals the oracle's return map
    (1e-8), and the solution agrees with the plain FP64 history to 1e-6."""
    n = 40
    m = pkg.box_mesh(n, n, n, 1.0, 1.0, 1.0)
    mesh = pkg.Mesh(m.points, m.cells_dict["hexahedron"])
    gmg = {"cg": {"precond": "gmg", "rtol": "adaptive", "atol": 0.0, "maxiter": 20000}}
    prob, sol, prev_state, start, bc, F, _ = _j2_history(pkg, cuda, mesh, 250.0, False, precision="mixed",
                                                         linear=gmg)
    u = sol.cpu().numpy().reshape(-1)
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, fo.Law("j2", E=70e3, nu=0.3, sig0=250.0, H=700.0),
                          dirichlet_bc_info=bc, internal_vars=[prev_state[0], prev_state[1], prev_state[2]])
    assert _rel_residual(op, u, start) <= 1e-8
    fo.j2_commit(op, u)
    sig = prob.internal_vars[0].cpu().numpy()
    assert np.abs(sig - op.internal_vars[0]).max() <= 1e-8 * np.abs(op.internal_vars[0]).max()
    _, sol_p, _, _, _, F_p, _ = _j2_history(pkg, cuda, mesh, 250.0, False)
    up = sol_p.cpu().numpy().reshape(-1)
    assert np.abs(u - up).max() <= 1e-6 * np.abs(up).max()
    assert abs(F - F_p) <= 1e-6 * abs(F_p)
