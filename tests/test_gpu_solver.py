"""Solver-level parity on the GPU: Krylov methods / preconditioners / error
codes, the mixed-precision path, the SIMP adjoint, and J2 with hardening over
load increments -- each against the FP64 oracle or scipy on the same input.

Tolerances: FP64 Krylov solutions 1e-8 relative to scipy spsolve of the same
matrix (rtol 1e-12 solves); mixed path within 1e-6 of the FP64 oracle (the
stated refinement tolerance); adjoint gradient 1e-8 vs the oracle's
implicit VJP and 1e-5 vs central finite differences (h = 1e-6)."""
import importlib
import math

import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

from helpers import make_problem, perturbed_box
from oracle import fem_oracle as fo


def _solver_mod():
    return importlib.import_module("jax_fem_b200.solver")


def _elastic_system(pkg, cuda, fp32=False, N=(5, 4, 6)):
    mesh = perturbed_box(pkg, N, seed=4)
    left = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    prob = make_problem(pkg, mesh, pkg.LinearElastic(70e3, 0.3), bc=[[left] * 3, [0, 1, 2], [lambda p: 0.0] * 3])
    A = prob.dev().new_matrix(torch.float32 if fp32 else torch.float64)
    u0 = torch.zeros(prob.num_total_dofs_all_vars, dtype=torch.float64, device=cuda)
    prob.assemble(u0, vals=A.vals, fp32=fp32)
    rng = np.random.default_rng(0)
    b = rng.normal(size=prob.num_total_dofs_all_vars)
    return prob, A, b


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["cg", "bicgstab"])
@pytest.mark.parametrize("precond", ["none", "jacobi", "block_jacobi"])
@pytest.mark.parametrize("fp32", [False, True])
def test_krylov_matches_direct_solve(pkg, cuda, method, precond, fp32):
    S = _solver_mod()
    prob, A, b = _elastic_system(pkg, cuda, fp32=fp32)
    dt = torch.float32 if fp32 else torch.float64
    K = A.to_scipy()
    xref = spla.spsolve(K.tocsc(), b)
    bd = torch.tensor(b, dtype=dt, device=cuda)
    x = torch.zeros_like(bd)
    cfg = S.resolve_linear({method: {"precond": precond, "rtol": 1e-5 if fp32 else 1e-12, "atol": 0.0,
                                     "maxiter": 20000}})
    it, rel = S.krylov_solve(A, bd, x, cfg)
    assert it > 0
    err = np.abs(x.double().cpu().numpy() - xref).max() / np.abs(xref).max()
    assert err < (1e-3 if fp32 else 1e-8), err
    # the reported relative residual is the true one, and it meets the tolerance
    r = b - K @ x.double().cpu().numpy()
    true_rel = np.linalg.norm(r) / np.linalg.norm(b)
    assert true_rel <= cfg.rtol * (1.0 + (1e-2 if fp32 else 1e-6))
    assert abs(true_rel - rel) <= (1e-6 if fp32 else 1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("precond", ["none", "jacobi", "block_jacobi"])
def test_mixed_reliable_cg_matches_direct_solve(pkg, cuda, precond):
    """FP32 matrix, FP64 b and x: reliable-update CG reaches 1e-10 on the
    true residual of the FP32-valued matrix (out of reach of FP32 CG alone),
    and the solution matches a direct FP64 solve of that matrix to 1e-8."""
    S = _solver_mod()
    prob, A32, b = _elastic_system(pkg, cuda, fp32=True)
    K = A32.to_scipy().astype(np.float64)
    xref = spla.spsolve(K.tocsc(), b)
    bd = torch.tensor(b, dtype=torch.float64, device=cuda)
    x = torch.zeros_like(bd)
    cfg = S.resolve_linear({"cg": {"precond": precond, "rtol": 1e-10, "atol": 0.0, "maxiter": 20000}})
    it, nrep, rel = S.reliable_solve(A32, bd, x, cfg, S._Workspaces())
    assert it > 0 and nrep > 0
    xs = x.cpu().numpy()
    assert np.abs(xs - xref).max() / np.abs(xref).max() < 1e-8
    true_rel = np.linalg.norm(b - K @ xs) / np.linalg.norm(b)
    assert true_rel <= 1e-10 * (1.0 + 1e-6)
    assert abs(true_rel - rel) <= 1e-3 * true_rel
    # a second solve from the converged x is immediate
    it2, _, _ = S.reliable_solve(A32, bd, x, cfg, S._Workspaces())
    assert it2 == 0


@pytest.mark.gpu
def test_mixed_reliable_cg_error_codes(pkg, cuda):
    S = _solver_mod()
    nat = pkg._native
    prob, A32, b = _elastic_system(pkg, cuda, fp32=True)
    bd = torch.tensor(b, dtype=torch.float64, device=cuda)
    x = torch.zeros_like(bd)
    with pytest.raises(nat.FEMNativeError) as ei:
        S.reliable_solve(A32, bd, x, S.resolve_linear({"cg": {"rtol": 1e-12, "maxiter": 5}}), S._Workspaces())
    assert ei.value.status == nat.FEM_ERR_NOT_CONVERGED
    with pytest.raises(nat.FEMNativeError) as ei:
        S.reliable_solve(A32, bd, x, S.resolve_linear({"cg": {"reliable_delta": 1.5}}), S._Workspaces())
    assert ei.value.status == nat.FEM_ERR_ARG
    bd[7] = float("nan")
    x.zero_()
    with pytest.raises(nat.FEMNativeError) as ei:
        S.reliable_solve(A32, bd, x, S.resolve_linear({"cg": {}}), S._Workspaces())
    assert ei.value.status == nat.FEM_ERR_NONFINITE


@pytest.mark.gpu
def test_krylov_error_codes(pkg, cuda):
    S = _solver_mod()
    nat = pkg._native
    prob, A, b = _elastic_system(pkg, cuda)
    bd = torch.tensor(b, device=cuda)
    x = torch.zeros_like(bd)
    with pytest.raises(nat.FEMNativeError) as ei:
        S.krylov_solve(A, bd, x, S.resolve_linear({"cg": {"rtol": 1e-14, "maxiter": 3}}))
    assert ei.value.status == nat.FEM_ERR_NOT_CONVERGED
    bd[5] = float("nan")
    x.zero_()
    with pytest.raises(nat.FEMNativeError) as ei:
        S.krylov_solve(A, bd, x, S.resolve_linear({"cg": {}}))
    assert ei.value.status == nat.FEM_ERR_NONFINITE
    # zero right-hand side converges immediately with x = 0
    x.zero_()
    it, rel = S.krylov_solve(A, torch.zeros_like(bd), x, S.resolve_linear({"cg": {}}))
    assert it == 0 and float(x.abs().max()) == 0.0


def _twist(pkg, n, deg):
    th = math.radians(deg)
    c, s = math.cos(th), math.sin(th)
    left = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    right = lambda p: np.isclose(p[0], 1.0, atol=1e-5)  # noqa: E731
    uy = lambda p: 0.5 + (p[1] - 0.5) * c - (p[2] - 0.5) * s - p[1]  # noqa: E731
    uz = lambda p: 0.5 + (p[1] - 0.5) * s + (p[2] - 0.5) * c - p[2]  # noqa: E731
    z = lambda p: 0.0 * p[0]  # noqa: E731
    return [[left] * 3 + [right] * 3, [0, 1, 2] * 2, [z, z, z, z, uy, uz]]


@pytest.mark.gpu
@pytest.mark.parametrize("precision,rtol,delta", [("fp64", 1e-10, 0.1), ("mixed", 1e-10, 0.1),
                                                  ("mixed", "adaptive", 0.1), ("mixed", "adaptive", 0.0)])
def test_newton_paths_match_oracle(pkg, cuda, precision, rtol, delta):
    """delta 0.1: mixed CG with reliable updates; delta 0: FP32 CG inside
    FP64 iterative refinement."""
    n = 6
    m = pkg.box_mesh(n, n, n, 1.0, 1.0, 1.0)
    mesh = pkg.Mesh(m.points, m.cells_dict["hexahedron"])
    bc = _twist(pkg, n, 20.0)
    prob = make_problem(pkg, mesh, pkg.NeoHookean(10.0, 0.3), bc=bc)
    opts = {"newton": {"rel_tol": 1e-8, "tol": 1e-14, "precision": precision,
                       "linear": {"cg": {"precond": "block_jacobi", "rtol": rtol, "atol": 0.0,
                                         "reliable_delta": delta}}}}
    sol = pkg.solver(prob, opts)[0].cpu().numpy().reshape(-1)
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, fo.Law("neo_hookean", E=10.0, nu=0.3), dirichlet_bc_info=bc)
    ref = fo.newton_solve(op, rel_tol=1e-12, tol=1e-14)
    err = np.abs(sol - ref).max() / np.abs(ref).max()
    assert err <= (1e-8 if precision == "fp64" else 1e-6), err
    # the oracle agrees that the GPU solution meets the Newton criterion
    r0 = np.linalg.norm(op.apply_bc_vec(op.residual(np.zeros(op.ndofs)), np.zeros(op.ndofs)))
    r = np.linalg.norm(op.apply_bc_vec(op.residual(sol), sol))
    assert r / r0 <= 1e-8


@pytest.mark.gpu
@pytest.mark.parametrize("precond", ["block_jacobi", "gmg"])
def test_arc_length_matches_oracle(pkg, cuda, precond):
    """Displacement-controlled arc-length continuation of a 30-degree twist
    (solver.py:521-597, 721-756): the load factor after every step equals the
    oracle's (direct solves) to 1e-8, the path reaches lambda >= 1, and the
    polished solution equals the oracle's Newton solution (1e-8)."""
    n = 4
    m = pkg.box_mesh(n, n, n, 1.0, 1.0, 1.0)
    mesh = pkg.Mesh(m.points, m.cells_dict["hexahedron"])
    bc = _twist(pkg, n, 30.0)
    prob = make_problem(pkg, mesh, pkg.NeoHookean(10.0, 0.3), bc=bc)
    lin = {"cg": {"precond": precond, "rtol": 1e-12, "atol": 0.0}}
    (sol,), info = pkg.solver(prob, {"arc_length": {"control": "displacement", "Delta_l": 0.3, "psi": 1.0,
                                                    "linear": lin, "return_info": True,
                                                    "newton": {"rel_tol": 1e-10, "tol": 1e-14}}})
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, fo.Law("neo_hookean", E=10.0, nu=0.3), dirichlet_bc_info=bc)
    ref_u, ref_lams = fo.arc_length_disp(op, Delta_l=0.3, psi=1.0)
    lams = [h["lam"] for h in info["history"]]
    assert len(lams) == len(ref_lams) and info["polished"] and lams[-1] >= 1.0
    np.testing.assert_allclose(lams, ref_lams, rtol=1e-8)
    sol = sol.cpu().numpy().reshape(-1)
    assert np.abs(sol - ref_u).max() <= 1e-8 * np.abs(ref_u).max()


@pytest.mark.gpu
def test_arc_length_force_control_matches_oracle(pkg, cuda):
    """Force-controlled arc-length (solver.py:607-685, 758-801) of a
    Neo-Hookean cantilever under an end traction: q_vec_aux is the residual
    at u = 0 of the same beam under the opposite traction (get_q_vec), so
    lambda = 0 is unloaded and lambda = 1 the full load.  Load factors step by
    step and the polished solution match the oracle (1e-8)."""
    S = _solver_mod()
    m = pkg.box_mesh(6, 2, 2, 3.0, 1.0, 1.0)
    mesh = pkg.Mesh(m.points, m.cells_dict["hexahedron"])
    left = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    right = lambda p: np.isclose(p[0], 3.0, atol=1e-5)  # noqa: E731
    z = lambda p: 0.0 * p[0]  # noqa: E731
    bc = [[left] * 3, [0, 1, 2], [z] * 3]
    T = 0.05
    law = pkg.NeoHookean(10.0, 0.3)
    prob = make_problem(pkg, mesh, law, bc=bc, location_fns=[right],
                        surface_maps=[lambda u, x: np.array([0.0, 0.0, T])])
    aux = make_problem(pkg, mesh, law, bc=bc, location_fns=[right],
                       surface_maps=[lambda u, x: np.array([0.0, 0.0, -T])])
    q = S.get_q_vec(aux)
    lin = {"cg": {"precond": "block_jacobi", "rtol": 1e-12, "atol": 0.0}}  # also the polishing solve's
    (sol,), info = pkg.solver(prob, {"arc_length": {"control": "force", "q_vec_aux": q, "Delta_l": 0.15,
                                                    "psi": 0.5, "return_info": True, "linear": lin,
                                                    "newton": {"rel_tol": 1e-10, "tol": 1e-14}}})
    olaw = fo.Law("neo_hookean", E=10.0, nu=0.3)
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, olaw, dirichlet_bc_info=bc, location_fns=[right],
                          surface_maps=[lambda u, x: np.array([0.0, 0.0, T])])
    oaux = fo.OracleProblem(mesh.points, mesh.cells, 3, olaw, dirichlet_bc_info=bc, location_fns=[right],
                            surface_maps=[lambda u, x: np.array([0.0, 0.0, -T])])
    qo = oaux.residual(np.zeros(oaux.ndofs))
    np.testing.assert_allclose(q.cpu().numpy(), qo, atol=1e-14)
    ref_u, ref_lams = fo.arc_length_force(op, qo, Delta_l=0.15, psi=0.5)
    lams = [h["lam"] for h in info["history"]]
    assert len(lams) == len(ref_lams) >= 5 and info["polished"] and info["control"] == "force"
    np.testing.assert_allclose(lams, ref_lams, rtol=1e-8)
    sol = sol.cpu().numpy().reshape(-1)
    assert np.abs(sol - ref_u).max() <= 1e-8 * np.abs(ref_u).max()
    with pytest.raises(ValueError):
        pkg.solver(prob, {"arc_length": {"control": "force"}})


@pytest.mark.gpu
@pytest.mark.parametrize("nkmat", [1000, 5])
def test_dynamic_relax_matches_oracle(pkg, cuda, nkmat):
    """Dynamic relaxation (solver.py:837-1047) of a 20-degree twist: the
    iteration count and the end point equal the oracle's (1e-9), and the end
    point is the Newton solution to within the tolerance (1e-6).  nKMat = 5
    also exercises the mass re-formed from a new tangent."""
    n = 3
    m = pkg.box_mesh(n, n, n, 1.0, 1.0, 1.0)
    mesh = pkg.Mesh(m.points, m.cells_dict["hexahedron"])
    bc = _twist(pkg, n, 20.0)
    prob = make_problem(pkg, mesh, pkg.NeoHookean(10.0, 0.3), bc=bc)
    (sol,) = pkg.solver(prob, {"dynamic_relax": {"tol": 1e-8, "nKMat": nkmat, "info": False, "info_force": False}})
    its = prob.last_solve_info["dr_iters"]
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, fo.Law("neo_hookean", E=10.0, nu=0.3), dirichlet_bc_info=bc)
    ref_u, ref_its = fo.dynamic_relax(op, tol=1e-8, nKMat=nkmat)
    sol = sol.cpu().numpy().reshape(-1)
    assert abs(its - ref_its) <= 1, (its, ref_its)
    assert np.abs(sol - ref_u).max() <= 1e-9 * np.abs(ref_u).max()
    newton = fo.newton_solve(op, rel_tol=1e-12, tol=1e-14)
    assert np.abs(sol - newton).max() <= 1e-6 * np.abs(newton).max()


@pytest.mark.gpu
def test_line_search_and_custom_solver(pkg, cuda):
    S = _solver_mod()
    n = 4
    m = pkg.box_mesh(n, n, n, 1.0, 1.0, 1.0)
    mesh = pkg.Mesh(m.points, m.cells_dict["hexahedron"])
    bc = _twist(pkg, n, 15.0)
    prob = make_problem(pkg, mesh, pkg.NeoHookean(10.0, 0.3), bc=bc)
    ref = pkg.solver(prob, {"newton": {"rel_tol": 1e-9, "tol": 1e-14, "linear": {"cg": {"rtol": 1e-12}}}})[0]
    ls = pkg.solver(prob, {"newton": {"rel_tol": 1e-9, "tol": 1e-14, "line_search_flag": True,
                                      "linear": {"cg": {"rtol": 1e-12}}}})[0]
    assert float((ls - ref).abs().max()) <= 1e-8 * float(ref.abs().max())
    calls = []

    def custom(A, b, x0, opts):
        calls.append(A.shape)
        x = x0.clone()
        S.krylov_solve(A, b, x, S.resolve_linear({"bicgstab": {"precond": "block_jacobi", "rtol": 1e-12}}))
        return x

    cs = pkg.solver(prob, {"newton": {"rel_tol": 1e-9, "tol": 1e-14, "linear": {"custom_solver": custom}}})[0]
    assert calls and float((cs - ref).abs().max()) <= 1e-8 * float(ref.abs().max())


def _cantilever(pkg, Nx=6, Ny=3, Nz=3):
    m = pkg.box_mesh(Nx, Ny, Nz, float(Nx), float(Ny), float(Nz))
    mesh = pkg.Mesh(m.points, m.cells_dict["hexahedron"])
    fixed = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    load = lambda p: np.isclose(p[0], float(Nx), atol=1e-5) & (p[2] <= 1.0 + 1e-5)  # noqa: E731
    bc = [[fixed] * 3, [0, 1, 2], [lambda p: 0.0 * p[0]] * 3]
    return mesh, bc, load


@pytest.mark.gpu
def test_simp_adjoint_matches_oracle_and_fd(pkg, cuda):
    mesh, bc, load = _cantilever(pkg)
    C = len(mesh.cells)
    smap = lambda u, x: np.array([0.0, 0.0, 1.0])  # noqa: E731  (unit downward traction)
    law = pkg.SIMPElastic(70e3, 70.0, 0.3, 3.0)

    class TO(pkg.Problem):
        def get_tensor_map(self):
            return law

        def get_surface_maps(self):
            return [smap]

        def set_params(self, params):
            self.internal_vars = [params[:, None, :].expand(C, 8, 1)]

    prob = TO(mesh, vec=3, dim=3, dirichlet_bc_info=bc, location_fns=[load])
    opts = {"newton": {"rel_tol": 1e-10, "tol": 1e-14,
                       "linear": {"cg": {"precond": "block_jacobi", "rtol": 1e-12, "atol": 0.0}}}}
    fwd = pkg.ad_wrapper(prob, opts, {"cg": {"precond": "block_jacobi", "rtol": 1e-12, "atol": 0.0}})
    rng = np.random.default_rng(5)
    rho0 = rng.uniform(0.2, 1.0, size=(C, 1))
    rho = torch.tensor(rho0, device=cuda, requires_grad=True)
    comp = pkg.compliance(prob, fwd(rho))
    comp.backward()
    g = rho.grad.cpu().numpy().reshape(-1)

    # oracle: the reference's implicit VJP with a direct solve
    th = np.repeat(rho0, 8, axis=1)
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, fo.Law("simp", E0=70e3, Emin=70.0, nu=0.3, penal=3.0),
                          dirichlet_bc_info=bc, location_fns=[load], surface_maps=[smap], internal_vars=[th])
    u = fo.newton_solve(op, rel_tol=1e-12, tol=1e-14)
    np.testing.assert_allclose(comp.item(), fo.compliance(op, u), rtol=1e-9)
    v = -op.surface_load()  # dC/du for C = -f_s . u
    gq = fo.implicit_vjp_cellwise(op, u, v)
    g_ref = gq.sum(axis=1)
    assert np.abs(g - g_ref).max() <= 1e-8 * np.abs(g_ref).max()

    # central finite differences on a few cells
    h = 1e-6
    for c in rng.choice(C, size=5, replace=False):
        vals = []
        for sgn in (1, -1):
            r = rho0.copy()
            r[c, 0] += sgn * h
            vals.append(pkg.compliance(prob, fwd(torch.tensor(r, device=cuda))).item())
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g[c]) <= 1e-5 * max(abs(g[c]), 1e-12 * abs(comp.item())), (c, fd, g[c])


@pytest.mark.gpu
def test_j2_hardening_increments_match_oracle(pkg, cuda):
    n = 4
    m = pkg.box_mesh(n, n, n, 1.0, 1.0, 1.0)
    mesh = pkg.Mesh(m.points, m.cells_dict["hexahedron"])
    C = len(mesh.cells)
    left = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    right = lambda p: np.isclose(p[0], 1.0, atol=1e-5)  # noqa: E731
    bc = [[left] * 3 + [right], [0, 1, 2, 0], [lambda p: 0.0] * 4]
    prob = make_problem(pkg, mesh, pkg.J2Plasticity(70e3, 0.3, 250.0, 700.0), bc=bc,
                        ivars=[torch.zeros(C, 8, 3, 3, dtype=torch.float64, device=cuda),
                               torch.zeros(C, 8, 3, 3, dtype=torch.float64, device=cuda),
                               torch.zeros(C, 8, dtype=torch.float64, device=cuda)])
    iv = [np.zeros((C, 8, 3, 3)), np.zeros((C, 8, 3, 3)), np.zeros((C, 8))]
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, fo.Law("j2", E=70e3, nu=0.3, sig0=250.0, H=700.0),
                          dirichlet_bc_info=bc, internal_vars=iv)
    opts = {"newton": {"rel_tol": 1e-10, "tol": 1e-12,
                       "linear": {"cg": {"precond": "block_jacobi", "rtol": 1e-13, "atol": 0.0}}}}
    for k in range(1, 5):
        d = 0.02 * k / 4
        bc[2][-1] = (lambda v: (lambda p: v))(d)
        prob.fes[0].update_Dirichlet_boundary_conditions(bc)
        op.update_dirichlet(bc)
        sol = pkg.solver(prob, opts)[0]
        prob.update_j2_state(sol)
        u = fo.newton_solve(op, rel_tol=1e-12, tol=1e-12)
        fo.j2_commit(op, u)
        assert np.abs(sol.cpu().numpy().reshape(-1) - u).max() <= 1e-8 * np.abs(u).max()
    sig = prob.internal_vars[0].cpu().numpy()
    alpha = prob.internal_vars[2].cpu().numpy()
    assert alpha.max() > 0  # the bar has yielded
    np.testing.assert_allclose(sig, op.internal_vars[0], rtol=0, atol=1e-7 * np.abs(op.internal_vars[0]).max())
    np.testing.assert_allclose(alpha, op.internal_vars[2], rtol=0, atol=1e-10)


def _oracle_j2_reaction(mesh, sig0, increments, total, mask):
    """Reaction force at the end of an oracle J2 load history (FP64, direct
    solves): the internal force summed over the dofs in ``mask``."""
    C = len(mesh.cells)
    left = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    right = lambda p: np.isclose(p[0], 1.0, atol=1e-5)  # noqa: E731
    bc = [[left] * 3 + [right], [0, 1, 2, 0], [lambda p: 0.0] * 4]
    iv = [np.zeros((C, 8, 3, 3)), np.zeros((C, 8, 3, 3)), np.zeros((C, 8))]
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, fo.Law("j2", E=70e3, nu=0.3, sig0=sig0, H=700.0),
                          dirichlet_bc_info=bc, internal_vars=iv)
    u = None
    for k in range(1, increments + 1):
        bc[2][-1] = (lambda v: (lambda p: v))(total * k / increments)
        op.update_dirichlet(bc)
        u = fo.newton_solve(op, initial_guess=u, rel_tol=1e-12, tol=1e-11)
        F = op.residual(u)[mask].sum()
        fo.j2_commit(op, u)
    return F


@pytest.mark.gpu
def test_j2_yield_sensitivity_matches_oracle_fd(pkg, cuda):
    """dF/dsigma_y of the end reaction of a 4-increment J2 history (4^3
    cells, plastic flow at the last three increments) from the direct
    sensitivity on the GPU vs a central difference of the oracle's history
    (h = 1e-2 on sigma_y = 250): 1e-6 relative.  The reaction itself matches
    the oracle's to 1e-9."""
    n, incs, total, sy = 4, 4, 0.02, 250.0
    m = pkg.box_mesh(n, n, n, 1.0, 1.0, 1.0)
    mesh = pkg.Mesh(m.points, m.cells_dict["hexahedron"])
    C = len(mesh.cells)
    left = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    right = lambda p: np.isclose(p[0], 1.0, atol=1e-5)  # noqa: E731
    bc = [[left] * 3 + [right], [0, 1, 2, 0], [lambda p: 0.0] * 4]
    prob = make_problem(pkg, mesh, pkg.J2Plasticity(70e3, 0.3, sy, 700.0), bc=bc,
                        ivars=[torch.zeros(C, 8, 3, 3, dtype=torch.float64, device=cuda),
                               torch.zeros(C, 8, 3, 3, dtype=torch.float64, device=cuda),
                               torch.zeros(C, 8, dtype=torch.float64, device=cuda)])
    mask_np = np.zeros(mesh.points.shape[0] * 3, dtype=bool)
    mask_np[np.flatnonzero(np.isclose(mesh.points[:, 0], 1.0, atol=1e-5)) * 3] = True
    mask = torch.from_numpy(mask_np).to(cuda)
    sens = pkg.J2YieldSensitivity(prob)
    opts = {"newton": {"rel_tol": 1e-11, "tol": 1e-12,
                       "linear": {"cg": {"precond": "block_jacobi", "rtol": 1e-13, "atol": 0.0}}}}
    sol = None
    for k in range(1, incs + 1):
        bc[2][-1] = (lambda v: (lambda p: v))(total * k / incs)
        prob.fes[0].update_Dirichlet_boundary_conditions(bc)
        sol = pkg.solver(prob, {"newton": dict(opts["newton"], initial_guess=sol)})[0]
        sens.step(sol)
        prob.update_j2_state(sol)
    F = float(pkg.j2_reaction(prob, mask))
    dF = float(sens.reaction(mask))
    assert prob.internal_vars[2].max().item() > 0.0
    F_ref = _oracle_j2_reaction(mesh, sy, incs, total, mask_np)
    assert abs(F - F_ref) <= 1e-9 * abs(F_ref), (F, F_ref)
    h = 1e-2
    fd = (_oracle_j2_reaction(mesh, sy + h, incs, total, mask_np)
          - _oracle_j2_reaction(mesh, sy - h, incs, total, mask_np)) / (2 * h)
    assert abs(dF - fd) <= 1e-6 * abs(fd), (dF, fd)
