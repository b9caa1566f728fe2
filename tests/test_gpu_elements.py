"""General-element path on the GPU (fem_assemble_elem_*, fem_j2_commit_elem,
fem_param_vjp_elem_f64 through ``Problem``): TET4, TET10, HEX20, HEX27 and
HEX8 with a 3x3x3 rule, each against the FP64 oracle on the same input.

- residual / BC-eliminated tangent / Dirichlet lift on curved (jittered)
  meshes against the oracle's complex-step cell Jacobians, 1e-11 relative;
  the FP32 tangent within 2e-5 of the matrix norm (the FP64 residual of
  both variants within 1e-13);
- HEX8 cells through the general kernel equal the HEX8 kernel's (1e-12);
- Newton on Neo-Hookean TET10 / HEX27 against the oracle's Newton with a
  direct solve, 1e-8 relative; the J2 commit, 1e-12;
- the SIMP adjoint on TET10 (theta per quadrature point) against the
  oracle's implicit VJP, 1e-8;
- the reference's convergence-rate study (manufactured Poisson solution,
  applications/convergence_rate/example.py): the GPU solutions give the
  oracle's errors (1e-8 relative) and the rates 2/1 (TET4), 3/2 (TET10,
  HEX27), 2/1.5 (HEX20, edge-mean dofs)."""
import numpy as np
import pytest
import torch

from helpers import element_box, face_fn, law_pair, make_problem, mms_bc, mms_errors, mms_mass_map
from oracle import fem_oracle as fo

CONFIGS = [("TET4", None), ("TET10", None), ("HEX20", None), ("HEX27", None), ("HEX8", 4)]
LAWS = ["laplace", "linear", "simp", "neo_hookean_scaled", "j2"]


def _problem(pkg, ele, order, law, ivars, bc=None, location_fns=None, vec=3, mass_map=None, surface_maps=None,
             mesh=None):
    class P(pkg.Problem):
        def get_tensor_map(self):
            return law

    if mass_map is not None:
        P.get_mass_map = lambda self: mass_map
    if surface_maps is not None:
        P.get_surface_maps = lambda self: surface_maps
    p = P(mesh, vec=vec, dim=3, ele_type=ele, quadrature_order=order, dirichlet_bc_info=bc,
          location_fns=location_fns)
    p.internal_vars = list(ivars)
    return p


def _setup(pkg, ele, order, kind, seed=0):
    rng = np.random.default_rng(seed)
    mesh = element_box(pkg, ele, (2, 2, 2), amp=0.12, seed=seed)
    C = len(mesh.cells)
    ov, og, ow = fo.element_tables(ele, order)
    law, olaw, iv, oiv = law_pair(pkg, kind, C, rng, Q=len(ow))
    bc = [[face_fn(0, 0.0)] * 3 + [face_fn(0, 1.0)], [0, 1, 2, 0], [lambda p: 0.0] * 3 + [lambda p: 0.02]]
    prob = _problem(pkg, ele, order, law, iv, bc=bc, mesh=mesh)
    oprob = fo.OracleProblem(mesh.points, mesh.cells, 3, olaw, dirichlet_bc_info=bc, internal_vars=oiv,
                             ele_type=ele, quadrature_order=order)
    # displacements that leave det F > 0 at every quadrature point of these
    # small curved cells (0.05 inverts some quadratic ones)
    scale = 0.02 if kind.startswith("neo") else 2e-3
    u = rng.normal(0, scale, size=prob.num_total_dofs_all_vars)
    assert np.linalg.det(fo.sol_to_grad(oprob, u) + np.eye(3)).min() > 0.1
    return prob, oprob, u


def _eliminate(A, rows):
    import scipy.sparse as sp
    keep = np.ones(A.shape[0], bool)
    keep[rows] = False
    D = sp.diags(keep.astype(float))
    return (D @ A.tocsr() @ D + sp.diags((~keep).astype(float))).tocsr()


def _assemble(prob, u, cuda, fp32=False):
    n = prob.num_total_dofs_all_vars
    ud = torch.tensor(u, device=cuda)
    mask, ubc = prob.dirichlet_device()
    dvec = torch.where(mask.bool(), ubc - ud, torch.zeros_like(ud))
    res = torch.empty(n, dtype=torch.float64, device=cuda)
    lift = torch.empty_like(res)
    A = prob.dev().new_matrix(torch.float32 if fp32 else torch.float64)
    prob.assemble(ud, res=res, vals=A.vals, lift=lift, dvec=dvec, fp32=fp32)
    torch.cuda.synchronize()
    return res.cpu().numpy(), A, lift.cpu().numpy(), dvec.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("ele,order", CONFIGS)
@pytest.mark.parametrize("kind", LAWS)
def test_elem_residual_tangent_lift(pkg, cuda, ele, order, kind):
    prob, oprob, u = _setup(pkg, ele, order, kind)
    assert not prob.hex8_kernel
    res, A, lift, dv = _assemble(prob, u, cuda)
    n = prob.num_total_dofs_all_vars
    cell_u = u.reshape(-1, 3)[oprob.cells]
    r_ref, jac = oprob.cell_residual_and_jacobian(cell_u, oprob.internal_vars)
    R_ref = np.zeros(n)
    np.add.at(R_ref, oprob.cell_dofs.reshape(-1), r_ref.reshape(-1))
    np.testing.assert_allclose(res, R_ref, rtol=0, atol=1e-11 * np.abs(R_ref).max())
    K = oprob.assemble_global(jac)
    rows = oprob.bc_rows()
    scale_k = np.abs(K.data).max()
    assert np.abs((A.to_scipy() - _eliminate(K, rows)).toarray()).max() <= 1e-11 * scale_k
    lift_ref = K @ dv
    lift_ref[rows] = 0.0
    lift[rows] = 0.0
    np.testing.assert_allclose(lift, lift_ref, rtol=0, atol=1e-11 * max(1.0, np.abs(lift_ref).max()))


@pytest.mark.gpu
@pytest.mark.parametrize("ele", ["TET10", "HEX27"])
def test_elem_fp32_tangent(pkg, cuda, ele):
    prob, _, u = _setup(pkg, ele, None, "neo_hookean_scaled")
    r64, A64, l64, _ = _assemble(prob, u, cuda)
    r32, A32, l32, _ = _assemble(prob, u, cuda, fp32=True)
    # the residual is FP64 in both (the two instantiations may contract FMAs differently)
    np.testing.assert_allclose(r32, r64, rtol=0, atol=1e-13 * np.abs(r64).max())
    K64 = A64.to_scipy()
    assert np.abs((A32.to_scipy() - K64).toarray()).max() <= 2e-5 * np.abs(K64.data).max()
    np.testing.assert_allclose(l32, l64, rtol=0, atol=2e-5 * max(1.0, np.abs(l64).max()))


@pytest.mark.gpu
def test_general_kernel_reproduces_hex8_kernel(pkg, cuda):
    from helpers import perturbed_box
    nat = pkg._native
    mesh = perturbed_box(pkg, (3, 4, 5), seed=2)
    law = pkg.NeoHookean(10.0, 0.3)
    bc = [[face_fn(0, 0.0)] * 3 + [face_fn(0, 1.0)], [0, 1, 2, 0], [lambda p: 0.0] * 3 + [lambda p: 0.02]]
    prob = make_problem(pkg, mesh, law, bc=bc)
    assert prob.hex8_kernel
    u = np.random.default_rng(1).normal(0, 0.05, size=prob.num_total_dofs_all_vars)
    r8, A8, l8, dv = _assemble(prob, u, cuda)
    # the same cells through fem_assemble_elem_f64 with the HEX8 tables
    d = prob.dev()
    gref, wq = prob.element_tables()
    ud = torch.tensor(u, device=cuda)
    dvec = torch.tensor(dv, device=cuda)
    mask, _ = prob.dirichlet_device()
    res = torch.empty_like(ud)
    lift = torch.empty_like(ud)
    A = d.new_matrix(torch.float64)
    pr, npar = nat.params_array(law.params())
    nat.check(nat.lib().fem_assemble_elem_f64(law.law_id, pr, npar, 3, 8, 8, nat.ptr(gref), nat.ptr(wq), d.num_cells,
                                              d.num_nodes, nat.ptr(d.cells), nat.ptr(d.points), nat.ptr(ud), None,
                                              None, None, nat.ptr(d.scatter), nat.ptr(d.diag), nat.ptr(d.transpose),
                                              d.nnzb, nat.ptr(mask), nat.ptr(dvec), nat.ptr(res), nat.ptr(lift),
                                              nat.ptr(A.vals), nat.stream_ptr()), "assemble_elem")
    torch.cuda.synchronize()
    np.testing.assert_allclose(res.cpu().numpy(), r8, rtol=0, atol=1e-12 * np.abs(r8).max())
    np.testing.assert_allclose(A.vals.cpu().numpy(), A8.vals.cpu().numpy(), rtol=0,
                               atol=1e-12 * A8.vals.abs().max().item())
    np.testing.assert_allclose(lift.cpu().numpy(), l8, rtol=0, atol=1e-12 * max(1.0, np.abs(l8).max()))


@pytest.mark.gpu
@pytest.mark.parametrize("ele", ["TET10", "HEX27"])
def test_elem_newton_matches_oracle(pkg, cuda, ele):
    mesh = element_box(pkg, ele, (3, 2, 2), amp=0.1, seed=3)
    bc = [[face_fn(0, 0.0)] * 3 + [face_fn(0, 1.0)] * 2, [0, 1, 2, 0, 1],
          [lambda p: 0.0] * 3 + [lambda p: 0.1, lambda p: 0.05]]
    prob = _problem(pkg, ele, None, pkg.NeoHookean(10.0, 0.3), [], bc=bc, mesh=mesh)
    opts = {"newton": {"rel_tol": 1e-11, "tol": 1e-14,
                       "linear": {"cg": {"precond": "block_jacobi", "rtol": 1e-13, "atol": 0.0, "maxiter": 20000}}}}
    sol = pkg.solver(prob, opts)[0].cpu().numpy().reshape(-1)
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, fo.Law("neo_hookean", E=10.0, nu=0.3), dirichlet_bc_info=bc,
                          ele_type=ele)
    ref = fo.newton_solve(op, rel_tol=1e-12, tol=1e-14)
    assert np.abs(sol - ref).max() <= 1e-8 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("ele", ["TET10", "HEX20"])
def test_elem_j2_commit_matches_oracle(pkg, cuda, ele):
    prob, oprob, u = _setup(pkg, ele, None, "j2", seed=4)
    u = u * 0.3  # with the random prior state, most points yield and a few stay elastic
    alpha0 = np.asarray(oprob.internal_vars[2]).copy()
    prob.update_j2_state([torch.tensor(u.reshape(-1, 3), device=cuda)])
    fo.j2_commit(oprob, u)
    for got, ref in zip(prob.internal_vars, oprob.internal_vars):
        ref = np.asarray(ref)
        np.testing.assert_allclose(got.cpu().numpy().reshape(ref.shape), ref, rtol=0,
                                   atol=1e-12 * max(1.0, np.abs(ref).max()))
    yielded = np.asarray(oprob.internal_vars[2]) > alpha0
    assert yielded.any() and not yielded.all()


@pytest.mark.gpu
def test_elem_simp_adjoint_matches_oracle(pkg, cuda):
    ele = "TET10"
    mesh = element_box(pkg, ele, (4, 2, 2), L=(2.0, 1.0, 1.0), amp=0.05, seed=5)
    C = len(mesh.cells)
    Q = 4
    bc = [[face_fn(0, 0.0)] * 3, [0, 1, 2], [lambda p: 0.0] * 3]
    load = lambda p: np.isclose(p[0], 2.0, atol=1e-5)  # noqa: E731
    smap = lambda u, x: np.array([0.0, 0.0, 1.0])  # noqa: E731
    law = pkg.SIMPElastic(70e3, 70.0, 0.3, 3.0)

    class TO(pkg.Problem):
        def get_tensor_map(self):
            return law

        def get_surface_maps(self):
            return [smap]

        def set_params(self, params):
            self.internal_vars = [params]

    prob = TO(mesh, vec=3, dim=3, ele_type=ele, dirichlet_bc_info=bc, location_fns=[load])
    lin = {"cg": {"precond": "block_jacobi", "rtol": 1e-12, "atol": 0.0, "maxiter": 20000}}
    fwd = pkg.ad_wrapper(prob, {"newton": {"rel_tol": 1e-10, "tol": 1e-14, "linear": lin}}, lin)
    rng = np.random.default_rng(6)
    th0 = rng.uniform(0.2, 1.0, size=(C, Q))
    th = torch.tensor(th0, device=cuda, requires_grad=True)
    comp = pkg.compliance(prob, fwd(th))
    comp.backward()
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, fo.Law("simp", E0=70e3, Emin=70.0, nu=0.3, penal=3.0),
                          dirichlet_bc_info=bc, location_fns=[load], surface_maps=[smap], internal_vars=[th0],
                          ele_type=ele)
    u = fo.newton_solve(op, rel_tol=1e-12, tol=1e-14)
    np.testing.assert_allclose(comp.item(), fo.compliance(op, u), rtol=1e-9)
    g_ref = fo.implicit_vjp_cellwise(op, u, -op.surface_load())
    g = th.grad.cpu().numpy()
    assert np.abs(g - g_ref).max() <= 1e-8 * np.abs(g_ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("ele,rates", [("TET4", (2, 1)), ("TET10", (3, 2)), ("HEX20", (2, 1.5)),
                                       ("HEX27", (3, 2))])
def test_convergence_study_matches_oracle(pkg, cuda, ele, rates):
    lin = {"cg": {"precond": "jacobi", "rtol": 1e-13, "atol": 0.0, "maxiter": 50000}}
    errs = []
    for N in (4, 8):
        mesh = element_box(pkg, ele, (N, N, N))
        prob = _problem(pkg, ele, None, pkg.Laplace(), [], bc=mms_bc(), vec=1, mass_map=mms_mass_map, mesh=mesh)
        sol = pkg.solver(prob, {"newton": {"rel_tol": 1e-10, "tol": 1e-10, "linear": lin}})[0]
        fe = prob.fes[0]
        errs.append(mms_errors(fe.points, fe.cells, fe.shape_vals, fe.shape_grads_ref, fe.quad_weights,
                               sol.cpu().numpy()))
        if N == 4:
            op = fo.OracleProblem(mesh.points, mesh.cells, 1, fo.Law("laplace", vec=1), dirichlet_bc_info=mms_bc(),
                                  mass_map=mms_mass_map, ele_type=ele)
            ref = fo.newton_solve(op, rel_tol=1e-10, tol=1e-10)
            assert np.abs(sol.cpu().numpy().reshape(-1) - ref).max() <= 1e-8 * np.abs(ref).max()
    l2_rate = np.log2(errs[0][0] / errs[1][0])
    h1_rate = np.log2(errs[0][1] / errs[1][1])
    assert abs(l2_rate - rates[0]) < 0.15 and abs(h1_rate - rates[1]) < 0.15, (l2_rate, h1_rate)


def _twist_bc(deg):
    import math
    th = math.radians(deg)
    c, s = math.cos(th), math.sin(th)
    uy = lambda p: 0.5 + (p[1] - 0.5) * c - (p[2] - 0.5) * s - p[1]  # noqa: E731
    uz = lambda p: 0.5 + (p[1] - 0.5) * s + (p[2] - 0.5) * c - p[2]  # noqa: E731
    z = lambda p: 0.0 * p[0]  # noqa: E731
    return [[face_fn(0, 0.0)] * 3 + [face_fn(0, 1.0)] * 3, [0, 1, 2] * 2, [z, z, z, z, uy, uz]]


@pytest.mark.gpu
def test_elem_arc_length_matches_oracle(pkg, cuda):
    """Displacement-controlled arc-length continuation (solver.py:521-597)
    of a 30-degree twist on TET10 cells: the load factor after every step
    equals the oracle's (1e-8) and the polished end point its Newton
    solution (1e-8)."""
    mesh = element_box(pkg, "TET10", (2, 2, 2))
    bc = _twist_bc(30.0)
    prob = _problem(pkg, "TET10", None, pkg.NeoHookean(10.0, 0.3), [], bc=bc, mesh=mesh)
    lin = {"cg": {"precond": "block_jacobi", "rtol": 1e-12, "atol": 0.0, "maxiter": 20000}}
    (sol,), info = pkg.solver(prob, {"arc_length": {"control": "displacement", "Delta_l": 0.3, "psi": 1.0,
                                                    "linear": lin, "return_info": True,
                                                    "newton": {"rel_tol": 1e-10, "tol": 1e-14}}})
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, fo.Law("neo_hookean", E=10.0, nu=0.3), dirichlet_bc_info=bc,
                          ele_type="TET10")
    ref_u, ref_lams = fo.arc_length_disp(op, Delta_l=0.3, psi=1.0)
    lams = [h["lam"] for h in info["history"]]
    assert len(lams) == len(ref_lams) and info["polished"] and lams[-1] >= 1.0
    np.testing.assert_allclose(lams, ref_lams, rtol=1e-8)
    sol = sol.cpu().numpy().reshape(-1)
    assert np.abs(sol - ref_u).max() <= 1e-8 * np.abs(ref_u).max()


@pytest.mark.gpu
def test_cell_path_dynamic_relax_matches_oracle(pkg, cuda):
    """Dynamic relaxation (solver.py:837-1047) through the cell-kernel path:
    a universal kernel restating the Neo-Hookean law on TET4 cells (scalar
    CSR tangent, mass from its absolute row sums) takes the oracle's
    iteration count (+-1) to the oracle's end point (1e-9)."""
    import kernels as K
    mesh = element_box(pkg, "TET4", (2, 2, 2))
    bc = _twist_bc(20.0)

    class Universal(pkg.Problem):
        def get_universal_kernel(self):
            return K.neo_hookean_universal(torch, 10.0, 0.3)

    prob = Universal(mesh, vec=3, dim=3, ele_type="TET4", dirichlet_bc_info=bc)
    assert prob.cell_path
    (sol,) = pkg.solver(prob, {"dynamic_relax": {"tol": 1e-8, "nKMat": 1000, "info": False, "info_force": False}})
    its = prob.last_solve_info["dr_iters"]
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, fo.Law("neo_hookean", E=10.0, nu=0.3), dirichlet_bc_info=bc,
                          ele_type="TET4")
    ref_u, ref_its = fo.dynamic_relax(op, tol=1e-8, nKMat=1000)
    sol = sol.cpu().numpy().reshape(-1)
    assert abs(its - ref_its) <= 1, (its, ref_its)
    assert np.abs(sol - ref_u).max() <= 1e-9 * np.abs(ref_u).max()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tet4_multigrid_matches_oracle(pkg, cuda, precision):
    """The lattice multigrid preconditioner on a TET4 box (Galerkin coarse
    operators from the TET4 tangent): Newton with gmg CG matches the oracle
    (1e-8 plain, 1e-6 mixed) in under a third of block-Jacobi's CG
    iterations (129 vs 472 on this 8x6x6 box; 166 vs 3579 at 50^3)."""
    mesh = element_box(pkg, "TET4", (8, 6, 6))
    bc = _twist_bc(20.0)
    prob = _problem(pkg, "TET4", None, pkg.NeoHookean(10.0, 0.3), [], bc=bc, mesh=mesh)
    its = {}
    for pc in ("gmg", "block_jacobi"):
        lin = {"cg": {"precond": pc, "rtol": 1e-10, "atol": 0.0, "maxiter": 20000}}
        opts = {"newton": {"rel_tol": 1e-10, "tol": 1e-14, "precision": precision, "linear": lin,
                           "return_info": True}}
        (sol,), info = pkg.solver(prob, opts)
        its[pc] = sum(info["krylov_iters"])
        if pc == "gmg":
            got = sol.cpu().numpy().reshape(-1)
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, fo.Law("neo_hookean", E=10.0, nu=0.3), dirichlet_bc_info=bc,
                          ele_type="TET4")
    ref = fo.newton_solve(op, rel_tol=1e-12, tol=1e-14)
    assert np.abs(got - ref).max() <= (1e-8 if precision == "fp64" else 1e-6) * np.abs(ref).max()
    assert its["gmg"] * 3 < its["block_jacobi"], its


@pytest.mark.gpu
@pytest.mark.parametrize("ele,precision", [("TET10", "fp64"), ("HEX27", "fp64"), ("HEX20", "fp64"),
                                           ("TET10", "mixed")])
def test_quadratic_pmultigrid_matches_oracle(pkg, cuda, ele, precision):
    """precond 'gmg' on quadratic cells runs p-multigrid (pmultigrid.py: the
    linear element on the corner-node lattice, its lattice hierarchy,
    Chebyshev / block-Jacobi smoothing on the fine level): Newton matches
    the oracle (1e-8 plain, 1e-6 mixed) in under a third of block-Jacobi's
    CG iterations (a CPU prototype of the same method: 15 / 19 / 29
    iterations vs 186 / 278 / 376 for HEX27 / TET10 / HEX20 on 6x4x4 boxes)."""
    mesh = element_box(pkg, ele, (6, 4, 4))
    bc = _twist_bc(20.0)
    prob = _problem(pkg, ele, None, pkg.NeoHookean(10.0, 0.3), [], bc=bc, mesh=mesh)
    its = {}
    for pc in ("gmg", "block_jacobi"):
        lin = {"cg": {"precond": pc, "rtol": 1e-10, "atol": 0.0, "maxiter": 20000}}
        opts = {"newton": {"rel_tol": 1e-10, "tol": 1e-14, "precision": precision, "linear": lin,
                           "return_info": True}}
        (sol,), info = pkg.solver(prob, opts)
        its[pc] = sum(info["krylov_iters"])
        if pc == "gmg":
            got = sol.cpu().numpy().reshape(-1)
    op = fo.OracleProblem(mesh.points, mesh.cells, 3, fo.Law("neo_hookean", E=10.0, nu=0.3), dirichlet_bc_info=bc,
                          ele_type=ele)
    ref = fo.newton_solve(op, rel_tol=1e-12, tol=1e-14)
    assert np.abs(got - ref).max() <= (1e-8 if precision == "fp64" else 1e-6) * np.abs(ref).max()
    assert its["gmg"] * 3 < its["block_jacobi"], its
