"""Pin the FP64 oracle to the reference's golden data (CPU only).

Each case restates one of the reference's integration tests
(tests/benchmarks/*/test_*.py) with the oracle and compares with the
FEniCSx fixtures at the reference's tolerances.  Also checks the oracle's
law derivatives (analytic P vs complex-step of psi) and the closed-form
rank-structured tangents the CUDA kernel uses against the oracle's
complex-step cell Jacobians.
"""
import numpy as np
import pytest

from helpers import golden
from oracle import fem_oracle as fo

left = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
right = lambda p: np.isclose(p[0], 1.0, atol=1e-5)  # noqa: E731
top = lambda p: np.isclose(p[2], 10.0, atol=1e-5)  # noqa: E731
bottom = lambda p: np.isclose(p[2], 0.0, atol=1e-5)  # noqa: E731


def test_poisson_golden():
    d = golden("linear_poisson")
    pb = fo.OracleProblem(d["points"], d["cells"], 1, fo.Law("laplace", vec=1),
                          dirichlet_bc_info=[[left, right], [0, 0], [lambda p: 0.0, lambda p: 1.0]])
    u = fo.newton_solve(pb)
    np.testing.assert_array_almost_equal(d["sol"].reshape(-1), u, decimal=5)


def test_cube_golden():
    d = golden("linear_elasticity_cube")
    pb = fo.OracleProblem(d["points"], d["cells"], 3, fo.Law("linear", E=70e3, nu=0.3),
                          dirichlet_bc_info=[[left] * 3, [0, 1, 2], [lambda p: 1.0] * 3], location_fns=[right],
                          mass_map=lambda u, x: -np.array([0.0, 10.0, 10.0]),
                          surface_maps=[lambda u, x: -np.array([10.0, 0.0, 0.0])])
    u = fo.newton_solve(pb)
    np.testing.assert_array_almost_equal(d["sol"].reshape(-1), u, decimal=5)


def test_cylinder_golden():
    d = golden("linear_elasticity_cylinder")
    pb = fo.OracleProblem(d["points"], d["cells"], 3, fo.Law("linear", E=70e3, nu=0.3),
                          dirichlet_bc_info=[[bottom] * 3, [0, 1, 2], [lambda p: 0.0] * 3], location_fns=[top],
                          mass_map=lambda u, x: -np.array([1e3 * x[0], 2e3 * x[1], 3e3 * x[2]]),
                          surface_maps=[lambda u, x: -np.array([1e3 * x[0] ** 2 + 1e3 * x[1] ** 2, 0.0, 0.0])])
    u = fo.newton_solve(pb)
    np.testing.assert_array_almost_equal(d["sol"].reshape(-1), u, decimal=3)
    area = fo.surface_integral(pb, top, lambda ug: np.ones_like(ug)[:, :, :, 0], u)[0]
    np.testing.assert_almost_equal(d["surface_area"], area, decimal=4)


def test_hyperelastic_golden():
    d = golden("hyperelasticity")
    z = lambda p: 0.0  # noqa: E731
    pb = fo.OracleProblem(d["points"], d["cells"], 3, fo.Law("neo_hookean", E=1e3, nu=0.3),
                          dirichlet_bc_info=[[bottom] * 3 + [top] * 3, [0, 1, 2] * 2, [z] * 5 + [lambda p: 1.0]])
    u = fo.newton_solve(pb)
    np.testing.assert_array_almost_equal(d["sol"].reshape(-1), u, decimal=5)
    tr = fo.surface_integral(pb, top, lambda ug: fo.stress_neo_hookean(ug, 1e3, 0.3) @ np.array([0.0, 0.0, 1.0]), u)
    np.testing.assert_almost_equal(d["traction"], tr[2], decimal=5)


@pytest.mark.slow
def test_plasticity_golden():
    d = golden("plasticity")
    C = len(d["cells"])
    bc = [[bottom] * 3 + [top] * 3, [0, 1, 2] * 2, [lambda p: 0.0] * 6]
    pb = fo.OracleProblem(d["points"], d["cells"], 3, fo.Law("j2", E=70e3, nu=0.3, sig0=250.0, H=0.0),
                          dirichlet_bc_info=bc,
                          internal_vars=[np.zeros((C, 8, 3, 3)), np.zeros((C, 8, 3, 3)), np.zeros((C, 8))])
    avg = []
    for disp in d["disps"]:
        bc[2][-1] = (lambda v: (lambda p: v))(float(disp))
        pb.update_dirichlet(bc)
        u = fo.newton_solve(pb)
        fo.j2_commit(pb, u)
        avg.append(fo.avg_stress(pb)[2, 2])
    np.testing.assert_array_almost_equal(d["sol"].reshape(-1), u, decimal=5)
    np.testing.assert_array_almost_equal(d["avg_stresses"], np.array(avg), decimal=3)


def test_neo_hookean_stress_is_gradient_of_energy():
    rng = np.random.default_rng(0)
    F = np.eye(3) + 0.2 * rng.standard_normal((5, 3, 3))
    P = fo.stress_neo_hookean(F - np.eye(3), 10.0, 0.3)
    h = 1e-30
    for i in range(3):
        for j in range(3):
            Fc = F.astype(complex)
            Fc[:, i, j] += 1j * h
            dpsi = np.imag(fo.psi_neo_hookean(Fc, 10.0, 0.3)) / h
            np.testing.assert_allclose(P[:, i, j], dpsi, rtol=1e-12, atol=1e-12)


def test_hex8_tables():
    vals, grads, w = fo.hex8_tables()
    np.testing.assert_allclose(vals.sum(axis=1), 1.0, atol=1e-15)      # partition of unity
    np.testing.assert_allclose(grads.sum(axis=1), 0.0, atol=1e-15)
    np.testing.assert_allclose(w.sum(), 1.0, atol=1e-15)
    # exact for trilinear-times-trilinear integrands: int x^2 y^2 z^2 over [0,1]^3 = 1/27
    p = np.array([[a, b, c] for a in fo.gauss_jacobi_01(2)[0] for b in fo.gauss_jacobi_01(2)[0]
                  for c in fo.gauss_jacobi_01(2)[0]])
    np.testing.assert_allclose((w * (p ** 2).prod(axis=1)).sum(), 1.0 / 27.0, rtol=1e-14)


def _closed_form_tangent(kind, g, jxw, ug, params, ivq=None):
    """The rank-structured per-quad tangent blocks the CUDA kernel evaluates
    (assemble.cu, pair_block), restated in numpy: K_ab (8,8,3,3)."""
    K = np.zeros((8, 8, 3, 3))
    dot = g @ g.T
    I = np.eye(3)
    if kind == "linear":
        E, nu = params
        lm, mu = fo.lame(E, nu)
        K = lm * np.einsum("ai,bk->abik", g, g) + mu * np.einsum("bi,ak->abik", g, g) + mu * dot[:, :, None, None] * I
    elif kind == "neo_hookean":
        E, nu = params
        mu = E / (2 * (1 + nu))
        kappa = E / (3 * (1 - 2 * nu))
        F = ug + I
        J = np.linalg.det(F)
        H = np.linalg.inv(F).T
        I1 = (F * F).sum()
        m = mu * J ** (-2.0 / 3.0)
        f = g @ F.T
        h = g @ H.T
        c2, c4, c5 = -2.0 / 3.0 * m, 2.0 / 9.0 * m * I1 + kappa * (2 * J - 1) * J, m * I1 / 3.0 - kappa * J * (J - 1)
        K = (m * dot[:, :, None, None] * I + c2 * (np.einsum("ai,bk->abik", f, h) + np.einsum("ai,bk->abik", h, f))
             + c4 * np.einsum("ai,bk->abik", h, h) + c5 * np.einsum("bi,ak->abik", h, h))
    elif kind == "j2":
        E, nu, sy, Hh = params
        so, eo, ao = ivq
        lm, mu = fo.lame(E, nu)
        de = 0.5 * (ug + ug.T) - eo
        st = lm * np.trace(de) * I + 2 * mu * de + so
        s = st - np.trace(st) / 3 * I
        q = np.sqrt(1.5 * (s * s).sum())
        syc = sy + Hh * ao
        beta = gam2 = 0.0
        if q - syc > 0:
            dg = (q - syc) / (3 * mu + Hh)
            beta = 3 * mu * dg / q
            gam2 = 9 * mu * mu * syc / ((3 * mu + Hh) * q ** 3)
        cII, ch = lm + 2 * mu * beta / 3, mu * (1 - beta)
        sg = g @ s.T
        K = (cII * np.einsum("ai,bk->abik", g, g) + ch * (dot[:, :, None, None] * I + np.einsum("bi,ak->abik", g, g))
             - gam2 * np.einsum("ai,bk->abik", sg, sg))
    return K * jxw


@pytest.mark.parametrize("kind", ["linear", "neo_hookean", "j2"])
def test_closed_form_tangent_matches_complex_step(kind):
    rng = np.random.default_rng(3)
    pts, cells = fo.box_mesh(2, 2, 2, 1.0, 1.0, 1.0)
    pts = pts + 0.05 * rng.uniform(-1, 1, pts.shape) * (np.abs(pts - 0.5) < 0.49)
    C = len(cells)
    if kind == "linear":
        law, params, iv = fo.Law("linear", E=70e3, nu=0.3), (70e3, 0.3), []
        u = rng.normal(0, 1e-3, (len(pts), 3))
    elif kind == "neo_hookean":
        law, params, iv = fo.Law("neo_hookean", E=10.0, nu=0.3), (10.0, 0.3), []
        u = rng.normal(0, 0.05, (len(pts), 3))
    else:
        so = rng.normal(0, 200.0, (C, 8, 3, 3))
        so = 0.5 * (so + np.swapaxes(so, -1, -2))
        eo = rng.normal(0, 1e-3, (C, 8, 3, 3))
        eo = 0.5 * (eo + np.swapaxes(eo, -1, -2))
        ao = rng.uniform(0, 0.01, (C, 8))
        iv = [so, eo, ao]
        law, params = fo.Law("j2", E=70e3, nu=0.3, sig0=250.0, H=700.0), (70e3, 0.3, 250.0, 700.0)
        u = rng.normal(0, 2e-3, (len(pts), 3))
    pb = fo.OracleProblem(pts, cells, 3, law, internal_vars=iv)
    _, jac = pb.cell_residual_and_jacobian(u[pb.cells], pb.internal_vars)
    ug = np.einsum("cai,cqaj->cqij", u[pb.cells], pb.shape_grads)
    for c in range(C):
        K = np.zeros((8, 8, 3, 3))
        for q in range(8):
            ivq = (iv[0][c, q], iv[1][c, q], iv[2][c, q]) if kind == "j2" else None
            K += _closed_form_tangent(kind, pb.shape_grads[c, q], pb.JxW[c, q], ug[c, q], params, ivq)
        Kf = K.transpose(0, 2, 1, 3).reshape(24, 24)
        np.testing.assert_allclose(Kf, jac[c], rtol=0, atol=1e-10 * np.abs(jac[c]).max())


def test_oracle_arc_length_reaches_newton_solution():
    """The oracle's displacement-controlled arc-length path (solver.py:521-597,
    721-756) climbs to lambda >= 1 in increasing steps, and its polished
    end point is the Newton solution of the full-load problem."""
    import math
    pts, cells = fo.box_mesh(3, 3, 3, 1.0, 1.0, 1.0)
    c, s = math.cos(math.radians(30.0)), math.sin(math.radians(30.0))
    left = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    right = lambda p: np.isclose(p[0], 1.0, atol=1e-5)  # noqa: E731
    uy = lambda p: 0.5 + (p[1] - 0.5) * c - (p[2] - 0.5) * s - p[1]  # noqa: E731
    uz = lambda p: 0.5 + (p[1] - 0.5) * s + (p[2] - 0.5) * c - p[2]  # noqa: E731
    z = lambda p: 0.0 * p[0]  # noqa: E731
    bc = [[left] * 3 + [right] * 3, [0, 1, 2] * 2, [z, z, z, z, uy, uz]]
    op = fo.OracleProblem(pts, cells, 3, fo.Law("neo_hookean", E=10.0, nu=0.3), dirichlet_bc_info=bc)
    u, lams = fo.arc_length_disp(op, Delta_l=0.3)
    assert lams[-1] >= 1.0 and all(b > a for a, b in zip(lams, lams[1:])) and len(lams) >= 4
    ref = fo.newton_solve(op, rel_tol=1e-12, tol=1e-14)
    assert np.abs(u - ref).max() <= 1e-12 * np.abs(ref).max()


def test_oracle_force_arc_length_reaches_newton_solution():
    """The oracle's force-controlled path (solver.py:607-685, 758-801) on a
    cantilever: counter-load q from the opposite traction, lambda climbs to 1,
    the polished end point is the Newton solution under the full load."""
    pts, cells = fo.box_mesh(6, 2, 2, 3.0, 1.0, 1.0)
    left = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    right = lambda p: np.isclose(p[0], 3.0, atol=1e-5)  # noqa: E731
    z = lambda p: 0.0 * p[0]  # noqa: E731
    bc = [[left] * 3, [0, 1, 2], [z] * 3]
    law = fo.Law("neo_hookean", E=10.0, nu=0.3)
    op = fo.OracleProblem(pts, cells, 3, law, dirichlet_bc_info=bc, location_fns=[right],
                          surface_maps=[lambda u, x: np.array([0.0, 0.0, 0.05])])
    aux = fo.OracleProblem(pts, cells, 3, law, dirichlet_bc_info=bc, location_fns=[right],
                           surface_maps=[lambda u, x: np.array([0.0, 0.0, -0.05])])
    u, lams = fo.arc_length_force(op, aux.residual(np.zeros(aux.ndofs)), Delta_l=0.15, psi=0.5)
    assert lams[-1] >= 1.0 and all(b > a for a, b in zip(lams, lams[1:]))
    ref = fo.newton_solve(op, rel_tol=1e-12, tol=1e-14)
    assert np.abs(u - ref).max() <= 1e-12 * np.abs(ref).max()


def test_oracle_dynamic_relax_reaches_newton_solution():
    """The oracle's dynamic relaxation (solver.py:837-1047) ends within its
    residual tolerance of the Newton solution."""
    import math
    pts, cells = fo.box_mesh(3, 3, 3, 1.0, 1.0, 1.0)
    c, s = math.cos(math.radians(20.0)), math.sin(math.radians(20.0))
    left = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    right = lambda p: np.isclose(p[0], 1.0, atol=1e-5)  # noqa: E731
    uy = lambda p: 0.5 + (p[1] - 0.5) * c - (p[2] - 0.5) * s - p[1]  # noqa: E731
    uz = lambda p: 0.5 + (p[1] - 0.5) * s + (p[2] - 0.5) * c - p[2]  # noqa: E731
    z = lambda p: 0.0 * p[0]  # noqa: E731
    bc = [[left] * 3 + [right] * 3, [0, 1, 2] * 2, [z, z, z, z, uy, uz]]
    op = fo.OracleProblem(pts, cells, 3, fo.Law("neo_hookean", E=10.0, nu=0.3), dirichlet_bc_info=bc)
    u, its = fo.dynamic_relax(op, tol=1e-8)
    assert 0 < its < 1000
    assert np.max(np.abs(np.delete(op.residual(u), op.bc_rows()))) <= 1e-8
    ref = fo.newton_solve(op, rel_tol=1e-12, tol=1e-14)
    assert np.abs(u - ref).max() <= 1e-6 * np.abs(ref).max()
