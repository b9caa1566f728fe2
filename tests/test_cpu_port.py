"""The C++/OpenMP restatement of the reference's method (oracle/fem_cpu.cpp,
the timed CPU baseline of bench.py) against the numpy oracle, on the CPU:

- residual (Dirichlet rows u - u_D) and row-zeroed tangent of the
  Neo-Hookean and linear-elastic laws at a random state of a 3^3 box equal
  the oracle's complex-step assembly (1e-12 relative);
- the 5-step Neo-Hookean twist on a 4^3 box, solved by its BiCGSTAB +
  Jacobi Newton loop to rel.res 1e-9 (its linear solves stop at 1e-10 of
  ||b||, the reference's tolerance, which floors Newton near 1e-10), equals
  the oracle's Newton solution (1e-7) and meets rel.res 1e-8 in the
  oracle's own residual;
- the 20^3 stretch (linear elasticity, u_x = 0.01 on x = 1) by its CG +
  Jacobi equals the oracle's direct solve (1e-8)."""
import numpy as np
import pytest

from oracle import fem_cpu as fc
from oracle import fem_oracle as fo


def _twist_bc(theta):
    c, s = np.cos(theta), np.sin(theta)
    left = lambda p: np.isclose(p[0], 0.0)  # noqa: E731
    right = lambda p: np.isclose(p[0], 1.0)  # noqa: E731
    zero = lambda p: 0.0 * p[0]  # noqa: E731
    uy = lambda p: 0.5 + (p[1] - 0.5) * c - (p[2] - 0.5) * s - p[1]  # noqa: E731
    uz = lambda p: 0.5 + (p[1] - 0.5) * s + (p[2] - 0.5) * c - p[2]  # noqa: E731
    return [[left] * 3 + [right] * 3, [0, 1, 2] * 2, [zero, zero, zero, zero, uy, uz]]


@pytest.fixture(scope="module")
def built():
    fc.build()
    return fc


@pytest.mark.parametrize("law", ["neo_hookean", "linear"])
def test_residual_and_tangent_match_oracle(built, law):
    n = 3
    E = 10.0 if law == "neo_hookean" else 70e3
    p = fc.CPUProblem(n, fc.LAW_NEO_HOOKEAN if law == "neo_hookean" else fc.LAW_LINEAR, E, 0.3, threads=2)
    theta = np.deg2rad(12.0)
    p.set_dirichlet(*fc.box_dirichlet(n, "twist", theta))
    u = np.random.default_rng(0).normal(0.0, 0.02, p.ndofs)
    res, A = p.residual_tangent(u)
    pts, cells = fo.box_mesh(n, n, n, 1.0, 1.0, 1.0)
    op = fo.OracleProblem(pts, cells, 3, fo.Law(law, E=E, nu=0.3), dirichlet_bc_info=_twist_bc(theta))
    r_o = op.apply_bc_vec(op.residual(u), u)
    op.newton_update(u)
    A_o = op.get_A()
    assert np.abs(res - r_o).max() <= 1e-12 * np.abs(r_o).max()
    assert abs(A - A_o).max() <= 1e-12 * abs(A_o).max()


def test_twist_newton_matches_oracle(built):
    n = 4
    p = fc.CPUProblem(n, fc.LAW_NEO_HOOKEAN, 10.0, 0.3, threads=2)
    u, st = fc.twist_solve(p, rel_tol=1e-9, tol=1e-14)
    assert st["newton"] >= 5 and st["krylov"] > 0
    pts, cells = fo.box_mesh(n, n, n, 1.0, 1.0, 1.0)
    ref = None
    for k in range(1, 6):
        op = fo.OracleProblem(pts, cells, 3, fo.Law("neo_hookean", E=10.0, nu=0.3),
                              dirichlet_bc_info=_twist_bc(np.deg2rad(6.0 * k)))
        ref = fo.newton_solve(op, initial_guess=ref, rel_tol=1e-12, tol=1e-14)
    assert np.abs(u - ref).max() <= 1e-7 * np.abs(ref).max()
    zero = np.zeros(op.ndofs)
    r = np.linalg.norm(op.apply_bc_vec(op.residual(u), u))
    r0 = np.linalg.norm(op.apply_bc_vec(op.residual(zero), zero))
    assert r <= 1e-8 * r0


def test_stretch_cg_matches_direct_solve(built):
    n = 20
    p = fc.CPUProblem(n, fc.LAW_LINEAR, 70e3, 0.3, threads=4)
    p.set_dirichlet(*fc.box_dirichlet(n, "stretch"))
    u = np.zeros(p.ndofs)
    st = p.newton(u, rel_tol=1e-8, tol=1e-14, method=fc.METHOD_CG, lin_tol=1e-10)
    assert st["newton"] >= 1
    pts, cells = fo.box_mesh(n, n, n, 1.0, 1.0, 1.0)
    left = lambda q: np.isclose(q[0], 0.0)  # noqa: E731
    right = lambda q: np.isclose(q[0], 1.0)  # noqa: E731
    bc = [[left] * 3 + [right], [0, 1, 2, 0], [lambda q: 0.0 * q[0]] * 3 + [lambda q: 0.01 + 0.0 * q[0]]]
    op = fo.OracleProblem(pts, cells, 3, fo.Law("linear", E=70e3, nu=0.3), dirichlet_bc_info=bc)
    ref = fo.newton_solve(op, tol=1e-14)
    assert np.abs(u - ref).max() <= 1e-8 * np.abs(ref).max()
