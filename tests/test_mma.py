"""The MMA outer loop (jax-fem_b200/mma.py) on the CPU.

- Svanberg's three-variable test problem (a convex objective, two convex
  constraints) solved by MMA iterations agrees with scipy's SLSQP (1e-5);
- every subproblem solve ends with its relaxed-KKT residual below 1e-6;
- the sensitivity filter matrix equals a brute-force construction of the
  reference's rule (20 nearest centroids, weights max(rmin - d, 0),
  rmin = 1.5 element sizes), and the filtered gradients its formula."""
import numpy as np
import pytest
import torch
from scipy.optimize import minimize

from __graft_entry__ import load_package


@pytest.fixture(scope="module")
def mma():
    load_package()
    import importlib
    return importlib.import_module("jax_fem_b200.mma")


def _toy(x):
    f0 = float((x ** 2).sum())
    df0 = 2 * x
    c1, c2 = torch.tensor([5.0, 2.0, 1.0], dtype=x.dtype), torch.tensor([3.0, 4.0, 3.0], dtype=x.dtype)
    fval = torch.stack([((x - c1) ** 2).sum() - 9.0, ((x - c2) ** 2).sum() - 9.0])
    dfdx = torch.stack([2 * (x - c1), 2 * (x - c2)])
    return f0, df0, fval, dfdx


def test_mma_toy_problem_matches_slsqp(mma):
    x = torch.tensor([4.0, 3.0, 2.0], dtype=torch.float64)
    opt = mma.MMA(torch.zeros(3, dtype=torch.float64), torch.full((3,), 5.0, dtype=torch.float64), move=1.0,
                  a0=1.0, c=[1000.0, 1000.0], d=[1.0, 1.0], num_constraints=2)
    for _ in range(60):
        f0, df0, fval, dfdx = _toy(x)
        x = opt.step(x, f0, df0, fval, dfdx)
        assert opt.last_kkt <= 1e-6
    cons = [{"type": "ineq", "fun": lambda v, c=c: 9.0 - ((v - np.array(c)) ** 2).sum(),
             "jac": lambda v, c=c: -2.0 * (v - np.array(c))} for c in ([5.0, 2.0, 1.0], [3.0, 4.0, 3.0])]
    ref = minimize(lambda v: (v ** 2).sum(), np.array([4.0, 3.0, 2.0]), jac=lambda v: 2.0 * v, method="SLSQP",
                   bounds=[(0, 5)] * 3, constraints=cons, options={"ftol": 1e-15, "maxiter": 500})
    # (SLSQP may end on a line-search status at the optimum: compare the point)
    assert abs(ref.fun - 8.7702) < 1e-3
    np.testing.assert_allclose(x.numpy(), ref.x, atol=1e-5)
    _, _, fval, _ = _toy(x)
    assert float(fval.max()) <= 1e-6


def test_filter_matches_brute_force(mma):
    pkg = load_package()
    m = pkg.box_mesh(6, 4, 3, 1.2, 0.8, 0.6)
    fe = pkg.fe.FiniteElement(pkg.Mesh(m.points, m.cells_dict["hexahedron"]), 3, 3)
    fe.flex_inds = np.arange(len(fe.cells))[::2]  # a subset of design cells
    H, Hs = mma.compute_filter_kd_tree(fe)
    cen = fe.points[fe.cells].mean(axis=1)[fe.flex_inds]
    n = len(cen)
    rmin = 1.5 * (fe.JxW().sum() / len(fe.cells)) ** (1 / 3)
    dist = np.linalg.norm(cen[:, None] - cen[None], axis=2)
    ref = np.zeros((n, n))
    for i in range(n):
        nn = np.argsort(dist[i], kind="stable")[:20]
        ref[i, nn] = np.maximum(rmin - dist[i, nn], 0.0)
    np.testing.assert_allclose(H.to_dense().numpy(), ref, atol=1e-14)
    np.testing.assert_allclose(Hs.numpy().reshape(-1), ref.sum(1), rtol=1e-14)
    rng = np.random.default_rng(0)
    rho = torch.tensor(rng.uniform(0, 1, (n, 1)))
    rho[0] = 1e-4  # below the 1e-3 floor
    dJ, dvc = torch.tensor(rng.normal(size=(n, 1))), torch.tensor(rng.normal(size=(2, n, 1)))
    fdJ, fdvc = mma.applySensitivityFilter({"H": H, "Hs": Hs}, rho, dJ, dvc)
    w = rho.numpy() / np.maximum(1e-3, rho.numpy()) / ref.sum(1)[:, None]
    np.testing.assert_allclose(fdJ.numpy(), ref @ (w * dJ.numpy()), rtol=1e-12)
    np.testing.assert_allclose(fdvc.numpy()[1], ref @ (w * dvc.numpy()[1]), rtol=1e-12)


def test_optimize_loop_on_host(mma):
    """The optimize() loop with numpy handles on the CPU: a separable
    objective sum (rho - t)^2 under mean(rho) <= 0.3 reaches the KKT point
    the filter and MMA allow (objective falls, constraint holds)."""
    pkg = load_package()
    m = pkg.box_mesh(4, 4, 4, 1.0, 1.0, 1.0)
    fe = pkg.fe.FiniteElement(pkg.Mesh(m.points, m.cells_dict["hexahedron"]), 3, 3)
    fe.flex_inds = np.arange(len(fe.cells))
    n = len(fe.cells)
    t = np.linspace(0.0, 1.0, n)[:, None]

    def obj(rho):
        assert isinstance(rho, np.ndarray) and rho.shape == (n, 1)
        return float(((rho - t) ** 2).sum()), 2.0 * (rho - t)

    def cons(rho, it):
        return np.array([rho.mean() / 0.3 - 1.0]), np.full((1, n, 1), 1.0 / (0.3 * n))

    rho0 = np.full((n, 1), 0.3)
    rho = mma.optimize(fe, rho0, {"maxIters": 30, "movelimit": 0.2}, obj, cons, 1, device=torch.device("cpu"))
    assert isinstance(rho, np.ndarray) and rho.shape == (n, 1)
    hist = mma.optimize.history
    assert obj(rho)[0] < 0.7 * hist[0]["J"]
    assert rho.mean() <= 0.3 * (1 + 1e-4)
    assert max(h["kkt"] for h in hist) <= 1e-6
