"""Smoothed-aggregation AMG (jax-fem_b200/amg.py, ``precond='amg'``, the
counterpart of the reference's AMGX path, solver.py:136-259) on the CPU.

- Aggregation covers every node that has a strong neighbour, each
  aggregate connected in the strength graph; the tentative prolongator has
  orthonormal columns and reproduces the near null space on the
  aggregated unknowns (T Bc = B); rigid-body modes are exact null vectors
  of an unconstrained linear-elastic tangent;
- AMG's own setup, Chebyshev V-cycle and device-scalar CG, run on CPU
  tensors with scipy standing in for the two library products (the
  problem's block-CSR operator and the scalar CSR levels / transfers),
  solve the oracle's eliminated tangents to the direct solution (1e-8):
  linear elasticity on a TET10 box whose nodes are randomly renumbered (no
  lattice: the geometric multigrid cannot run there), in under a fifth of
  block-Jacobi PCG's iterations, and Poisson on curved QUAD8 cells at two
  mesh sizes, where AMG-CG's iteration count stays nearly flat while Jacobi
  PCG's doubles; a second full setup on a changed tangent reuses the
  aggregates and still converges."""
import importlib
import types

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

from helpers import element_box, face_fn, planar_box
from oracle import fem_oracle as fo


@pytest.fixture(scope="module")
def amg(pkg):
    return importlib.import_module("jax_fem_b200.amg")


def _eliminated(op):
    op.newton_update(np.zeros(op.ndofs))
    free = np.ones(op.ndofs)
    free[op.bc_rows()] = 0.0
    A = (sp.diags(free) @ op.assemble_global() @ sp.diags(free) + sp.diags(1.0 - free)).tocsr()
    return A, free


def _renumbered_tet10(pkg, seed=3):
    m = element_box(pkg, "TET10", (4, 3, 3), amp=0.1, seed=1)
    perm = np.random.default_rng(seed).permutation(len(m.points))
    inv = np.argsort(perm)
    return m.points[perm], inv[m.cells].astype(np.int64)


def test_aggregation_and_tentative_prolongator(pkg, amg):
    points, cells = _renumbered_tet10(pkg)
    law = fo.Law("linear", E=70e3, nu=0.3)
    op = fo.OracleProblem(points, cells, 3, law, ele_type="TET10")
    op.newton_update(np.zeros(op.ndofs))
    A = op.assemble_global().tocsr()
    n_nodes = len(points)
    free = np.ones(3 * n_nodes)
    B = amg.near_null_space(points, 3, free)
    assert B.shape == (3 * n_nodes, 6)
    assert np.abs(A @ B).max() <= 1e-9 * np.abs(A).max()  # rigid-body modes: null vectors
    dof_node = np.arange(3 * n_nodes) // 3
    S = amg.strength(A, dof_node, n_nodes, 0.08)
    agg, na = amg.aggregate(S)
    assert (agg >= 0).all() and 1 < na < n_nodes
    for a in range(na):  # every aggregate is connected in the strength graph
        nodes = np.flatnonzero(agg == a)
        sub = S[nodes][:, nodes]
        assert sp.csgraph.connected_components(sub, directed=False)[0] == 1
    T, Bc, owner = amg.tentative(agg, na, dof_node, B)
    np.testing.assert_allclose((T.T @ T).toarray(), np.eye(T.shape[1]), rtol=0, atol=1e-12)
    np.testing.assert_allclose(T @ Bc, B, rtol=0, atol=1e-12)
    assert len(owner) == T.shape[1] and set(owner) == set(range(na))
    # eliminated unknowns stay out of every aggregate
    dn = dof_node.copy()
    dn[:30] = -1
    T2, _, _ = amg.tentative(agg, na, dn, B * (dn >= 0)[:, None])
    assert T2[:30].nnz == 0


def _amg_on_cpu(amg, monkeypatch, A, free, points, vec, block):
    """(AMG set up on CPU tensors, its operator stand-in)."""
    n = A.shape[0]

    def csr_apply(self, x, y):
        M = sp.csr_matrix((self.vals.numpy(), self.col_idx.numpy(), self.row_ptr.numpy()), shape=self.shape)
        return y.copy_(torch.from_numpy(M @ x.numpy()))

    monkeypatch.setattr(amg._CSR, "apply", csr_apply)
    Ab = A.tobsr(blocksize=(block, block))
    Ab.sort_indices()
    diag = np.array([Ab.indptr[i] + np.searchsorted(Ab.indices[Ab.indptr[i]:Ab.indptr[i + 1]], i)
                     for i in range(n // block)])

    def matvec(x, out=None):
        y = torch.from_numpy(A @ x.numpy())
        return y if out is None else out.copy_(y)

    Aop = types.SimpleNamespace(vals=torch.from_numpy(Ab.data.reshape(-1).copy()), diag=torch.from_numpy(diag),
                                row_ptr=torch.from_numpy(Ab.indptr.astype(np.int32)),
                                col_idx=torch.from_numpy(Ab.indices.astype(np.int32)),
                                n_brows=n // block, vec=block, matvec=matvec, to_scipy=lambda: A)
    mask = torch.from_numpy((1.0 - free).astype(np.uint8))
    fe = types.SimpleNamespace(vec=vec, points=points)
    problem = types.SimpleNamespace(num_vars=1, fes=[fe], dirichlet_device=lambda: (mask, None),
                                    dev=lambda: types.SimpleNamespace(device=torch.device("cpu")))
    g = amg.AMG(problem, coarse_size=60)
    g.setup(Aop)
    return g, Aop


def _run_amg(amg, monkeypatch, A, free, points, vec, block, min_transfers=2):
    """AMG's solve on CPU tensors; returns (iterations, solution, rhs)."""
    n = A.shape[0]
    g, Aop = _amg_on_cpu(amg, monkeypatch, A, free, points, vec, block)
    assert len(g.T) >= min_transfers
    b = np.random.default_rng(1).normal(size=n) * free
    x = torch.zeros(n, dtype=torch.float64)
    its, rel = g.solve(Aop, torch.from_numpy(b), x, rtol=1e-10, maxiter=300)
    assert rel <= 1e-10
    ref = spla.spsolve(A.tocsc(), b)
    np.testing.assert_allclose(x.numpy(), ref, rtol=0, atol=1e-8 * np.abs(ref).max())
    return its, g, Aop, b


def _pcg_iterations(A, b, block):
    n = A.shape[0]
    D = np.stack([A[block * i:block * i + block, block * i:block * i + block].toarray() for i in range(n // block)])
    Dinv = np.linalg.inv(D)
    count = []
    spla.cg(A, b, rtol=1e-10, atol=0.0, maxiter=50000,
            M=spla.LinearOperator((n, n), lambda v: np.einsum("nij,nj->ni", Dinv, v.reshape(-1, block)).reshape(-1)),
            callback=lambda xk: count.append(1))
    return len(count)


def test_amg_cg_on_renumbered_tet10_elasticity(pkg, amg, monkeypatch):
    points, cells = _renumbered_tet10(pkg)
    bc = [[face_fn(0, 0.0)] * 3, [0, 1, 2], [lambda p: 0.0] * 3]
    law = fo.Law("linear", E=70e3, nu=0.3)
    A, free = _eliminated(fo.OracleProblem(points, cells, 3, law, dirichlet_bc_info=bc, ele_type="TET10"))
    its, g, Aop, b = _run_amg(amg, monkeypatch, A, free, points, 3, 3)
    assert its * 5 < _pcg_iterations(A, b, 3), its
    # a changed tangent: full setup again (aggregates and T kept), fine-only setup
    T0 = g.T
    A2 = (A @ sp.diags(np.where(free > 0, 1.0, 0.0)) * 2.0 + sp.diags(1.0 - free)).tocsr()
    A2 = (0.5 * (A2 + A2.T)).tocsr()
    Ab = A2.tobsr(blocksize=(3, 3))
    Ab.sort_indices()
    Aop.vals = torch.from_numpy(Ab.data.reshape(-1).copy())
    Aop.matvec = lambda x, out=None: (torch.from_numpy(A2 @ x.numpy()) if out is None
                                      else out.copy_(torch.from_numpy(A2 @ x.numpy())))
    Aop.to_scipy = lambda: A2
    for fine_only in (False, True):
        g.setup(Aop, fine_only=fine_only)
        assert g.T is T0
        x = torch.zeros(len(b), dtype=torch.float64)
        its2, rel = g.solve(Aop, torch.from_numpy(b), x, rtol=1e-10, maxiter=300)
        assert rel <= 1e-10 and its2 <= its + 5
        ref = spla.spsolve(A2.tocsc(), b)
        np.testing.assert_allclose(x.numpy(), ref, rtol=0, atol=1e-8 * np.abs(ref).max())


def test_amg_cg_on_quad8_poisson(pkg, amg, monkeypatch):
    """Poisson on curved QUAD8 cells at two mesh sizes: AMG-CG's iteration
    count stays nearly flat (measured 36 -> 44) while Jacobi PCG's doubles
    (180 -> 385)."""
    counts = []
    for N in ((12, 10), (24, 20)):
        m = planar_box(pkg, "QUAD8", N, amp=0.05, seed=2)
        _, gref, _ = fo.element_tables("QUAD8")
        assert (np.linalg.det(np.einsum("cai,qaj->cqij", m.points[m.cells], gref)) > 0).all()  # no inverted cell
        bnd = lambda p: np.isclose(p[0], 0.0) | np.isclose(p[0], 1.0)  # noqa: E731
        kp = fo.KernelProblem([dict(points=m.points, cells=m.cells, vec=1, ele_type="QUAD8",
                                    dirichlet=[[bnd], [0], [lambda p: 0.0]])], tensor_map=lambda g: g)
        _, K = kp.residual_and_tangent(np.zeros(kp.ndofs))
        rows, _ = kp.bc_rows()
        free = np.ones(kp.ndofs)
        free[rows] = 0.0
        A = (sp.diags(free) @ K @ sp.diags(free) + sp.diags(1.0 - free)).tocsr()
        A = (0.5 * (A + A.T)).tocsr()
        its, _, _, b = _run_amg(amg, monkeypatch, A, free, m.points, 1, 1, min_transfers=1)
        counts.append((its, _pcg_iterations(A, b, 1)))
    (a0, j0), (a1, j1) = counts
    assert a1 <= 1.3 * a0 and j1 >= 1.9 * j0 and 5 * a1 < j1, counts


def test_amg_cg_failures_are_reported(pkg, amg, monkeypatch):
    """A failed AMG-CG solve raises the native error codes the Newton loop
    acts on: FEM_ERR_BREAKDOWN on an indefinite operator (Newton then
    retries with BiCGSTAB), FEM_ERR_NOT_CONVERGED at maxiter; with
    strict=False (the reference's AMGX call, which returns its last iterate)
    the solve returns its true residual instead."""
    nat = importlib.import_module("jax_fem_b200._native")
    points, cells = _renumbered_tet10(pkg)
    bc = [[face_fn(0, 0.0)] * 3, [0, 1, 2], [lambda p: 0.0] * 3]
    A, free = _eliminated(fo.OracleProblem(points, cells, 3, fo.Law("linear", E=70e3, nu=0.3),
                                           dirichlet_bc_info=bc, ele_type="TET10"))
    n = A.shape[0]
    b = torch.from_numpy(np.random.default_rng(1).normal(size=n) * free)
    g, Aop = _amg_on_cpu(amg, monkeypatch, A, free, points, 3, 3)
    x = torch.zeros(n, dtype=torch.float64)
    with pytest.raises(nat.FEMNativeError) as e:
        g.solve(Aop, b, x, rtol=1e-10, maxiter=3)
    assert e.value.status == nat.FEM_ERR_NOT_CONVERGED
    x.zero_()
    its, rel = g.solve(Aop, b, x, rtol=1e-10, maxiter=3, strict=False)
    assert its == 3 and 1e-10 < rel < 1.0
    r = b.numpy() - A @ x.numpy()
    assert abs(np.linalg.norm(r) / np.linalg.norm(b.numpy()) - rel) <= 1e-12
    # shift the free block by minus its median eigenvalue: indefinite
    lam = np.sort(np.linalg.eigvalsh(A.toarray()[np.ix_(free > 0, free > 0)]))
    shift = lam[len(lam) // 2]
    A2 = (A - shift * sp.diags(free)).tocsr()
    g2, Aop2 = _amg_on_cpu(amg, monkeypatch, A2, free, points, 3, 3)
    x = torch.zeros(n, dtype=torch.float64)
    with pytest.raises(nat.FEMNativeError) as e:
        g2.solve(Aop2, b, x, rtol=1e-10, maxiter=200)
    assert e.value.status == nat.FEM_ERR_BREAKDOWN
    assert torch.isfinite(x).all()


def test_device_galerkin_matches_scipy(pkg, amg):
    """The Galerkin products as torch sparse products (the form setup runs on
    the operator's device) equal scipy's: P = (I - omega D^-1 A) T and
    P^T A P (symmetrised), 1e-12 relative; the fine operator gathered from
    block-CSR values into scalar CSR equals the block matrix."""
    points, cells = _renumbered_tet10(pkg)
    A = fo.OracleProblem(points, cells, 3, fo.Law("linear", E=70e3, nu=0.3), ele_type="TET10")
    A.newton_update(np.zeros(A.ndofs))
    K = A.assemble_global().tocsr()
    Kb = K.tobsr(blocksize=(3, 3))
    Kb.sort_indices()
    Aop = types.SimpleNamespace(vals=torch.from_numpy(Kb.data.reshape(-1).copy()),
                                row_ptr=torch.from_numpy(Kb.indptr.astype(np.int32)),
                                col_idx=torch.from_numpy(Kb.indices.astype(np.int32)), vec=3)
    g = amg.AMG.__new__(amg.AMG)
    Kt = g._fine_csr(Aop)
    assert abs(amg._t_scipy(Kt) - K).max() == 0.0
    n_nodes = len(points)
    free = np.ones(3 * n_nodes)
    dof_node = np.arange(3 * n_nodes) // 3
    agg, na = amg.aggregate(amg.strength(K, dof_node, n_nodes, 0.08))
    T, _, _ = amg.tentative(agg, na, dof_node, amg.near_null_space(points, 3, free))
    P_t, Ac_t = amg.galerkin_t(Kt, amg._t_csr(T, "cpu"))
    d = K.diagonal()
    dinv = 1.0 / d
    omega = 4.0 / (3.0 * amg._t_spectral_radius(Kt, torch.from_numpy(dinv)))
    P = (T - sp.diags(omega * dinv) @ (K @ T)).tocsr()
    Ac = P.T @ K @ P
    Ac = 0.5 * (Ac + Ac.T)
    assert abs(amg._t_scipy(P_t) - P).max() <= 1e-12 * abs(P).max()
    assert abs(amg._t_scipy(Ac_t) - Ac).max() <= 1e-12 * abs(Ac).max()
