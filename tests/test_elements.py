"""Element types besides the HEX8 fast path (TET4, TET10, HEX20, HEX27), on
the CPU: tabulation, quadrature, structured meshes, the nen-node block
pattern, load vectors, and the oracle's own convergence study.

- The product's tables (jax-fem_b200/basis.py: written in mesh node order)
  equal the oracle's (basix numbering moved to mesh order with the
  reference's re_order, basis.py:53-76, dual bases by inverting the dof
  functionals) to round-off;
- shape functions: partition of unity, exact reproduction of linear
  fields, the Kronecker property at the nodes (Lagrange types) and, for
  HEX20, at its dofs (vertex values and edge means);
- the simplex rules integrate every monomial of their degree exactly;
- box meshes are conforming and positively oriented;
- the oracle reproduces the reference's convergence-rate study
  (applications/convergence_rate/example.py: TET4 and TET10 on N = 8, 16
  here at N = 4, 8): L2 / H1 rates 2 / 1 (TET4, HEX8) and 3 / 2 (TET10,
  HEX27).  HEX20 gets 2 / 1.5: basix's serendipity dofs on edges are edge
  means, while Dirichlet data are values at the midside nodes."""
import importlib
import math

import numpy as np
import pytest

from helpers import element_box, face_fn, mms_bc, mms_errors, mms_mass_map
from oracle import fem_oracle as fo

TYPES = ["HEX8", "TET4", "TET10", "HEX20", "HEX27"]


@pytest.fixture(scope="module")
def B(pkg):
    return importlib.import_module("jax_fem_b200.basis")


@pytest.mark.parametrize("ele", TYPES)
def test_tables_match_oracle(B, ele):
    v1, g1, w1 = B.get_shape_vals_and_grads(ele)
    v2, g2, w2 = fo.element_tables(ele) if ele != "HEX8" else fo.hex8_tables()
    np.testing.assert_allclose(v1, v2, rtol=0, atol=1e-12)
    np.testing.assert_allclose(g1, g2, rtol=0, atol=1e-12)
    np.testing.assert_allclose(w1, w2, rtol=0, atol=1e-15)
    f1 = B.get_face_shape_vals_and_grads(ele)
    f2 = fo.element_face_tables(ele)
    for a, b in zip(f1, f2):
        np.testing.assert_allclose(np.asarray(a, float), np.asarray(b, float), rtol=0, atol=1e-12)


@pytest.mark.parametrize("ele", TYPES)
def test_shape_function_properties(B, ele):
    rng = np.random.default_rng(3)
    xi = rng.uniform(0, 1, size=(50, 3))
    if ele.startswith("TET"):
        xi = xi[xi.sum(axis=1) <= 1.0]
    v, g = B.shape_fn(ele, xi)
    X = B.node_coords(ele)
    np.testing.assert_allclose(v.sum(axis=1), 1.0, atol=1e-13)
    np.testing.assert_allclose(g.sum(axis=1), 0.0, atol=1e-12)
    np.testing.assert_allclose(v @ X, xi, atol=1e-13)  # linear fields are reproduced
    np.testing.assert_allclose(np.einsum("nad,ai->nid", g, X), np.broadcast_to(np.eye(3), (len(xi), 3, 3)),
                               atol=1e-12)
    vn, _ = B.shape_fn(ele, X)
    if ele != "HEX20":
        np.testing.assert_allclose(vn, np.eye(len(X)), atol=1e-13)
    else:  # dofs: corner values and edge means
        np.testing.assert_allclose(vn[:8], np.eye(20)[:8], atol=1e-13)
        t, w = B.gauss_legendre_01(3)
        for e, (i, j) in enumerate(B.HEX_EDGES):
            pts = X[i][None] + t[:, None] * (X[j] - X[i])[None]
            np.testing.assert_allclose(w @ B.shape_fn(ele, pts)[0], np.eye(20)[8 + e], atol=1e-13)


def test_simplex_rules_exact(B):
    for order, deg in ((0, 1), (1, 1), (2, 2)):
        pts, w = B.volume_quadrature("TET4", order)
        for a in range(deg + 1):
            for b in range(deg + 1 - a):
                for c in range(deg + 1 - a - b):
                    exact = math.factorial(a) * math.factorial(b) * math.factorial(c) / math.factorial(a + b + c + 3)
                    got = w @ (pts[:, 0] ** a * pts[:, 1] ** b * pts[:, 2] ** c)
                    assert abs(got - exact) < 1e-15, (order, a, b, c)
        _, fpts, fw, _ = B.face_rule("TET4", order)
        # face 3 is z = 0 with unit reference area scaling: the triangle rule itself
        for a in range(deg + 1):
            for b in range(deg + 1 - a):
                exact = math.factorial(a) * math.factorial(b) / math.factorial(a + b + 2)
                got = fw[3] @ (fpts[3][:, 0] ** a * fpts[3][:, 1] ** b)
                assert abs(got - exact) < 1e-15
    with pytest.raises(NotImplementedError):
        B.volume_quadrature("TET10", 3)


@pytest.mark.parametrize("ele", ["TET4", "TET10", "HEX20", "HEX27"])
def test_box_mesh_conforming(pkg, B, ele):
    m = element_box(pkg, ele, (3, 2, 2), L=(1.5, 1.0, 1.0))
    pts, cells = m.points, m.cells
    vals, grads, w = B.get_shape_vals_and_grads(ele)
    J = np.einsum("cai,qaj->cqij", pts[cells], grads)
    det = np.linalg.det(J)
    assert det.min() > 0
    np.testing.assert_allclose((det * w).sum(), 1.5, rtol=1e-13)
    # every face of a cell is shared by exactly two cells, or lies on the boundary
    finds = B.get_face_shape_vals_and_grads(ele)[4]
    keys = np.sort(cells[:, finds].reshape(-1, finds.shape[1]), axis=1)
    _, counts = np.unique(keys, axis=0, return_counts=True)
    assert counts.max() == 2
    nb = (counts == 1).sum()
    per_face = 2 if ele.startswith("TET") else 1
    assert nb == per_face * 2 * (3 * 2 + 3 * 2 + 2 * 2)
    # every node is used; quadratic nodes sit at their isoparametric positions
    assert len(np.unique(cells)) == len(pts)
    lin = "TET4" if ele.startswith("TET") else "HEX8"
    vn = B.shape_fn(lin, B.node_coords(ele))[0]  # (nen, corners)
    mapped = np.einsum("ka,cai->cki", vn, pts[cells[:, :vn.shape[1]]])
    np.testing.assert_allclose(mapped, pts[cells], atol=1e-13)


@pytest.mark.parametrize("ele", ["TET4", "TET10", "HEX27"])
def test_pattern_nen_matches_adjacency(pkg, ele):
    import ctypes
    nat = pkg._native
    m = element_box(pkg, ele, (2, 2, 1))
    cells = np.ascontiguousarray(m.cells, dtype=np.int32)
    C, nen = cells.shape
    N = len(m.points)
    lib = nat.lib()
    rp = np.zeros(N + 1, dtype=np.int32)
    nnzb = nat.I64(0)
    nat.check(lib.fem_bsr_pattern_nen(cells.ctypes.data, C, nen, N, rp.ctypes.data, ctypes.byref(nnzb), None, 0,
                                      None, None), "count")
    col = np.zeros(nnzb.value, dtype=np.int32)
    sc = np.zeros((C, nen * nen), dtype=np.int32)
    dg = np.zeros(N, dtype=np.int32)
    nat.check(lib.fem_bsr_pattern_nen(cells.ctypes.data, C, nen, N, rp.ctypes.data, ctypes.byref(nnzb),
                                      col.ctypes.data, col.size, sc.ctypes.data, dg.ctypes.data), "fill")
    adj = [set() for _ in range(N)]
    for c in cells:
        for a in c:
            adj[a].update(int(b) for b in c)
    for n in range(N):
        assert list(col[rp[n]:rp[n + 1]]) == sorted(adj[n])
        assert col[dg[n]] == n
    for c in range(C):
        for a in range(nen):
            for b in range(nen):
                k = sc[c, a * nen + b]
                assert rp[cells[c, a]] <= k < rp[cells[c, a] + 1] and col[k] == cells[c, b]


def test_load_vectors_match_oracle_tet10(pkg):
    m = element_box(pkg, "TET10", (2, 2, 2), amp=0.1)
    top = lambda p: np.isclose(p[2], 1.0, atol=1e-5)  # noqa: E731
    smap = lambda u, x: np.array([x[0], 2.0 * x[1], -1.0])  # noqa: E731
    bmap = lambda u, x: np.array([x[2], 1.0, x[0] * x[1]])  # noqa: E731
    fe = pkg.fe.FiniteElement(m, 3, 3, ele_type="TET10")
    binds = fe.get_boundary_conditions_inds([top])[0]
    assert len(binds) == 2 * 2 * 2
    op = fo.OracleProblem(m.points, m.cells, 3, fo.Law("linear", E=1.0, nu=0.3), location_fns=[top],
                          mass_map=bmap, surface_maps=[smap], ele_type="TET10")
    np.testing.assert_allclose(fe.surface_load(smap, binds), op.surface_load(), rtol=0, atol=1e-14)
    np.testing.assert_allclose(fe.body_load(bmap), op.body_load(), rtol=0, atol=1e-14)


@pytest.mark.parametrize("ele,rates", [("HEX8", (2, 1)), ("TET4", (2, 1)), ("TET10", (3, 2)),
                                       ("HEX20", (2, 1.5)), ("HEX27", (3, 2))])
def test_oracle_convergence_rates(pkg, ele, rates):
    errs = []
    for N in (4, 8):
        m = element_box(pkg, ele, (N, N, N))
        op = fo.OracleProblem(m.points, m.cells, 1, fo.Law("laplace", vec=1), dirichlet_bc_info=mms_bc(),
                              mass_map=mms_mass_map, ele_type=ele)
        u = fo.newton_solve(op, rel_tol=1e-10, tol=1e-10)
        errs.append(mms_errors(op.points, op.cells, op.vals, op.grads_ref, op.weights, u))
    l2_rate = np.log2(errs[0][0] / errs[1][0])
    h1_rate = np.log2(errs[0][1] / errs[1][1])
    assert abs(l2_rate - rates[0]) < 0.15 and abs(h1_rate - rates[1]) < 0.15, (l2_rate, h1_rate)


def test_multigrid_accepts_tet4_lattices_only(pkg):
    """precond 'gmg' needs lattice nodes in box_mesh numbering and a fine
    pattern inside the 27-point stencil: TET4 boxes qualify (each node
    couples to at most 14 lattice neighbours), quadratic types do not."""
    import ctypes
    mg = importlib.import_module("jax_fem_b200.multigrid")
    nat = pkg._native
    m = element_box(pkg, "TET4", (3, 2, 4))
    n, _ = mg.lattice_of(m.points)
    assert n == (4, 3, 5) and mg.lattice_of(m.points, m.cells) is None  # not HEX8 cells
    cells = np.ascontiguousarray(m.cells, dtype=np.int32)
    N = len(m.points)
    rp = np.zeros(N + 1, dtype=np.int32)
    nnzb = nat.I64(0)
    nat.check(nat.lib().fem_bsr_pattern_nen(cells.ctypes.data, len(cells), 4, N, rp.ctypes.data, ctypes.byref(nnzb),
                                            None, 0, None, None), "count")
    col = np.zeros(nnzb.value, dtype=np.int32)
    nat.check(nat.lib().fem_bsr_pattern_nen(cells.ctypes.data, len(cells), 4, N, rp.ctypes.data, ctypes.byref(nnzb),
                                            col.ctypes.data, col.size, None, None), "fill")
    st = mg.stencil_of(n, rp, col)
    assert (st >= 0).sum(axis=1).max() == 15 and (st[:, 13] >= 0).all()
    for ele in ("TET10", "HEX20", "HEX27"):
        assert mg.lattice_of(element_box(pkg, ele, (2, 2, 2)).points) is None


@pytest.mark.parametrize("ele", ["TET10", "HEX20", "HEX27"])
def test_pmultigrid_prolongation(pkg, ele):
    """p-multigrid's prolongation (pmultigrid.coarse_space) reproduces every
    linear field on all nodes from its corner values, its rows sum to one,
    and the corner nodes of box meshes form a lattice."""
    pm = importlib.import_module("jax_fem_b200.pmultigrid")
    mg = importlib.import_module("jax_fem_b200.multigrid")
    import scipy.sparse as sp
    m = element_box(pkg, ele, (3, 2, 2), amp=0.0)
    corners, cc, (r, c, w) = pm.coarse_space(ele, m.points, np.asarray(m.cells, dtype=np.int64))
    P = sp.csr_matrix((w, (r, c)), shape=(len(m.points), len(corners)))
    f = lambda X: 1.0 + 2.0 * X[:, 0] - X[:, 1] + 0.5 * X[:, 2]  # noqa: E731
    np.testing.assert_allclose(P @ f(m.points[corners]), f(m.points), atol=1e-14)
    np.testing.assert_allclose(np.asarray(P.sum(axis=1)).ravel(), 1.0, atol=1e-14)
    assert mg.lattice_of(m.points[corners]) is not None
    assert cc.shape == (len(m.cells), 4 if ele == "TET10" else 8)


@pytest.mark.parametrize("ele", ["TET10", "HEX27"])
def test_pmultigrid_method_on_oracle_tangents(pkg, ele):
    """The p-multigrid method of pmultigrid.py -- Chebyshev smoothing in the
    3x3 block-Jacobi-scaled operator (degree 2, [lmax/25, lmax]), the
    prolongation of coarse_space, the linear element re-discretised on the
    corner nodes (an exact coarse solve here), Dirichlet dofs projected out
    -- restated with scipy on the oracle's eliminated linear-elastic
    tangent: PCG reaches 1e-10 in under a fifth of block-Jacobi PCG's
    iterations, with the same solution."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    pm = importlib.import_module("jax_fem_b200.pmultigrid")
    m = element_box(pkg, ele, (4, 3, 3))
    bc = [[face_fn(0, 0.0)] * 3, [0, 1, 2], [lambda p: 0.0] * 3]
    law = fo.Law("linear", E=70e3, nu=0.3)
    op = fo.OracleProblem(m.points, m.cells, 3, law, dirichlet_bc_info=bc, ele_type=ele)
    op.newton_update(np.zeros(op.ndofs))
    K = op.assemble_global().tocsr()
    free = np.ones(op.ndofs)
    free[op.bc_rows()] = 0.0
    A = (sp.diags(free) @ K @ sp.diags(free) + sp.diags(1.0 - free)).tocsr()
    corners, cc, (r, c, w) = pm.coarse_space(ele, m.points, np.asarray(m.cells, dtype=np.int64))
    lin = "TET4" if ele == "TET10" else "HEX8"
    opc = fo.OracleProblem(m.points[corners], cc, 3, law, ele_type=lin)
    opc.newton_update(np.zeros(opc.ndofs))
    cd = (corners[:, None] * 3 + np.arange(3)).reshape(-1)
    fc = free[cd]
    Ac = (sp.diags(fc) @ opc.assemble_global() @ sp.diags(fc) + sp.diags(1.0 - fc)).tocsc()
    P = sp.kron(sp.csr_matrix((w, (r, c)), shape=(len(m.points), len(corners))), sp.eye(3)).tocsr()
    n = op.ndofs
    D = np.stack([A[3 * i:3 * i + 3, 3 * i:3 * i + 3].toarray() for i in range(n // 3)])
    Dinv = np.linalg.inv(D)
    jac = lambda v: np.einsum("nij,nj->ni", Dinv, v.reshape(-1, 3)).reshape(-1)  # noqa: E731
    x = np.random.default_rng(0).random(n)
    for _ in range(12):
        x /= np.linalg.norm(x)
        z = jac(A @ x)
        lam, x = x @ z, z
    lmax, ratio, nu = 1.1 * lam, 25.0, 2

    def cheb(b, z):
        lmin = lmax / ratio
        th, de = 0.5 * (lmax + lmin), 0.5 * (lmax - lmin)
        sig = th / de
        rho = 1.0 / sig
        rr = b - A @ z
        d = jac(rr) / th
        for k in range(nu):
            z = z + d
            if k == nu - 1:
                break
            rr = rr - A @ d
            rn = 1.0 / (2.0 * sig - rho)
            d = rn * rho * d + 2.0 * rn / de * jac(rr)
            rho = rn
        return z

    lu = spla.splu(Ac)

    def pmg(rv):
        z = cheb(rv, np.zeros(n))
        zc = lu.solve((P.T @ ((rv - A @ z) * free)) * fc) * fc
        z = z + (P @ zc) * free
        return cheb(rv, z) * free

    def pcg(M, b):
        x = np.zeros(n)
        rv = b.copy()
        z = M(rv)
        p = z.copy()
        rz = rv @ z
        for it in range(1, 5000):
            q = A @ p
            a = rz / (p @ q)
            x += a * p
            rv -= a * q
            if np.linalg.norm(rv) <= 1e-10 * np.linalg.norm(b):
                return x, it
            z = M(rv)
            rz, rz_old = rv @ z, rz
            p = z + rz / rz_old * p
        raise AssertionError("no convergence")

    b = np.random.default_rng(1).normal(size=n) * free
    x1, it_pmg = pcg(pmg, b)
    x2, it_bj = pcg(lambda v: jac(v) * free + v * (1.0 - free), b)
    assert it_pmg * 5 < it_bj, (it_pmg, it_bj)
    np.testing.assert_allclose(x1, x2, rtol=0, atol=1e-8 * np.abs(x2).max())


def test_pmultigrid_solver_code_on_cpu(pkg):
    """PMultigrid's own code -- setup (block-Jacobi inverse, power
    iteration), the Chebyshev smoother, the two-level apply with Dirichlet
    projection and the device-scalar CG -- run on CPU tensors with stand-ins
    for its library calls (operator and transfer products through scipy, an
    exact coarse solve for the V-cycle): on the oracle's eliminated TET10
    linear-elastic tangent it converges to the direct solution (1e-8) in
    under a fifth of block-Jacobi PCG's iterations (counted by scipy)."""
    import types

    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    import torch
    pm = importlib.import_module("jax_fem_b200.pmultigrid")
    ele = "TET10"
    m = element_box(pkg, ele, (4, 3, 3))
    bc = [[face_fn(0, 0.0)] * 3, [0, 1, 2], [lambda p: 0.0] * 3]
    law = fo.Law("linear", E=70e3, nu=0.3)
    op = fo.OracleProblem(m.points, m.cells, 3, law, dirichlet_bc_info=bc, ele_type=ele)
    op.newton_update(np.zeros(op.ndofs))
    free = np.ones(op.ndofs)
    free[op.bc_rows()] = 0.0
    A = (sp.diags(free) @ op.assemble_global() @ sp.diags(free) + sp.diags(1.0 - free)).tocsr()
    corners, cc, (r, c, w) = pm.coarse_space(ele, m.points, np.asarray(m.cells, dtype=np.int64))
    opc = fo.OracleProblem(m.points[corners], cc, 3, law, ele_type="TET4")
    opc.newton_update(np.zeros(opc.ndofs))
    cd = (corners[:, None] * 3 + np.arange(3)).reshape(-1)
    fc = free[cd]
    lu = spla.splu((sp.diags(fc) @ opc.assemble_global() @ sp.diags(fc) + sp.diags(1.0 - fc)).tocsc())
    P = sp.kron(sp.csr_matrix((w, (r, c)), shape=(len(m.points), len(corners))), sp.eye(3)).tocsr()
    n = op.ndofs
    Ab = A.tobsr(blocksize=(3, 3))
    Ab.sort_indices()
    diag = np.array([Ab.indptr[i] + np.searchsorted(Ab.indices[Ab.indptr[i]:Ab.indptr[i + 1]], i)
                     for i in range(n // 3)])

    def product(M):
        return lambda x, y: y.copy_(torch.from_numpy(M @ x.numpy()))

    Aop = types.SimpleNamespace(vals=torch.from_numpy(Ab.data.reshape(-1).copy()), diag=torch.from_numpy(diag),
                                n_brows=n // 3, vec=3, matvec=product(A))
    g = pm.PMultigrid.__new__(pm.PMultigrid)
    g.vec, g.fp32, g.lmax, g.dinv = 3, False, None, None
    g.corner_dofs = torch.from_numpy(cd)
    g.P = types.SimpleNamespace(n_brows=len(m.points), apply=product(P))
    g.PT = types.SimpleNamespace(n_brows=len(corners), apply=product(P.T.tocsr()))
    g.mg = types.SimpleNamespace(vcycle=lambda rhs, z, **kw: z.copy_(torch.from_numpy(lu.solve(rhs.numpy()))))
    mask = torch.from_numpy((1.0 - free).astype(np.uint8))
    g.problem = types.SimpleNamespace(dirichlet_device=lambda: (mask, torch.zeros(n, dtype=torch.float64)))
    g.setup(Aop, fine_only=True)
    b = np.random.default_rng(1).normal(size=n) * free
    x = torch.zeros(n, dtype=torch.float64)
    its, rel = g.solve(Aop, torch.from_numpy(b), x, rtol=1e-10, maxiter=500)
    ref = spla.spsolve(A.tocsc(), b)
    assert rel <= 1e-10
    np.testing.assert_allclose(x.numpy(), ref, rtol=0, atol=1e-8 * np.abs(ref).max())
    bj = []
    D = np.stack([A[3 * i:3 * i + 3, 3 * i:3 * i + 3].toarray() for i in range(n // 3)])
    Dinv = np.linalg.inv(D)
    spla.cg(A, b, rtol=1e-10, atol=0.0, maxiter=20000,
            M=spla.LinearOperator((n, n), lambda v: np.einsum("nij,nj->ni", Dinv, v.reshape(-1, 3)).reshape(-1)),
            callback=lambda xk: bj.append(1))
    assert its * 5 < len(bj), (its, len(bj))
