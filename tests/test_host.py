"""Host-side logic without a GPU: the C ABI loads and exports every declared
symbol, the pattern builder, mesh numbering, Dirichlet/face discovery, load
vectors, law recognition and solver-option resolution."""
import ctypes
import os
import re

import numpy as np
import pytest
import scipy.sparse as sp

from helpers import golden
from oracle import fem_oracle as fo

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg._native.load()
    header = open(os.path.join(ROOT, "include", "jaxfem_b200.h")).read()
    declared = set(re.findall(r"FEM_API\s+[\w\s\*]+?\b(fem_\w+)\s*\(", header))
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(lib, name), name
    assert declared == set(pkg._native.exported_symbols())
    assert pkg._native.version().startswith("jaxfem_b200")


def _pattern(pkg, cells, N):
    lib = pkg._native.load()
    C = len(cells)
    cells = np.ascontiguousarray(cells, dtype=np.int32)
    rp = np.zeros(N + 1, dtype=np.int32)
    nnzb = ctypes.c_int64(0)
    assert lib.fem_bsr_pattern(cells.ctypes.data, C, N, rp.ctypes.data, nnzb, None, 0, None, None) == 0
    col = np.zeros(nnzb.value, dtype=np.int32)
    sc = np.zeros((C, 64), dtype=np.int32)
    dg = np.zeros(N, dtype=np.int32)
    assert lib.fem_bsr_pattern(cells.ctypes.data, C, N, rp.ctypes.data, nnzb, col.ctypes.data, col.size,
                               sc.ctypes.data, dg.ctypes.data) == 0
    return rp, col, sc, dg, nnzb.value


@pytest.mark.parametrize("shape", [(1, 1, 1), (3, 2, 4), (20, 20, 20)])
def test_pattern_matches_node_adjacency(pkg, shape):
    pts, cells = fo.box_mesh(*shape, 1.0, 1.0, 1.0)
    N = len(pts)
    rp, col, sc, dg, nnzb = _pattern(pkg, cells, N)
    rows = np.repeat(cells[:, :, None], 8, axis=2).reshape(-1)
    cols = np.repeat(cells[:, None, :], 8, axis=1).reshape(-1)
    A = sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(N, N))
    A.sum_duplicates()
    A.sort_indices()
    np.testing.assert_array_equal(rp, A.indptr)
    np.testing.assert_array_equal(col, A.indices)
    # scatter map points at the (cells[c,a], cells[c,b]) block
    c = np.arange(len(cells))[:, None, None]
    a = np.arange(8)[None, :, None]
    b = np.arange(8)[None, None, :]
    blk = sc.reshape(-1, 8, 8)
    np.testing.assert_array_equal(col[blk], np.broadcast_to(cells[c, b], blk.shape))
    row_of_blk = np.searchsorted(rp, blk, side="right") - 1
    np.testing.assert_array_equal(row_of_blk, np.broadcast_to(cells[c, a], blk.shape))
    np.testing.assert_array_equal(col[dg], np.arange(N))
    Nx, Ny, Nz = shape
    assert nnzb == (3 * Nx + 1) * (3 * Ny + 1) * (3 * Nz + 1)  # prod(3 n_i - 2) over node counts


@pytest.mark.parametrize("shape", [(1, 1, 1), (3, 2, 4)])
def test_transpose_map_pairs_blocks(pkg, shape):
    """tmap[k] is the block (j, i) of block k = (i, j); it is an involution,
    and tmap[k] < k exactly for the lower-triangle blocks."""
    lib = pkg._native.load()
    pts, cells = fo.box_mesh(*shape, 1.0, 1.0, 1.0)
    N = len(pts)
    rp, col, _, _, nnzb = _pattern(pkg, cells, N)
    tmap = np.full(nnzb, -7, dtype=np.int32)
    assert lib.fem_bsr_transpose_map(rp.ctypes.data, col.ctypes.data, N, tmap.ctypes.data) == 0
    row = np.searchsorted(rp, np.arange(nnzb), side="right") - 1
    np.testing.assert_array_equal(col[tmap], row)
    np.testing.assert_array_equal(row[tmap], col)
    np.testing.assert_array_equal(tmap[tmap], np.arange(nnzb))
    np.testing.assert_array_equal(tmap < np.arange(nnzb), row > col)
    # a pattern without the partner of block (0, 1) is rejected
    rp2 = np.array([0, 2, 3], dtype=np.int32)
    col2 = np.array([0, 1, 1], dtype=np.int32)
    t2 = np.zeros(3, dtype=np.int32)
    assert lib.fem_bsr_transpose_map(rp2.ctypes.data, col2.ctypes.data, 2, t2.ctypes.data) == -1
    assert b"partner" in lib.fem_last_error()


def test_pattern_rejects_bad_node(pkg):
    lib = pkg._native.load()
    cells = np.arange(8, dtype=np.int32).reshape(1, 8)
    cells[0, 3] = 99
    rp = np.zeros(9, dtype=np.int32)
    n = ctypes.c_int64(0)
    assert lib.fem_bsr_pattern(cells.ctypes.data, 1, 8, rp.ctypes.data, n, None, 0, None, None) == -1
    assert b"outside" in lib.fem_last_error()


def test_box_mesh_numbering_matches_reference(pkg):
    m = pkg.box_mesh(3, 4, 5, 3.0, 2.0, 1.0)
    p, c = fo.box_mesh(3, 4, 5, 3.0, 2.0, 1.0)
    np.testing.assert_array_equal(m.points, p)
    np.testing.assert_array_equal(m.cells_dict["hexahedron"], c)


def test_dirichlet_discovery_batched_and_pointwise(pkg):
    d = golden("hyperelasticity")
    mesh = pkg.Mesh(d["points"], d["cells"])
    top = lambda p: np.isclose(p[2], 10.0, atol=1e-5)  # noqa: E731
    # a function that cannot be batched (uses Python control flow per point)
    def ring(p):
        return bool(p[0] ** 2 + p[1] ** 2 > 16.0) and bool(np.isclose(p[2], 0.0, atol=1e-5))
    val = lambda p: 0.1 * p[0]  # noqa: E731
    fe = pkg.fe.FiniteElement(mesh, 3, 3, dirichlet_bc_info=[[top, ring], [2, 0], [val, val]])
    n_ref, v_ref, val_ref = fo.dirichlet_bcs(d["points"], [[top, ring], [2, 0], [val, val]])
    for a, b in zip(fe.node_inds_list, n_ref):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(fe.vals_list, val_ref):
        np.testing.assert_allclose(a, b, rtol=0, atol=0)


def test_dirichlet_compact_matches_full_arrays(pkg):
    """The compact form a Dirichlet refresh copies to the device (constrained
    dofs and their values) equals the full-length mask and values, with the
    later condition winning where conditions overlap."""
    m = pkg.box_mesh(4, 3, 3, 1.0, 1.0, 1.0)
    left = lambda p: np.isclose(p[0], 0.0)  # noqa: E731
    low = lambda p: p[1] < 0.5  # overlaps the left face  # noqa: E731
    bc = [[left, left, low, left], [0, 1, 0, 2],
          [lambda p: 1.0 + p[1], lambda p: 0.0 * p[0], lambda p: -2.0 + 0.0 * p[0], lambda p: 3.0 * p[2]]]

    class P(pkg.Problem):
        def get_tensor_map(self):
            return pkg.LinearElastic(1.0, 0.3)

    p = P(pkg.Mesh(m.points, m.cells_dict["hexahedron"]), vec=3, dim=3, dirichlet_bc_info=bc)
    dofs, vals = p._dirichlet_compact()
    mask, full = p.fes[0].dirichlet_arrays()
    np.testing.assert_array_equal(dofs, np.flatnonzero(mask))
    np.testing.assert_array_equal(vals, full[dofs])
    assert np.all(np.diff(dofs) > 0)
    assert np.any(np.isclose(vals, -2.0))  # the later condition where it overlaps the left face


def test_batched_confirmation_by_code(pkg):
    """A value function rebuilt with new closure numbers (one per load step)
    reuses its code's batched confirmation with a two-point check; a closure
    value under which batching is wrong still ends in point-wise values."""
    fe_mod = pkg.fe
    pts = np.random.default_rng(1).uniform(size=(50, 3))

    def make(c, k=0):
        def f(p):
            return c * p[1] + (p[0].sum() if k else 0.0)  # k: sums over every point when batched
        return f

    first = fe_mod._batched_or_pointwise(make(0.5), (pts,), ())
    np.testing.assert_array_equal(first, 0.5 * pts[:, 1])
    assert any(key[0] is make(0.0).__code__ for key in fe_mod._BATCHED_CODE)
    again = fe_mod._batched_or_pointwise(make(-2.0), (pts,), ())
    np.testing.assert_array_equal(again, -2.0 * pts[:, 1])
    wrong = fe_mod._batched_or_pointwise(make(1.0, 1), (pts,), ())
    np.testing.assert_allclose(wrong, pts[:, 1] + pts[:, 0], rtol=1e-15)
    # only plain numbers in the closure qualify for the two-point check
    arr = np.array([1.0, 2.0])
    flag = True
    assert fe_mod._code_key(lambda p: arr[0] * p[0], ()) is None
    assert fe_mod._code_key(lambda p: p[0] if flag else p[1], ()) is None
    assert fe_mod._code_key(np.sin, ()) is None  # no Python code object
    assert fe_mod._code_key(make(2.0), ()) is not None


def _hierarchy_levels(nat, nodes, fp32, dense=True, half_level=0):
    """A FemMGLevel array with the node counts of a lattice hierarchy and
    stand-in (never dereferenced) pointers, for the host-only tail query."""
    levels = (nat.FemMGLevel * len(nodes))()
    for l, n in enumerate(nodes):
        L = levels[l]
        L.nodes[0], L.nodes[1], L.nodes[2] = n
        L.n_brows = n[0] * n[1] * n[2]
        for f in ("row_ptr", "col_idx", "stencil", "vals", "dinv", "x", "b", "r", "d0", "d1", "lmax"):
            setattr(L, f, 4096 * (l + 1))
        if l > 0:
            L.cpos, L.ilo, L.whi = 4096, 4096, 4096
    if dense:
        levels[len(nodes) - 1].cinv = 8192
    if fp32 and half_level is not None:
        levels[half_level].vals_lo, levels[half_level].lo_scale = 8192, 8192
    levels[0].nu = 1
    return levels


def test_mg_tail_plan(pkg):
    """Where the V-cycle's coarse end runs as one CTA over shared memory, for
    the 50^3 lattice hierarchy (51^3 ... 3^3 nodes): from the 5^3 level, in
    the FP32 layout that ran on the B200 (167,632 bytes) and in FP64; not
    when the smoothed coarsest level needs more Chebyshev steps than the
    coefficient tables hold, nor through a level with an FP16 copy."""
    import ctypes
    nat = pkg._native
    fn = nat.lib().fem_mg_tail_plan
    nodes = [(51, 51, 51), (26, 26, 26), (14, 14, 14), (8, 8, 8), (5, 5, 5), (3, 3, 3)]

    def plan(levels, fp32, nu=2, coarse_steps=8):
        s, b = ctypes.c_int(-2), ctypes.c_size_t(1)
        nat.check(fn(3, len(nodes), ctypes.byref(levels), int(fp32), nu, coarse_steps, ctypes.byref(s),
                     ctypes.byref(b)), "tail_plan")
        return s.value, b.value

    assert plan(_hierarchy_levels(nat, nodes, True), True) == (4, 167632)
    s64, b64 = plan(_hierarchy_levels(nat, nodes, False), False)
    assert s64 == 4 and 167632 < b64 <= 226 * 1024 and b64 % 16 == 0
    # a smoothed coarsest level: its steps must fit the tables (32)
    assert plan(_hierarchy_levels(nat, nodes, True, dense=False), True, coarse_steps=8)[0] == 4
    assert plan(_hierarchy_levels(nat, nodes, True, dense=False), True, coarse_steps=40) == (-1, 0)
    # the dense inverse makes coarse_steps irrelevant
    assert plan(_hierarchy_levels(nat, nodes, True), True, coarse_steps=40)[0] == 4
    # a level with an FP16 copy stays with the per-level kernels
    assert plan(_hierarchy_levels(nat, nodes, True, half_level=4), True) == (-1, 0)
    with pytest.raises(nat.FEMNativeError):
        plan(_hierarchy_levels(nat, nodes, True), True, nu=0)


_XCUT = 2.0


def _below_cut(p):
    return p[0] < _XCUT


def test_location_node_sets_reused_only_while_unchanged(pkg, monkeypatch):
    """A location function's node set is reused across Dirichlet updates
    while the function and what it reads are unchanged, and recomputed when a
    global or a closure array it reads changes; a function reading a mutable
    container is evaluated at every update."""
    global _XCUT
    fe_mod = pkg.fe
    d = golden("hyperelasticity")
    mesh = pkg.Mesh(d["points"], d["cells"])
    calls = []
    real = fe_mod._location_flags
    monkeypatch.setattr(fe_mod, "_location_flags", lambda fn, pts: calls.append(fn) or real(fn, pts))
    zero = lambda p: 0.0 * p[0]  # noqa: E731
    fe = fe_mod.FiniteElement(mesh, 3, 3, dirichlet_bc_info=[[_below_cut], [0], [zero]])
    first = fe.node_inds_list[0].copy()
    fe.update_Dirichlet_boundary_conditions([[_below_cut], [0], [zero]])
    assert len(calls) == 1  # reused
    np.testing.assert_array_equal(fe.node_inds_list[0], first)
    old = _XCUT
    try:
        _XCUT = 5.0  # a global the function reads
        fe.update_Dirichlet_boundary_conditions([[_below_cut], [0], [zero]])
        assert len(calls) == 2
        np.testing.assert_array_equal(fe.node_inds_list[0], np.flatnonzero(d["points"][:, 0] < 5.0))
    finally:
        _XCUT = old
    box = np.array([1.0, 3.0])
    inside = lambda p: (p[0] > box[0]) & (p[0] < box[1])  # noqa: E731
    fe.update_Dirichlet_boundary_conditions([[inside], [0], [zero]])
    box[1] = 6.0  # mutated in place
    fe.update_Dirichlet_boundary_conditions([[inside], [0], [zero]])
    assert len(calls) == 4  # evaluated again after the mutation
    np.testing.assert_array_equal(fe.node_inds_list[0],
                                  np.flatnonzero((d["points"][:, 0] > 1.0) & (d["points"][:, 0] < 6.0)))
    lims = [1.0]
    right_of = lambda p: p[0] > lims[0]  # noqa: E731
    for _ in range(2):
        fe.update_Dirichlet_boundary_conditions([[right_of], [0], [zero]])
    assert len(calls) == 6  # a list is never trusted
    assert fe_mod.function_state(right_of) is None and fe_mod.function_state(_below_cut) is not None


def test_load_vectors_match_oracle(pkg):
    d = golden("linear_elasticity_cylinder")
    mesh = pkg.Mesh(d["points"], d["cells"])
    top = lambda p: np.isclose(p[2], 10.0, atol=1e-5)  # noqa: E731
    mass = lambda u, x: -np.array([1e3 * x[0], 2e3 * x[1], 3e3 * x[2]])  # noqa: E731
    surf = lambda u, x: -np.array([1e3 * x[0] ** 2 + 1e3 * x[1] ** 2, 0.0, 0.0])  # noqa: E731
    fe = pkg.fe.FiniteElement(mesh, 3, 3)
    binds = fe.get_boundary_conditions_inds([top])
    op = fo.OracleProblem(d["points"], d["cells"], 3, fo.Law("linear", E=1.0, nu=0.3), location_fns=[top],
                          mass_map=mass, surface_maps=[surf])
    np.testing.assert_array_equal(binds[0], op.boundary_inds[0])
    fb = fe.body_load(mass)
    fs = fe.surface_load(surf, binds[0])
    np.testing.assert_allclose(fb, op.body_load(), rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(fs, op.surface_load(), rtol=1e-12, atol=1e-9)


def test_u_dependent_maps_are_rejected(pkg):
    m = pkg.box_mesh(2, 2, 2, 1.0, 1.0, 1.0)
    fe = pkg.fe.FiniteElement(pkg.Mesh(m.points, m.cells_dict["hexahedron"]), 3, 3)
    with pytest.raises(NotImplementedError):
        fe.body_load(lambda u, x: -u)


def test_law_recognition(pkg):
    assert isinstance(pkg.laws.as_law(lambda x: x, 1), pkg.Laplace)

    def stress(u_grad):
        E, nu = 70e3, 0.3
        mu = E / (2.0 * (1.0 + nu))
        lmbda = E * nu / ((1 + nu) * (1 - 2 * nu))
        eps = 0.5 * (u_grad + u_grad.T)
        return lmbda * np.trace(eps) * np.eye(3) + 2 * mu * eps

    law = pkg.laws.as_law(stress, 3)
    assert isinstance(law, pkg.LinearElastic)
    assert abs(law.E - 70e3) < 1e-6 and abs(law.nu - 0.3) < 1e-12
    with pytest.raises(NotImplementedError):
        pkg.laws.as_law(lambda F: F @ F.T, 3)  # nonlinear: must be a registered law
    with pytest.raises(NotImplementedError):
        pkg.laws.as_law(lambda u, th: u, 3)   # internal variables: must be registered


def test_solver_option_resolution(pkg):
    import importlib
    s = importlib.import_module("jax_fem_b200.solver")
    assert s._resolve_solver_options({}) == ("newton", {})
    m, cfg = s._resolve_solver_options({"petsc_solver": {}, "tol": 1e-5})
    assert m == "newton" and cfg["tol"] == 1e-5 and "petsc_solver" in cfg["linear"]
    lc = s.resolve_linear({})
    assert lc.method == pkg._native.KRYLOV_BICGSTAB and lc.precond == pkg._native.PRECOND_JACOBI
    assert lc.rtol == 1e-10 and lc.atol == 1e-10 and lc.maxiter == 10000
    lc = s.resolve_linear({"petsc_solver": {"ksp_type": "cg", "pc_type": "jacobi"}})
    assert lc.method == pkg._native.KRYLOV_CG and lc.precond == pkg._native.PRECOND_JACOBI
    with pytest.raises(ValueError):
        s._resolve_solver_options({"newton": {}, "arc_length": {}})
    # the reference's AMGX key: CG with the smoothed-aggregation AMG to an
    # absolute residual of 1e-10 (its built-in configuration's tolerance)
    lc = s.resolve_linear({"amgx_solver": {}})
    assert lc.method == pkg._native.KRYLOV_CG and lc.gmg and lc.mg["amg"] and lc.atol == 1e-10 and lc.rtol == 0.0
    with pytest.warns(UserWarning, match="configuration files"):
        s.resolve_linear({"amgx_solver": {"cfg_path": "amgx.json"}})
    lc = s.resolve_linear({"cg": {"precond": "amg", "mg_nu": 3}})
    assert lc.gmg and lc.mg["amg"] and lc.mg["nu"] == 3 and lc.with_rtol(1e-6).mg["amg"]
    assert not s.resolve_linear({"cg": {"precond": "gmg"}}).mg["amg"]
    with pytest.raises(ValueError, match="'cg' only"):
        s.resolve_linear({"bicgstab": {"precond": "amg"}})
    lc = s.resolve_linear({"cg": {"precond": "gmg", "rtol": "adaptive", "mg_lag": 4, "mg_nu_fine": 2, "mg_nu": 3}})
    assert lc.gmg and lc.adaptive and lc.eta_max == 1e-3
    assert lc.mg["lag"] == 4 and lc.mg["nu_fine"] == 2 and lc.mg["nu"] == 3 and lc.mg["coarse_steps"] == 8
    assert s.resolve_linear({"cg": {"precond": "gmg"}}).mg["nu_fine"] == 1


def test_no_gpu_means_loud_failure(pkg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    m = pkg.box_mesh(1, 1, 1, 1.0, 1.0, 1.0)

    class P(pkg.Problem):
        def get_tensor_map(self):
            return pkg.LinearElastic(1.0, 0.3)

    p = P(pkg.Mesh(m.points, m.cells_dict["hexahedron"]), vec=3, dim=3)
    with pytest.raises(pkg._native.FEMNativeError):
        pkg.solver(p)


def test_multigrid_lattice_hierarchy(pkg):
    """Host side of the multigrid: lattice detection, 1-D coarsening (the
    prolongation reproduces linear functions of the coordinates exactly, on
    graded lattices and odd cell counts) and the 27-point stencil map."""
    import importlib
    mg = importlib.import_module("jax_fem_b200.multigrid")
    m = pkg.box_mesh(5, 4, 6, 1.0, 2.0, 0.5)
    lat = mg.lattice_of(m.points, m.cells_dict["hexahedron"])
    assert lat is not None and lat[0] == (6, 5, 7)
    bent = m.points.copy()
    bent[7, 0] += 1e-3
    assert mg.lattice_of(bent, m.cells_dict["hexahedron"]) is None
    for coords in (np.linspace(0.0, 1.0, 6), np.linspace(0.0, 1.0, 9) ** 2, np.array([0.0, 0.3, 1.0])):
        cc, cpos, ilo, whi = mg.coarsen_1d(coords)
        np.testing.assert_array_equal(cc, coords[cpos])
        assert cpos[0] == 0 and cpos[-1] == len(coords) - 1
        P = np.zeros((len(coords), len(cc)))
        P[np.arange(len(coords)), ilo] += 1.0 - whi
        P[np.arange(len(coords)), ilo + 1] += whi
        np.testing.assert_allclose(P @ (2.0 - 3.0 * cc), 2.0 - 3.0 * coords, atol=1e-14)
        np.testing.assert_allclose(P.sum(axis=1), 1.0)
        assert ((whi >= 0) & (whi <= 1)).all()
    n = lat[0]
    rp, col, _, _, _ = _pattern(pkg, mg.lattice_cells(n), n[0] * n[1] * n[2])
    st = mg.stencil_of(n, rp, col)
    assert (st[:, 13] >= 0).all() and (col[st[:, 13]] == np.arange(len(st))).all()
    interior = (1 * n[1] + 1) * n[2] + 1
    assert (st[interior] >= 0).all()
    assert (st >= 0).sum() == len(col)
    # a mesh that is not a box lattice is refused before any device work
    with pytest.raises(NotImplementedError):
        mg.Multigrid(None, bent, m.cells_dict["hexahedron"])
    # the multigrid preconditioner is a CG preconditioner only
    S = importlib.import_module("jax_fem_b200.solver")
    with pytest.raises(ValueError):
        S.resolve_linear({"bicgstab": {"precond": "gmg"}})
    assert S.resolve_linear({"cg": {"precond": "gmg"}}).eta_max == 1e-3
