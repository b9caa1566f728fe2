"""Cell-kernel parity: GPU residual / BC-eliminated tangent / Dirichlet lift
against the FP64 oracle (complex-step cell Jacobians, PETSc-style COO sum),
on jittered meshes so every cell is a general trilinear hexahedron, and on
graded box lattices (every cell an axis-aligned box of its own size, the
kernel's box-cell geometry).

Tolerances: FP64 path 1e-11 relative (round-off of two differently ordered
FP64 computations); FP32 tangent 2e-5 relative to the matrix norm."""
import numpy as np
import pytest
import torch

from helpers import law_pair, make_problem, perturbed_box
from oracle import fem_oracle as fo

LAWS = ["laplace", "linear", "simp", "neo_hookean", "neo_hookean_scaled", "j2"]


def graded_lattice(pkg, N, seed=0):
    """Box lattice with randomly graded spacing per direction: every cell is
    an axis-aligned box, each of its own size (the kernel's box-cell
    geometry path)."""
    rng = np.random.default_rng(seed)
    axes = [np.concatenate([[0.0], np.cumsum(rng.uniform(0.5, 1.5, n))]) for n in N]
    axes = [a / a[-1] for a in axes]
    m = pkg.box_mesh(N[0], N[1], N[2], 1.0, 1.0, 1.0)
    n1 = [n + 1 for n in N]
    idx = np.arange(np.prod(n1))
    i, j, k = idx // (n1[1] * n1[2]), (idx // n1[2]) % n1[1], idx % n1[2]
    pts = np.stack([axes[0][i], axes[1][j], axes[2][k]], axis=1)
    return pkg.Mesh(pts, m.cells_dict["hexahedron"])


def _setup(pkg, kind, N=(3, 4, 5), seed=0, cells="jittered"):
    rng = np.random.default_rng(seed)
    mesh = perturbed_box(pkg, N, seed=seed) if cells == "jittered" else graded_lattice(pkg, N, seed=seed)
    C = len(mesh.cells)
    law, olaw, iv, oiv = law_pair(pkg, kind, C, rng)
    left = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    right = lambda p: np.isclose(p[0], 1.0, atol=1e-5)  # noqa: E731
    bc = [[left] * 3 + [right], [0, 1, 2, 0], [lambda p: 0.0] * 3 + [lambda p: 0.02]]
    prob = make_problem(pkg, mesh, law, bc=bc, ivars=iv)
    oprob = fo.OracleProblem(mesh.points, mesh.cells, 3, olaw, dirichlet_bc_info=bc, internal_vars=oiv)
    scale = 0.05 if kind.startswith("neo") else 2e-3
    u = rng.normal(0, scale, size=prob.num_total_dofs_all_vars)
    return prob, oprob, u


def _eliminate(A, rows):
    A = A.tolil()
    keep = np.ones(A.shape[0], bool)
    keep[rows] = False
    import scipy.sparse as sp
    D = sp.diags(keep.astype(float))
    out = D @ A.tocsr() @ D
    out = out + sp.diags((~keep).astype(float))
    return out.tocsr()


@pytest.mark.gpu
@pytest.mark.parametrize("cells", ["jittered", "boxes"])
@pytest.mark.parametrize("kind", LAWS)
def test_residual_tangent_lift_f64(pkg, cuda, kind, cells):
    prob, oprob, u = _setup(pkg, kind, cells=cells)
    n = prob.num_total_dofs_all_vars
    ud = torch.tensor(u, device=cuda)
    mask, ubc = prob.dirichlet_device()
    dvec = torch.where(mask.bool(), ubc - ud, torch.zeros_like(ud))
    res = torch.empty(n, dtype=torch.float64, device=cuda)
    lift = torch.empty_like(res)
    A = prob.dev().new_matrix(torch.float64)
    prob.assemble(ud, res=res, vals=A.vals, lift=lift, dvec=dvec)
    torch.cuda.synchronize()

    cell_u = u.reshape(-1, 3)[oprob.cells]
    r_ref, jac = oprob.cell_residual_and_jacobian(cell_u, oprob.internal_vars)
    R_ref = np.zeros(n)
    np.add.at(R_ref, oprob.cell_dofs.reshape(-1), r_ref.reshape(-1))
    K = oprob.assemble_global(jac)
    rows = oprob.bc_rows()
    scale_r = np.abs(R_ref).max()
    np.testing.assert_allclose(res.cpu().numpy(), R_ref, rtol=0, atol=1e-11 * scale_r)

    Kg = A.to_scipy()
    Ke = _eliminate(K, rows)
    scale_k = np.abs(K.data).max()
    assert np.abs((Kg - Ke).toarray()).max() <= 1e-11 * scale_k

    dv = dvec.cpu().numpy()
    lift_ref = K @ dv
    lift_ref[rows] = 0.0
    got = lift.cpu().numpy()
    got[rows] = 0.0
    np.testing.assert_allclose(got, lift_ref, rtol=0, atol=1e-11 * max(1.0, np.abs(lift_ref).max()))


@pytest.mark.gpu
@pytest.mark.parametrize("cells", ["jittered", "boxes"])
@pytest.mark.parametrize("kind", ["linear", "neo_hookean", "j2"])
def test_tangent_f32(pkg, cuda, kind, cells):
    """The FP32-tangent pass: tangent within FP32 rounding of the FP64 one,
    residual FP64 (as the FP64 pass gives it), lift from the FP32 tangent."""
    prob, oprob, u = _setup(pkg, kind, seed=1, cells=cells)
    ud = torch.tensor(u, device=cuda)
    n = ud.numel()
    mask, _ = prob.dirichlet_device()
    dvec = torch.where(mask.bool(), torch.full_like(ud, 1e-3), torch.zeros_like(ud))
    A32 = prob.dev().new_matrix(torch.float32)
    r32, l32 = torch.empty(n, dtype=torch.float64, device=cuda), torch.empty(n, dtype=torch.float64, device=cuda)
    prob.assemble(ud, res=r32, vals=A32.vals, lift=l32, dvec=dvec, fp32=True)
    A64 = prob.dev().new_matrix(torch.float64)
    r64, l64 = torch.empty_like(r32), torch.empty_like(l32)
    prob.assemble(ud, res=r64, vals=A64.vals, lift=l64, dvec=dvec)
    torch.cuda.synchronize()
    d = (A32.vals.double() - A64.vals).abs().max().item()
    assert d <= 1e-5 * A64.vals.abs().max().item()
    assert (r32 - r64).abs().max().item() <= 1e-13 * r64.abs().max().item()
    assert (l32 - l64).abs().max().item() <= 1e-5 * max(l64.abs().max().item(), 1e-300)


@pytest.mark.gpu
def test_tangent_symmetric(pkg, cuda):
    for kind in ["linear", "neo_hookean", "j2"]:
        prob, _, u = _setup(pkg, kind, seed=2)
        A = prob.dev().new_matrix(torch.float64)
        prob.assemble(torch.tensor(u, device=cuda), vals=A.vals)
        K = A.to_scipy()
        assert abs(K - K.T).max() <= 1e-12 * abs(K).max()


@pytest.mark.gpu
def test_empty_and_single_cell(pkg, cuda):
    # one cell, no BCs: residual of a rigid translation vanishes
    m = pkg.box_mesh(1, 1, 1, 1.0, 1.0, 1.0)
    mesh = pkg.Mesh(m.points, m.cells_dict["hexahedron"])
    prob = make_problem(pkg, mesh, pkg.NeoHookean(10.0, 0.3))
    u = torch.full((24,), 0.3, dtype=torch.float64, device=cuda)
    r = prob.compute_residual([u.reshape(8, 3)])[0]
    assert r.abs().max().item() < 1e-13
