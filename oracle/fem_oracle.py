"""FP64 numpy restatement of the reference's assemble-and-solve path (HEX8,
and the TET4, TET10, HEX20, HEX27 and 2D QUAD4, QUAD8, TRI3, TRI6 element
types).

TEST INFRASTRUCTURE ONLY: the parity checker and the CPU baseline.  The
product (``jax-fem_b200``) never imports this module.

Every function cites the reference file:line it restates (paths inside the
reference project).  Arithmetic is float64 (the reference forces x64 when
``jax_fem.solver`` is imported, solver.py:10-11).  The per-cell Jacobian is
computed the way the reference does it -- forward-mode derivatives of the
weak-form kernel along the 24 cell dofs (problem.py:262-266, ``jax.jvp``
over an identity basis) -- here by complex-step differentiation, which gives
the same directional derivatives to round-off for these analytic kernels.
The GPU path uses closed-form tangents instead and is checked against this.

Third-party arithmetic restated here (absent from the reference tree):
basix 0.10.0 (HEX8 Lagrange tabulation, Gauss-Jacobi quadrature; see
``hex8_tables``) and PETSc 3.25.1 COO summation / ``zeroRows`` (see
``assemble_global``).
"""
import itertools

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

# --------------------------------------------------------------------------
# Basis and quadrature (basis.py:19-57, 117-124, 141-250)
# --------------------------------------------------------------------------

# basix hexahedron vertices on [0,1]^3, x fastest (basix cell geometry).
BASIX_HEX_VERTICES = np.array(
    [[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0],
     [0, 0, 1], [1, 0, 1], [0, 1, 1], [1, 1, 1]], dtype=np.float64)
# VTK/meshio -> basix node permutation for HEX8 (basis.py:53).
HEX8_REORDER = np.array([0, 1, 3, 2, 4, 5, 7, 6])
# basix hexahedron facets (sub-entity connectivity, dim 2) and outward normals.
BASIX_HEX_FACETS = np.array(
    [[0, 1, 2, 3], [0, 1, 4, 5], [0, 2, 4, 6], [1, 3, 5, 7], [2, 3, 6, 7], [4, 5, 6, 7]])
BASIX_HEX_NORMALS = np.array(
    [[0, 0, -1], [0, -1, 0], [-1, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.float64)


def gauss_jacobi_01(m):
    """m-point Gauss-Legendre rule on [0,1], points ascending (basix GJ rule)."""
    x, w = np.polynomial.legendre.leggauss(m)
    return 0.5 + 0.5 * x, 0.5 * w


def hex8_shape(xi):
    """Trilinear shape values/gradients at points xi (n,3), VTK node order.

    Returns vals (n,8), grads (n,8,3).  Equivalent to basix P1 hexahedron
    tabulation followed by ``[:, :, re_order]`` (basis.py:170-173).
    """
    X = BASIX_HEX_VERTICES[HEX8_REORDER]  # VTK node positions
    xi = np.atleast_2d(xi)
    f = X[None, :, :] * xi[:, None, :] + (1 - X[None, :, :]) * (1 - xi[:, None, :])  # (n,8,3)
    df = (2 * X - 1)[None, :, :] * np.ones_like(f)
    vals = f.prod(axis=2)
    grads = np.stack([df[:, :, 0] * f[:, :, 1] * f[:, :, 2],
                      f[:, :, 0] * df[:, :, 1] * f[:, :, 2],
                      f[:, :, 0] * f[:, :, 1] * df[:, :, 2]], axis=2)
    return vals, grads


def hex8_tables(quadrature_order=2):
    """shape_vals (Q,8), shape_grads_ref (Q,8,3), weights (Q,) (basis.py:141-175).

    basix ``make_quadrature(hexahedron, order)`` with the default Gauss-Jacobi
    rule uses m = (order+2)//2 points per axis, tensor product with the x
    coordinate slowest and z fastest.
    """
    m = (quadrature_order + 2) // 2
    p, w = gauss_jacobi_01(m)
    pts = np.array([[a, b, c] for a in p for b in p for c in p])
    wts = np.array([wa * wb * wc for wa in w for wb in w for wc in w])
    vals, grads = hex8_shape(pts)
    return vals, grads, wts


def hex8_face_tables(quadrature_order=2):
    """Face tables (basis.py:178-250): vals (6,F,8), grads (6,F,8,3),
    weights (6,F), normals (6,3), face_inds (6,4) in VTK node numbering."""
    m = (quadrature_order + 2) // 2
    p, w = gauss_jacobi_01(m)
    qpts = np.array([[a, b] for a in p for b in p])
    qw = np.array([wa * wb for wa in w for wb in w])
    s, t = qpts[:, 0], qpts[:, 1]
    lag = np.stack([(1 - s) * (1 - t), s * (1 - t), (1 - s) * t, s * t], axis=1)  # P1 quad map
    fpts, fw, finds = [], [], []
    for facet in BASIX_HEX_FACETS:
        v = BASIX_HEX_VERTICES[facet]
        fpts.append(lag @ v)
        jac = np.stack([v[1] - v[0], v[2] - v[0]], axis=1)
        fw.append(qw * np.linalg.norm(np.cross(jac[:, 0], jac[:, 1])))
        finds.append([int(np.argwhere(HEX8_REORDER == i)[0, 0]) for i in facet])
    fpts = np.stack(fpts)
    vals, grads = hex8_shape(fpts.reshape(-1, 3))
    nf, nq = fpts.shape[:2]
    return (vals.reshape(nf, nq, 8), grads.reshape(nf, nq, 8, 3), np.stack(fw),
            BASIX_HEX_NORMALS.copy(), np.array(finds))


# --------------------------------------------------------------------------
# Other element types (basis.py:19-114): TET4, TET10, HEX20, HEX27
# --------------------------------------------------------------------------
# Restated from basix's element definitions in basix numbering, then moved
# to mesh order with the reference's re_order tables, the way
# get_shape_vals_and_grads does (basis.py:168-173).  Each element is the
# dual basis of its degrees of freedom in its polynomial space, computed by
# inverting the functionals applied to a monomial basis:
#   P1/P2 on the tetrahedron, Q2 on the hexahedron: point values at the
#   vertices, edge midpoints, face centres and cell centre (basix's dof
#   entity order: vertices, edges, faces, interior);
#   serendipity degree 2 on the hexahedron: vertex values and edge means
#   (moments against the degree-0 DPC space on each edge).
BASIX_TET_VERTICES = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.float64)
BASIX_TET_EDGES = np.array([[2, 3], [1, 3], [1, 2], [0, 3], [0, 2], [0, 1]])
BASIX_TET_FACETS = np.array([[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]])
BASIX_TET_NORMALS = np.array([[1, 1, 1], [-1, 0, 0], [0, -1, 0], [0, 0, -1]], dtype=np.float64)
BASIX_TET_NORMALS[0] /= np.sqrt(3.0)
BASIX_HEX_EDGES = np.array([[0, 1], [0, 2], [0, 4], [1, 3], [1, 5], [2, 3], [2, 6], [3, 7],
                            [4, 5], [4, 6], [5, 7], [6, 7]])
# basix quadrilateral / triangle: vertices, edges (= facets) and the
# facets' outward normals.
BASIX_QUAD_VERTICES = np.array([[0, 0], [1, 0], [0, 1], [1, 1]], dtype=np.float64)
BASIX_QUAD_EDGES = np.array([[0, 1], [0, 2], [1, 3], [2, 3]])
BASIX_QUAD_NORMALS = np.array([[0, -1], [-1, 0], [1, 0], [0, 1]], dtype=np.float64)
BASIX_TRI_VERTICES = np.array([[0, 0], [1, 0], [0, 1]], dtype=np.float64)
BASIX_TRI_EDGES = np.array([[1, 2], [0, 2], [0, 1]])
BASIX_TRI_NORMALS = np.array([[1, 1], [-1, 0], [0, -1]], dtype=np.float64) / np.array([[np.sqrt(2.0)], [1], [1]])
# re_order of basis.py:53-107 (mesh position -> basix dof)
RE_ORDER = {
    "HEX8": [0, 1, 3, 2, 4, 5, 7, 6],
    "HEX27": [0, 1, 3, 2, 4, 5, 7, 6, 8, 11, 13, 9, 16, 18, 19, 17, 10, 12, 15, 14, 22, 23, 21, 24, 20, 25, 26],
    "HEX20": [0, 1, 3, 2, 4, 5, 7, 6, 8, 11, 13, 9, 16, 18, 19, 17, 10, 12, 15, 14],
    "TET4": [0, 1, 2, 3],
    "TET10": [0, 1, 2, 3, 9, 6, 8, 7, 5, 4],
    "QUAD4": [0, 1, 3, 2],
    "QUAD8": [0, 1, 3, 2, 4, 6, 7, 5],
    "TRI3": [0, 1, 2],
    "TRI6": [0, 1, 2, 5, 3, 4],
}
DEFAULT_QUADRATURE_ORDER = {"HEX8": 2, "HEX27": 10, "HEX20": 2, "TET4": 0, "TET10": 2,
                            "QUAD4": 2, "QUAD8": 2, "TRI3": 0, "TRI6": 2}


def element_dim(ele_type):
    return 2 if ele_type[:3] in ("QUA", "TRI") else 3


def _monomial_table(pts, exps):
    """Values (n, m) and gradients (n, m, dim) of monomials x^e at points."""
    pts = np.atleast_2d(pts)
    n, m, dim = len(pts), len(exps), pts.shape[1]
    vals = np.ones((n, m))
    grads = np.zeros((n, m, dim))
    for k, e in enumerate(exps):
        vals[:, k] = np.prod([pts[:, d] ** e[d] for d in range(dim)], axis=0)
        for d in range(dim):
            if e[d] == 0:
                continue
            g = e[d] * pts[:, d] ** (e[d] - 1)
            for o in range(dim):
                if o != d:
                    g = g * pts[:, o] ** e[o]
            grads[:, k, d] = g
    return vals, grads


def _element_space(ele_type):
    """Monomial exponents of the element's polynomial space."""
    d = element_dim(ele_type)
    if ele_type in ("TET4", "TRI3"):
        return [e for e in np.ndindex(*(2,) * d) if sum(e) <= 1]
    if ele_type in ("TET10", "TRI6"):
        return [e for e in np.ndindex(*(3,) * d) if sum(e) <= 2]
    if ele_type in ("HEX27",):
        return list(np.ndindex(3, 3, 3))
    if ele_type == "QUAD4":
        return list(np.ndindex(2, 2))
    if ele_type in ("HEX20", "QUAD8"):  # superlinear degree (degree minus linearly entering variables) <= 2
        return [e for e in np.ndindex(*(4,) * d) if sum(e) - sum(x == 1 for x in e) <= 2]
    raise ValueError(ele_type)


def _basix_vertices_edges(ele_type):
    return {"TET": (BASIX_TET_VERTICES, BASIX_TET_EDGES), "HEX": (BASIX_HEX_VERTICES, BASIX_HEX_EDGES),
            "QUA": (BASIX_QUAD_VERTICES, BASIX_QUAD_EDGES), "TRI": (BASIX_TRI_VERTICES, BASIX_TRI_EDGES)}[ele_type[:3]]


def _basix_dof_functionals(ele_type):
    """The element's dofs in basix order, each (points, weights): a point
    value is one point with weight 1; an edge mean is a Gauss rule on the edge."""
    V, E = _basix_vertices_edges(ele_type)
    dofs = [(V[i][None], np.ones(1)) for i in range(len(V))]
    if ele_type in ("TET10", "HEX27", "TRI6"):
        dofs += [(0.5 * (V[a] + V[b])[None], np.ones(1)) for a, b in E]
    if ele_type in ("HEX20", "QUAD8"):
        t, w = gauss_jacobi_01(3)
        dofs += [(V[a][None] + t[:, None] * (V[b] - V[a])[None], w) for a, b in E]
    if ele_type == "HEX27":
        dofs += [(V[f].mean(axis=0)[None], np.ones(1)) for f in BASIX_HEX_FACETS]
        dofs += [(np.full((1, 3), 0.5), np.ones(1))]
    return dofs


def element_shape(ele_type, xi):
    """vals (n, nen), grads (n, nen, 3) in mesh node order at points xi."""
    if ele_type == "HEX8":
        return hex8_shape(xi)
    exps = _element_space(ele_type)
    dofs = _basix_dof_functionals(ele_type)
    assert len(exps) == len(dofs), (ele_type, len(exps), len(dofs))
    L = np.array([w @ _monomial_table(p, exps)[0] for p, w in dofs])  # (dof, monomial)
    C = np.linalg.inv(L)  # column k: coefficients of basis function k
    v, g = _monomial_table(xi, exps)
    vals, grads = v @ C, np.einsum("nmd,mk->nkd", g, C)
    ro = RE_ORDER[ele_type]
    return vals[:, ro], grads[:, ro]


def simplex_quadrature(dim, order):
    """basix default (Xiao-Gimbutas) rules of orders 0-2 on the reference
    triangle / tetrahedron."""
    if dim == 3:
        if order <= 1:
            return np.array([[0.25, 0.25, 0.25]]), np.array([1.0 / 6.0])
        a = 0.1381966011250105
        b = 1.0 - 3.0 * a
        return np.array([[a, a, a], [b, a, a], [a, b, a], [a, a, b]]), np.full(4, 1.0 / 24.0)
    if order <= 1:
        return np.array([[1.0 / 3.0, 1.0 / 3.0]]), np.array([0.5])
    return np.array([[1 / 6, 1 / 6], [2 / 3, 1 / 6], [1 / 6, 2 / 3]]), np.full(3, 1.0 / 6.0)


def element_tables(ele_type, quadrature_order=None):
    """shape_vals (Q,nen), shape_grads_ref (Q,nen,dim), weights (Q,) (basis.py:141-175)."""
    order = DEFAULT_QUADRATURE_ORDER[ele_type] if quadrature_order is None else quadrature_order
    dim = element_dim(ele_type)
    if ele_type[:3] in ("TET", "TRI"):
        pts, wts = simplex_quadrature(dim, order)
    else:
        m = (order + 2) // 2
        p, w = gauss_jacobi_01(m)
        pts = np.array(list(itertools.product(p, repeat=dim)))
        wts = np.array([np.prod(c) for c in itertools.product(w, repeat=dim)])
    vals, grads = element_shape(ele_type, pts)
    return vals, grads, wts


def _edge_face_tables(ele_type, order):
    """2D cells: facets are edges, the Gauss-Jacobi rule of the order on
    each, weights times the edge length (basis.py:225-233)."""
    p, w = gauss_jacobi_01((order + 2) // 2)
    V, E = _basix_vertices_edges(ele_type)
    normals = BASIX_TRI_NORMALS if ele_type.startswith("TRI") else BASIX_QUAD_NORMALS
    ro = np.array(RE_ORDER[ele_type])
    fpts = np.stack([np.outer(1 - p, V[a]) + np.outer(p, V[b]) for a, b in E])
    fw = np.stack([w * np.linalg.norm(V[b] - V[a]) for a, b in E])
    finds = np.array([[int(np.argwhere(ro == i)[0, 0]) for i in e] for e in E])
    nf, nq = fpts.shape[:2]
    vals, grads = element_shape(ele_type, fpts.reshape(-1, 2))
    nen = vals.shape[1]
    return vals.reshape(nf, nq, nen), grads.reshape(nf, nq, nen, 2), fw, normals.copy(), finds


def element_face_tables(ele_type, quadrature_order=None):
    """Face tables (basis.py:178-250) for any element type: vals (nf,F,nen),
    grads (nf,F,nen,dim), weights (nf,F), normals (nf,dim), face_inds (nf,nfv)."""
    order = DEFAULT_QUADRATURE_ORDER[ele_type] if quadrature_order is None else quadrature_order
    if element_dim(ele_type) == 2:
        return _edge_face_tables(ele_type, order)
    if ele_type.startswith("TET"):
        qp, qw = simplex_quadrature(2, order)
        s, t = qp[:, 0], qp[:, 1]
        lag = np.stack([1 - s - t, s, t], axis=1)
        V, facets, normals = BASIX_TET_VERTICES, BASIX_TET_FACETS, BASIX_TET_NORMALS
    else:
        m = (order + 2) // 2
        p, w = gauss_jacobi_01(m)
        qp = np.array([[a, b] for a in p for b in p])
        qw = np.array([wa * wb for wa in w for wb in w])
        s, t = qp[:, 0], qp[:, 1]
        lag = np.stack([(1 - s) * (1 - t), s * (1 - t), (1 - s) * t, s * t], axis=1)
        V, facets, normals = BASIX_HEX_VERTICES, BASIX_HEX_FACETS, BASIX_HEX_NORMALS
    ro = np.array(RE_ORDER[ele_type])
    fpts, fw, finds = [], [], []
    for facet in facets:
        v = V[facet]
        fpts.append(lag @ v)
        fw.append(qw * np.linalg.norm(np.cross(v[1] - v[0], v[2] - v[0])))
        finds.append([int(np.argwhere(ro == i)[0, 0]) for i in facet])
    fpts = np.stack(fpts)
    nf, nq = fpts.shape[:2]
    vals, grads = element_shape(ele_type, fpts.reshape(-1, 3))
    nen = vals.shape[1]
    return (vals.reshape(nf, nq, nen), grads.reshape(nf, nq, nen, 3), np.stack(fw), normals.copy(),
            np.array(finds))


# --------------------------------------------------------------------------
# Mesh (generate_mesh.py:151-189)
# --------------------------------------------------------------------------

def box_mesh(Nx, Ny, Nz, Lx, Ly, Lz):
    x = np.linspace(0, Lx, Nx + 1)
    y = np.linspace(0, Ly, Ny + 1)
    z = np.linspace(0, Lz, Nz + 1)
    xv, yv, zv = np.meshgrid(x, y, z, indexing="ij")
    points = np.stack((xv, yv, zv), axis=3).reshape(-1, 3)
    ind = np.arange(len(points)).reshape(Nx + 1, Ny + 1, Nz + 1)
    cells = np.stack((ind[:-1, :-1, :-1], ind[1:, :-1, :-1], ind[1:, 1:, :-1], ind[:-1, 1:, :-1],
                      ind[:-1, :-1, 1:], ind[1:, :-1, 1:], ind[1:, 1:, 1:], ind[:-1, 1:, 1:]),
                     axis=3).reshape(-1, 8)
    return points, cells.astype(np.int32)


# --------------------------------------------------------------------------
# Geometry (fe.py:112-218)
# --------------------------------------------------------------------------

def shape_grads(points, cells, grads_ref, weights):
    """Physical shape gradients (C,Q,8,3) and JxW (C,Q) (fe.py:112-141)."""
    X = points[cells]  # (C,8,3)
    J = np.einsum("cai,qaj->cqij", X, grads_ref)
    det = np.linalg.det(J)
    Jinv = np.linalg.inv(J)
    g = np.einsum("qaj,cqjk->cqak", grads_ref, Jinv)
    return g, det * weights[None, :]


def physical_quad_points(points, cells, vals):
    return np.einsum("qa,cai->cqi", vals, points[cells])


def eval_pointwise(fn, *args):
    """Evaluate a per-point user function over leading axes of ``args``.

    The reference evaluates location/value/mass/surface functions one point
    at a time under ``jax.vmap`` (fe.py:252-254, problem.py:230,253).  Here a
    Python loop plays the role of vmap.
    """
    n = len(args[0])
    out = [np.asarray(fn(*[a[i] for a in args])) for i in range(n)]
    return np.array(out)


def dirichlet_bcs(points, bc_info):
    """node_inds, vec_inds, vals lists (fe.py:220-258)."""
    nodes, vecs, vals = [], [], []
    if bc_info is None:
        return nodes, vecs, vals
    loc_fns, vec_list, val_fns = bc_info
    for lf, v, vf in zip(loc_fns, vec_list, val_fns):
        nargs = lf.__code__.co_argcount
        if nargs == 1:
            flags = np.array([bool(lf(p)) for p in points])
        else:
            flags = np.array([bool(lf(p, i)) for i, p in enumerate(points)])
        ni = np.argwhere(flags).reshape(-1)
        nodes.append(ni)
        vecs.append(np.full(len(ni), v, dtype=np.int64))
        vals.append(np.array([float(vf(points[i])) for i in ni], dtype=np.float64).reshape(-1))
    return nodes, vecs, vals


def boundary_faces(points, cells, location_fns, face_inds):
    """(num_selected_faces, 2) [cell, local face] per location fn (fe.py:271-322)."""
    out = []
    if location_fns is None:
        return out
    for lf in location_fns:
        nargs = lf.__code__.co_argcount
        if nargs == 1:
            flag = np.array([bool(lf(p)) for p in points])
        else:
            flag = np.array([bool(lf(p, i)) for i, p in enumerate(points)])
        cf = flag[cells[:, face_inds]]  # (C,6,4)
        out.append(np.argwhere(cf.all(axis=2)))
    return out


def face_geometry(points, cells, binds, fgrads_ref, fweights, normals):
    """face shape grads and Nanson scale (fe.py:143-183)."""
    X = points[cells][binds[:, 0]]
    gr = fgrads_ref[binds[:, 1]]  # (F,q,8,3)
    J = np.einsum("fai,fqaj->fqij", X, gr)
    det = np.linalg.det(J)
    Jinv = np.linalg.inv(J)
    n = normals[binds[:, 1]]
    nJ = np.einsum("fi,fqij->fqj", n, Jinv)
    scale = np.linalg.norm(nJ, axis=-1) * det * fweights[binds[:, 1]]
    return scale


# --------------------------------------------------------------------------
# Constitutive laws (complex-step safe)
# --------------------------------------------------------------------------

def _eye(shape):
    return np.broadcast_to(np.eye(3), shape + (3, 3))


def lame(E, nu):
    mu = E / (2.0 * (1.0 + nu))
    lmbda = E * nu / ((1 + nu) * (1 - 2 * nu))
    return lmbda, mu


def stress_linear(u_grad, E, nu):
    """Isotropic linear elasticity (test_linear_elasticity_cube.py:16-25)."""
    lmbda, mu = lame(E, nu)
    eps = 0.5 * (u_grad + np.swapaxes(u_grad, -1, -2))
    tr = np.trace(eps, axis1=-2, axis2=-1)
    return lmbda * tr[..., None, None] * _eye(tr.shape) + 2 * mu * eps


def simp_modulus(theta, E0, Emin, penal):
    """E = Emin + (E0-Emin) theta^p (top_opt/fem_model.py:67-80)."""
    return Emin + (E0 - Emin) * theta ** penal


def stress_simp(u_grad, theta, E0, Emin, nu, penal):
    E = simp_modulus(theta, E0, Emin, penal)
    lmbda, mu = lame(E, nu)
    eps = 0.5 * (u_grad + np.swapaxes(u_grad, -1, -2))
    tr = np.trace(eps, axis1=-2, axis2=-1)
    return (lmbda * tr)[..., None, None] * _eye(tr.shape) + (2 * mu)[..., None, None] * eps


def _det3(F):
    return (F[..., 0, 0] * (F[..., 1, 1] * F[..., 2, 2] - F[..., 1, 2] * F[..., 2, 1])
            - F[..., 0, 1] * (F[..., 1, 0] * F[..., 2, 2] - F[..., 1, 2] * F[..., 2, 0])
            + F[..., 0, 2] * (F[..., 1, 0] * F[..., 2, 1] - F[..., 1, 1] * F[..., 2, 0]))


def _cof3(F):
    """Cofactor matrix (det(F) F^{-T}), complex-safe."""
    c = np.empty(F.shape, dtype=F.dtype)
    c[..., 0, 0] = F[..., 1, 1] * F[..., 2, 2] - F[..., 1, 2] * F[..., 2, 1]
    c[..., 0, 1] = F[..., 1, 2] * F[..., 2, 0] - F[..., 1, 0] * F[..., 2, 2]
    c[..., 0, 2] = F[..., 1, 0] * F[..., 2, 1] - F[..., 1, 1] * F[..., 2, 0]
    c[..., 1, 0] = F[..., 0, 2] * F[..., 2, 1] - F[..., 0, 1] * F[..., 2, 2]
    c[..., 1, 1] = F[..., 0, 0] * F[..., 2, 2] - F[..., 0, 2] * F[..., 2, 0]
    c[..., 1, 2] = F[..., 0, 1] * F[..., 2, 0] - F[..., 0, 0] * F[..., 2, 1]
    c[..., 2, 0] = F[..., 0, 1] * F[..., 1, 2] - F[..., 0, 2] * F[..., 1, 1]
    c[..., 2, 1] = F[..., 0, 2] * F[..., 1, 0] - F[..., 0, 0] * F[..., 1, 2]
    c[..., 2, 2] = F[..., 0, 0] * F[..., 1, 1] - F[..., 0, 1] * F[..., 1, 0]
    return c


def psi_neo_hookean(F, E, nu):
    """Strain energy (test_hyper_elasticity.py:17-27; scalability/hyperelastic3d_common.py:152-169)."""
    mu = E / (2.0 * (1.0 + nu))
    kappa = E / (3.0 * (1.0 - 2.0 * nu))
    J = _det3(F)
    I1 = np.einsum("...ij,...ij->...", F, F)
    return (mu / 2.0) * (J ** (-2.0 / 3.0) * I1 - 3.0) + (kappa / 2.0) * (J - 1.0) ** 2


def stress_neo_hookean(u_grad, E, nu, scale=None):
    """First Piola stress P = dpsi/dF, F = I + grad u (jax.grad of psi in the reference).

    ``scale`` multiplies psi (the density-scaled variant,
    scalability/hyperelastic3d_common.py:186-202).
    """
    mu = E / (2.0 * (1.0 + nu))
    kappa = E / (3.0 * (1.0 - 2.0 * nu))
    F = u_grad + _eye(u_grad.shape[:-2])
    J = _det3(F)
    H = _cof3(F) / J[..., None, None]  # F^{-T}
    I1 = np.einsum("...ij,...ij->...", F, F)
    m = mu * J ** (-2.0 / 3.0)
    P = m[..., None, None] * (F - (I1 / 3.0)[..., None, None] * H) \
        + (kappa * J * (J - 1.0))[..., None, None] * H
    if scale is not None:
        P = scale[..., None, None] * P
    return P


def safe_sqrt(x):
    return np.where(np.real(x) > 0.0, np.sqrt(np.where(np.real(x) > 0.0, x, 1.0)), 0.0)


def safe_divide(x, y):
    return np.where(np.real(y) == 0.0, 0.0, x / np.where(np.real(y) == 0.0, 1.0, y))


def j2_return_map(u_grad, sigma_old, eps_old, alpha_old, E, nu, sig0, H):
    """Small-strain J2 radial return (test_plasticity.py:42-64).

    The reference's map has no hardening; with linear isotropic hardening
    modulus H and equivalent plastic strain alpha the yield stress is
    sig0 + H*alpha_old and the plastic multiplier is f/(3 mu + H) (radial
    return, Simo & Hughes, Computational Inelasticity, Box 3.1).  With H=0
    this is exactly the reference's map.  Returns (sigma, alpha_new).
    """
    lmbda, mu = lame(E, nu)
    eps = 0.5 * (u_grad + np.swapaxes(u_grad, -1, -2))
    deps = eps - eps_old
    tr = np.trace(deps, axis1=-2, axis2=-1)
    sig_tr = lmbda * tr[..., None, None] * _eye(tr.shape) + 2 * mu * deps + sigma_old
    trs = np.trace(sig_tr, axis1=-2, axis2=-1)
    s = sig_tr - (trs / 3.0)[..., None, None] * _eye(trs.shape)
    q = safe_sqrt(1.5 * np.einsum("...ij,...ij->...", s, s))
    f = q - (sig0 + H * alpha_old)
    fp = np.where(np.real(f) > 0.0, f, 0.0)
    dgam = fp / (3.0 * mu + H)
    sigma = sig_tr - safe_divide((3.0 * mu * dgam)[..., None, None] * s, q[..., None, None])
    return sigma, alpha_old + dgam


class Law:
    """A tensor map P(u_grad, *ivars) over (..., vec, 3) arrays (problem.py:203-210)."""

    def __init__(self, kind, vec=3, **params):
        self.kind, self.vec, self.params = kind, vec, params

    def __call__(self, u_grad, ivars):
        p = self.params
        if self.kind == "laplace":
            return u_grad
        if self.kind == "linear":
            return stress_linear(u_grad, p["E"], p["nu"])
        if self.kind == "simp":
            return stress_simp(u_grad, ivars[0], p["E0"], p["Emin"], p["nu"], p["penal"])
        if self.kind == "neo_hookean":
            return stress_neo_hookean(u_grad, p["E"], p["nu"], ivars[0] if ivars else None)
        if self.kind == "j2":
            sig, _ = j2_return_map(u_grad, ivars[0], ivars[1], ivars[2],
                                   p["E"], p["nu"], p["sig0"], p["H"])
            return sig
        raise ValueError(self.kind)


# --------------------------------------------------------------------------
# Problem (problem.py) -- cell kernels, assembly, residual
# --------------------------------------------------------------------------

class OracleProblem:
    """Single-variable HEX8 problem mirroring ``Problem`` (problem.py:15-128).

    ``mass_map(u, x)`` and ``surface_maps[i](u, x)`` follow the reference's
    per-quad-point signatures (problem.py:216-259); ``law`` replaces the
    traced ``get_tensor_map`` callable.
    """

    def __init__(self, points, cells, vec, law, dirichlet_bc_info=None, location_fns=None,
                 mass_map=None, surface_maps=None, internal_vars=(), ele_type="HEX8", quadrature_order=None):
        self.points = np.asarray(points, dtype=np.float64)
        self.cells = np.asarray(cells, dtype=np.int64)
        self.vec, self.law = vec, law
        self.ele_type = ele_type
        self.num_cells, self.num_nodes = len(self.cells), len(self.points)
        self.ndofs = self.num_nodes * vec
        if ele_type == "HEX8" and quadrature_order in (None, 2):
            self.vals, self.grads_ref, self.weights = hex8_tables()
            (self.fvals, self.fgrads_ref, self.fweights, self.normals,
             self.face_inds) = hex8_face_tables()
        else:
            self.vals, self.grads_ref, self.weights = element_tables(ele_type, quadrature_order)
            (self.fvals, self.fgrads_ref, self.fweights, self.normals,
             self.face_inds) = element_face_tables(ele_type, quadrature_order)
        self.nen = self.vals.shape[1]
        self.num_quads = self.vals.shape[0]
        self.shape_grads, self.JxW = shape_grads(self.points, self.cells, self.grads_ref, self.weights)
        self.quad_points = physical_quad_points(self.points, self.cells, self.vals)
        self.bc_info = dirichlet_bc_info
        self.node_inds, self.vec_inds, self.bc_vals = dirichlet_bcs(self.points, dirichlet_bc_info)
        self.location_fns = location_fns
        self.boundary_inds = boundary_faces(self.points, self.cells, location_fns, self.face_inds)
        self.mass_map, self.surface_maps = mass_map, surface_maps or []
        self.internal_vars = list(internal_vars)
        # dof index table (problem.py:86-97)
        self.cell_dofs = (vec * self.cells[:, :, None] + np.arange(vec)[None, None, :]).reshape(
            self.num_cells, -1)

    def update_dirichlet(self, bc_info):
        """fe.py:260-269."""
        self.bc_info = bc_info
        self.node_inds, self.vec_inds, self.bc_vals = dirichlet_bcs(self.points, bc_info)

    def bc_rows(self):
        return np.concatenate([n * self.vec + v for n, v in zip(self.node_inds, self.vec_inds)]
                              ) if self.node_inds else np.zeros(0, dtype=np.int64)

    # -- kernels ---------------------------------------------------------
    def cell_residual(self, cell_u, ivars):
        """Laplace-kernel residual (problem.py:189-214) for all cells.

        cell_u (C,8,vec) -> (C,8,vec).
        """
        u_grad = np.einsum("cai,cqaj->cqij", cell_u, self.shape_grads)
        P = self.law(u_grad, ivars)
        return np.einsum("cqij,cqaj,cq->cai", P, self.shape_grads, self.JxW)

    def cell_residual_and_jacobian(self, cell_u, ivars, h=1e-30):
        """Residual (C,nen*vec) and Jacobian (C,nen*vec,nen*vec) via forward
        directional derivatives along each cell dof (problem.py:262-266,299-301)."""
        C, n = self.num_cells, self.nen * self.vec
        r = self.cell_residual(cell_u, ivars).reshape(C, n)
        jac = np.empty((C, n, n))
        base = cell_u.reshape(C, n).astype(np.complex128)
        civars = [np.asarray(v, dtype=np.complex128) for v in ivars]
        for d in range(n):
            up = base.copy()
            up[:, d] += 1j * h
            jac[:, :, d] = np.imag(self.cell_residual(up.reshape(C, self.nen, self.vec), civars).reshape(C, n)) / h
        return r, jac

    def body_load(self):
        """Mass-kernel vector (problem.py:216-236) for u-independent maps."""
        f = np.zeros((self.num_nodes, self.vec))
        if self.mass_map is None:
            return f.reshape(-1)
        x = self.quad_points.reshape(-1, 3)
        u0 = np.zeros((len(x), self.vec))
        val = eval_pointwise(self.mass_map, u0, x).reshape(self.num_cells, self.num_quads, self.vec)
        r = np.einsum("cqi,qa,cq->cai", val, self.vals, self.JxW)
        np.add.at(f, self.cells.reshape(-1), r.reshape(-1, self.vec))
        return f.reshape(-1)

    def surface_load(self):
        """Surface-kernel vector (problem.py:238-259, 398-424) for u-independent maps."""
        f = np.zeros((self.num_nodes, self.vec))
        for binds, smap in zip(self.boundary_inds, self.surface_maps):
            if len(binds) == 0:
                continue
            scale = face_geometry(self.points, self.cells, binds, self.fgrads_ref,
                                  self.fweights, self.normals)
            fv = self.fvals[binds[:, 1]]  # (F,q,8)
            xq = np.einsum("fqa,fai->fqi", fv, self.points[self.cells[binds[:, 0]]])
            u0 = np.zeros((xq.shape[0] * xq.shape[1], self.vec))
            val = eval_pointwise(smap, u0, xq.reshape(-1, 3)).reshape(xq.shape[0], xq.shape[1], self.vec)
            r = np.einsum("fqi,fqa,fq->fai", val, fv, scale)
            np.add.at(f, self.cells[binds[:, 0]].reshape(-1), r.reshape(-1, self.vec))
        return f.reshape(-1)

    def external_load(self):
        if not hasattr(self, "_fext"):
            self._fext = self.body_load() + self.surface_load()
        return self._fext

    def residual(self, dofs):
        """compute_residual (problem.py:426-445,462-475), flattened."""
        cell_u = dofs.reshape(self.num_nodes, self.vec)[self.cells]
        r = self.cell_residual(cell_u, self.internal_vars)
        R = np.zeros((self.num_nodes, self.vec))
        np.add.at(R, self.cells.reshape(-1), r.reshape(-1, self.vec))
        return R.reshape(-1) + self.external_load()

    def newton_update(self, dofs):
        """compute_newton_vars (problem.py:447-460): residual + COO values V."""
        cell_u = dofs.reshape(self.num_nodes, self.vec)[self.cells]
        r, jac = self.cell_residual_and_jacobian(cell_u, self.internal_vars)
        R = np.zeros(self.ndofs)
        np.add.at(R, self.cell_dofs.reshape(-1), r.reshape(-1))
        self.V = jac
        return R + self.external_load()

    def assemble_global(self, jac=None):
        """PETSc COO -> AIJ with duplicate summation (solver.py:466-491, problem.py:94-107)."""
        jac = self.V if jac is None else jac
        n = jac.shape[1]
        I = np.repeat(self.cell_dofs[:, :, None], n, axis=2).reshape(-1)
        J = np.repeat(self.cell_dofs[:, None, :], n, axis=1).reshape(-1)
        return sp.csr_matrix((jac.reshape(-1), (I, J)), shape=(self.ndofs, self.ndofs))

    def get_A(self):
        """Tangent with BC rows zeroed and unit diagonal, columns kept (solver.py:485-491)."""
        A = self.assemble_global()
        keep = np.ones(self.ndofs)
        rows = self.bc_rows()
        keep[rows] = 0.0
        unit = np.zeros(self.ndofs)
        unit[rows] = 1.0
        A = sp.diags(keep) @ A + sp.diags(unit)
        return A.tocsr()

    # -- BCs (solver.py:290-363) ------------------------------------------
    def apply_bc_vec(self, res, dofs, scale=1.0):
        res = res.copy()
        for n, v, val in zip(self.node_inds, self.vec_inds, self.bc_vals):
            rows = n * self.vec + v
            res[rows] = dofs[rows] - val * scale
        return res

    def assign_bc(self, dofs):
        dofs = dofs.copy()
        for n, v, val in zip(self.node_inds, self.vec_inds, self.bc_vals):
            dofs[n * self.vec + v] = val
        return dofs

    def copy_bc(self, dofs):
        out = np.zeros_like(dofs)
        rows = self.bc_rows()
        out[rows] = dofs[rows]
        return out


class KernelProblem:
    """Multi-variable problem with user kernels (problem.py:56-128, 130-190,
    189-340, 426-483): cell residual = laplace kernel of ``tensor_map`` on
    the first variable + mass kernel of ``mass_map`` + ``universal_kernel``;
    face residual = surface kernel of ``surface_maps[i]`` + universal surface
    kernel ``universal_surface[i]``.  Kernels are numpy functions with the
    reference's per-cell signatures (complex-step safe); a Python loop over
    cells stands in for jax.vmap.  Jacobians by complex step along each
    cell dof (the reference's forward JVPs), COO assembly with the variables'
    dof offsets, BC rows zeroed (solver.py:466-491).

    ``vars``: list of dicts with points, cells, vec, ele_type, order and
    dirichlet (a [location_fns, vecs, value_fns] triple or None)."""

    def __init__(self, vars, tensor_map=None, mass_map=None, universal_kernel=None, location_fns=None,
                 surface_maps=None, universal_surface=None, internal_vars=(), internal_vars_surfaces=()):
        self.vars = []
        off = 0
        for v in vars:
            ele, order = v.get("ele_type", "HEX8"), v.get("order")
            if ele == "HEX8" and order in (None, 2):
                vals, grads_ref, w = hex8_tables()
                fv, fg, fw, normals, finds = hex8_face_tables()
            else:
                vals, grads_ref, w = element_tables(ele, order)
                fv, fg, fw, normals, finds = element_face_tables(ele, order)
            pts = np.asarray(v["points"], dtype=np.float64)
            cells = np.asarray(v["cells"], dtype=np.int64)
            g, jxw = shape_grads(pts, cells, grads_ref, w)
            nodes, vecs, bvals = dirichlet_bcs(pts, v.get("dirichlet"))
            self.vars.append(dict(points=pts, cells=cells, vec=v["vec"], vals=vals, grads_ref=grads_ref, w=w,
                                  fvals=fv, fgrads=fg, fw=fw, normals=normals, face_inds=finds, g=g, jxw=jxw,
                                  off=off, nodes=nodes, vecs=vecs, bvals=bvals))
            off += len(pts) * v["vec"]
        self.ndofs = off
        v0 = self.vars[0]
        self.num_cells = len(v0["cells"])
        # (C, nd) global dofs of each cell (problem.py:86-97)
        self.cell_dofs = np.hstack([(v["vec"] * v["cells"][:, :, None] + np.arange(v["vec"])[None, None, :]
                                     + v["off"]).reshape(self.num_cells, -1) for v in self.vars])
        self.shape_grads = np.concatenate([v["g"] for v in self.vars], axis=2)          # (C,Q,sum nen,3)
        self.JxW = np.stack([v["jxw"] for v in self.vars], axis=1)                      # (C,V,Q)
        self.v_grads_JxW = np.concatenate([v["g"][:, :, :, None, :] * v["jxw"][:, :, None, None, None]
                                           for v in self.vars], axis=2)
        self.x = np.einsum("qa,cai->cqi", v0["vals"], v0["points"][v0["cells"]])
        self.tensor_map, self.mass_map, self.universal = tensor_map, mass_map, universal_kernel
        self.surface_maps, self.universal_surface = surface_maps, universal_surface
        self.internal_vars = list(internal_vars)
        self.internal_vars_surfaces = list(internal_vars_surfaces)
        self.boundary_inds = boundary_faces(v0["points"], v0["cells"], location_fns, v0["face_inds"])
        self.faces = []
        for binds in self.boundary_inds:
            fvals, fgrads, scales = [], [], []
            for v in self.vars:
                X = v["points"][v["cells"][binds[:, 0]]]
                gr = v["fgrads"][binds[:, 1]]
                Jf = np.einsum("fai,fqaj->fqij", X, gr)
                fgrads.append(np.einsum("fqaj,fqjk->fqak", gr, np.linalg.inv(Jf)))
                scales.append(face_geometry(v["points"], v["cells"], binds, v["fgrads"], v["fw"], v["normals"]))
                fvals.append(v["fvals"][binds[:, 1]])
            xs = np.einsum("fqa,fai->fqi", v0["fvals"][binds[:, 1]], v0["points"][v0["cells"][binds[:, 0]]])
            self.faces.append(dict(binds=binds, vals=np.concatenate(fvals, axis=2),
                                   grads=np.concatenate(fgrads, axis=2), nanson=np.stack(scales, axis=1), x=xs))

    def unflatten_fn_dof(self, flat):
        out, k = [], 0
        for v in self.vars:
            n = v["vals"].shape[1] * v["vec"]
            out.append(flat[k:k + n].reshape(-1, v["vec"]))
            k += n
        return out

    def _first(self, val, nd):
        out = np.zeros(nd, dtype=val.dtype)
        out[: val.size] = val.reshape(-1)
        return out

    def cell_kernel(self, c, sol, ivars):
        """problem.py:278-300 for cell c."""
        v0 = self.vars[0]
        n0 = v0["vals"].shape[1]
        nd = sol.size
        val = np.zeros(nd, dtype=sol.dtype)
        u = sol[: n0 * v0["vec"]].reshape(n0, v0["vec"])
        iv = [np.asarray(a)[c] for a in ivars]
        if self.tensor_map is not None:  # laplace kernel, problem.py:189-214
            ug = np.einsum("ai,qaj->qij", u, self.shape_grads[c][:, :n0, :])
            P = np.array([self.tensor_map(ug[q], *[a[q] for a in iv]) for q in range(ug.shape[0])])
            val = val + self._first(np.einsum("qij,qaj->ai", P, self.v_grads_JxW[c][:, :n0, 0, :]), nd)
        if self.mass_map is not None:  # mass kernel, problem.py:216-236
            uq = np.einsum("ai,qa->qi", u, v0["vals"])
            m = np.array([self.mass_map(uq[q], self.x[c][q], *[a[q] for a in iv]) for q in range(uq.shape[0])])
            val = val + self._first(np.einsum("qi,qa,q->ai", m, v0["vals"], self.JxW[c][0]), nd)
        if self.universal is not None:
            val = val + self.universal(sol, self.x[c], self.shape_grads[c], self.JxW[c], self.v_grads_JxW[c], *iv)
        return val

    def face_kernel(self, i, f, sol, ivars):
        """problem.py:305-332 for face f of surface i."""
        face = self.faces[i]
        v0 = self.vars[0]
        n0 = v0["vals"].shape[1]
        nd = sol.size
        val = np.zeros(nd, dtype=sol.dtype)
        iv = [np.asarray(a)[f] for a in ivars]
        fsv = face["vals"][f]
        if self.surface_maps is not None:  # surface kernel, problem.py:238-259
            u = sol[: n0 * v0["vec"]].reshape(n0, v0["vec"])
            uq = np.einsum("ai,qa->qi", u, fsv[:, :n0])
            t = np.array([self.surface_maps[i](uq[q], face["x"][f][q], *[a[q] for a in iv])
                          for q in range(uq.shape[0])])
            val = val + self._first(np.einsum("qi,qa,q->ai", t, fsv[:, :n0], face["nanson"][f][0]), nd)
        if self.universal_surface is not None:
            val = val + self.universal_surface[i](sol, face["x"][f], fsv, face["grads"][f], face["nanson"][f], *iv)
        return val

    def _items(self):
        """(global dofs, kernel(sol) -> residual) of every cell and selected face."""
        out = []
        for c in range(self.num_cells):
            out.append((self.cell_dofs[c], lambda s, c=c: self.cell_kernel(c, s, self.internal_vars)))
        for i, face in enumerate(self.faces):
            ivs = self.internal_vars_surfaces[i] if i < len(self.internal_vars_surfaces) else ()
            for f, (c, _) in enumerate(face["binds"]):
                out.append((self.cell_dofs[c], lambda s, i=i, f=f, ivs=ivs: self.face_kernel(i, f, s, ivs)))
        return out

    def residual(self, dofs):
        R = np.zeros(self.ndofs)
        for idx, k in self._items():
            np.add.at(R, idx, k(dofs[idx]))
        return R

    def residual_and_tangent(self, dofs, h=1e-30):
        R = np.zeros(self.ndofs)
        I, J, V = [], [], []
        for idx, k in self._items():
            base = dofs[idx].astype(np.complex128)
            np.add.at(R, idx, k(dofs[idx]))
            nd = len(idx)
            jac = np.empty((nd, nd))
            for d in range(nd):
                up = base.copy()
                up[d] += 1j * h
                jac[:, d] = np.imag(k(up)) / h
            I.append(np.repeat(idx, nd))
            J.append(np.tile(idx, nd))
            V.append(jac.reshape(-1))
        K = sp.csr_matrix((np.concatenate(V), (np.concatenate(I), np.concatenate(J))), shape=(self.ndofs,) * 2)
        return R, K

    def bc_rows(self):
        rows, vals = [], []
        for v in self.vars:
            for n, vi, bv in zip(v["nodes"], v["vecs"], v["bvals"]):
                rows.append(v["off"] + n * v["vec"] + vi)
                vals.append(bv)
        if not rows:
            return np.zeros(0, dtype=np.int64), np.zeros(0)
        return np.concatenate(rows), np.concatenate(vals)

    def newton(self, rel_tol=1e-10, tol=1e-12, max_iter=30):
        """The Newton loop of solver.py:1232-1318 with spsolve and zeroRows."""
        rows, bvals = self.bc_rows()
        dofs = np.zeros(self.ndofs)

        def system(d):
            R, K = self.residual_and_tangent(d)
            R[rows] = d[rows] - bvals
            keep = np.ones(self.ndofs)
            keep[rows] = 0.0
            unit = 1.0 - keep
            return R, (sp.diags(keep) @ K + sp.diags(unit)).tocsc()

        R, K = system(dofs)
        r0 = np.linalg.norm(R)
        it = 0
        while np.linalg.norm(R) > tol and np.linalg.norm(R) / r0 > rel_tol and it < max_iter:
            dofs = dofs + spla.spsolve(K, -R)
            R, K = system(dofs)
            it += 1
        return dofs


def newton_solve(problem, initial_guess=None, rel_tol=1e-8, tol=1e-6, linear="spsolve",
                 max_iter=50, return_info=False):
    """Newton loop of ``solver`` (solver.py:1232-1318) with the step of
    ``newton_step`` (solver.py:390-421).  ``linear='spsolve'`` is the
    reference's ``spsolve_solver`` (solver.py:94-107)."""
    dofs = np.zeros(problem.ndofs) if initial_guess is None else np.asarray(initial_guess, dtype=np.float64).reshape(-1).copy()

    def update(d):
        res = problem.newton_update(d)
        res = problem.apply_bc_vec(res, d)
        return res, problem.get_A()

    res, A = update(dofs)
    r0 = np.linalg.norm(res)
    rel = 1.0 if r0 > 0 else 0.0
    hist = [r0]
    it = 0
    while rel > rel_tol and np.linalg.norm(res) > tol and it < max_iter:
        it += 1
        b = -res
        x0 = problem.assign_bc(np.zeros(problem.ndofs)) - problem.copy_bc(dofs)
        if linear == "spsolve":
            inc = spla.spsolve(A.tocsc(), b)
        else:
            inc, _ = spla.bicgstab(A, b, x0=x0, rtol=1e-12, atol=1e-14, maxiter=20000)
        dofs = dofs + inc
        res, A = update(dofs)
        hist.append(np.linalg.norm(res))
        rel = hist[-1] / r0
    assert np.all(np.isfinite(dofs))
    if return_info:
        return dofs, dict(iters=it, res_hist=hist)
    return dofs


def arc_length_disp(problem, Delta_l=0.1, psi=1.0, max_steps=600, tol=1e-6):
    """Displacement-controlled arc-length continuation (solver.py:521-597,
    721-756): Dirichlet values scaled by lambda, Crisfield's spherical
    constraint, direct solves; then a Newton solve at full load
    (solver.py:686-718).  Returns (u, [lambda after each step])."""
    u = np.zeros(problem.ndofs)
    lam, du_dir, dl_dir = 0.0, np.zeros_like(u), 0.0
    u_b = problem.assign_bc(np.zeros_like(u))
    ub2 = float(np.sum(u_b ** 2))
    lams = []
    for _ in range(max_steps):
        u_prev, l_prev = u.copy(), lam
        res_val = 1.0
        while res_val > tol:
            R = problem.newton_update(u)
            res = problem.apply_bc_vec(R, u, lam)
            A = problem.get_A().tocsc()
            res_val = np.linalg.norm(res)
            du_bar = spla.spsolve(A, -res)
            du_t = spla.spsolve(A, u_b)
            w = u - u_prev + du_bar
            Dl = lam - l_prev
            a1 = np.sum(du_t ** 2) + psi ** 2 * ub2
            a2 = 2.0 * np.sum(w * du_t) + 2.0 * psi ** 2 * Dl * ub2
            a3 = np.sum(w ** 2) + psi ** 2 * Dl ** 2 * ub2 - Delta_l ** 2
            disc = np.sqrt(a2 ** 2 - 4.0 * a1 * a3)
            roots = ((-a2 + disc) / (2.0 * a1), (-a2 - disc) / (2.0 * a1))
            dots = [np.sum(du_dir * (w + dl * du_t)) + psi ** 2 * dl_dir * (Dl + dl) * ub2 for dl in roots]
            if abs(dots[0]) < 1e-10 and abs(dots[1]) < 1e-10:
                dl = max(roots)
            else:
                dl = roots[0] if dots[0] > dots[1] else roots[1]
            lam += dl
            u = u + du_bar + dl * du_t
            du_dir, dl_dir = u - u_prev, lam - l_prev
        lams.append(lam)
        if lam >= 1.0:
            break
    if lams[-1] >= 1.0:
        u = newton_solve(problem, initial_guess=u, rel_tol=1e-12, tol=1e-14)
    return u, lams


def arc_length_force(problem, q_aux, Delta_l=0.1, psi=0.5, Delta_l_late=1.0, switch_step=200, max_steps=500,
                     tol=1e-6):
    """Force-controlled arc-length continuation (solver.py:607-685, 758-801):
    residual R(u) + (1 - lambda) q with q = q_aux zeroed on Dirichlet rows,
    direct solves; then a Newton solve at full load.  Returns (u, lambdas)."""
    u = np.zeros(problem.ndofs)
    lam, du_dir, dl_dir = 0.0, np.zeros_like(u), 0.0
    q = np.asarray(q_aux, dtype=np.float64).reshape(-1).copy()
    q[problem.bc_rows()] = 0.0
    q2 = float(np.sum(q ** 2))
    lams = []
    for step in range(max_steps):
        dl_len = Delta_l if step < switch_step else Delta_l_late
        u_prev, l_prev = u.copy(), lam
        res_val = 1.0
        while res_val > tol:
            R = problem.newton_update(u)
            res = problem.apply_bc_vec(R, u) + (1.0 - lam) * q
            A = problem.get_A().tocsc()
            res_val = np.linalg.norm(res)
            du_bar = spla.spsolve(A, -res)
            du_t = spla.spsolve(A, q)
            w = u - u_prev + du_bar
            Dl = lam - l_prev
            a1 = np.sum(du_t ** 2) + psi ** 2 * q2
            a2 = 2.0 * np.sum(w * du_t) + 2.0 * psi ** 2 * Dl * q2
            a3 = np.sum(w ** 2) + psi ** 2 * Dl ** 2 * q2 - dl_len ** 2
            disc = np.sqrt(a2 ** 2 - 4.0 * a1 * a3)
            roots = ((-a2 + disc) / (2.0 * a1), (-a2 - disc) / (2.0 * a1))
            dots = [np.sum(du_dir * (w + dl * du_t)) + psi ** 2 * dl_dir * (Dl + dl) * q2 for dl in roots]
            if abs(dots[0]) < 1e-10 and abs(dots[1]) < 1e-10:
                dl = max(roots)
            else:
                dl = roots[0] if dots[0] > dots[1] else roots[1]
            lam += dl
            u = u + du_bar + dl * du_t
            du_dir, dl_dir = u - u_prev, lam - l_prev
        lams.append(lam)
        if lam >= 1.0:
            break
    if lams[-1] >= 1.0:
        u = newton_solve(problem, initial_guess=u, rel_tol=1e-12, tol=1e-14)
    return u, lams


def dynamic_relax(problem, tol=1e-6, nKMat=1000, initial_guess=None, max_iters=1000000):  # noqa: N803
    """Dynamic relaxation (solver.py:837-1047): one direct Newton step from
    u = 0 (or the initial guess with its Dirichlet values), then the damped
    pseudo-dynamic march until max |R| <= tol.  Returns (u, iterations)."""
    dofs = np.zeros(problem.ndofs)
    res = problem.apply_bc_vec(problem.newton_update(dofs), dofs)
    dofs = dofs + spla.spsolve(problem.get_A().tocsc(), -res)
    if initial_guess is not None:
        dofs = problem.assign_bc(np.asarray(initial_guess, dtype=np.float64).reshape(-1))
    rows = problem.bc_rows()
    cmin, cmax, h_tilde, h = 1e-3, 3.9, 1.1, 1.0

    def residual(d):
        r = problem.residual(d)
        r[rows] = 0.0
        return r

    def mass(d):
        problem.newton_update(d)
        return h_tilde ** 2 / 4.0 * np.asarray(abs(problem.get_A()).sum(axis=1)).reshape(-1)

    R = residual(dofs)
    M = mass(dofs)
    q = dofs.copy()
    qdot = -h / 2.0 * R / M
    qdotdot, qdotdot_old = np.zeros_like(q), np.zeros_like(q)
    n_iters, i_kmat = 0, 0
    error = np.max(np.abs(R))
    while error > tol and n_iters < max_iters:
        q_old, R_old = q.copy(), R.copy()
        q = q + h * qdot
        R = residual(q)
        n_iters += 1
        i_kmat += 1
        error = np.max(np.abs(R))
        t = np.dot((R - R_old) / h, qdot) / np.sum(qdot * M * qdot)
        c = min(max(2.0 * np.sqrt(max(t, 0.0)), cmin), cmax)
        dq = q - q_old
        eps = h_tilde ** 2 / 4.0 * np.abs(np.divide(qdotdot - qdotdot_old, dq, out=np.zeros_like(dq), where=dq != 0))
        if np.max(eps) > 1 and i_kmat > nKMat:
            i_kmat = 0
            M = mass(q)
        qdot_old, qdotdot_old = qdot.copy(), qdotdot.copy()
        qdot = (2.0 - c * h) / (2.0 + c * h) * qdot_old - 2.0 * h / (2.0 + c * h) * R / M
        qdotdot = (qdot - qdot_old) / h
    return q, n_iters


# --------------------------------------------------------------------------
# Plasticity state commit (test_plasticity.py:67-78, fe.py:366-382)
# --------------------------------------------------------------------------

def sol_to_grad(problem, dofs):
    cell_u = dofs.reshape(problem.num_nodes, problem.vec)[problem.cells]
    return np.einsum("cai,cqaj->cqij", cell_u, problem.shape_grads)


def j2_commit(problem, dofs):
    p = problem.law.params
    sig_old, eps_old, alpha_old = problem.internal_vars
    ug = sol_to_grad(problem, dofs)
    sig, alpha = j2_return_map(ug, sig_old, eps_old, alpha_old, p["E"], p["nu"], p["sig0"], p["H"])
    eps = 0.5 * (ug + np.swapaxes(ug, -1, -2))
    problem.internal_vars = [sig, eps, alpha]


def avg_stress(problem):
    sig = problem.internal_vars[0]
    return np.einsum("cqij,cq->ij", sig, problem.JxW) / problem.JxW.sum()


# --------------------------------------------------------------------------
# Adjoint (solver.py:1324-1380)
# --------------------------------------------------------------------------

def implicit_vjp_cellwise(problem, dofs, v, h=1e-30):
    """-(dc/dtheta)^T lambda for a per-cell scalar internal variable theta
    stored per quad in ``internal_vars[0]`` (shape (C,Q)).

    A^T lambda = v with the BC-row-zeroed tangent at the solution
    (solver.py:1358-1371); the parameter VJP is taken through the residual
    with BC rows replaced (BC rows do not depend on theta).  Each cell's
    residual depends only on its own theta, so one complex-step evaluation
    with every theta perturbed gives all per-cell partials at once.
    Returns dJ/dtheta per (cell, quad).
    """
    problem.newton_update(dofs)
    A = problem.get_A()
    lam = spla.spsolve(A.T.tocsc(), v)
    lam[problem.bc_rows()] = 0.0  # BC rows of dc/dtheta vanish
    cell_u = dofs.reshape(problem.num_nodes, problem.vec)[problem.cells]
    cell_lam = lam.reshape(problem.num_nodes, problem.vec)[problem.cells]
    theta = np.asarray(problem.internal_vars[0], dtype=np.float64)
    Q = theta.shape[1]
    grads = np.zeros_like(theta)
    others = [np.asarray(x, dtype=np.complex128) for x in problem.internal_vars[1:]]
    for q in range(Q):
        tp = theta.astype(np.complex128)
        tp[:, q] += 1j * h
        dr = np.imag(problem.cell_residual(cell_u.astype(np.complex128), [tp] + others)) / h
        grads[:, q] = -np.einsum("cai,cai->c", dr, cell_lam)
    return grads


def compliance(problem, dofs, surface_index=0):
    """C = int t . u ds with t = -surface_map (topology_optimization cell 9)."""
    binds = problem.boundary_inds[surface_index]
    smap = problem.surface_maps[surface_index]
    scale = face_geometry(problem.points, problem.cells, binds, problem.fgrads_ref,
                          problem.fweights, problem.normals)
    fv = problem.fvals[binds[:, 1]]
    cu = dofs.reshape(problem.num_nodes, problem.vec)[problem.cells[binds[:, 0]]]
    uq = np.einsum("fqa,fai->fqi", fv, cu)
    xq = np.einsum("fqa,fai->fqi", fv, problem.points[problem.cells[binds[:, 0]]])
    t = -eval_pointwise(smap, uq.reshape(-1, problem.vec), xq.reshape(-1, 3)).reshape(uq.shape)
    return float(np.sum(t * uq * scale[:, :, None]))


def surface_integral(problem, location_fn, surface_fn, dofs):
    """Post-processing face integral of f(u_grad) used by the reference tests
    (test_hyper_elasticity.py:36-45, test_linear_elasticity_cylinder.py:40-66)."""
    binds = boundary_faces(problem.points, problem.cells.astype(np.int64), [location_fn], problem.face_inds)[0]
    X = problem.points[problem.cells[binds[:, 0]]]
    gr = problem.fgrads_ref[binds[:, 1]]
    J = np.einsum("fai,fqaj->fqij", X, gr)
    Jinv = np.linalg.inv(J)
    g = np.einsum("fqaj,fqjk->fqak", gr, Jinv)
    scale = face_geometry(problem.points, problem.cells, binds, problem.fgrads_ref,
                          problem.fweights, problem.normals)
    cu = dofs.reshape(problem.num_nodes, problem.vec)[problem.cells[binds[:, 0]]]
    ug = np.einsum("fai,fqaj->fqij", cu, g)
    val = surface_fn(ug)
    return np.sum(val * scale[:, :, None], axis=(0, 1))
