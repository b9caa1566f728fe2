"""Element tabulation: shape functions, quadrature and face tables of the
element types of the reference's basis.py:19-114 (HEX8, HEX20, HEX27, TET4,
TET10 and the 2D QUAD4, QUAD8, TRI3, TRI6), in mesh (VTK/meshio) node order.

The reference tabulates with basix 0.10 (``get_shape_vals_and_grads``,
basis.py:141-175; ``get_face_shape_vals_and_grads``, basis.py:178-250) and
permutes basix's dof order into the mesh's with ``re_order``.  Here each
element is written directly in mesh order from its definition:

- HEX8, HEX27, QUAD4: tensor-product Lagrange of degree 1 and 2 on
  [0,1]^d (basix P on the hexahedron / quadrilateral; at degree <= 2 every
  Lagrange variant puts the nodes at vertices, edge midpoints, face centres
  and the centre);
- TET4, TET10, TRI3, TRI6: Lagrange P1 / P2 on the unit simplex, written
  in barycentric coordinates (corner L(2L-1), edge 4 L_i L_j);
- HEX20, QUAD8: basix's serendipity element of degree 2, whose degrees of
  freedom are the vertex values and the edge means (moments against the
  constant on each unit edge), not midpoint values.  Its basis is the dual
  basis of those functionals in the serendipity space (superlinear degree
  <= 2: 20 monomials on the cube, 8 on the square), computed once by
  solving a 20x20 / 8x8 system.

Quadrature follows basix's default rule (basis.py:117-124): Gauss-Jacobi
(Gauss-Legendre on [0,1]) with (order+2)//2 points per axis on hexahedra
and quadrilaterals; on tetrahedra and triangles the Xiao-Gimbutas rules,
of which the orders the element types use by default are restated here:
order 0 and 1 the centroid, order 2 the symmetric 4-point (tetrahedron)
and 3-point (triangle) rules.  Faces of 2D cells are edges, integrated with
the Gauss-Legendre rule of the same order.
"""
import functools

import numpy as np

# meshio cell type of each element (generate_mesh.py:83-117)
MESHIO_CELL_TYPE = {"HEX8": "hexahedron", "HEX20": "hexahedron20", "HEX27": "hexahedron27",
                    "TET4": "tetra", "TET10": "tetra10", "QUAD4": "quad", "QUAD8": "quad8",
                    "TRI3": "triangle", "TRI6": "triangle6"}
# default quadrature order (basis.py:52-107)
DEFAULT_ORDER = {"HEX8": 2, "HEX20": 2, "HEX27": 10, "TET4": 0, "TET10": 2,
                 "QUAD4": 2, "QUAD8": 2, "TRI3": 0, "TRI6": 2}
NODES_PER_CELL = {"HEX8": 8, "HEX20": 20, "HEX27": 27, "TET4": 4, "TET10": 10,
                  "QUAD4": 4, "QUAD8": 8, "TRI3": 3, "TRI6": 6}
# spatial dimension of each element type
ELEMENT_DIM = {e: (2 if e[:3] in ("QUA", "TRI") else 3) for e in NODES_PER_CELL}

# ---- reference cells ----------------------------------------------------------
# VTK hexahedron corners on [0,1]^3
_HEX_CORNERS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                         [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.float64)
# VTK quadratic-hexahedron edges (nodes 8..19) as corner pairs
HEX_EDGES = np.array([[0, 1], [1, 2], [2, 3], [3, 0], [4, 5], [5, 6], [6, 7], [7, 4],
                      [0, 4], [1, 5], [2, 6], [3, 7]])
# VTK triquadratic-hexahedron face centres (nodes 20..25): -x, +x, -y, +y, -z, +z
HEX_FACE_CORNERS = np.array([[0, 3, 7, 4], [1, 2, 6, 5], [0, 1, 5, 4], [3, 2, 6, 7],
                             [0, 1, 2, 3], [4, 5, 6, 7]])
_TET_CORNERS = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.float64)
# VTK quadratic-tetrahedron edges (nodes 4..9)
TET_EDGES = np.array([[0, 1], [1, 2], [0, 2], [0, 3], [1, 3], [2, 3]])

# Element faces in basix's facet order with their basix vertex lists mapped
# to mesh corner numbers, and the reference outward normals
# (basix.cell.sub_entity_connectivity / facet_outward_normals).
_HEX_FACETS_BASIX = np.array([[0, 1, 2, 3], [0, 1, 4, 5], [0, 2, 4, 6],
                              [1, 3, 5, 7], [2, 3, 6, 7], [4, 5, 6, 7]])
_HEX8_REORDER = np.array([0, 1, 3, 2, 4, 5, 7, 6])  # basis.py:53, its own inverse
HEX_FACE_INDS = _HEX8_REORDER[_HEX_FACETS_BASIX]
HEX_FACE_NORMALS = np.array([[0, 0, -1], [0, -1, 0], [-1, 0, 0],
                             [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.float64)
TET_FACE_INDS = np.array([[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]])
TET_FACE_NORMALS = np.array([[1, 1, 1], [-1, 0, 0], [0, -1, 0], [0, 0, -1]], dtype=np.float64)
TET_FACE_NORMALS[0] /= np.sqrt(3.0)

# 2D cells.  VTK quadrilateral corners on [0,1]^2 and its quadratic edges
# (nodes 4..7); VTK triangle corners and its quadratic edges (nodes 3..5).
_QUAD_CORNERS = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], dtype=np.float64)
QUAD_EDGES = np.array([[0, 1], [1, 2], [2, 3], [3, 0]])
_TRI_CORNERS = np.array([[0, 0], [1, 0], [0, 1]], dtype=np.float64)
TRI_EDGES = np.array([[0, 1], [1, 2], [2, 0]])
# Faces (edges) in basix's facet order as mesh corner numbers, and normals:
# basix's quadrilateral facets [0,1], [0,2], [1,3], [2,3] under QUAD4's
# re_order [0,1,3,2]; the triangle's [1,2], [0,2], [0,1].
QUAD_FACE_INDS = np.array([[0, 1], [0, 3], [1, 2], [3, 2]])
QUAD_FACE_NORMALS = np.array([[0, -1], [-1, 0], [1, 0], [0, 1]], dtype=np.float64)
TRI_FACE_INDS = np.array([[1, 2], [0, 2], [0, 1]])
TRI_FACE_NORMALS = np.array([[1, 1], [-1, 0], [0, -1]], dtype=np.float64)
TRI_FACE_NORMALS[0] /= np.sqrt(2.0)


def check_ele_type(ele_type):
    if ele_type not in NODES_PER_CELL:
        raise NotImplementedError(
            f"element {ele_type!r}: the types {', '.join(NODES_PER_CELL)} are supported")
    return ele_type


def node_coords(ele_type):
    """Reference coordinates (nen, dim) of the nodes in mesh order."""
    check_ele_type(ele_type)
    if ELEMENT_DIM[ele_type] == 2:
        X, E = (_TRI_CORNERS, TRI_EDGES) if ele_type.startswith("TRI") else (_QUAD_CORNERS, QUAD_EDGES)
        if ele_type in ("QUAD8", "TRI6"):
            X = np.vstack([X, 0.5 * (X[E[:, 0]] + X[E[:, 1]])])
        return X.copy()
    if ele_type.startswith("TET"):
        X = _TET_CORNERS
        if ele_type == "TET10":
            X = np.vstack([X, 0.5 * (X[TET_EDGES[:, 0]] + X[TET_EDGES[:, 1]])])
        return X.copy()
    X = _HEX_CORNERS
    if ele_type in ("HEX20", "HEX27"):
        X = np.vstack([X, 0.5 * (X[HEX_EDGES[:, 0]] + X[HEX_EDGES[:, 1]])])
    if ele_type == "HEX27":
        X = np.vstack([X, _HEX_CORNERS[HEX_FACE_CORNERS].mean(axis=1), [[0.5, 0.5, 0.5]]])
    return X.copy()


# ---- shape functions ----------------------------------------------------------------
def _lagrange1d(nodes, t):
    """Values and derivatives (n, len(nodes)) of the 1D Lagrange basis on nodes."""
    t = np.asarray(t, dtype=np.float64)[:, None]
    k = len(nodes)
    vals = np.ones((t.shape[0], k))
    ders = np.zeros((t.shape[0], k))
    for i, xi in enumerate(nodes):
        others = [xj for j, xj in enumerate(nodes) if j != i]
        den = np.prod([xi - xj for xj in others])
        vals[:, i] = np.prod([t[:, 0] - xj for xj in others], axis=0) / den
        ders[:, i] = sum(np.prod([t[:, 0] - xm for m, xm in enumerate(others) if m != l], axis=0)
                         for l in range(len(others))) / den
    return vals, ders


def _tensor_lagrange(X, xi, nodes1d):
    """Tensor-product Lagrange basis at points xi (n,d) with node coordinates X (nen,d)."""
    idx = np.rint(X * (len(nodes1d) - 1)).astype(int)  # index of each coordinate in nodes1d
    d = X.shape[1]
    v, dv = [], []
    for ax in range(d):
        va, da = _lagrange1d(nodes1d, xi[:, ax])
        v.append(va[:, idx[:, ax]])
        dv.append(da[:, idx[:, ax]])
    vals = np.prod(v, axis=0)
    grads = np.stack([np.prod([dv[b] if b == ax else v[b] for b in range(d)], axis=0) for ax in range(d)],
                     axis=2)
    return vals, grads


def _simplex_shape(ele_type, xi):
    """P1 / P2 on the unit simplex from barycentric coordinates L."""
    d = xi.shape[1]
    L = np.concatenate([1.0 - xi.sum(axis=1, keepdims=True), xi], axis=1)  # (n, d+1)
    dL = np.vstack([-np.ones((1, d)), np.eye(d)])  # (d+1, d)
    if ele_type in ("TET4", "TRI3"):
        return L, np.broadcast_to(dL, (len(xi), d + 1, d)).copy()
    edges = TET_EDGES if d == 3 else TRI_EDGES
    nen = d + 1 + len(edges)
    vals = np.empty((len(xi), nen))
    grads = np.empty((len(xi), nen, d))
    for a in range(d + 1):
        vals[:, a] = L[:, a] * (2.0 * L[:, a] - 1.0)
        grads[:, a] = (4.0 * L[:, a] - 1.0)[:, None] * dL[a]
    for e, (i, j) in enumerate(edges):
        vals[:, d + 1 + e] = 4.0 * L[:, i] * L[:, j]
        grads[:, d + 1 + e] = 4.0 * (L[:, j][:, None] * dL[i] + L[:, i][:, None] * dL[j])
    return vals, grads


# Serendipity spaces of degree 2 (superlinear degree <= 2).  Cube: P2 plus
# xyz, the six x_i^2 x_j and the three x_i^2 x_j x_k; square: P2 plus x^2 y
# and x y^2 (exponent tuples).
_SERENDIPITY_EXPONENTS = {3: np.array(
    [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [2, 0, 0], [0, 2, 0], [0, 0, 2], [1, 1, 0], [0, 1, 1],
     [1, 0, 1], [1, 1, 1], [2, 1, 0], [2, 0, 1], [1, 2, 0], [0, 2, 1], [1, 0, 2], [0, 1, 2], [2, 1, 1],
     [1, 2, 1], [1, 1, 2]]),
    2: np.array([[0, 0], [1, 0], [0, 1], [2, 0], [1, 1], [0, 2], [2, 1], [1, 2]])}


def _monomials(xi, E):
    """Values (n, m) and gradients (n, m, d) of monomials x^E (E: (m, d))."""
    xi = np.asarray(xi, dtype=np.float64)
    d = E.shape[1]
    pw = [xi[:, a:a + 1] ** E[:, a] for a in range(d)]
    vals = np.prod(pw, axis=0)
    grads = np.empty(vals.shape + (d,))
    for ax in range(d):
        e = E[:, ax]
        dax = np.where(e > 0, e * xi[:, ax:ax + 1] ** np.maximum(e - 1, 0), 0.0)
        grads[:, :, ax] = dax * np.prod([pw[b] for b in range(d) if b != ax], axis=0)
    return vals, grads


@functools.lru_cache(maxsize=None)
def _serendipity_coefficients(d):
    """Coefficients C (monomials x nodes) of the dual basis of basix's
    degree-2 serendipity dofs on [0,1]^d: phi_k = sum_m C[m, k]
    (x - 1/2)^E_m with l_j(phi_k) = delta_jk, l_j = value at corner j or
    mean over an edge (VTK corner and edge order)."""
    E = _SERENDIPITY_EXPONENTS[d]
    corners, edges = (_HEX_CORNERS, HEX_EDGES) if d == 3 else (_QUAD_CORNERS, QUAD_EDGES)
    t, w = gauss_legendre_01(3)  # exact for the cubic restrictions to an edge
    n = len(E)
    Lmat = np.empty((n, n))
    nc = len(corners)
    Lmat[:nc] = _monomials(corners - 0.5, E)[0]
    for e, (i, j) in enumerate(edges):
        pts = corners[i][None] + t[:, None] * (corners[j] - corners[i])[None]
        Lmat[nc + e] = w @ _monomials(pts - 0.5, E)[0]
    return np.linalg.solve(Lmat, np.eye(n))


def shape_fn(ele_type, xi):
    """Shape values (n, nen) and reference gradients (n, nen, dim) at points xi (n, dim)."""
    check_ele_type(ele_type)
    xi = np.atleast_2d(np.asarray(xi, dtype=np.float64))
    if xi.shape[1] != ELEMENT_DIM[ele_type]:
        raise ValueError(f"{ele_type} points have {ELEMENT_DIM[ele_type]} coordinates, got {xi.shape[1]}")
    if ele_type[:3] in ("TET", "TRI"):
        return _simplex_shape(ele_type, xi)
    if ele_type in ("HEX8", "QUAD4"):
        return _tensor_lagrange(node_coords(ele_type), xi, [0.0, 1.0])
    if ele_type == "HEX27":
        return _tensor_lagrange(node_coords("HEX27"), xi, [0.0, 0.5, 1.0])
    d = ELEMENT_DIM[ele_type]
    C = _serendipity_coefficients(d)
    mv, mg = _monomials(xi - 0.5, _SERENDIPITY_EXPONENTS[d])  # centred monomials (the space is shift-invariant)
    return mv @ C, np.einsum("nmd,mk->nkd", mg, C)


# ---- quadrature ---------------------------------------------------------------
def gauss_legendre_01(m):
    """m-point Gauss-Legendre rule on [0, 1] (basix Gauss-Jacobi with alpha = 0)."""
    x, w = np.polynomial.legendre.leggauss(m)
    return 0.5 + 0.5 * x, 0.5 * w


_TET4PT = (5.0 - np.sqrt(5.0)) / 20.0


def _simplex_rule(dim, order):
    """Xiao-Gimbutas rules of orders 0-2 on the unit triangle / tetrahedron."""
    if order < 0 or order > 2:
        raise NotImplementedError(
            f"quadrature order {order} on a simplex: orders 0-2 (the element defaults) are supported")
    if dim == 3:
        if order <= 1:
            return np.full((1, 3), 0.25), np.array([1.0 / 6.0])
        a, b = _TET4PT, 1.0 - 3.0 * _TET4PT
        pts = np.array([[a, a, a], [b, a, a], [a, b, a], [a, a, b]])
        return pts, np.full(4, 1.0 / 24.0)
    if order <= 1:
        return np.full((1, 2), 1.0 / 3.0), np.array([0.5])
    pts = np.array([[1.0 / 6.0, 1.0 / 6.0], [2.0 / 3.0, 1.0 / 6.0], [1.0 / 6.0, 2.0 / 3.0]])
    return pts, np.full(3, 1.0 / 6.0)


def _tensor_rule(dim, order):
    p, w = gauss_legendre_01((order + 2) // 2)
    grids = np.meshgrid(*([p] * dim), indexing="ij")  # first axis slowest
    wgrid = np.meshgrid(*([w] * dim), indexing="ij")
    pts = np.stack([g.reshape(-1) for g in grids], axis=1)
    return pts, np.prod(np.stack([g.reshape(-1) for g in wgrid], axis=1), axis=1)


def volume_quadrature(ele_type, order=None):
    """Quadrature points (nq, dim) and weights (nq,) of the element's cell."""
    order = DEFAULT_ORDER[check_ele_type(ele_type)] if order is None else int(order)
    d = ELEMENT_DIM[ele_type]
    return _simplex_rule(d, order) if ele_type[:3] in ("TET", "TRI") else _tensor_rule(d, order)


def face_rule(ele_type, order=None):
    """Per-face quadrature (basis.py:178-250): face_inds (nf, nfv) corner
    numbers, points (nf, nfq, dim) in reference coordinates, weights
    (nf, nfq) times the facet's reference area (edge length in 2D),
    normals (nf, dim)."""
    order = DEFAULT_ORDER[check_ele_type(ele_type)] if order is None else int(order)
    if ELEMENT_DIM[ele_type] == 2:
        t, fw = gauss_legendre_01((order + 2) // 2)  # basix's default rule on the interval
        lag = np.stack([1.0 - t, t], axis=1)
        if ele_type.startswith("TRI"):
            corners, finds, normals = _TRI_CORNERS, TRI_FACE_INDS, TRI_FACE_NORMALS
        else:
            corners, finds, normals = _QUAD_CORNERS, QUAD_FACE_INDS, QUAD_FACE_NORMALS
        pts = np.stack([lag @ corners[f] for f in finds])
        wts = np.stack([fw * np.linalg.norm(corners[f[1]] - corners[f[0]]) for f in finds])
        return finds.copy(), pts, wts, normals.copy()
    tet = ele_type.startswith("TET")
    if tet:
        fp, fw = _simplex_rule(2, order)
        lag = np.stack([1.0 - fp[:, 0] - fp[:, 1], fp[:, 0], fp[:, 1]], axis=1)
        corners, finds, normals = _TET_CORNERS, TET_FACE_INDS, TET_FACE_NORMALS
    else:
        fp, fw = _tensor_rule(2, order)
        s, t = fp[:, 0], fp[:, 1]
        lag = np.stack([(1 - s) * (1 - t), s * (1 - t), (1 - s) * t, s * t], axis=1)
        corners, finds, normals = _HEX_CORNERS, HEX_FACE_INDS, HEX_FACE_NORMALS
    pts, wts = [], []
    for f in finds:
        v = corners[f]
        pts.append(lag @ v)
        area = np.linalg.norm(np.cross(v[1] - v[0], v[2] - v[0]))
        wts.append(fw * area)
    return finds.copy(), np.stack(pts), np.stack(wts), normals.copy()


def get_shape_vals_and_grads(ele_type, quadrature_order=None):
    """shape_vals (nq, nen), shape_grads_ref (nq, nen, dim), weights (nq,)
    (basis.py:141-175)."""
    pts, w = volume_quadrature(ele_type, quadrature_order)
    vals, grads = shape_fn(ele_type, pts)
    return vals, grads, w


def get_face_shape_vals_and_grads(ele_type, quadrature_order=None):
    """face_shape_vals (nf, nfq, nen), face_shape_grads_ref (nf, nfq, nen, dim),
    face_weights (nf, nfq), face_normals (nf, dim), face_inds (nf, nfv)
    (basis.py:178-250)."""
    finds, pts, wts, normals = face_rule(ele_type, quadrature_order)
    nf, nfq, d = pts.shape
    vals, grads = shape_fn(ele_type, pts.reshape(-1, d))
    nen = vals.shape[1]
    return (vals.reshape(nf, nfq, nen), grads.reshape(nf, nfq, nen, d), wts, normals, finds)
