"""Element tabulation: shape functions, quadrature and face tables of the
3D element types of the reference's basis.py:19-114 (HEX8, HEX20, HEX27,
TET4, TET10), in mesh (VTK/meshio) node order.

The reference tabulates with basix 0.10 (``get_shape_vals_and_grads``,
basis.py:141-175; ``get_face_shape_vals_and_grads``, basis.py:178-250) and
permutes basix's dof order into the mesh's with ``re_order``.  Here each
element is written directly in mesh order from its definition:

- HEX8, HEX27: tensor-product Lagrange of degree 1 and 2 on [0,1]^3
  (basix P on the hexahedron; at degree <= 2 every Lagrange variant puts
  the nodes at vertices, edge midpoints, face centres and the centre);
- TET4, TET10: Lagrange P1 / P2 on the unit tetrahedron, written in
  barycentric coordinates (corner L(2L-1), edge 4 L_i L_j);
- HEX20: basix's serendipity element of degree 2, whose degrees of freedom
  are the 8 vertex values and the 12 edge means (moments against the
  constant on each unit edge), not midpoint values.  Its basis is the dual
  basis of those 20 functionals in the 20-dimensional serendipity space,
  computed once by solving a 20x20 system.

Quadrature follows basix's default rule (basis.py:117-124): Gauss-Jacobi
(Gauss-Legendre on [0,1]) with (order+2)//2 points per axis on hexahedra
and quadrilaterals; on tetrahedra and triangles the Xiao-Gimbutas rules,
of which the orders the element types use by default are restated here:
order 0 and 1 the centroid, order 2 the symmetric 4-point (tetrahedron)
and 3-point (triangle) rules.
"""
import functools

import numpy as np

# meshio cell type of each element (generate_mesh.py:83-117)
MESHIO_CELL_TYPE = {"HEX8": "hexahedron", "HEX20": "hexahedron20", "HEX27": "hexahedron27",
                    "TET4": "tetra", "TET10": "tetra10"}
# default quadrature order (basis.py:52-89)
DEFAULT_ORDER = {"HEX8": 2, "HEX20": 2, "HEX27": 10, "TET4": 0, "TET10": 2}
NODES_PER_CELL = {"HEX8": 8, "HEX20": 20, "HEX27": 27, "TET4": 4, "TET10": 10}

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


def check_ele_type(ele_type):
    if ele_type not in NODES_PER_CELL:
        raise NotImplementedError(
            f"element {ele_type!r}: the 3D types HEX8, HEX20, HEX27, TET4 and TET10 are supported")
    return ele_type


def node_coords(ele_type):
    """Reference coordinates (nen, 3) of the nodes in mesh order."""
    check_ele_type(ele_type)
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
    """Tensor-product Lagrange basis at points xi (n,3) with node coordinates X."""
    idx = np.rint(X * (len(nodes1d) - 1)).astype(int)  # index of each coordinate in nodes1d
    v = []
    d = []
    for ax in range(3):
        va, da = _lagrange1d(nodes1d, xi[:, ax])
        v.append(va[:, idx[:, ax]])
        d.append(da[:, idx[:, ax]])
    vals = v[0] * v[1] * v[2]
    grads = np.stack([d[0] * v[1] * v[2], v[0] * d[1] * v[2], v[0] * v[1] * d[2]], axis=2)
    return vals, grads


def _tet_shape(ele_type, xi):
    L = np.stack([1.0 - xi.sum(axis=1), xi[:, 0], xi[:, 1], xi[:, 2]], axis=1)  # (n,4)
    dL = np.array([[-1, -1, -1], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.float64)  # (4,3)
    if ele_type == "TET4":
        return L, np.broadcast_to(dL, (len(xi), 4, 3)).copy()
    vals = np.empty((len(xi), 10))
    grads = np.empty((len(xi), 10, 3))
    for a in range(4):
        vals[:, a] = L[:, a] * (2.0 * L[:, a] - 1.0)
        grads[:, a] = (4.0 * L[:, a] - 1.0)[:, None] * dL[a]
    for e, (i, j) in enumerate(TET_EDGES):
        vals[:, 4 + e] = 4.0 * L[:, i] * L[:, j]
        grads[:, 4 + e] = 4.0 * (L[:, j][:, None] * dL[i] + L[:, i][:, None] * dL[j])
    return vals, grads


# Serendipity space of degree 2 on the cube: P2 plus xyz, the six x_i^2 x_j
# and the three x_i^2 x_j x_k (exponent triples).
_SERENDIPITY_EXPONENTS = np.array(
    [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [2, 0, 0], [0, 2, 0], [0, 0, 2], [1, 1, 0], [0, 1, 1],
     [1, 0, 1], [1, 1, 1], [2, 1, 0], [2, 0, 1], [1, 2, 0], [0, 2, 1], [1, 0, 2], [0, 1, 2], [2, 1, 1],
     [1, 2, 1], [1, 1, 2]])


def _monomials(xi, E):
    """Values (n, m) and gradients (n, m, 3) of monomials x^E."""
    xi = np.asarray(xi, dtype=np.float64)
    pw = lambda k, a: xi[:, a:a + 1] ** k  # noqa: E731
    vals = pw(E[:, 0], 0) * pw(E[:, 1], 1) * pw(E[:, 2], 2)
    grads = np.empty(vals.shape + (3,))
    for ax in range(3):
        e = E[:, ax]
        dax = np.where(e > 0, e * xi[:, ax:ax + 1] ** np.maximum(e - 1, 0), 0.0)
        other = [b for b in range(3) if b != ax]
        grads[:, :, ax] = dax * pw(E[:, other[0]], other[0]) * pw(E[:, other[1]], other[1])
    return vals, grads


@functools.lru_cache(maxsize=None)
def _hex20_coefficients():
    """Coefficients C (20 monomials x 20 nodes) of the dual basis of basix's
    degree-2 serendipity dofs: phi_k = sum_m C[m, k] (x - 1/2)^E_m with
    l_j(phi_k) = delta_jk, l_j = value at corner j (j < 8) or mean over
    edge j-8 (VTK edge order)."""
    E = _SERENDIPITY_EXPONENTS
    t, w = gauss_legendre_01(3)  # exact for the cubic restrictions to an edge
    Lmat = np.empty((20, 20))
    Lmat[:8] = _monomials(_HEX_CORNERS - 0.5, E)[0]
    for e, (i, j) in enumerate(HEX_EDGES):
        pts = _HEX_CORNERS[i][None] + t[:, None] * (_HEX_CORNERS[j] - _HEX_CORNERS[i])[None]
        Lmat[8 + e] = w @ _monomials(pts - 0.5, E)[0]
    return np.linalg.solve(Lmat, np.eye(20))


def shape_fn(ele_type, xi):
    """Shape values (n, nen) and reference gradients (n, nen, 3) at points xi (n, 3)."""
    check_ele_type(ele_type)
    xi = np.atleast_2d(np.asarray(xi, dtype=np.float64))
    if ele_type.startswith("TET"):
        return _tet_shape(ele_type, xi)
    if ele_type == "HEX8":
        return _tensor_lagrange(node_coords("HEX8"), xi, [0.0, 1.0])
    if ele_type == "HEX27":
        return _tensor_lagrange(node_coords("HEX27"), xi, [0.0, 0.5, 1.0])
    C = _hex20_coefficients()
    mv, mg = _monomials(xi - 0.5, _SERENDIPITY_EXPONENTS)  # centred monomials (the space is shift-invariant)
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
    """Quadrature points (nq, 3) and weights (nq,) of the element's cell."""
    order = DEFAULT_ORDER[check_ele_type(ele_type)] if order is None else int(order)
    return _simplex_rule(3, order) if ele_type.startswith("TET") else _tensor_rule(3, order)


def face_rule(ele_type, order=None):
    """Per-face quadrature (basis.py:178-250): face_inds (nf, nfv) corner
    numbers, points (nf, nfq, 3) in reference coordinates, weights
    (nf, nfq) times the facet's reference area, normals (nf, 3)."""
    order = DEFAULT_ORDER[check_ele_type(ele_type)] if order is None else int(order)
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
    """shape_vals (nq, nen), shape_grads_ref (nq, nen, 3), weights (nq,)
    (basis.py:141-175)."""
    pts, w = volume_quadrature(ele_type, quadrature_order)
    vals, grads = shape_fn(ele_type, pts)
    return vals, grads, w


def get_face_shape_vals_and_grads(ele_type, quadrature_order=None):
    """face_shape_vals (nf, nfq, nen), face_shape_grads_ref (nf, nfq, nen, 3),
    face_weights (nf, nfq), face_normals (nf, 3), face_inds (nf, nfv)
    (basis.py:178-250)."""
    finds, pts, wts, normals = face_rule(ele_type, quadrature_order)
    nf, nfq = pts.shape[:2]
    vals, grads = shape_fn(ele_type, pts.reshape(-1, 3))
    nen = vals.shape[1]
    return (vals.reshape(nf, nfq, nen), grads.reshape(nf, nfq, nen, 3), wts, normals, finds)
