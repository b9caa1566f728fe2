"""Host-side finite-element setup: element tables, Dirichlet and
boundary-face discovery, face geometry and the (u-independent) body/surface
load vectors.

Mirrors ``FiniteElement`` (fe.py:20-322 in the reference) for what runs once
per problem or per load step.  Nothing here is on the per-iteration path:
cell kernels, assembly and solves run in libjaxfem_b200.

User location/value/mass/surface functions are evaluated the way the
reference's ``jax.vmap`` does -- one point at a time semantically -- but
batched: a function is first called once with the coordinate axes as arrays
(``point[0]`` is the vector of all x coordinates) and the batched answer is
kept only if it agrees with point-by-point calls on a sample; otherwise it is
called point by point.

A location function that is a plain Python function is evaluated once per
function object: its node set is reused by later Dirichlet updates while its
code, defaults, closure values and the module globals it names are unchanged
(values compared by content: numbers, strings, tuples, small arrays; modules
and functions by identity).  One that reads anything that can change in place
unseen (a list, a dict, an object's attributes) is evaluated at every update,
as the reference does.
"""
import types
import weakref

import numpy as np

from . import basis

# Functions whose batched evaluation was confirmed against point-wise calls
# (a property of the function's code): later calls with the same function
# object skip the point-wise sample.  Weak keys: no id reuse after collection.
_BATCHED_OK = weakref.WeakKeyDictionary()
# Code objects confirmed on a full sample, with the kinds of their closure
# and default values: a new function object with the same code and plain
# number closure values (a boundary condition rebuilt at every load step) is
# checked at its first and last point only.
_BATCHED_CODE = {}


def _code_key(fn, key):
    code = getattr(fn, "__code__", None)
    if code is None:
        return None
    kinds = []
    for c in getattr(fn, "__closure__", None) or ():
        try:
            v = c.cell_contents
        except ValueError:  # an empty cell
            return None
        if not isinstance(v, (int, float, np.floating, np.integer)) or isinstance(v, bool):
            return None
        kinds.append(type(v).__name__)
    for v in getattr(fn, "__defaults__", None) or ():
        if not isinstance(v, (int, float, np.floating, np.integer)) or isinstance(v, bool):
            return None
        kinds.append(type(v).__name__)
    return (code, tuple(kinds), key)


def _batched_or_pointwise(fn, args, out_tail, sample=8):
    """Evaluate fn over leading axis of each array in ``args`` (see module doc)."""
    n = len(args[0])
    if n == 0:
        return np.zeros((0,) + out_tail)

    def pointwise(idx):
        out = [np.asarray(fn(*[a[i] for a in args]), dtype=np.float64) for i in idx]
        return np.array(out).reshape((len(idx),) + out_tail)

    batched = None
    try:
        r = np.asarray(fn(*[a.T for a in args]), dtype=np.float64)
        if r.shape == out_tail:  # constant answer
            batched = np.broadcast_to(r, (n,) + out_tail)
        elif r.shape == out_tail + (n,):  # one answer per point, point axis last
            batched = np.moveaxis(r, -1, 0)
    except Exception:  # noqa: BLE001 - fall back to point-by-point
        batched = None
    key = (len(args), out_tail)
    try:
        if batched is not None and key in _BATCHED_OK.get(fn, ()):
            return np.array(batched)
    except TypeError:  # not weak-referenceable
        pass
    ck = _code_key(fn, key) if batched is not None else None
    if ck is not None and ck in _BATCHED_CODE:
        idx = np.unique(np.array([0, n - 1]))
        if np.array_equal(np.asarray(batched[idx], dtype=np.float64), pointwise(idx)):
            return np.array(batched)
    rng = np.random.default_rng(0)
    idx = np.unique(np.concatenate([[0, n - 1], rng.integers(0, n, size=min(sample, n))]))
    ref = pointwise(idx)
    if batched is not None and np.array_equal(np.asarray(batched[idx], dtype=np.float64), ref):
        try:
            _BATCHED_OK.setdefault(fn, set()).add(key)
        except TypeError:
            pass
        if ck is not None:
            if len(_BATCHED_CODE) >= 256:
                _BATCHED_CODE.clear()
            _BATCHED_CODE[ck] = True
        return np.array(batched)
    return pointwise(np.arange(n))


_PLAIN = (int, float, complex, str, bytes, bool, type(None), np.generic)


def _code_names(code):
    names = set(code.co_names)
    for c in code.co_consts:
        if isinstance(c, types.CodeType):
            names |= _code_names(c)
    return names


def _value_state(v, depth):
    if isinstance(v, types.ModuleType):
        return ("module", v)
    if isinstance(v, _PLAIN):
        return ("value", type(v), v)
    if isinstance(v, np.ndarray):
        return ("array", v.dtype.str, v.shape, v.tobytes()) if v.nbytes <= (1 << 20) else None
    if isinstance(v, tuple):
        parts = tuple(_value_state(x, depth) for x in v)
        return None if any(p is None for p in parts) else ("tuple", parts)
    if isinstance(v, types.FunctionType):
        st = function_state(v, depth - 1)
        return None if st is None else ("function", v, st)
    if isinstance(v, (types.BuiltinFunctionType, np.ufunc)):
        return ("builtin", v)
    return None


def function_state(fn, depth=2):
    """What a plain Python function's answer can depend on besides its
    arguments, as a comparable value: its code, defaults, closure values and
    the globals it names.  None when fn is not a plain function or some of
    that state could change in place unseen."""
    if not isinstance(fn, types.FunctionType) or depth < 0:
        return None
    vals = list(fn.__defaults__ or ()) + list((fn.__kwdefaults__ or {}).values())
    for cell in fn.__closure__ or ():
        try:
            vals.append(cell.cell_contents)
        except ValueError:  # empty cell
            return None
    g = fn.__globals__
    vals += [g[nm] for nm in sorted(_code_names(fn.__code__)) if nm in g]
    state = [fn.__code__]
    for v in vals:
        st = _value_state(v, depth)
        if st is None:
            return None
        state.append(st)
    return tuple(state)


def _location_flags(fn, points):
    nargs = getattr(getattr(fn, "__code__", None), "co_argcount", 1)
    if nargs == 1:
        args = (points,)
        f = fn
    elif nargs == 2:
        args = (points, np.arange(len(points)))
        f = fn
    else:
        raise ValueError(f"Wrong number of arguments for location_fn: must be 1 or 2, get {nargs}")
    return _batched_or_pointwise(f, args, ()).astype(bool)


class FiniteElement:
    """One field on a mesh of one element type (fe.py:20-110), 3D or 2D.
    Holds the element tables (basis.py) and Dirichlet data as host arrays."""

    def __init__(self, mesh, vec, dim, ele_type="HEX8", quadrature_rule=None, quadrature_order=None,
                 dirichlet_bc_info=None):
        basis.check_ele_type(ele_type)
        if dim != basis.ELEMENT_DIM[ele_type]:
            raise ValueError(f"{ele_type} is a {basis.ELEMENT_DIM[ele_type]}D element, the problem has dim={dim}")
        if mesh.points.shape[1] != dim:
            raise ValueError(f"dim={dim} needs points of {dim} coordinates, the mesh has {mesh.points.shape[1]}")
        if quadrature_rule not in (None, "default"):
            raise NotImplementedError("only basix's default quadrature rule is supported")
        if mesh.cells.shape[1] != basis.NODES_PER_CELL[ele_type]:
            raise ValueError(f"{ele_type} needs cells of {basis.NODES_PER_CELL[ele_type]} nodes, "
                             f"the mesh has {mesh.cells.shape[1]}")
        self.mesh = mesh
        self.points = mesh.points
        self.cells = mesh.cells
        self.vec, self.dim, self.ele_type = vec, dim, ele_type
        self.quadrature_order = basis.DEFAULT_ORDER[ele_type] if quadrature_order is None else int(quadrature_order)
        self.num_cells = len(self.cells)
        self.num_total_nodes = len(self.points)
        self.num_total_dofs = self.num_total_nodes * vec
        self.shape_vals, self.shape_grads_ref, self.quad_weights = basis.get_shape_vals_and_grads(
            ele_type, self.quadrature_order)
        (self.face_shape_vals, self.face_shape_grads_ref, self.face_quad_weights, self.face_normals,
         self.face_inds) = basis.get_face_shape_vals_and_grads(ele_type, self.quadrature_order)
        self.num_quads, self.num_nodes = self.shape_vals.shape
        self.num_faces, self.num_face_quads = self.face_quad_weights.shape
        self.dirichlet_bc_info = dirichlet_bc_info
        self.bc_version = 0
        self.node_inds_list, self.vec_inds_list, self.vals_list = self.Dirichlet_boundary_conditions(
            dirichlet_bc_info)

    # -- Dirichlet (fe.py:220-269) -------------------------------------------
    def Dirichlet_boundary_conditions(self, dirichlet_bc_info):
        node_inds_list, vec_inds_list, vals_list = [], [], []
        if dirichlet_bc_info is not None:
            location_fns, vecs, value_fns = dirichlet_bc_info
            assert len(location_fns) == len(value_fns) and len(value_fns) == len(vecs)
            seen_loc, seen_val = {}, {}  # the same function object is evaluated once
            for lf, v, vf in zip(location_fns, vecs, value_fns):
                if id(lf) not in seen_loc:
                    seen_loc[id(lf)] = self._location_nodes(lf)
                node_inds = seen_loc[id(lf)]
                key = (id(vf), id(lf))
                if key not in seen_val:
                    seen_val[key] = _batched_or_pointwise(vf, (self._node_points(lf, node_inds),), ())
                vals = seen_val[key]
                node_inds_list.append(node_inds)
                vec_inds_list.append(np.full(len(node_inds), int(v), dtype=np.int32))
                vals_list.append(np.asarray(vals, dtype=np.float64).reshape(-1))
        return node_inds_list, vec_inds_list, vals_list

    def _location_nodes(self, lf):
        """Nodes where the location function holds (reused while its state,
        ``function_state``, is unchanged)."""
        memo = self.__dict__.setdefault("_location_memo", {})
        state = function_state(lf)
        hit = memo.get(id(lf))
        try:
            if state is not None and hit is not None and hit[0] is lf and hit[1] == state:
                return hit[2].copy()
        except (TypeError, ValueError):  # a state that does not compare plainly
            pass
        nodes = np.argwhere(_location_flags(lf, self.points)).reshape(-1)
        if state is not None:
            if len(memo) >= 64:
                memo.clear()
            memo[id(lf)] = (lf, state, nodes.copy())
        return nodes

    def _node_points(self, lf, nodes):
        """points[nodes] for a location function's node set, kept while the
        set is unchanged (load steps re-evaluate values on the same nodes)."""
        memo = self.__dict__.setdefault("_node_points_memo", {})
        hit = memo.get(id(lf))
        if hit is not None and hit[0] is lf and np.array_equal(hit[1], nodes):
            return hit[2].copy()  # a value function may write into its argument
        pts = self.points[nodes]
        if len(memo) >= 64:
            memo.clear()
        memo[id(lf)] = (lf, np.array(nodes), pts.copy())
        return pts

    def update_Dirichlet_boundary_conditions(self, dirichlet_bc_info):
        self.dirichlet_bc_info = dirichlet_bc_info
        self.node_inds_list, self.vec_inds_list, self.vals_list = self.Dirichlet_boundary_conditions(
            dirichlet_bc_info)
        self.bc_version += 1

    def dirichlet_arrays(self):
        """(mask uint8 (ndofs,), values (ndofs,)); later conditions win on overlap
        (the reference applies them in order, solver.py:297-300)."""
        mask = np.zeros(self.num_total_dofs, dtype=np.uint8)
        vals = np.zeros(self.num_total_dofs, dtype=np.float64)
        for n, v, val in zip(self.node_inds_list, self.vec_inds_list, self.vals_list):
            d = n * self.vec + v
            mask[d] = 1
            vals[d] = val
        return mask, vals

    # -- boundary faces (fe.py:271-322) ---------------------------------------
    def get_boundary_conditions_inds(self, location_fns):
        out = []
        if location_fns is None:
            return out
        for lf in location_fns:
            flags = _location_flags(lf, self.points)
            cf = flags[self.cells[:, self.face_inds]]  # (C, faces, face vertices)
            out.append(np.argwhere(cf.all(axis=2)))
        return out

    def get_face_shape_grads(self, boundary_inds):
        """Physical face shape gradients (F,fq,nen,dim) and Nanson scale (F,fq) (fe.py:143-183)."""
        binds = np.asarray(boundary_inds).reshape(-1, 2)
        F = len(binds)
        if F == 0:
            return np.zeros((0, self.num_face_quads, self.num_nodes, self.dim)), np.zeros((0, self.num_face_quads))
        gref = self.face_shape_grads_ref[binds[:, 1]]  # (F,fq,nen,dim)
        X = self.points[self.cells[binds[:, 0]]]
        J = np.einsum("fai,fqaj->fqij", X, gref)
        Jinv = np.linalg.inv(J)
        grads = np.einsum("fqaj,fqjk->fqak", gref, Jinv)
        nJ = np.einsum("fi,fqij->fqj", self.face_normals[binds[:, 1]], Jinv)
        scale = np.linalg.norm(nJ, axis=-1) * np.linalg.det(J) * self.face_quad_weights[binds[:, 1]]
        return grads, scale

    def face_shape_vals_at(self, faces):
        return self.face_shape_vals[np.asarray(faces, dtype=np.int64)]

    # -- load vectors of u-independent maps (problem.py:216-259) ---------------
    def _check_u_independent(self, fn, x):
        rng = np.random.default_rng(7)
        k = min(4, len(x))
        for i in range(k):
            a = np.asarray(fn(np.zeros(self.vec), x[i]), dtype=np.float64)
            b = np.asarray(fn(rng.standard_normal(self.vec), x[i]), dtype=np.float64)
            if not np.array_equal(a, b):
                raise NotImplementedError(
                    "mass/surface maps that depend on u are not supported on this path; "
                    "only u-independent loads (evaluated once into a load vector) are")

    def depends_on_u(self, fn):
        """Whether a mass / surface map's value changes with u (checked at a
        few nodes with random u): such maps go to the cell-kernel path."""
        try:
            self._check_u_independent(fn, self.points[: min(4, len(self.points))])
        except NotImplementedError:
            return True
        except Exception:  # noqa: BLE001 - needs internal variables or torch input: user code
            return True
        return False

    def body_load(self, mass_map):
        """int mass_map(u, x) . v dx as a (ndofs,) vector."""
        X = self.points[self.cells]  # (C,nen,dim)
        J = np.einsum("cai,qaj->cqij", X, self.shape_grads_ref)
        jxw = np.linalg.det(J) * self.quad_weights[None]
        xq = np.einsum("qa,cai->cqi", self.shape_vals, X).reshape(-1, self.dim)
        self._check_u_independent(mass_map, xq)
        u0 = np.zeros((len(xq), self.vec))
        val = _batched_or_pointwise(mass_map, (u0, xq), (self.vec,)).reshape(self.num_cells, self.num_quads,
                                                                             self.vec)
        r = np.einsum("cqi,qa,cq->cai", val, self.shape_vals, jxw)
        f = np.zeros((self.num_total_nodes, self.vec))
        np.add.at(f, self.cells.reshape(-1), r.reshape(-1, self.vec))
        return f.reshape(-1)

    def surface_load(self, surface_map, boundary_inds):
        """int surface_map(u, x) . v ds over the selected faces as a (ndofs,) vector."""
        f = np.zeros((self.num_total_nodes, self.vec))
        binds = np.asarray(boundary_inds).reshape(-1, 2)
        if len(binds) == 0:
            return f.reshape(-1)
        _, scale = self.get_face_shape_grads(binds)
        fv = self.face_shape_vals_at(binds[:, 1])  # (F,fq,nen)
        X = self.points[self.cells[binds[:, 0]]]
        xq = np.einsum("fqa,fai->fqi", fv, X).reshape(-1, self.dim)
        self._check_u_independent(surface_map, xq)
        u0 = np.zeros((len(xq), self.vec))
        val = _batched_or_pointwise(surface_map, (u0, xq), (self.vec,)).reshape(len(binds), self.num_face_quads,
                                                                                self.vec)
        r = np.einsum("fqi,fqa,fq->fai", val, fv, scale)
        np.add.at(f, self.cells[binds[:, 0]].reshape(-1), r.reshape(-1, self.vec))
        return f.reshape(-1)

    def JxW(self):
        X = self.points[self.cells]
        J = np.einsum("cai,qaj->cqij", X, self.shape_grads_ref)
        return np.linalg.det(J) * self.quad_weights[None]
