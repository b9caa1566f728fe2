"""Problem builders shared by the tests: the same problem in the product
(``jax_fem_b200``) and in the FP64 oracle."""
import numpy as np

from oracle import fem_oracle as fo


def perturbed_box(pkg, N, L=(1.0, 1.0, 1.0), amp=0.15, seed=0):
    """Structured box with interior nodes jittered (general trilinear cells)."""
    m = pkg.box_mesh(N[0], N[1], N[2], *L)
    pts = m.points.copy()
    rng = np.random.default_rng(seed)
    h = np.array(L) / np.array(N)
    interior = np.all((pts > 1e-9) & (pts < np.array(L) - 1e-9), axis=1)
    pts[interior] += amp * h * rng.uniform(-1, 1, size=(interior.sum(), 3))
    return pkg.Mesh(pts, m.cells_dict["hexahedron"])


def law_pair(pkg, kind, C, rng, Q=8):
    """(product law, oracle law, product ivars, oracle ivars) for a law kind;
    internal variables per (cell, quadrature point), Q points per cell."""
    if kind == "laplace":
        return pkg.Laplace(), fo.Law("laplace", vec=3), [], []
    if kind == "linear":
        return pkg.LinearElastic(70e3, 0.3), fo.Law("linear", E=70e3, nu=0.3), [], []
    if kind == "simp":
        th = rng.uniform(0.05, 1.0, size=(C, Q))
        return (pkg.SIMPElastic(70e3, 70.0, 0.3, 3.0), fo.Law("simp", E0=70e3, Emin=70.0, nu=0.3, penal=3.0),
                [th], [th])
    if kind == "neo_hookean":
        return pkg.NeoHookean(10.0, 0.3), fo.Law("neo_hookean", E=10.0, nu=0.3), [], []
    if kind == "neo_hookean_scaled":
        s = rng.uniform(0.5, 1.5, size=(C, Q))
        return pkg.NeoHookean(10.0, 0.3), fo.Law("neo_hookean", E=10.0, nu=0.3), [s], [s]
    if kind == "j2":
        # a history with some points yielded: random prior stress / strain
        so = rng.normal(0, 150.0, size=(C, Q, 3, 3))
        so = 0.5 * (so + np.swapaxes(so, -1, -2))
        eo = rng.normal(0, 2e-3, size=(C, Q, 3, 3))
        eo = 0.5 * (eo + np.swapaxes(eo, -1, -2))
        ao = rng.uniform(0, 0.01, size=(C, Q))
        return (pkg.J2Plasticity(70e3, 0.3, 250.0, 700.0), fo.Law("j2", E=70e3, nu=0.3, sig0=250.0, H=700.0),
                [so, eo, ao], [so, eo, ao])
    raise ValueError(kind)


def make_problem(pkg, mesh, law, vec=3, bc=None, location_fns=None, ivars=(), mass_map=None,
                 surface_maps=None):
    class P(pkg.Problem):
        def get_tensor_map(self):
            return law

    if mass_map is not None:
        P.get_mass_map = lambda self: mass_map
    if surface_maps is not None:
        P.get_surface_maps = lambda self: surface_maps
    p = P(mesh, vec=vec, dim=3, dirichlet_bc_info=bc, location_fns=location_fns)
    p.internal_vars = list(ivars)
    return p


def element_box(pkg, ele_type, N, L=(1.0, 1.0, 1.0), amp=0.0, seed=0):
    """Structured box mesh of one element type; with amp > 0 every node off
    the boundary moves by up to amp * h (curved, general cells)."""
    import importlib
    gm = importlib.import_module("jax_fem_b200.generate_mesh")
    m = gm.box_mesh_gmsh(N[0], N[1], N[2], *L, None, ele_type)
    pts = m.points.copy()
    if amp > 0:
        rng = np.random.default_rng(seed)
        h = np.array(L) / np.array(N)
        inner = np.all((pts > 1e-9) & (pts < np.array(L) - 1e-9), axis=1)
        pts[inner] += amp * h * rng.uniform(-1, 1, size=(inner.sum(), 3))
    return pkg.Mesh(pts, m.cells_dict[gm.get_meshio_cell_type(ele_type)], ele_type)


def planar_box(pkg, ele_type, N, L=(1.0, 1.0), amp=0.0, seed=0):
    """Structured rectangle mesh of one 2D element type; with amp > 0 every
    node off the boundary moves by up to amp * h (curved, general cells)."""
    m = pkg.rectangle_mesh(N[0], N[1], L[0], L[1], ele_type=ele_type)
    pts = m.points.copy()
    if amp > 0:
        rng = np.random.default_rng(seed)
        h = np.array(L) / np.array(N)
        inner = np.all((pts > 1e-9) & (pts < np.array(L) - 1e-9), axis=1)
        pts[inner] += amp * h * rng.uniform(-1, 1, size=(inner.sum(), 2))
    return pkg.Mesh(pts, m.cells_dict[pkg.get_meshio_cell_type(ele_type)], ele_type)


def face_fn(axis, value):
    """Location function of the plane x[axis] = value."""
    return lambda p: np.isclose(p[axis], value, atol=1e-5)


# Manufactured Poisson solution of the reference's convergence-rate study
# (applications/convergence_rate/example.py:56-61): -lap u = -f with
# f = lap u_true as the mass map and u = u_true on the six faces.
def mms_u(p):
    x, y, z = p[..., 0], p[..., 1], p[..., 2]
    return 1e2 * ((x - 0.5) ** 3 + 2.0 * (y - 0.5) ** 3 + 1e1 * np.exp(-(z - 0.5) ** 2))


def mms_grad(p):
    x, y, z = p[..., 0], p[..., 1], p[..., 2]
    return 1e2 * np.stack([3.0 * (x - 0.5) ** 2, 6.0 * (y - 0.5) ** 2,
                           -2e1 * (z - 0.5) * np.exp(-(z - 0.5) ** 2)], axis=-1)


def mms_lap(p):
    x, y, z = p[..., 0], p[..., 1], p[..., 2]
    s = z - 0.5
    return 1e2 * (6.0 * (x - 0.5) + 12.0 * (y - 0.5) + 1e1 * (4.0 * s * s - 2.0) * np.exp(-s * s))


def mms_bc():
    """Dirichlet data of the study; the value function takes one point, or
    the coordinate arrays (p[0] = all x) in a batched call."""
    faces = [face_fn(a, v) for a in range(3) for v in (0.0, 1.0)]
    return [faces, [0] * 6, [lambda p: mms_u(np.stack([p[0], p[1], p[2]], axis=-1))] * 6]


def mms_mass_map(u, x):
    """mass_map of the study: lap u_true at x (one point or coordinate arrays)."""
    return np.array([mms_lap(np.stack([x[0], x[1], x[2]], axis=-1))])


def mms_errors(points, cells, vals, grads_ref, weights, sol):
    """L2 and H1 errors of sol against the manufactured solution, with the
    element's own quadrature, as compute_l2_norm_error / compute_h1_norm_error
    of the study (example.py:21-49; H1 = L2 of u plus L2 of grad u)."""
    X = points[cells]
    J = np.einsum("cai,qaj->cqij", X, grads_ref)
    jxw = np.linalg.det(J) * weights[None]
    g = np.einsum("qaj,cqjk->cqak", grads_ref, np.linalg.inv(J))
    cu = np.asarray(sol).reshape(-1)[cells]
    xq = np.einsum("qa,cai->cqi", vals, X)
    uq = np.einsum("qa,ca->cq", vals, cu)
    gq = np.einsum("ca,cqaj->cqj", cu, g)
    l2 = np.sqrt(np.sum((uq - mms_u(xq)) ** 2 * jxw))
    return l2, l2 + np.sqrt(np.sum(((gq - mms_grad(xq)) ** 2).sum(-1) * jxw))


def golden(name):
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    return dict(np.load(os.path.join(here, "golden", name + ".npz")))


def thermo_meshes(pkg):
    """A 2x1x1 box (length 2) of TET10 cells and the TET4 mesh of its corner nodes."""
    m10 = element_box(pkg, "TET10", (2, 1, 1), L=(2.0, 1.0, 1.0))
    ncorner = int(m10.cells[:, :4].max()) + 1
    m4 = pkg.Mesh(m10.points[:ncorner], m10.cells[:, :4], "TET4")
    return m10, m4


def thermo_problem(pkg, m10, m4, h=2.0, T_inf=1.0):
    """The two-variable thermo-elastic problem (u on TET10, T on TET4) with a
    Robin condition on x = 2, as a product Problem (torch kernels) and an
    oracle KernelProblem (numpy kernels)."""
    import torch

    import kernels as K
    bc_u = [[face_fn(0, 0.0)] * 3, [0, 1, 2], [lambda p: 0.0] * 3]
    bc_T = [[face_fn(0, 0.0)], [0], [lambda p: 0.0]]
    right = face_fn(0, 2.0)

    class Thermo(pkg.Problem):
        def get_universal_kernel(self):
            return K.thermoelastic_universal(torch, 10, self.fes[1].shape_vals_t, 100.0, 0.3, 2.0, 3.0, 1.0)

        def get_universal_kernels_surface(self):
            return [K.robin_surface(torch, 10, h, T_inf)]

    p = Thermo([m10, m4], vec=[3, 1], dim=3, ele_type=["TET10", "TET4"], quadrature_order=[2, 2],
               dirichlet_bc_info=[bc_u, bc_T], location_fns=[right])
    oracle = fo.KernelProblem(
        [dict(points=m10.points, cells=m10.cells, vec=3, ele_type="TET10", order=2, dirichlet=bc_u),
         dict(points=m4.points, cells=m4.cells, vec=1, ele_type="TET4", order=2, dirichlet=bc_T)],
        universal_kernel=K.thermoelastic_universal(np, 10, fo.element_tables("TET4", 2)[0], 100.0, 0.3, 2.0, 3.0,
                                                   1.0),
        location_fns=[right], universal_surface=[K.robin_surface(np, 10, h, T_inf)])
    return p, oracle, bc_u, bc_T
