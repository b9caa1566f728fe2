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


def law_pair(pkg, kind, C, rng):
    """(product law, oracle law, product ivars, oracle ivars) for a law kind."""
    if kind == "laplace":
        return pkg.Laplace(), fo.Law("laplace", vec=3), [], []
    if kind == "linear":
        return pkg.LinearElastic(70e3, 0.3), fo.Law("linear", E=70e3, nu=0.3), [], []
    if kind == "simp":
        th = rng.uniform(0.05, 1.0, size=(C, 8))
        return (pkg.SIMPElastic(70e3, 70.0, 0.3, 3.0), fo.Law("simp", E0=70e3, Emin=70.0, nu=0.3, penal=3.0),
                [th], [th])
    if kind == "neo_hookean":
        return pkg.NeoHookean(10.0, 0.3), fo.Law("neo_hookean", E=10.0, nu=0.3), [], []
    if kind == "neo_hookean_scaled":
        s = rng.uniform(0.5, 1.5, size=(C, 8))
        return pkg.NeoHookean(10.0, 0.3), fo.Law("neo_hookean", E=10.0, nu=0.3), [s], [s]
    if kind == "j2":
        # a history with some points yielded: random prior stress / strain
        so = rng.normal(0, 150.0, size=(C, 8, 3, 3))
        so = 0.5 * (so + np.swapaxes(so, -1, -2))
        eo = rng.normal(0, 2e-3, size=(C, 8, 3, 3))
        eo = 0.5 * (eo + np.swapaxes(eo, -1, -2))
        ao = rng.uniform(0, 0.01, size=(C, 8))
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


def golden(name):
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    return dict(np.load(os.path.join(here, "golden", name + ".npz")))
