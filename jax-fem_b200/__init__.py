"""jax_fem_b200: JAX-FEM's assemble-and-solve path on B200 (sm_100a), for
HEX8 cells and the other 3D element types (TET4, TET10, HEX20, HEX27).

Drop-in for the reference's ``Problem`` / ``solver`` / ``ad_wrapper``
(jax_fem/problem.py, jax_fem/solver.py): Python host code on PyTorch calls
hand-written CUDA kernels in ``lib/libjaxfem_b200.so`` through a C ABI
(include/jaxfem_b200.h).  There is no CPU fallback.

The package directory is ``jax-fem_b200/``; it is imported under the module
name ``jax_fem_b200`` by ``load_package()`` in the repository root's
``__graft_entry__.py`` (a hyphen cannot appear in an import statement).
"""
from . import _native
from .generate_mesh import Mesh, box_mesh, box_mesh_gmsh, check_mesh_TET4, get_meshio_cell_type, rectangle_mesh
from .laws import J2Plasticity, Laplace, LinearElastic, NeoHookean, SIMPElastic
from .problem import BSRMatrix, Problem, compliance
from .solver import (J2YieldSensitivity, ad_wrapper, get_A, get_q_vec, j2_reaction, reset_multigrid, solver,
                     stress_divergence)
from .utils import read_mesh, save_sol

__all__ = ["Mesh", "box_mesh", "box_mesh_gmsh", "check_mesh_TET4", "get_meshio_cell_type", "rectangle_mesh",
           "Problem", "solver", "ad_wrapper", "get_A",
           "BSRMatrix", "compliance", "Laplace", "LinearElastic", "SIMPElastic", "NeoHookean",
           "J2Plasticity", "J2YieldSensitivity", "j2_reaction", "stress_divergence", "save_sol", "read_mesh",
           "get_q_vec", "reset_multigrid",
           "_native"]
