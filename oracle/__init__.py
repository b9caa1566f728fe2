"""CPU FP64 oracle for the HEX8 assemble-and-solve path (test infrastructure).

This package is the parity checker of the project, not part of the product.
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import it.  The product path (``jax-fem_b200/``) never calls it: it
runs on the CUDA library and fails loudly when that library is missing.

Parity status: pinned.  ``fem_oracle`` is checked against the five FEniCSx
golden fixtures the reference's own tests hold
(tests/benchmarks/*/test_*.py in the reference), converted to
``tests/golden/*.npz`` by ``tests/golden/make_fixtures.py``.  The reference
itself (JAX + basix + PETSc) cannot be imported in this environment, so no
output of the reference is compared directly.
"""
