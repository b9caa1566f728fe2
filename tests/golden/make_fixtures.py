"""Convert the reference's FEniCSx golden data into compact .npz fixtures.

The reference pins its HEX8 path with five integration tests whose expected
results are FEniCSx solutions stored as ASCII VTU files plus a few .npy
scalars (tests/benchmarks/*/fenicsx/ in the reference).  This script reads
those files (it is the only committed file that reads the reference tree) and
writes one ``<case>.npz`` per test with the arrays the parity tests need:

- ``points`` (num_nodes, 3) float64, ``cells`` (num_cells, 8) int32 in VTK
  HEX8 order (the order meshio hands to ``Mesh`` in the reference tests),
- ``sol`` (num_nodes, vec) float64, the FEniCSx solution,
- case-specific scalars (``traction``, ``surface_area``, ``disps``,
  ``avg_stresses``).

Usage: python tests/golden/make_fixtures.py REFERENCE_ROOT

REFERENCE_ROOT is the root of a checkout of the reference project (the
directory that holds its ``tests/benchmarks``).
"""
import os
import re
import sys

import numpy as np

CASES = {
    "linear_poisson": [],
    "linear_elasticity_cube": [],
    "linear_elasticity_cylinder": ["surface_area"],
    "hyperelasticity": ["traction"],
    "plasticity": ["disps", "avg_stresses"],
}


def read_vtu_ascii(path):
    """Parse the ASCII UnstructuredGrid VTU written by dolfinx (version 2.2)."""
    text = open(path).read()
    arrays = {}
    for m in re.finditer(r"<DataArray([^>]*)>(.*?)</DataArray>", text, re.S):
        attrs, body = m.group(1), m.group(2)
        name = re.search(r'Name="([^"]*)"', attrs)
        typ = re.search(r'type="([^"]*)"', attrs).group(1)
        ncomp = re.search(r'NumberOfComponents="(\d+)"', attrs)
        dtype = np.float64 if typ.startswith("Float") else np.int64
        data = np.array(body.split(), dtype=dtype)
        if ncomp is not None:
            data = data.reshape(-1, int(ncomp.group(1)))
        key = name.group(1) if name else "points"
        # Points come first and carry no Name; keep the first unnamed array.
        if key in arrays and key == "points":
            continue
        if key == "vtkGhostType" and key in arrays:
            key = "vtkGhostType_points"
        arrays[key] = data
    return arrays


def main(ref_root):
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for case, extras in CASES.items():
        d = os.path.join(ref_root, "tests", "benchmarks", case, "fenicsx")
        a = read_vtu_ascii(os.path.join(d, "sol_p0_000000.vtu"))
        types = a["types"]
        assert np.all(types == 72), "expected order-1 VTK Lagrange hexahedra"
        cells = a["connectivity"].reshape(-1, 8).astype(np.int32)
        sol = a["sol"]
        if sol.ndim == 1:
            sol = sol[:, None]
        out = dict(points=a["points"].astype(np.float64), cells=cells, sol=sol.astype(np.float64))
        for e in extras:
            out[e] = np.load(os.path.join(d, e + ".npy"))
        np.savez_compressed(os.path.join(out_dir, case + ".npz"), **out)
        print(case, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py REFERENCE_ROOT")
    main(sys.argv[1])
