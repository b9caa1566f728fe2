"""ctypes binding of ``fem_cpu.cpp``: the reference's HEX8 assemble-and-solve
path restated in C++ / OpenMP (FP64).

TEST INFRASTRUCTURE ONLY: the timed CPU baseline of ``bench.py`` (its
``--impl reference`` arm and the ``cpu_baseline`` leg) and the tests that
check it against the numpy oracle.  The product (``jax-fem_b200``) never
imports, links or runs it.

``build()`` compiles ``oracle/lib/libfem_cpu.so`` with the recipe in
``oracle/Makefile`` (g++, x86-64-v3: AVX2 and FMA, so a library built on one
x86 host runs on any current one).
"""
import ctypes as _c
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "fem_cpu.cpp")
LIB = os.path.join(HERE, "lib", "libfem_cpu.so")

LAW_LINEAR, LAW_NEO_HOOKEAN = 0, 1
METHOD_BICGSTAB, METHOD_CG = 0, 1  # jax_solve's BiCGSTAB + Jacobi; PETSc CG + Jacobi

_lib = None


def build(force=False):
    """Compile the library (when the source is newer than it, or ``force``)."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    subprocess.run(["make", "-B" if force else "-s", "-C", HERE], check=True, capture_output=True, text=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = _c.CDLL(LIB)
        P, I64, D, I = _c.c_void_p, _c.c_int64, _c.c_double, _c.c_int
        L.fcpu_create.restype = P
        L.fcpu_create.argtypes = [I, I, I, D, D, D, I, D, D, I]
        L.fcpu_destroy.argtypes = [P]
        L.fcpu_ndofs.restype = I64
        L.fcpu_ndofs.argtypes = [P]
        L.fcpu_nnz.restype = I64
        L.fcpu_nnz.argtypes = [P]
        L.fcpu_threads.restype = I
        L.fcpu_threads.argtypes = [P]
        L.fcpu_set_dirichlet.restype = I
        L.fcpu_set_dirichlet.argtypes = [P, I64, P, P]
        L.fcpu_newton.restype = I
        L.fcpu_newton.argtypes = [P, P, D, D, I, D, D, I, I]
        L.fcpu_stats.argtypes = [P, _c.POINTER(I), _c.POINTER(I), _c.POINTER(D), _c.POINTER(D)]
        L.fcpu_residual_tangent.restype = D
        L.fcpu_residual_tangent.argtypes = [P, P, P, P, P, P]
        _lib = L
    return _lib


def box_dirichlet(n, kind, theta=0.0):
    """Dirichlet dofs and values of the benchmark boxes (box_mesh numbering,
    unit cube, n^3 cells): 'twist' = x=0 clamped, x=1 with u_x = 0 and (y, z)
    rotated by theta about (0.5, 0.5); 'stretch' = x=0 clamped, u_x = 0.01 on
    x=1.  Evaluated on the host, as the reference evaluates its Python value
    functions (fe.py:220-269)."""
    N = n + 1
    idx = np.arange(N ** 3)
    i, j, k = idx // (N * N), (idx // N) % N, idx % N
    y, z = j / n, k / n
    left, right = idx[i == 0], idx[i == n]
    dofs = [3 * left, 3 * left + 1, 3 * left + 2, 3 * right]
    vals = [np.zeros(len(left))] * 3
    if kind == "twist":
        c, s = np.cos(theta), np.sin(theta)
        yr, zr = y[right], z[right]
        vals = vals + [np.zeros(len(right))]
        dofs += [3 * right + 1, 3 * right + 2]
        vals += [0.5 + (yr - 0.5) * c - (zr - 0.5) * s - yr, 0.5 + (yr - 0.5) * s + (zr - 0.5) * c - zr]
    elif kind == "stretch":
        vals = vals + [np.full(len(right), 0.01)]
    else:
        raise ValueError(kind)
    return np.concatenate(dofs).astype(np.int64), np.concatenate(vals).astype(np.float64)


class CPUProblem:
    """One n^3 HEX8 unit-cube problem on the CPU (see fem_cpu.cpp)."""

    def __init__(self, n, law, E, nu, threads=0):
        self.n = n
        self.h = lib().fcpu_create(n, n, n, 1.0, 1.0, 1.0, law, E, nu, threads)
        if not self.h:
            raise ValueError("fcpu_create failed")
        self.ndofs = lib().fcpu_ndofs(self.h)
        self.nnz = lib().fcpu_nnz(self.h)
        self.threads = lib().fcpu_threads(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().fcpu_destroy(self.h)
            self.h = None

    def set_dirichlet(self, dofs, vals):
        self._bc = (np.ascontiguousarray(dofs, np.int64), np.ascontiguousarray(vals, np.float64))
        st = lib().fcpu_set_dirichlet(self.h, len(self._bc[0]), self._bc[0].ctypes.data, self._bc[1].ctypes.data)
        if st != 0:
            raise ValueError("Dirichlet dof out of range")

    def newton(self, u, rel_tol=1e-8, tol=1e-12, method=METHOD_BICGSTAB, lin_tol=1e-10, lin_atol=1e-10,
               lin_maxiter=10000, max_iter=50):
        """Newton solve of the current load step; u (float64, ndofs) in/out.
        Returns {newton, krylov, assembly_s, linear_s}."""
        assert u.dtype == np.float64 and u.flags.c_contiguous and u.size == self.ndofs
        st = lib().fcpu_newton(self.h, u.ctypes.data, rel_tol, tol, method, lin_tol, lin_atol, lin_maxiter,
                               max_iter)
        if st != 0:
            raise RuntimeError(f"fcpu_newton failed with status {st}")
        return self.stats()

    def stats(self):
        nw, kr, ta, tl = _c.c_int(0), _c.c_int(0), _c.c_double(0.0), _c.c_double(0.0)
        lib().fcpu_stats(self.h, _c.byref(nw), _c.byref(kr), _c.byref(ta), _c.byref(tl))
        return {"newton": nw.value, "krylov": kr.value, "assembly_s": ta.value, "linear_s": tl.value}

    def residual_tangent(self, u):
        """(residual with Dirichlet rows u - u_D, row-zeroed CSR tangent) at u."""
        import scipy.sparse as sp
        u = np.ascontiguousarray(u, np.float64)
        res = np.empty(self.ndofs)
        rp = np.empty(self.ndofs + 1, np.int64)
        col = np.empty(self.nnz, np.int32)
        vals = np.empty(self.nnz)
        lib().fcpu_residual_tangent(self.h, u.ctypes.data, res.ctypes.data, rp.ctypes.data, col.ctypes.data,
                                    vals.ctypes.data)
        return res, sp.csr_matrix((vals, col, rp), shape=(self.ndofs, self.ndofs))


def twist_solve(prob, steps=5, total_deg=30.0, **newton_kw):
    """The 5-step twist load history with the reference's practice of
    starting each load step from the previous solution.  Returns (u, stats
    summed over the steps)."""
    u = np.zeros(prob.ndofs)
    tot = {"newton": 0, "krylov": 0, "assembly_s": 0.0, "linear_s": 0.0}
    for s in range(1, steps + 1):
        prob.set_dirichlet(*box_dirichlet(prob.n, "twist", np.deg2rad(total_deg * s / steps)))
        st = prob.newton(u, **newton_kw)
        for k in tot:
            tot[k] += st[k]
    return u, tot
