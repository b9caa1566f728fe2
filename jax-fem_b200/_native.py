"""ctypes bindings of libjaxfem_b200.so (the C ABI declared in include/jaxfem_b200.h).

The library is the only compute path: importing this module without the
built library, or calling a device entry point without a CUDA device, raises
``FEMNativeError`` -- there is no CPU fallback.
"""
import ctypes
import os
import threading

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libjaxfem_b200.so")

FEM_OK = 0
FEM_ERR_ARG = -1
FEM_ERR_CUDA = -2
FEM_ERR_NOT_CONVERGED = -3
FEM_ERR_BREAKDOWN = -4
FEM_ERR_NONFINITE = -5
FEM_ERR_CAPACITY = -6

LAW_LAPLACE, LAW_LINEAR, LAW_SIMP, LAW_NEO_HOOKEAN, LAW_J2 = 0, 1, 2, 3, 4
KRYLOV_CG, KRYLOV_BICGSTAB = 0, 1
PRECOND_NONE, PRECOND_JACOBI, PRECOND_BLOCK_JACOBI = 0, 1, 2
PRECOND_GMG = 100  # host-side selector: CG preconditioned by a multigrid V-cycle (multigrid.py)


class FemMGLevel(ctypes.Structure):
    """Mirror of ``FemMGLevel`` in include/jaxfem_b200.h."""
    _fields_ = [("nodes", ctypes.c_int64 * 3), ("n_brows", ctypes.c_int64),
                ("row_ptr", ctypes.c_void_p), ("col_idx", ctypes.c_void_p), ("stencil", ctypes.c_void_p),
                ("vals", ctypes.c_void_p), ("dinv", ctypes.c_void_p), ("x", ctypes.c_void_p),
                ("b", ctypes.c_void_p), ("r", ctypes.c_void_p), ("d0", ctypes.c_void_p), ("d1", ctypes.c_void_p),
                ("cpos", ctypes.c_void_p), ("ilo", ctypes.c_void_p), ("whi", ctypes.c_void_p),
                ("lmax", ctypes.c_void_p), ("cinv", ctypes.c_void_p), ("nu", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("vals_lo", ctypes.c_void_p), ("lo_scale", ctypes.c_void_p)]

FEM_MG_DENSE_MAX = 128  # largest coarsest level (n_brows * vec) solved by a dense inverse

_STATUS_NAMES = {
    FEM_ERR_ARG: "invalid argument",
    FEM_ERR_CUDA: "CUDA error",
    FEM_ERR_NOT_CONVERGED: "not converged",
    FEM_ERR_BREAKDOWN: "Krylov breakdown",
    FEM_ERR_NONFINITE: "non-finite value",
    FEM_ERR_CAPACITY: "capacity exceeded",
}


class FEMNativeError(RuntimeError):
    """A call into libjaxfem_b200 failed (or the library is missing)."""

    def __init__(self, status, message):
        super().__init__(f"[{_STATUS_NAMES.get(status, status)}] {message}")
        self.status = status


_c = ctypes
P = _c.c_void_p
I32 = _c.c_int
I64 = _c.c_int64
F64 = _c.c_double
SZ = _c.c_size_t
DP = _c.POINTER(_c.c_double)
IP = _c.POINTER(_c.c_int)

# name -> (restype, argtypes)
_SIGS = {
    "fem_version": (_c.c_char_p, []),
    "fem_last_error": (_c.c_char_p, []),
    "fem_launch_count": (I64, []),
    "fem_bsr_pattern": (I32, [P, I64, I64, P, _c.POINTER(I64), P, I64, P, P]),
    "fem_assemble_f64": (I32, [I32, DP, I32, I32, I64, I64, P, P, P, P, P, P, P, P, P, I64, P, P, P, P, P, P]),
    "fem_assemble_f32": (I32, [I32, DP, I32, I32, I64, I64, P, P, P, P, P, P, P, P, P, I64, P, P, P, P, P, P]),
    "fem_bsr_pattern_nen": (I32, [P, I64, I32, I64, P, _c.POINTER(I64), P, I64, P, P]),
    "fem_assemble_elem_f64": (I32, [I32, DP, I32, I32, I32, I32, P, P, I64, I64, P, P, P, P, P, P, P, P, P, I64, P,
                                    P, P, P, P, P]),
    "fem_assemble_elem_f32": (I32, [I32, DP, I32, I32, I32, I32, P, P, I64, I64, P, P, P, P, P, P, P, P, P, I64, P,
                                    P, P, P, P, P]),
    "fem_j2_commit_elem": (I32, [DP, I32, I32, I32, P, I64, P, P, P, P, P, P, P, P, P, P]),
    "fem_param_vjp_elem_f64": (I32, [I32, DP, I32, I32, I32, P, P, I64, P, P, P, P, P, P, P]),
    "fem_scatter_cells_f64": (I32, [I32, I64, P, P, P, P, P, P, P, P, P, P, P]),
    "fem_scatter_cells_f32": (I32, [I32, I64, P, P, P, P, P, P, P, P, P, P, P]),
    "fem_bsr_bc_diag_f64": (I32, [I32, I64, P, P, P, P]),
    "fem_bsr_bc_diag_f32": (I32, [I32, I64, P, P, P, P]),
    "fem_bsr_transpose_map": (I32, [P, P, I64, P]),
    "fem_j2_commit": (I32, [DP, I32, I64, P, P, P, P, P, P, P, P, P, P]),
    "fem_j2_sensitivity": (I32, [DP, I32, I64, P, P, P, P, P, P, P, P, P, P, P, P, P, P]),
    "fem_stress_divergence": (I32, [I64, P, P, P, P, P]),
    "fem_mg_setup_scratch_bytes": (SZ, [I32, I64, I32]),
    "fem_mg_setup_f64": (I32, [I32, I32, P, P, SZ, P]),
    "fem_mg_setup_f32": (I32, [I32, I32, P, P, P, SZ, P]),
    "fem_mg_vcycle_f64": (I32, [I32, I32, P, I32, I32, F64, P, P, P]),
    "fem_mg_vcycle_f32": (I32, [I32, I32, P, I32, I32, F64, P, P, P]),
    "fem_mg_tail_plan": (I32, [I32, I32, P, I32, I32, I32, IP, _c.POINTER(SZ)]),
    "fem_mg_pcg_workspace_bytes": (SZ, [I32, I64]),
    "fem_mg_pcg_solve": (I32, [I32, I64, P, P, P, P, P, F64, F64, I32, I32, I32, P, I32, I32, I32, F64, P, SZ, IP,
                               DP, P]),
    "fem_mg_pcg_solve_mixed": (I32, [I32, I64, P, P, P, P, P, F64, F64, I32, I32, I32, P, I32, I32, I32, F64, P, SZ, IP,
                               DP, P]),
    "fem_param_vjp_f64": (I32, [I32, DP, I32, I64, P, P, P, P, P, P, P]),
    "fem_bsr_spmv_f64": (I32, [I32, I64, P, P, P, P, P, P]),
    "fem_bsr_spmv_f32": (I32, [I32, I64, P, P, P, P, P, P]),
    "fem_bsr_residual_mixed": (I32, [I32, I64, P, P, P, P, P, P, P]),
    "fem_krylov_workspace_bytes": (SZ, [I32, I32, I32, I64, I32]),
    "fem_krylov_solve_f64": (I32, [I32, I32, I32, I64, P, P, P, P, P, P, F64, F64, I32, I32, P, SZ, IP, DP, P]),
    "fem_krylov_solve_f32": (I32, [I32, I32, I32, I64, P, P, P, P, P, P, F64, F64, I32, I32, P, SZ, IP, DP, P]),
    "fem_krylov_mixed_workspace_bytes": (SZ, [I32, I32, I64]),
    "fem_krylov_solve_mixed": (I32, [I32, I32, I64, P, P, P, P, P, P, F64, F64, I32, I32, F64, P, SZ, IP, IP,
                                     DP, P]),
    "fem_newton_rhs": (I32, [I64, P, P, P, P, P, P, P, P, DP, P, SZ, P]),
    "fem_dot_workspace_bytes": (SZ, [I64]),
    "fem_dot_f64": (I32, [I64, P, P, DP, P, SZ, P]),
    "fem_dot_f64_noalloc": (I32, [I64, P, P, P, P]),
    "fem_conv3d_fwd_bf16": (I32, [P, P, P, P, I32, I32, I32, I32, I32, I32, I32, P]),
    "fem_gemm_bf16_tn_f32": (I32, [P, P, P, I32, I32, I32, I32, I32, P]),
    "fem_tc_error": (I32, [IP, I32]),
    "fem_conv3d_im2col_t_bf16": (I32, [P, P, I32, I32, I32, I32, I32, P]),
    "fem_transpose_bf16": (I32, [P, P, I64, I32, P]),
    "fem_conv3d_flip_weights_bf16": (I32, [P, P, I32, I32, P]),
    "fem_relu_mask_bf16": (I32, [P, P, P, I64, P]),
}

_lib = None
_lock = threading.Lock()


def load():
    """Load the shared library once; raise FEMNativeError if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise FEMNativeError(FEM_ERR_ARG, f"{LIB_PATH} is missing: build it with "
                                 "`python jax-fem_b200/build.py` (no CPU fallback exists)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def exported_symbols():
    return list(_SIGS)


def lib():
    return load()


def check(status, what):
    if status != FEM_OK:
        msg = load().fem_last_error().decode(errors="replace")
        raise FEMNativeError(status, f"{what}: {msg}")


def ptr(t):
    """Device/host pointer of a tensor (None -> NULL)."""
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def params_array(values):
    arr = (ctypes.c_double * max(1, len(values)))(*[float(v) for v in values])
    return arr, len(values)


def require_cuda(t, name, dtype=None):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise FEMNativeError(FEM_ERR_ARG, f"{name} must be a CUDA tensor")
    if dtype is not None and t.dtype != dtype:
        raise FEMNativeError(FEM_ERR_ARG, f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise FEMNativeError(FEM_ERR_ARG, f"{name} must be contiguous")
    return t


def launch_count():
    return int(load().fem_launch_count())


def version():
    return load().fem_version().decode()
