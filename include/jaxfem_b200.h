/*
 * jaxfem_b200.h -- C ABI of the B200 (sm_100a) assemble-and-solve library
 * (HEX8 fast path; TET4, TET10, HEX20, HEX27 through the general element
 * entry points).
 *
 * The reference (JAX-FEM) is pure Python: its hot path is a chain of Python
 * functions with no foreign-function boundary.  Each entry point below
 * replaces one of those functions; the comment above it cites the reference
 * interface (file:line inside the reference project) whose role it takes.
 *
 * Conventions
 *  - Plain pointers and sizes only.  Pointers named d_* are device pointers,
 *    h_* are host pointers.  `stream` is a cudaStream_t passed as void*
 *    (NULL = legacy default stream).
 *  - Every function returns an int status: FEM_OK (0) or a negative code.
 *    No exception crosses the ABI.  fem_last_error() returns a message for
 *    the last failure on the calling thread.
 *  - The caller owns every buffer.  Workspaces are passed in with their size
 *    (query with the *_workspace_bytes functions).  A workspace must not be
 *    shared by two calls that may run concurrently.
 *  - Layouts: points (num_nodes,3) f64 row-major; cells (num_cells,8) int32
 *    in VTK/meshio HEX8 order ((num_cells,nen) for the general element
 *    entry points); dof = node*vec + component; block-CSR (BSR)
 *    matrices with vec x vec row-major blocks, sorted columns per block row.
 *  - Per-quadrature-point data is (num_cells, 8, ...) with the quadrature
 *    points in basix order (2x2x2 Gauss-Legendre on [0,1]^3, x slowest);
 *    (num_cells, nq, ...) for the general element entry points.
 */
#ifndef JAXFEM_B200_H
#define JAXFEM_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FEM_API __attribute__((visibility("default")))
#else
#define FEM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define FEM_OK 0
#define FEM_ERR_ARG (-1)           /* invalid argument / unsupported combination */
#define FEM_ERR_CUDA (-2)          /* a CUDA runtime call failed */
#define FEM_ERR_NOT_CONVERGED (-3) /* Krylov hit maxiter before the tolerance */
#define FEM_ERR_BREAKDOWN (-4)     /* Krylov breakdown (p.Ap <= 0, rho == 0, ...) */
#define FEM_ERR_NONFINITE (-5)     /* NaN/Inf met in a reduction */
#define FEM_ERR_CAPACITY (-6)      /* output buffer too small */

/* ---- constitutive laws (the registered replacements for get_tensor_map) --
 * Each law maps the displacement gradient at a quadrature point to the
 * stress of the weak form, with its exact (consistent) tangent.
 *   FEM_LAW_LAPLACE     P = grad u                       params: -
 *   FEM_LAW_LINEAR      sigma = lmbda tr(eps) I + 2 mu eps    params: E, nu
 *   FEM_LAW_SIMP        as LINEAR with E = Emin + (E0-Emin) theta^penal
 *                       params: E0, Emin, nu, penal; ivar0 = theta (C,8)
 *   FEM_LAW_NEO_HOOKEAN P = dpsi/dF, psi = mu/2 (J^-2/3 I1 - 3) + kappa/2 (J-1)^2
 *                       params: E, nu; ivar0 = optional psi scale (C,8) or NULL
 *   FEM_LAW_J2          small-strain radial return, linear isotropic hardening
 *                       params: E, nu, sigma_y, H;
 *                       ivar0 = sigma_old (C,8,3,3), ivar1 = eps_old (C,8,3,3),
 *                       ivar2 = alpha_old (C,8)
 * ------------------------------------------------------------------------ */
#define FEM_LAW_LAPLACE 0
#define FEM_LAW_LINEAR 1
#define FEM_LAW_SIMP 2
#define FEM_LAW_NEO_HOOKEAN 3
#define FEM_LAW_J2 4

/* Krylov methods and preconditioners. */
#define FEM_KRYLOV_CG 0
#define FEM_KRYLOV_BICGSTAB 1
#define FEM_PRECOND_NONE 0
#define FEM_PRECOND_JACOBI 1
#define FEM_PRECOND_BLOCK_JACOBI 2

/* Library version string and a message for the last failure on this thread. */
FEM_API const char* fem_version(void);
FEM_API const char* fem_last_error(void);
/* Number of kernels this library has launched since load (all threads). */
FEM_API int64_t fem_launch_count(void);

/* ---- sparsity pattern (host, one-off setup) -----------------------------
 * Replaces the COO pattern of Problem.__post_init__ (problem.py:86-107) and
 * PETSc's setPreallocationCOO (solver.py:469-475): instead of num_cells*576
 * duplicated (I, J) pairs it builds the node-adjacency block-CSR pattern and a
 * cell -> block scatter map, so assembly never sorts.
 *   pass 1: h_col_idx == NULL  -> fills h_row_ptr (num_nodes+1), *h_nnzb
 *   pass 2: h_col_idx != NULL  -> fills h_col_idx (capacity >= nnzb),
 *           h_scatter (num_cells*64: block index of local pair (a,b) at
 *           [c*64 + a*8 + b]) and h_diag (num_nodes: index of block (n,n)).
 * ------------------------------------------------------------------------ */
FEM_API int fem_bsr_pattern(const int32_t* h_cells, int64_t num_cells, int64_t num_nodes,
                    int32_t* h_row_ptr, int64_t* h_nnzb, int32_t* h_col_idx,
                    int64_t col_capacity, int32_t* h_scatter, int32_t* h_diag);
/* The same for cells of nen nodes (the element types of basis.py:19-114:
 * TET4 4, HEX8 8, TET10 10, HEX20 20, HEX27 27); h_cells is (num_cells, nen)
 * and h_scatter (num_cells, nen*nen) with the block index of local pair
 * (a, b) at [c*nen*nen + a*nen + b].  fem_bsr_pattern is the nen = 8 case.
 * 1 <= nen <= 256 (the cell-kernel path passes cell dof tables). */
FEM_API int fem_bsr_pattern_nen(const int32_t* h_cells, int64_t num_cells, int nen, int64_t num_nodes,
                    int32_t* h_row_ptr, int64_t* h_nnzb, int32_t* h_col_idx,
                    int64_t col_capacity, int32_t* h_scatter, int32_t* h_diag);
/* Block transpose map (host, one-off): h_tmap[k] = index of block (j, i) for
 * block k = (i, j) of a row-sorted, structurally symmetric pattern (as
 * fem_bsr_pattern builds).  Assembly writes the lower block triangle from
 * the upper one through it.  Part of the same pattern setup as above. */
FEM_API int fem_bsr_transpose_map(const int32_t* h_row_ptr, const int32_t* h_col_idx, int64_t n_brows,
                    int32_t* h_tmap);

/* ---- cell assembly ------------------------------------------------------
 * Replaces Problem.newton_update / compute_residual (problem.py:439-491): the
 * per-cell weak-form kernel and its jacfwd (problem.py:189-214, 262-266,
 * 299-301), the residual scatter (problem.py:426-437) and the PETSc COO value
 * insertion + zeroRows of get_A (solver.py:485-491).
 *
 * Residual:   d_res[dof] = sum_cells int P(grad u) : grad v   (zeroed first)
 * Tangent:    d_vals (BSR, value type per suffix) = dR/du with Dirichlet rows
 *             AND columns eliminated (unit diagonal), zeroed first.
 * Lift:       d_lift = K_full * d_dvec restricted to free rows, where d_dvec
 *             holds the prescribed Dirichlet increment (zero at free dofs);
 *             the eliminated system A x = b with b_free = -(R_free + lift),
 *             b_bc = dvec has the solution of the reference's row-zeroed
 *             system (solver.py:390-421) while staying symmetric for CG.
 * Any of d_res / d_lift / d_vals may be NULL to skip that output.  d_bc_mask
 * (uint8 per dof, 1 = Dirichlet) may be NULL (no elimination).
 * The element tangents of every law here are symmetric: the kernel forms the
 * 36 node pairs a <= b of each cell into the upper block triangle and a
 * transpose pass fills the lower one, using d_transpose, the block transpose
 * map of the pattern (fem_bsr_transpose_map; needed with d_vals).
 * d_params: host array of law parameters (see FEM_LAW_*), n_params entries.
 * d_ivar0..2: per-law internal variables (device, f64) or NULL.
 * ------------------------------------------------------------------------ */
FEM_API int fem_assemble_f64(int law, const double* h_params, int n_params, int vec,
                     int64_t num_cells, int64_t num_nodes, const int32_t* d_cells,
                     const double* d_points, const double* d_u,
                     const double* d_ivar0, const double* d_ivar1, const double* d_ivar2,
                     const int32_t* d_scatter, const int32_t* d_diag,
                     const int32_t* d_transpose, int64_t nnzb,
                     const uint8_t* d_bc_mask, const double* d_dvec,
                     double* d_res, double* d_lift, double* d_vals, void* stream);
/* Same with the tangent computed and stored in FP32 (mixed-precision path).
 * Geometry, the constitutive update and d_res are FP64 as in _f64 (the
 * Newton residual is exact); d_lift is accumulated in FP64 from the FP32
 * tangent. */
FEM_API int fem_assemble_f32(int law, const double* h_params, int n_params, int vec,
                     int64_t num_cells, int64_t num_nodes, const int32_t* d_cells,
                     const double* d_points, const double* d_u,
                     const double* d_ivar0, const double* d_ivar1, const double* d_ivar2,
                     const int32_t* d_scatter, const int32_t* d_diag,
                     const int32_t* d_transpose, int64_t nnzb,
                     const uint8_t* d_bc_mask, const double* d_dvec,
                     double* d_res, double* d_lift, float* d_vals, void* stream);

/* ---- general elements ---------------------------------------------------
 * The same cell assembly for the element types of basis.py:19-114 other than
 * the HEX8 fast path above (TET4, TET10, HEX20, HEX27; HEX8 is accepted too).
 * The element enters through its tabulation (get_shape_vals_and_grads,
 * basis.py:141-175): d_gref (nq, nen, 3) f64, the reference shape gradients
 * at the quadrature points in mesh node order, and d_wq (nq) the weights.
 *   nen in {4, 8, 10, 20, 27}; 1 <= nq <= 4096
 *   d_cells (num_cells, nen); d_scatter (num_cells, nen*nen) from
 *   fem_bsr_pattern_nen; internal variables are per (cell, quadrature
 *   point): theta / psi scale (num_cells, nq), J2 state (num_cells, nq, 3, 3)
 *   and (num_cells, nq).
 * Outputs, Dirichlet elimination and the lift are those of fem_assemble_*.
 * The _f32 variant accumulates the tangent in FP64 and stores it in FP32. */
FEM_API int fem_assemble_elem_f64(int law, const double* h_params, int n_params, int vec, int nen, int nq,
                     const double* d_gref, const double* d_wq, int64_t num_cells, int64_t num_nodes,
                     const int32_t* d_cells, const double* d_points, const double* d_u,
                     const double* d_ivar0, const double* d_ivar1, const double* d_ivar2,
                     const int32_t* d_scatter, const int32_t* d_diag, const int32_t* d_transpose,
                     int64_t nnzb, const uint8_t* d_bc_mask, const double* d_dvec,
                     double* d_res, double* d_lift, double* d_vals, void* stream);
FEM_API int fem_assemble_elem_f32(int law, const double* h_params, int n_params, int vec, int nen, int nq,
                     const double* d_gref, const double* d_wq, int64_t num_cells, int64_t num_nodes,
                     const int32_t* d_cells, const double* d_points, const double* d_u,
                     const double* d_ivar0, const double* d_ivar1, const double* d_ivar2,
                     const int32_t* d_scatter, const int32_t* d_diag, const int32_t* d_transpose,
                     int64_t nnzb, const uint8_t* d_bc_mask, const double* d_dvec,
                     double* d_res, double* d_lift, float* d_vals, void* stream);
/* fem_j2_commit for these elements (state arrays (num_cells, nq, ...)). */
FEM_API int fem_j2_commit_elem(const double* h_params, int n_params, int nen, int nq, const double* d_gref,
                     int64_t num_cells, const int32_t* d_cells, const double* d_points, const double* d_u,
                     const double* d_sigma_old, const double* d_eps_old, const double* d_alpha_old,
                     double* d_sigma_new, double* d_eps_new, double* d_alpha_new, void* stream);
/* fem_param_vjp_f64 for these elements: d_grad (num_cells, nq). */
FEM_API int fem_param_vjp_elem_f64(int law, const double* h_params, int n_params, int nen, int nq,
                     const double* d_gref, const double* d_wq, int64_t num_cells, const int32_t* d_cells,
                     const double* d_points, const double* d_u, const double* d_ivar0,
                     const double* d_lambda, double* d_grad, void* stream);

/* ---- cell-kernel path ---------------------------------------------------
 * For problems whose weak form is user code evaluated by the host on the
 * device (universal kernels, multi-variable problems, tensor maps that are
 * not registered laws; problem.py:260-300): the global system is a scalar
 * CSR matrix over all dofs (a BSR with vec = 1), its pattern from
 * fem_bsr_pattern_nen with the cell dof table (num_cells, nd) as "cells".
 * fem_scatter_cells_* replaces the residual scatter of
 * compute_residual_vars_helper (problem.py:471-483) and the COO insertion +
 * zeroRows of get_A (solver.py:466-491).  It ACCUMULATES (the caller zeroes
 * d_res / d_lift / d_vals once, then calls it for the cells and for each
 * set of boundary faces):
 *   d_item_res (items, nd), d_item_jac (items, nd, nd) row-major (NULL: no
 *   tangent or lift); item i belongs to cell d_item_cell[i] (NULL: cell i),
 *   whose dofs are d_cell_dofs[cell] and whose scatter row is
 *   d_scatter[cell] (nd*nd entries);
 *   d_res[dofs[a]] += res[i, a];
 *   d_vals[scatter[cell, a*nd+b]] += jac[i, a, b] unless dofs[a] or dofs[b]
 *   is a Dirichlet dof (d_bc_mask);
 *   d_lift[dofs[a]] += jac[i, a, b] * d_dvec[dofs[b]] for free dofs[a].
 * No symmetry is assumed.  1 <= nd <= 256.
 * fem_bsr_bc_diag_* then writes the unit diagonal at Dirichlet dofs. */
FEM_API int fem_scatter_cells_f64(int nd, int64_t num_items, const int32_t* d_item_cell,
                     const int32_t* d_cell_dofs, const int32_t* d_scatter, const double* d_item_res,
                     const double* d_item_jac, const uint8_t* d_bc_mask, const double* d_dvec,
                     double* d_res, double* d_lift, double* d_vals, void* stream);
FEM_API int fem_scatter_cells_f32(int nd, int64_t num_items, const int32_t* d_item_cell,
                     const int32_t* d_cell_dofs, const int32_t* d_scatter, const double* d_item_res,
                     const double* d_item_jac, const uint8_t* d_bc_mask, const double* d_dvec,
                     double* d_res, double* d_lift, float* d_vals, void* stream);
FEM_API int fem_bsr_bc_diag_f64(int vec, int64_t n_brows, const uint8_t* d_bc_mask, const int32_t* d_diag,
                     double* d_vals, void* stream);
FEM_API int fem_bsr_bc_diag_f32(int vec, int64_t n_brows, const uint8_t* d_bc_mask, const int32_t* d_diag,
                     float* d_vals, void* stream);

/* ---- J2 state commit ----------------------------------------------------
 * Replaces the reference plasticity update (test_plasticity.py:67-78 with
 * fe.py:366-382): at every quadrature point run the return map at the
 * converged u and write sigma_new, eps_new = sym grad u, alpha_new. */
FEM_API int fem_j2_commit(const double* h_params, int n_params, int64_t num_cells,
                  const int32_t* d_cells, const double* d_points, const double* d_u,
                  const double* d_sigma_old, const double* d_eps_old, const double* d_alpha_old,
                  double* d_sigma_new, double* d_eps_new, double* d_alpha_new, void* stream);

/* ---- J2 yield-stress sensitivity ----------------------------------------
 * No counterpart in the reference: its ad_wrapper (solver.py:1383-1417)
 * differentiates one static solve, not a load history.  The derivative of
 * the return map above (stress_return_map, test_plasticity.py:42-64, with
 * linear hardening) w.r.t. the initial yield stress sigma_y, given d_du =
 * du/dsigma_y (NULL = 0: the explicit part) and the committed state's
 * sensitivities (NULL = 0: the first increment).  Writes dsigma (C,8,9),
 * deps = sym grad du (C,8,9; NULL to skip) and dalpha (C,8).  Carried over
 * the increments this gives d(reaction)/d(sigma_y) with one extra linear
 * solve per increment (the direct method; for a single parameter it costs
 * what the adjoint does and needs no stored history). */
FEM_API int fem_j2_sensitivity(const double* h_params, int n_params, int64_t num_cells,
                  const int32_t* d_cells, const double* d_points, const double* d_u,
                  const double* d_du, const double* d_sigma_old, const double* d_eps_old,
                  const double* d_alpha_old, const double* d_dsigma_old, const double* d_deps_old,
                  const double* d_dalpha_old, double* d_dsigma, double* d_deps, double* d_dalpha,
                  void* stream);

/* The internal force of a quadrature-point stress field: d_out[node*3+i] +=
 * sum over cells and quadrature points of stress_ij dN_node/dx_j JxW (the
 * residual of problem.py:189-214 with the stress supplied instead of
 * computed from u).  d_stress is (C,8,9) f64; d_out (N*3) f64 accumulates. */
FEM_API int fem_stress_divergence(int64_t num_cells, const int32_t* d_cells, const double* d_points,
                  const double* d_stress, double* d_out, void* stream);

/* ---- adjoint parameter VJP ----------------------------------------------
 * Replaces jax.vjp of the BC-applied residual w.r.t. internal variables in
 * implicit_vjp (solver.py:1340-1356, 1376-1378):
 *   d_grad[c,q] = - (dR/dtheta_{c,q})^T lambda
 * for the law's per-quad scalar parameter (SIMP: theta; NEO_HOOKEAN: psi
 * scale).  lambda must be zero at Dirichlet dofs (their residual rows do not
 * depend on theta).  d_grad is (num_cells, 8) f64, overwritten. */
FEM_API int fem_param_vjp_f64(int law, const double* h_params, int n_params, int64_t num_cells,
                      const int32_t* d_cells, const double* d_points, const double* d_u,
                      const double* d_ivar0, const double* d_lambda, double* d_grad,
                      void* stream);

/* ---- block-CSR operators ------------------------------------------------
 * Replace the BCOO mat-vec inside jax.scipy bicgstab (solver.py:63-92).
 * y (n_brows*vec) = A x; x is read only at the column indices, so A may be
 * rectangular (p-multigrid's transfers between node sets). */
FEM_API int fem_bsr_spmv_f64(int vec, int64_t n_brows, const int32_t* d_row_ptr, const int32_t* d_col_idx,
                     const double* d_vals, const double* d_x, double* d_y, void* stream);
FEM_API int fem_bsr_spmv_f32(int vec, int64_t n_brows, const int32_t* d_row_ptr, const int32_t* d_col_idx,
                     const float* d_vals, const float* d_x, float* d_y, void* stream);
/* r = b - A x with FP32 matrix values, FP64 vectors and FP64 accumulation
 * (the refinement residual of the mixed path). */
FEM_API int fem_bsr_residual_mixed(int vec, int64_t n_brows, const int32_t* d_row_ptr,
                           const int32_t* d_col_idx, const float* d_vals, const double* d_x,
                           const double* d_b, double* d_r, void* stream);

/* ---- Krylov solvers -----------------------------------------------------
 * Replace linear_solver / jax_solve (solver.py:63-92, 261-284): solve
 * A x = b to ||b - A x|| <= max(rtol ||b||, atol), starting from the x passed
 * in.  The iteration runs on the device; the host polls a status word every
 * `check_every` iterations.  When the recursively updated residual meets the
 * tolerance the true residual b - A x is recomputed; if it does not meet the
 * tolerance the recurrence restarts from it; a breakdown (zero or
 * non-positive denominator, typically round-off near the attainable
 * accuracy) also restarts from the true residual.  After 3 restarts the call
 * returns FEM_ERR_NOT_CONVERGED.  *h_iters = total iterations, *h_relres = the last
 * true (or, while iterating, recursive) ||r||/||b||.  Returns
 * FEM_ERR_NOT_CONVERGED / FEM_ERR_BREAKDOWN / FEM_ERR_NONFINITE with x
 * holding the last iterate.
 * _f64: values/vectors f64.  _f32: values/vectors f32, dot products and
 * their reductions in f64 (an FP32 solve cannot push the true residual much
 * below ~1e-6 relative; the mixed path refines in FP64 around it).
 * d_work must hold fem_krylov_workspace_bytes() bytes. */
FEM_API size_t fem_krylov_workspace_bytes(int method, int precond, int vec, int64_t n_brows, int fp32);
FEM_API int fem_krylov_solve_f64(int method, int precond, int vec, int64_t n_brows,
                         const int32_t* d_row_ptr, const int32_t* d_col_idx,
                         const int32_t* d_diag, const double* d_vals, const double* d_b,
                         double* d_x, double rtol, double atol, int maxiter, int check_every,
                         void* d_work, size_t work_bytes, int* h_iters, double* h_relres,
                         void* stream);
FEM_API int fem_krylov_solve_f32(int method, int precond, int vec, int64_t n_brows,
                         const int32_t* d_row_ptr, const int32_t* d_col_idx,
                         const int32_t* d_diag, const float* d_vals, const float* d_b,
                         float* d_x, double rtol, double atol, int maxiter, int check_every,
                         void* d_work, size_t work_bytes, int* h_iters, double* h_relres,
                         void* stream);

/* Mixed-precision CG of the same linear solve (jax_solve / linear_solver,
 * solver.py:63-92, 261-284): FP32 matrix values and FP32 iteration vectors,
 * FP64 right-hand side d_b and FP64 solution d_x (initial guess in, result
 * out), reductions in FP64.  Reliable updates: when the recursive residual
 * has fallen below delta times its largest value since the last update
 * (0 < delta < 1; 0.1 is the usual choice), the FP32 increment is added to
 * d_x and the residual is replaced by the true one, b - A x with FP64
 * accumulation; the search direction is kept.  Convergence, ||b - A x|| <=
 * max(rtol ||b||, atol), is always confirmed on the true residual, which
 * *h_relres reports.  Only method CG; needs fem_krylov_mixed_workspace_bytes
 * of workspace.  *h_replacements counts the residual replacements. */
FEM_API size_t fem_krylov_mixed_workspace_bytes(int precond, int vec, int64_t n_brows);
FEM_API int fem_krylov_solve_mixed(int precond, int vec, int64_t n_brows,
                         const int32_t* d_row_ptr, const int32_t* d_col_idx,
                         const int32_t* d_diag, const float* d_vals, const double* d_b,
                         double* d_x, double rtol, double atol, int maxiter, int check_every,
                         double delta, void* d_work, size_t work_bytes, int* h_iters,
                         int* h_replacements, double* h_relres, void* stream);

/* ---- vector helpers of the Newton loop ----------------------------------
 * fem_newton_rhs: the BC handling of newton_update_helper + newton_step
 * (solver.py:290-304, 390-409).  With R = res + f_ext:
 *   d_rbc[dof] = R[dof] at free dofs, u[dof] - ubc[dof] at Dirichlet dofs
 *               (the reference's BC-applied residual vector, whose norm is the
 *               Newton criterion)
 *   d_rhs[dof] = -(R + lift) at free dofs, ubc - u at Dirichlet dofs
 * and *h_norm2 (optional, synchronous) = ||d_rbc||^2 in f64. */
FEM_API int fem_newton_rhs(int64_t ndofs, const double* d_res, const double* d_fext,
                   const double* d_lift, const uint8_t* d_bc_mask, const double* d_u,
                   const double* d_ubc, double* d_rbc, double* d_rhs, double* h_norm2,
                   void* d_work, size_t work_bytes, void* stream);
/* Deterministic f64 dot product: *h_out = x . y (synchronous). d_work needs
 * fem_dot_workspace_bytes(n) bytes (per-block partial sums). */
FEM_API size_t fem_dot_workspace_bytes(int64_t n);
FEM_API int fem_dot_f64(int64_t n, const double* d_x, const double* d_y, double* h_out,
                void* d_work, size_t work_bytes, void* stream);

/* ---- learned warm start: tensor-core 3D convolution ----------------------
 * No counterpart in the reference (its only network is an unrelated MLP
 * energy surrogate, applications/surrogate_model/train.py).  BF16 operands,
 * FP32 accumulation in TMEM (tcgen05), TMA tile loads.  Activations are
 * NDHWC bf16, 16-byte aligned.
 * fem_conv3d_fwd_bf16: out = [relu](conv3x3x3_pad1(in, w) + bias), w is
 *   (Cout, 27, Cin) with tap = 9 kd + 3 kh + kw; Cin a multiple of 16,
 *   Cout in {16,32,64,128}; N*D*H*W must tile into 128-voxel bricks (W, H, D
 *   powers of two are fine).  bias (Cout f32) may be NULL.  The input
 *   gradient is the same call on the output gradient with weights from
 *   fem_conv3d_flip_weights_bf16.
 * fem_gemm_bf16_tn_f32: C[M,N] += A[M,K] B[N,K]^T (row-major, K contiguous),
 *   K a multiple of 16, N in {16,32,64} or a multiple of 128, split over K
 *   into split_k slices accumulated with FP32 atomics (C must be zeroed by
 *   the caller).  With A = im2col^T(X) (fem_conv3d_im2col_t_bf16) and
 *   B = dZ^T (fem_transpose_bf16) this is the weight gradient dW^T.
 * fem_tc_error: reads (and optionally resets) the device flag the tensor-core
 *   kernels set when a pipeline wait times out (0 = none). */
FEM_API int fem_conv3d_fwd_bf16(const void* d_in, const void* d_w, const float* d_bias, void* d_out,
                                int N, int D, int H, int W, int Cin, int Cout, int relu, void* stream);
FEM_API int fem_gemm_bf16_tn_f32(const void* d_a, const void* d_b, float* d_c, int M, int N, int K,
                                 int ldc, int split_k, void* stream);
FEM_API int fem_tc_error(int* h_err, int reset);
FEM_API int fem_conv3d_im2col_t_bf16(const void* d_x, void* d_col, int N, int D, int H, int W, int C,
                                     void* stream);
FEM_API int fem_transpose_bf16(const void* d_in, void* d_out, int64_t rows, int cols, void* stream);
FEM_API int fem_conv3d_flip_weights_bf16(const void* d_w, void* d_wt, int Cout, int Cin, void* stream);
FEM_API int fem_relu_mask_bf16(const void* d_dy, const void* d_y, void* d_dz, int64_t n, void* stream);

/* ---- geometric multigrid on box lattices ---------------------------------
 * Replaces the reference's optional AMGX preconditioner path
 * (solver.py:136-259) for meshes that are tensor lattices numbered as
 * box_mesh numbers them (generate_mesh.py:151-189): node (i, j, k) =
 * (i*ny + j)*nz + k with nx, ny, nz nodes per direction.  Levels coarsen 2:1
 * per direction (a last odd interval stays 1 fine cell wide); prolongation
 * is trilinear interpolation on the coarse lattice; coarse operators are
 * Galerkin products P^T A P of the Dirichlet-eliminated fine operator, so
 * they stay symmetric positive definite.  The smoother is Chebyshev
 * iteration on the Jacobi-scaled operator over [lmax/ratio, lmax], lmax a
 * Gershgorin bound; pre- and post-smoothing are the same polynomial and the
 * coarsest level takes a longer one, so a V-cycle is a fixed symmetric
 * operator and can precondition CG.
 *
 * A level describes its lattice, pattern, values and work vectors (device
 * pointers, each n_brows*vec entries of the call's type).  stencil[(n,27)]
 * holds the block index of neighbour (dx,dy,dz) at (dx+1)*9 + (dy+1)*3 +
 * (dz+1), or -1.  Levels >= 1 also hold, per direction d, cpos (the fine
 * lattice index of each coarse node), ilo (for each node of the finer level,
 * the coarse node at or below it) and whi (the interpolation weight of the
 * coarse node ilo+1), all concatenated over x, y, z. */
typedef struct FemMGLevel {
  int64_t nodes[3];
  int64_t n_brows;
  const int32_t* row_ptr;
  const int32_t* col_idx;
  const int32_t* stencil;
  void* vals;
  void* dinv;
  void* x;
  void* b;
  void* r;
  void* d0;
  void* d1;
  const int32_t* cpos;
  const int32_t* ilo;
  const double* whi;
  void* lmax;             /* device, 8 bytes: the level's Gershgorin bound (FP64), written by setup */
  double* cinv;           /* coarsest level only, or NULL: device, (n_brows*vec)^2 FP64 entries
                             (n_brows*vec <= FEM_MG_DENSE_MAX), the dense inverse of its operator,
                             written by setup; the V-cycle then solves that level exactly */
  int32_t nu;             /* smoothing steps on this level; 0: the call's nu */
  int32_t reserved;
  void* vals_lo;          /* FP32 hierarchies only, or NULL: device, 16-byte aligned, nnzb*vec*vec FP16
                             values, written by setup as the level's values times a power of two s
                             (max |a| s < 2^14); the V-cycle's smoothing and residual products on this
                             level then read them (half the bytes of FP32) */
  double* lo_scale;       /* with vals_lo: device, 2 doubles; setup writes 1/s to [0] ([1] is its scratch) */
} FemMGLevel;
#define FEM_MG_DENSE_MAX 128

/* Setup (once per operator, launches only): coarse values by Galerkin
 * products P^T (A P), the Jacobi scaling and the bound lmax of every level.
 * d_scratch holds A P of one level (levels[0].n_brows * 27 * vec*vec values
 * of the call's type; fem_mg_setup_scratch_bytes).  _f32: with d_fine_f64
 * non-NULL, level 0's values are first rounded from that FP64 operator. */
FEM_API size_t fem_mg_setup_scratch_bytes(int vec, int64_t fine_n_brows, int fp32);
FEM_API int fem_mg_setup_f64(int vec, int nlevels, const FemMGLevel* levels, void* d_scratch,
                             size_t scratch_bytes, void* stream);
FEM_API int fem_mg_setup_f32(int vec, int nlevels, const FemMGLevel* levels, const double* d_fine_f64,
                             void* d_scratch, size_t scratch_bytes, void* stream);
/* z = V(rhs): one V-cycle with nu Chebyshev steps before and after on each
 * level and coarse_steps on the coarsest; ratio sets the smoothed interval
 * [lmax/ratio, lmax].  Launches only (no synchronization). */
FEM_API int fem_mg_vcycle_f64(int vec, int nlevels, const FemMGLevel* levels, int nu, int coarse_steps,
                              double ratio, const double* d_rhs, double* d_z, void* stream);
FEM_API int fem_mg_vcycle_f32(int vec, int nlevels, const FemMGLevel* levels, int nu, int coarse_steps,
                              double ratio, const float* d_rhs, float* d_z, void* stream);
/* The V-cycle's coarse end (host query, no GPU work): *start = the first
 * level (>= 1) from which fem_mg_vcycle_* and the multigrid CG run the rest
 * of each V-cycle as one kernel on one CTA, its data in shared memory, and
 * *smem_bytes = the shared memory it takes; *start = -1 (and 0 bytes) when
 * every level runs as launches per step.  It depends on the levels' node
 * counts, FP16 copies, dense inverse and nu, on the call's nu and
 * coarse_steps, on fp32 (the hierarchy's type) and on FEM_MG_TAIL=0 in the
 * environment, which turns it off. */
FEM_API int fem_mg_tail_plan(int vec, int nlevels, const FemMGLevel* levels, int fp32, int nu, int coarse_steps,
                             int* start, size_t* smem_bytes);
/* CG on the FP64 operator (row_ptr, col_idx, vals) preconditioned by one
 * V-cycle per iteration, the linear solve of solver.py:63-92 / 261-284 with
 * a multigrid preconditioner.  levels_fp32 != 0: the hierarchy is FP32 (the
 * V-cycle runs in FP32 on a rounded copy of r; CG, its vectors and
 * reductions stay FP64, so the attainable accuracy is FP64's).  x holds the
 * initial guess.  Stops when ||b - A x|| <= max(rtol ||b||, atol) on the
 * recursive residual, then reports the true one in *h_relres. */
FEM_API size_t fem_mg_pcg_workspace_bytes(int vec, int64_t n_brows);
FEM_API int fem_mg_pcg_solve(int vec, int64_t n_brows, const int32_t* d_row_ptr, const int32_t* d_col_idx,
                             const double* d_vals, const double* d_b, double* d_x, double rtol, double atol,
                             int maxiter, int check_every, int nlevels, const FemMGLevel* levels,
                             int levels_fp32, int nu, int coarse_steps, double ratio, void* d_work,
                             size_t work_bytes, int* h_iters, double* h_relres, void* stream);
/* The same CG on an FP32 operator (an FP32-assembled tangent): the products
 * A p read FP32 values and accumulate in FP64, every vector and reduction is
 * FP64.  The solve is exact for the FP32 operator; for a Newton step that
 * operator is the tangent rounded to FP32. */
FEM_API int fem_mg_pcg_solve_mixed(int vec, int64_t n_brows, const int32_t* d_row_ptr, const int32_t* d_col_idx,
                                   const float* d_vals, const double* d_b, double* d_x, double rtol, double atol,
                                   int maxiter, int check_every, int nlevels, const FemMGLevel* levels,
                                   int levels_fp32, int nu, int coarse_steps, double ratio, void* d_work,
                                   size_t work_bytes, int* h_iters, double* h_relres, void* stream);

/* ---- dot product that allocates nothing ---------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory: code whose device memory is owned by a host framework's pool that
 * forbids raw cudaMalloc, or real-time loops that must not allocate once
 * running.  Same reduction as fem_dot_f64, but its scratch (per-block
 * partial sums, completion counter, result slot) is a file-scope static
 * __device__ array inside the library, and the result goes to the caller's
 * device double *d_out, asynchronously on `stream`.
 *  - n <= 16,777,216; larger n returns FEM_ERR_ARG.
 *  - The array (~32 KB) stays resident on every GPU that loads the library.
 *  - All calls share it: calls whose kernels overlap on the GPU race.
 *  - The first call on a device looks up the array's address
 *    (cudaGetSymbolAddress); make it before any stream capture.
 *  - `stream` must belong to the current device; a stream of another device
 *    returns FEM_ERR_ARG.
 * ------------------------------------------------------------------------ */
FEM_API int fem_dot_f64_noalloc(int64_t n, const double* d_x, const double* d_y, double* d_out,
                                void* stream);

#ifdef __cplusplus
}
#endif
#endif /* JAXFEM_B200_H */
