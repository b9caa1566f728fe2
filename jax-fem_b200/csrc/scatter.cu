// Scatter of dense cell residuals and cell matrices into the global residual
// and a scalar (1x1-block) CSR tangent, for the cell-kernel path: problems
// whose weak form is user code (universal kernels, multi-variable problems,
// tensor maps other than the registered laws) evaluated on the device by the
// host, with the cell Jacobians from forward-mode differentiation.
//
// Replaces, for that path, the residual scatter of
// compute_residual_vars_helper (problem.py:471-483) and the PETSc COO value
// insertion + zeroRows of get_A (solver.py:466-491): every cell matrix entry
// (a, b) adds into the CSR value of (dofs[a], dofs[b]) through the
// precomputed cell -> entry map (fem_bsr_pattern_nen with the cell dof table
// as "cells"), Dirichlet rows and columns eliminated, K_ab d_b added to the
// lift of free row a for prescribed columns b.  No symmetry is assumed.
//
// One thread per (item, a, b): consecutive threads read consecutive entries
// of the item's nd x nd matrix (coalesced) and of its scatter-map row.
#include "common.cuh"
#include "tangent.cuh"

namespace fem {
namespace {

template <typename T>
__global__ void __launch_bounds__(256) scatter_cells_kernel(int nd, int64_t items, const int32_t* __restrict__ item_cell,
                                                            const int32_t* __restrict__ cell_dofs,
                                                            const int32_t* __restrict__ scatter,
                                                            const double* __restrict__ item_res,
                                                            const double* __restrict__ item_jac,
                                                            const uint8_t* __restrict__ bc,
                                                            const double* __restrict__ dvec, double* res, double* lift,
                                                            T* vals) {
  const int64_t nn = int64_t(nd) * nd;
  const int64_t total = items * nn;
  for (int64_t w = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; w < total;
       w += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = w / nn;
    const int e = int(w - i * nn);
    const int a = e / nd, b = e - (e / nd) * nd;
    const int64_t c = item_cell != nullptr ? int64_t(item_cell[i]) : i;
    const int32_t ra = cell_dofs[c * nd + a];
    if (b == 0 && res != nullptr && item_res != nullptr) atomicAdd(res + ra, item_res[i * nd + a]);
    if (item_jac == nullptr) continue;
    const double K = item_jac[w];
    const int32_t rb = cell_dofs[c * nd + b];
    const bool bra = bc != nullptr && bc[ra];
    const bool brb = bc != nullptr && bc[rb];
    if (lift != nullptr && !bra && dvec[rb] != 0.0) atomicAdd(lift + ra, K * dvec[rb]);
    if (vals != nullptr && !bra && !brb) atomicAdd(vals + scatter[c * nn + e], T(K));
  }
}

template <typename T>
int scatter_impl(int nd, int64_t num_items, const int32_t* d_item_cell, const int32_t* d_cell_dofs,
                 const int32_t* d_scatter, const double* d_item_res, const double* d_item_jac, const uint8_t* d_bc,
                 const double* d_dvec, double* d_res, double* d_lift, T* d_vals, void* stream) {
  FEM_CHECK_ARG(nd >= 1 && nd <= 256, "cell dofs %d outside [1, 256]", nd);
  FEM_CHECK_ARG(num_items >= 0, "negative size");
  FEM_CHECK_ARG(num_items == 0 || d_cell_dofs != nullptr, "cell dof table is NULL");
  FEM_CHECK_ARG(d_vals == nullptr || (d_scatter != nullptr && d_item_jac != nullptr),
                "tangent values need the scatter map and the cell matrices");
  FEM_CHECK_ARG(d_lift == nullptr || (d_dvec != nullptr && d_item_jac != nullptr),
                "lift needs dvec and the cell matrices");
  FEM_CHECK_ARG(d_res == nullptr || d_item_res != nullptr, "residual needs the cell residuals");
  if (num_items == 0) return FEM_OK;
  const int64_t total = num_items * nd * nd;
  const int64_t blocks = (total + 255) / 256;
  const unsigned grid = unsigned(blocks < int64_t(num_sms()) * 32 ? blocks : int64_t(num_sms()) * 32);
  scatter_cells_kernel<T><<<grid, 256, 0, as_stream(stream)>>>(nd, num_items, d_item_cell, d_cell_dofs, d_scatter,
                                                                d_item_res, d_item_jac, d_bc, d_dvec, d_res, d_lift,
                                                                d_vals);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}

template <typename T>
int bc_diag_impl(int vec, int64_t n_brows, const uint8_t* d_bc, const int32_t* d_diag, T* d_vals, void* stream) {
  FEM_CHECK_ARG(vec >= 1 && vec <= 3, "vec %d", vec);
  FEM_CHECK_ARG(n_brows >= 0, "negative size");
  FEM_CHECK_ARG(n_brows == 0 || (d_bc != nullptr && d_diag != nullptr && d_vals != nullptr), "NULL pointer");
  const int64_t ndofs = n_brows * vec;
  if (ndofs == 0) return FEM_OK;
  bc_diag_kernel<T><<<unsigned((ndofs + 255) / 256), 256, 0, as_stream(stream)>>>(vec, ndofs, d_bc, d_diag, d_vals);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}

}  // namespace
}  // namespace fem

extern "C" int fem_scatter_cells_f64(int nd, int64_t num_items, const int32_t* d_item_cell,
                                     const int32_t* d_cell_dofs, const int32_t* d_scatter, const double* d_item_res,
                                     const double* d_item_jac, const uint8_t* d_bc_mask, const double* d_dvec,
                                     double* d_res, double* d_lift, double* d_vals, void* stream) {
  return fem::scatter_impl<double>(nd, num_items, d_item_cell, d_cell_dofs, d_scatter, d_item_res, d_item_jac,
                                   d_bc_mask, d_dvec, d_res, d_lift, d_vals, stream);
}

extern "C" int fem_scatter_cells_f32(int nd, int64_t num_items, const int32_t* d_item_cell,
                                     const int32_t* d_cell_dofs, const int32_t* d_scatter, const double* d_item_res,
                                     const double* d_item_jac, const uint8_t* d_bc_mask, const double* d_dvec,
                                     double* d_res, double* d_lift, float* d_vals, void* stream) {
  return fem::scatter_impl<float>(nd, num_items, d_item_cell, d_cell_dofs, d_scatter, d_item_res, d_item_jac,
                                  d_bc_mask, d_dvec, d_res, d_lift, d_vals, stream);
}

extern "C" int fem_bsr_bc_diag_f64(int vec, int64_t n_brows, const uint8_t* d_bc_mask, const int32_t* d_diag,
                                   double* d_vals, void* stream) {
  return fem::bc_diag_impl<double>(vec, n_brows, d_bc_mask, d_diag, d_vals, stream);
}

extern "C" int fem_bsr_bc_diag_f32(int vec, int64_t n_brows, const uint8_t* d_bc_mask, const int32_t* d_diag,
                                   float* d_vals, void* stream) {
  return fem::bc_diag_impl<float>(vec, n_brows, d_bc_mask, d_diag, d_vals, stream);
}
