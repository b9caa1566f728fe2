// Passes shared by the cell-assembly kernels (assemble.cu: HEX8; element.cu:
// the other element types) after they have written the upper block triangle
// of the tangent.
#pragma once

#include "common.cuh"

namespace fem {
namespace {

// Node flag beside the Dirichlet bits 0..2: d != 0 at the node (the node
// contributes to the Dirichlet lift).
constexpr int kLiftBit = 8;

// Lower-triangle blocks as transposes of their upper partners: block k of
// row i, column j < i, takes block tmap[k] = (j, i) transposed.  In the
// row-sorted layout tmap[k] < k holds exactly for those blocks.  One thread
// per value word: consecutive threads store consecutive words (coalesced),
// and the VEC*VEC threads of a block read one partner block.
template <int VEC, typename T>
__global__ void mirror_lower_kernel(int64_t nnzb, const int32_t* __restrict__ tmap, T* vals) {
  constexpr int VV = VEC * VEC;
  const int64_t nwords = nnzb * VV;
  for (int64_t w = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; w < nwords;
       w += int64_t(gridDim.x) * blockDim.x) {
    const int64_t k = w / VV;
    const int e = int(w - k * VV);
    const int64_t p = tmap[k];
    if (p >= k) continue;
    const int r = e / VEC, c = e - (e / VEC) * VEC;
    vals[w] = vals[p * VV + c * VEC + r];
  }
}

// Unit diagonal at Dirichlet dofs of the eliminated tangent.
template <typename T>
__global__ void bc_diag_kernel(int vec, int64_t ndofs, const uint8_t* bc, const int32_t* diag,
                               T* vals) {
  const int64_t d = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (d >= ndofs || !bc[d]) return;
  const int64_t node = d / vec;
  const int i = int(d % vec);
  vals[int64_t(diag[node]) * vec * vec + i * vec + i] = T(1);
}

// The two passes above, in order, on stream st.
template <typename T>
int finish_tangent(int vec, int64_t nnzb, int64_t ndofs, const int32_t* d_transpose,
                   const uint8_t* d_bc, const int32_t* d_diag, T* d_vals, cudaStream_t st) {
  const int64_t blocks = (nnzb * vec * vec + 255) / 256;
  const unsigned grid = unsigned(blocks < int64_t(num_sms()) * 16 ? blocks : int64_t(num_sms()) * 16);
  if (grid > 0) {
    if (vec == 3)
      mirror_lower_kernel<3, T><<<grid, 256, 0, st>>>(nnzb, d_transpose, d_vals);
    else
      mirror_lower_kernel<1, T><<<grid, 256, 0, st>>>(nnzb, d_transpose, d_vals);
    FEM_LAUNCH_CHECK();
  }
  if (d_bc != nullptr && ndofs > 0) {
    bc_diag_kernel<T><<<unsigned((ndofs + 255) / 256), 256, 0, st>>>(vec, ndofs, d_bc, d_diag, d_vals);
    FEM_LAUNCH_CHECK();
  }
  return FEM_OK;
}

}  // namespace
}  // namespace fem
