// Block-CSR row kernels shared by the SpMV entry points and the Krylov solvers.
#pragma once
#include "common.cuh"

namespace fem {

constexpr int kRowThreads = 256;  // 8 warps per block, one warp per block row

// One warp computes out = sum_k A(row, k) x(col_k) for one block row; lane l
// owns blocks l, l+32, ... of the row (a HEX8 interior row has 27 blocks, so
// one pass).  XF fetches x by dof index so callers can form x on the fly.
template <int VEC, typename VT, typename AT, class XF>
__device__ __forceinline__ void bsr_row(int64_t row, int lane, const int32_t* __restrict__ rp,
                                        const int32_t* __restrict__ ci,
                                        const VT* __restrict__ vals, XF xf, AT out[VEC]) {
  AT acc[VEC];
#pragma unroll
  for (int r = 0; r < VEC; ++r) acc[r] = AT(0);
  const int s = rp[row], e = rp[row + 1];
  for (int k = s + lane; k < e; k += 32) {
    const int64_t col = ci[k];
    AT xv[VEC];
#pragma unroll
    for (int c = 0; c < VEC; ++c) xv[c] = AT(xf(col * VEC + c));
    const VT* bv = vals + int64_t(k) * (VEC * VEC);
#pragma unroll
    for (int r = 0; r < VEC; ++r)
#pragma unroll
      for (int c = 0; c < VEC; ++c) acc[r] = fma(AT(__ldg(bv + r * VEC + c)), xv[c], acc[r]);
  }
#pragma unroll
  for (int r = 0; r < VEC; ++r) out[r] = warp_sum(acc[r]);
}

inline unsigned row_grid(int64_t n_brows) {
  // grid-stride: at most 8 resident blocks per SM worth of warps
  const int64_t blocks_needed = (n_brows + (kRowThreads / 32) - 1) / (kRowThreads / 32);
  const int64_t cap = int64_t(num_sms()) * 8;
  return unsigned(blocks_needed < cap ? (blocks_needed > 0 ? blocks_needed : 1) : cap);
}

inline unsigned vec_grid(int64_t n) {
  const int64_t blocks_needed = (n + 255) / 256;
  const int64_t cap = int64_t(num_sms()) * 8;
  return unsigned(blocks_needed < cap ? (blocks_needed > 0 ? blocks_needed : 1) : cap);
}

// Block-wide sum of NV doubles; result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double v[NV], double* sred /* 32*NV */) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = warp_sum(v[i]);
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < NV; ++i) sred[wid * NV + i] = v[i];
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = lane < nw ? sred[lane * NV + i] : 0.0;
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = warp_sum(v[i]);
  }
}

// Deterministic two-stage reduction: every block stores its partial sums,
// the last block to finish adds them in block order and returns true (in
// thread 0 only, with the totals in tot[]).
template <int NV>
__device__ __forceinline__ bool last_block_reduce(double v[NV], double* partials,
                                                  unsigned int* counter, double tot[NV]) {
  __shared__ double sred[32 * NV];
  __shared__ bool is_last;
  block_sum<NV>(v, sred);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) partials[blockIdx.x * NV + i] = v[i];
    __threadfence();
    const unsigned int done = atomicAdd(counter, 1u);
    is_last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  double acc[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) acc[i] = 0.0;
  // fixed-order sum: thread t adds blocks t, t+blockDim, ... then tree
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
    for (int i = 0; i < NV; ++i) acc[i] += ((volatile double*)partials)[b * NV + i];
  __syncthreads();
  block_sum<NV>(acc, sred);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) tot[i] = acc[i];
    *counter = 0u;
  }
  return threadIdx.x == 0;
}

}  // namespace fem
