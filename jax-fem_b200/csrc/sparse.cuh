// Block-CSR row kernels shared by the SpMV entry points and the Krylov solvers.
#pragma once
#include <cuda_fp16.h>

#include "common.cuh"

namespace fem {

// Compile-time tuning of the row kernels (defaults measured on B200).
#ifndef FEM_ROW_STAGE_BYTES
#define FEM_ROW_STAGE_BYTES 4096
#endif
#ifndef FEM_ROW_BLOCKS_PER_SM
#define FEM_ROW_BLOCKS_PER_SM 4
#endif
#ifndef FEM_ROW_GROUP_F32
#define FEM_ROW_GROUP_F32 4
#endif
#ifndef FEM_ROW_GROUP_F64
#define FEM_ROW_GROUP_F64 2
#endif
#ifndef FEM_ROW_GROUP_MIXED
#define FEM_ROW_GROUP_MIXED 3
#endif

constexpr int kRowThreads = 256;   // 8 warps per block
constexpr int kStageBytes = FEM_ROW_STAGE_BYTES;     // per-warp shared-memory stage for matrix values
constexpr int kRowBlocksPerSM = FEM_ROW_BLOCKS_PER_SM;  // resident blocks per SM the row kernels are sized for

// Block rows per warp group: ~3.9 KB of FP32 or FP64 3x3 blocks; FP32
// values with FP64 accumulation take 3 rows, the most that stay within the
// registers of kRowBlocksPerSM resident blocks without spills (3 measured
// ~1 % faster per multigrid CG iteration than 2 on the 50^3 tangent).
template <typename VT, typename AT = VT>
__host__ __device__ constexpr int rows_per_warp() {
  return (sizeof(VT) <= 4 && sizeof(AT) == 4) ? FEM_ROW_GROUP_F32  // FP32 or FP16 values, FP32 sums
         : (sizeof(VT) == 4)                      ? FEM_ROW_GROUP_MIXED
                                                  : FEM_ROW_GROUP_F64;
}

// Dynamic shared memory a bsr_rows kernel needs (one stage per warp).
constexpr size_t bsr_rows_smem() { return size_t(kRowThreads / 32) * (kStageBytes + 16); }

// The row kernels copy matrix values with 16-byte cp.async transfers: the
// values must start on a 16-byte boundary (and the column indices, read as
// int32, on a 4-byte one).
inline bool bsr_aligned(const void* vals, const void* col_idx) {
  return (reinterpret_cast<uintptr_t>(vals) & 15u) == 0 && (reinterpret_cast<uintptr_t>(col_idx) & 3u) == 0;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Grid-stride loop in which each warp owns groups of R consecutive block rows
// (R = rows_per_warp<VT>()).  The values of a group are one contiguous byte
// range; the warp copies it into its shared-memory stage with 16-byte
// cp.async transfers (fully coalesced, no registers), and while those are in
// flight it gathers the column indices and x values.  Lane l then handles
// blocks l, l+32, ... of each row from shared memory (a HEX8 interior row has
// 27 blocks).  XF fetches x by dof index (callers may form x on the fly);
// EPI(row, out[VEC], lane) consumes the warp-reduced row result.  Groups too
// large for the stage (very high-degree rows) read values directly.
template <int VEC, typename VT, typename AT, class XF, class EPI>
__device__ __forceinline__ void bsr_rows(int64_t n_brows, const int32_t* __restrict__ rp,
                                         const int32_t* __restrict__ ci,
                                         const VT* __restrict__ vals, XF xf, EPI epi) {
  constexpr int R = rows_per_warp<VT, AT>();
  constexpr int VV = VEC * VEC;
  extern __shared__ __align__(16) unsigned char bsr_smem[];
  unsigned char* stage = bsr_smem + (threadIdx.x >> 5) * (kStageBytes + 16);
  const int lane = threadIdx.x & 31;
  const int64_t gw = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int64_t ngw = int64_t(gridDim.x) * (blockDim.x >> 5);
  const int64_t total_bytes = int64_t(rp[n_brows]) * VV * int64_t(sizeof(VT));
  const int64_t full_chunks = total_bytes >> 4;  // 16-byte chunks entirely inside vals
  for (int64_t g = gw; g * R < n_brows; g += ngw) {
    const int64_t row0 = g * R;
    // rp[row0 .. row0+R] with one coalesced load
    const int64_t nr = (n_brows - row0) < R ? (n_brows - row0) : R;
    const int rpv = lane <= nr ? rp[row0 + lane] : 0;
    int s[R + 1];
#pragma unroll
    for (int r = 0; r <= R; ++r) s[r] = __shfl_sync(0xffffffffu, rpv, r <= nr ? r : int(nr));
    const int64_t byte0 = int64_t(s[0]) * VV * int64_t(sizeof(VT));
    const int64_t byte1 = int64_t(s[R]) * VV * int64_t(sizeof(VT));
    const int64_t c0 = byte0 >> 4, c1 = (byte1 + 15) >> 4;
    const bool staged = (c1 - c0) * 16 <= kStageBytes;
    if (staged) {
      const unsigned char* gsrc = reinterpret_cast<const unsigned char*>(vals);
      for (int64_t c = c0 + lane; c < c1; c += 32) {
        unsigned char* dst = stage + (c - c0) * 16;
        if (c < full_chunks) {
          cp_async16(dst, gsrc + c * 16);
        } else {  // ragged tail of the array: element-wise, inside bounds only
          for (int k = 0; k < 16 / int(sizeof(VT)); ++k) {
            const int64_t byte = c * 16 + k * int64_t(sizeof(VT));
            if (byte < total_bytes)
              reinterpret_cast<VT*>(dst)[k] = __ldg(reinterpret_cast<const VT*>(gsrc + byte));
          }
        }
      }
    }
    // gathers while the stage fills
    int64_t col[R];
    AT xv[R][VEC];
    int maxlen = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) maxlen = max(maxlen, s[r + 1] - s[r]);
    AT acc[R][VEC];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int i = 0; i < VEC; ++i) acc[r][i] = AT(0);
    for (int off = 0; off < maxlen; off += 32) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int k = s[r] + off + lane;
        col[r] = k < s[r + 1] ? int64_t(ci[k]) : -1;
      }
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int c = 0; c < VEC; ++c) xv[r][c] = col[r] >= 0 ? AT(xf(col[r] * VEC + c)) : AT(0);
      if (staged && off == 0) {
        cp_async_wait_all();
        __syncwarp();
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (col[r] < 0) continue;
        const int k = s[r] + off + lane;
        const VT* bv = staged ? reinterpret_cast<const VT*>(stage + (int64_t(k) * VV * int64_t(sizeof(VT)) - c0 * 16))
                              : vals + int64_t(k) * VV;
#pragma unroll
        for (int i = 0; i < VEC; ++i)
#pragma unroll
          for (int c = 0; c < VEC; ++c) acc[r][i] = fma(AT(bv[i * VEC + c]), xv[r][c], acc[r][i]);
      }
    }
    if (staged && maxlen == 0) {
      cp_async_wait_all();
    }
    __syncwarp();  // stage reused by the next group
    // Transposed reduction of the NV = R*VEC row sums: each halving step
    // trades half of the values with the partner lane, so NV sums cost
    // P-1 + (5 - log2 P) shuffles (P = NV rounded up to a power of two)
    // instead of 5 NV.  Value j ends in lanes j * 2^(5 - log2 P) onwards.
    constexpr int NV = R * VEC;
    constexpr int P = NV <= 2 ? 2 : NV <= 4 ? 4 : NV <= 8 ? 8 : NV <= 16 ? 16 : 32;
    constexpr int L = P == 2 ? 1 : P == 4 ? 2 : P == 8 ? 3 : P == 16 ? 4 : 5;
    static_assert(NV <= 32, "at most 32 row sums per group");
    AT v[P];
#pragma unroll
    for (int j = 0; j < P; ++j) v[j] = j < NV ? acc[j / VEC][j % VEC] : AT(0);
#pragma unroll
    for (int step = 0; step < L; ++step) {
      const int o = 16 >> step;
      const bool up = (lane & o) != 0;
      const int half = P >> (step + 1);
#pragma unroll
      for (int i = 0; i < half; ++i) {
        const AT send = up ? v[i] : v[i + half];
        const AT keep = up ? v[i + half] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
      }
    }
    AT t = v[0];
#pragma unroll
    for (int o = (16 >> L); o >= 1; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    const int j = (lane >> (5 - L)) & (P - 1);
    if ((lane & ((1 << (5 - L)) - 1)) == 0 && j < NV) {
      const int64_t row = row0 + j / VEC;
      if (row < n_brows) epi(row, j % VEC, t);
    }
  }
}

// Opt a bsr_rows kernel into its dynamic shared memory (> 48 KB) once per
// kernel and device.
int ensure_smem_attr_ptr(const void* kernel);
template <typename K>
inline int ensure_smem_attr(K* kernel) {
  return ensure_smem_attr_ptr(reinterpret_cast<const void*>(kernel));
}

template <typename VT>
inline unsigned row_grid(int64_t n_brows) {
  const int64_t groups = (n_brows + rows_per_warp<VT>() - 1) / rows_per_warp<VT>();
  const int64_t blocks_needed = (groups + (kRowThreads / 32) - 1) / (kRowThreads / 32);
  const int64_t cap = int64_t(num_sms()) * kRowBlocksPerSM;
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
