// 3D convolution (3x3x3, padding 1, stride 1) and GEMM on the 5th-generation
// tensor cores (tcgen05 + TMEM + TMA) for the learned warm-start network.
//
// One kernel template serves both:
//  MODE_CONV  implicit GEMM, out[v, co] = sum_{tap, ci} in[v + tap - 1, ci] W[co, tap, ci]
//             M = voxels (a 128-voxel brick per CTA), N = C_out, K = 27 C_in.
//             The A tile of each (tap, channel chunk) is one 5-D TMA box of
//             the NDHWC activation tensor shifted by the tap; TMA's zero fill
//             of out-of-range coordinates is the convolution's zero padding.
//             Epilogue: + bias, optional ReLU, BF16 store (NDHWC).
//             The input gradient (dgrad) is this same kernel applied to the
//             output gradient with tap-flipped, transposed weights.
//  MODE_GEMM  C[M, N] += A[M, K] B[N, K]^T (both K-major), split-K over
//             gridDim.z with FP32 atomic accumulation: the weight gradient
//             dW^T = im2col(X)^T dZ.
// Warp roles (128 threads): warp 0 lane 0 issues TMA loads into a 4-stage
// ring, warp 1 lane 0 issues tcgen05.mma (BF16 in, FP32 accumulate in TMEM)
// and commits each stage back to the producer, warp 2 owns the TMEM
// allocation, all 4 warps run the epilogue (tcgen05.ld of their 32 lanes).
// Every mbarrier wait is bounded; a timeout sets *err and the CTA skips the
// rest of its work, waits (bounded) for its own copies and frees its TMEM.
#include <cuda.h>

#include <mutex>

#include "common.cuh"
#include "tc_gemm.cuh"

namespace fem {
namespace {

constexpr int MODE_CONV = 0;
constexpr int MODE_GEMM = 1;
constexpr int kStages = 4;

struct TcParams {
  // conv geometry (MODE_CONV)
  int N, D, H, W, Cin;
  int bw, bh, bd, bn;  // 128-voxel brick
  int tw, th, td;      // bricks per dimension
  // gemm geometry (MODE_GEMM)
  int M, Ng, K;
  int kchunks_per_split;
  int ldc;
  // epilogue
  const float* bias;
  int relu;
  __nv_bfloat16* out;  // MODE_CONV: (voxels, BN)
  float* C;            // MODE_GEMM
  int* err;
};

template <int BN, int BK>
struct TcSmem {
  static constexpr int A_BYTES = 128 * BK * 2;
  static constexpr int B_BYTES = BN * BK * 2;
  static constexpr int A_STRIDE = (A_BYTES + 1023) / 1024 * 1024;
  static constexpr int B_STRIDE = (B_BYTES + 1023) / 1024 * 1024;
  static constexpr int STAGE = A_STRIDE + B_STRIDE;
  static constexpr int BAR_OFF = kStages * STAGE;
  static constexpr int TOTAL = BAR_OFF + 256 + 1024;  // barriers + tmem slot + alignment slack
};

template <int BN, int BK, int MODE>
__global__ void __launch_bounds__(128, 1) tc_kernel(const __grid_constant__ CUtensorMap tmA,
                                                    const __grid_constant__ CUtensorMap tmB,
                                                    const TcParams p) {
  using S = TcSmem<BN, BK>;
  constexpr int TMEM_COLS = BN < 32 ? 32 : BN;
  constexpr uint32_t IDESC = tc::idesc_bf16_f32(128, BN);
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                         ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S::BAR_OFF);
  uint64_t* empty = full + kStages;
  uint64_t* done = empty + kStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // ---- K iteration range ----
  int k_begin = 0, k_iters = 0;
  int n0 = 0, m0 = 0, d0 = 0, h0 = 0, w0 = 0;
  if constexpr (MODE == MODE_CONV) {
    k_iters = 27 * (p.Cin / BK);
    int t = blockIdx.x;
    const int wi = t % p.tw;
    t /= p.tw;
    const int hi = t % p.th;
    t /= p.th;
    const int di = t % p.td;
    const int ni = t / p.td;
    w0 = wi * p.bw;
    h0 = hi * p.bh;
    d0 = di * p.bd;
    n0 = ni * p.bn;
  } else {
    m0 = blockIdx.x * 128;
    n0 = blockIdx.y * BN;
    const int kc_total = (p.K + BK - 1) / BK;
    k_begin = blockIdx.z * p.kchunks_per_split;
    const int k_end = min(kc_total, k_begin + p.kchunks_per_split);
    k_iters = max(0, k_end - k_begin);
  }

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(done, 1);
    *abort_flag = 0;
    tc::fence_barrier_init();
    tc::prefetch_tmap(&tmA);
    tc::prefetch_tmap(&tmB);
  }
  if (warp == 2) tc::tmem_alloc(tmem_slot, TMEM_COLS);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer ----
    int armed = 0;
    for (int it = 0; it < k_iters; ++it) {
      const int s = it % kStages;
      if (it >= kStages && !tc::mbar_wait(&empty[s], ((it / kStages) - 1) & 1)) {
        atomicExch(p.err, 1);
        *((volatile int*)abort_flag) = 1;
        break;
      }
      if (*((volatile int*)abort_flag)) break;
      unsigned char* a_dst = smem + s * S::STAGE;
      unsigned char* b_dst = a_dst + S::A_STRIDE;
      tc::mbar_arrive_expect_tx(&full[s], S::A_BYTES + S::B_BYTES);
      if constexpr (MODE == MODE_CONV) {
        const int cpt = p.Cin / BK;
        const int tap = it / cpt;
        const int c0 = (it % cpt) * BK;
        const int kd = tap / 9, kh = (tap / 3) % 3, kw = tap % 3;
        tc::tma_load_5d(a_dst, &tmA, c0, w0 + kw - 1, h0 + kh - 1, d0 + kd - 1, n0, &full[s]);
        tc::tma_load_2d(b_dst, &tmB, tap * p.Cin + c0, 0, &full[s]);
      } else {
        const int kk = (k_begin + it) * BK;
        tc::tma_load_2d(a_dst, &tmA, kk, m0, &full[s]);
        tc::tma_load_2d(b_dst, &tmB, kk, n0, &full[s]);
      }
      armed = it + 1;
    }
    if (*((volatile int*)abort_flag)) {
      // let the copies this thread started land before the CTA exits
      for (int it = (armed > kStages ? armed - kStages : 0); it < armed; ++it)
        tc::mbar_wait(&full[it % kStages], (it / kStages) & 1);
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    bool ok = true;
    for (int it = 0; it < k_iters; ++it) {
      const int s = it % kStages;
      if (!tc::mbar_wait(&full[s], (it / kStages) & 1)) {
        atomicExch(p.err, 2);
        *((volatile int*)abort_flag) = 1;
        ok = false;
        break;
      }
      tc::tc_fence_after();
      const uint32_t a_addr = tc::smem_u32(smem + s * S::STAGE);
      const uint32_t b_addr = a_addr + S::A_STRIDE;
#pragma unroll
      for (int j = 0; j < BK / 16; ++j) {
        const uint64_t ad = tc::sdesc_kmajor(a_addr + j * 32, BK * 2);
        const uint64_t bd = tc::sdesc_kmajor(b_addr + j * 32, BK * 2);
        tc::umma_bf16(tmem, ad, bd, IDESC, (it > 0 || j > 0) ? 1u : 0u);
      }
      tc::umma_commit(&empty[s]);
    }
    if (ok) tc::umma_commit(done);
  }
  __syncwarp();

  // ---- epilogue: all 4 warps, thread = accumulator row ----
  bool have = k_iters > 0;
  if (have) {
    if (!tc::mbar_wait(done, 0)) {
      atomicExch(p.err, 3);
      have = false;
    }
  }
  if (*((volatile int*)abort_flag)) have = false;
  tc::tc_fence_after();
  const int r = warp * 32 + lane;
  const uint32_t trow = tmem + (uint32_t(warp * 32) << 16);
  if constexpr (MODE == MODE_CONV) {
    const int rw = r % p.bw, rh = (r / p.bw) % p.bh, rd = (r / (p.bw * p.bh)) % p.bd,
              rn = r / (p.bw * p.bh * p.bd);
    const int64_t vox = ((int64_t(n0 + rn) * p.D + (d0 + rd)) * p.H + (h0 + rh)) * p.W + (w0 + rw);
    __nv_bfloat16* dst = p.out + vox * BN;
#pragma unroll
    for (int c = 0; c < BN; c += 16) {
      float v[16];
      if (have) {
        tc::tmem_ld16(trow + c, v);
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = 0.0f;
      }
      if (p.bias != nullptr)
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] += p.bias[c + i];
      if (p.relu)
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i], 0.0f);
      uint4 pk[2];
      __nv_bfloat162* h2 = reinterpret_cast<__nv_bfloat162*>(pk);
#pragma unroll
      for (int i = 0; i < 8; ++i) h2[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
      reinterpret_cast<uint4*>(dst + c)[0] = pk[0];
      reinterpret_cast<uint4*>(dst + c)[1] = pk[1];
    }
  } else {
    const int m = m0 + r;
    if (have) {
#pragma unroll
      for (int c = 0; c < BN; c += 16) {
        float v[16];
        tc::tmem_ld16(trow + c, v);
        if (m < p.M) {
#pragma unroll
          for (int i = 0; i < 16; ++i)
            if (n0 + c + i < p.Ng) atomicAdd(p.C + int64_t(m) * p.ldc + n0 + c + i, v[i]);
        }
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 2) tc::tmem_dealloc(tmem, TMEM_COLS);
}

// ---- host helpers -----------------------------------------------------------
int* err_flag_device() {
  static std::mutex mu;
  static int* flags[64] = {nullptr};
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (flags[dev] == nullptr) {
    if (cudaMalloc(&flags[dev], sizeof(int)) != cudaSuccess) return nullptr;
    cudaMemset(flags[dev], 0, sizeof(int));
  }
  return flags[dev];
}

// cuTensorMapEncodeTiled through the runtime's driver entry-point lookup, so
// the library does not link libcuda (and loads on hosts without a driver).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static std::mutex mu;
  static EncodeTiledFn fn = nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (fn == nullptr) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

CUtensorMapSwizzle swizzle_for(int row_bytes) {
  return row_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                          : (row_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B);
}

int make_map_2d(CUtensorMap* m, const void* base, uint64_t inner, uint64_t outer, uint32_t box_inner,
                uint32_t box_outer) {
  const cuuint64_t dims[2] = {inner, outer};
  const cuuint64_t strides[1] = {inner * 2};
  const cuuint32_t box[2] = {box_inner, box_outer};
  const cuuint32_t es[2] = {1, 1};
  EncodeTiledFn enc = encode_tiled();
  if (enc == nullptr) {
    set_error("cuTensorMapEncodeTiled is unavailable (driver entry point lookup failed)");
    return FEM_ERR_CUDA;
  }
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims,
                                      strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(box_inner * 2),
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled(2d %llux%llu box %ux%u) failed: %d", (unsigned long long)inner,
              (unsigned long long)outer, box_inner, box_outer, int(r));
    return FEM_ERR_CUDA;
  }
  return FEM_OK;
}

int make_map_5d(CUtensorMap* m, const void* base, int C, int W, int H, int D, int N, uint32_t bc, uint32_t bw,
                uint32_t bh, uint32_t bd, uint32_t bn) {
  const cuuint64_t dims[5] = {cuuint64_t(C), cuuint64_t(W), cuuint64_t(H), cuuint64_t(D), cuuint64_t(N)};
  const cuuint64_t strides[4] = {cuuint64_t(C) * 2, cuuint64_t(W) * C * 2, cuuint64_t(H) * W * C * 2,
                                 cuuint64_t(D) * H * W * C * 2};
  const cuuint32_t box[5] = {bc, bw, bh, bd, bn};
  const cuuint32_t es[5] = {1, 1, 1, 1, 1};
  EncodeTiledFn enc = encode_tiled();
  if (enc == nullptr) {
    set_error("cuTensorMapEncodeTiled is unavailable (driver entry point lookup failed)");
    return FEM_ERR_CUDA;
  }
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(base), dims,
                                      strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(bc * 2),
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled(5d) failed: %d", int(r));
    return FEM_ERR_CUDA;
  }
  return FEM_OK;
}

template <int BN, int BK, int MODE>
int launch_tc(const CUtensorMap& a, const CUtensorMap& b, const TcParams& p, dim3 grid, cudaStream_t st) {
  using S = TcSmem<BN, BK>;
  auto k = tc_kernel<BN, BK, MODE>;
  static std::mutex mu;
  static bool set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  {
    std::lock_guard<std::mutex> lock(mu);
    if (!set[dev]) {
      FEM_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, S::TOTAL));
      set[dev] = true;
    }
  }
  k<<<grid, 128, S::TOTAL, st>>>(a, b, p);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}

// Dispatch on (BN, BK); BN in {16,32,64,128}, BK in {16,32,64}.
template <int MODE>
int dispatch_tc(int BN, int BK, const CUtensorMap& a, const CUtensorMap& b, const TcParams& p, dim3 grid,
                cudaStream_t st) {
#define FEM_TC_CASE(bn, bk) \
  if (BN == bn && BK == bk) return launch_tc<bn, bk, MODE>(a, b, p, grid, st);
  FEM_TC_CASE(16, 16) FEM_TC_CASE(16, 32) FEM_TC_CASE(16, 64)
  FEM_TC_CASE(32, 16) FEM_TC_CASE(32, 32) FEM_TC_CASE(32, 64)
  FEM_TC_CASE(64, 16) FEM_TC_CASE(64, 32) FEM_TC_CASE(64, 64)
  FEM_TC_CASE(128, 16) FEM_TC_CASE(128, 32) FEM_TC_CASE(128, 64)
#undef FEM_TC_CASE
  set_error("unsupported tile BN=%d BK=%d", BN, BK);
  return FEM_ERR_ARG;
}

int bk_for(int K) { return K % 64 == 0 ? 64 : (K % 32 == 0 ? 32 : 16); }

// ---- small layout kernels -------------------------------------------------------
// col_t[(tap*Cin + ci) * V + v] = x[v + tap - 1, ci] (zero outside the grid)
__global__ void im2col_t_kernel(const __nv_bfloat16* x, __nv_bfloat16* col, int N, int D, int H, int W, int C,
                                int64_t V) {
  const int64_t total = int64_t(27) * C * V;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t v = i % V;
    const int64_t row = i / V;
    const int ci = int(row % C), tap = int(row / C);
    int64_t t = v;
    const int w = int(t % W);
    t /= W;
    const int h = int(t % H);
    t /= H;
    const int d = int(t % D);
    const int n = int(t / D);
    const int dd = d + tap / 9 - 1, hh = h + (tap / 3) % 3 - 1, ww = w + tap % 3 - 1;
    __nv_bfloat16 val = __float2bfloat16(0.0f);
    if (dd >= 0 && dd < D && hh >= 0 && hh < H && ww >= 0 && ww < W)
      val = x[((((int64_t(n) * D + dd) * H + hh) * W + ww) * C) + ci];
    col[i] = val;
  }
}

__global__ void transpose_kernel(const __nv_bfloat16* in, __nv_bfloat16* out, int64_t rows, int cols) {
  const int64_t total = rows * cols;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = i / cols;
    const int c = int(i % cols);
    out[int64_t(c) * rows + r] = in[i];
  }
}

// wt[ci, tap, co] = w[co, 26 - tap, ci]  (dgrad weights)
__global__ void flip_weights_kernel(const __nv_bfloat16* w, __nv_bfloat16* wt, int Cout, int Cin) {
  const int total = Cout * 27 * Cin;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int ci = i % Cin, tap = (i / Cin) % 27, co = i / (Cin * 27);
    wt[(int64_t(ci) * 27 + (26 - tap)) * Cout + co] = w[i];
  }
}

__global__ void relu_mask_kernel(const __nv_bfloat16* dy, const __nv_bfloat16* y, __nv_bfloat16* dz, int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    dz[i] = __bfloat162float(y[i]) > 0.0f ? dy[i] : __float2bfloat16(0.0f);
}

unsigned grid_for(int64_t n) {
  const int64_t b = (n + 255) / 256;
  const int64_t cap = int64_t(num_sms()) * 16;
  return unsigned(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace
}  // namespace fem

using namespace fem;

extern "C" int fem_conv3d_fwd_bf16(const void* d_in, const void* d_w, const float* d_bias, void* d_out, int N,
                                   int D, int H, int W, int Cin, int Cout, int relu, void* stream) {
  FEM_CHECK_ARG(N > 0 && D > 0 && H > 0 && W > 0, "empty tensor");
  FEM_CHECK_ARG(Cin % 16 == 0 && Cin >= 16 && Cin <= 4096, "Cin must be a multiple of 16 (got %d)", Cin);
  FEM_CHECK_ARG(Cout == 16 || Cout == 32 || Cout == 64 || Cout == 128, "Cout must be 16/32/64/128 (got %d)", Cout);
  FEM_CHECK_ARG(d_in && d_w && d_out, "NULL tensor");
  FEM_CHECK_ARG((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_w) |
                 reinterpret_cast<uintptr_t>(d_out)) % 16 == 0, "tensors must be 16-byte aligned");
  // 128-voxel brick: whole rows of W first, then H, D, N
  TcParams p{};
  p.N = N; p.D = D; p.H = H; p.W = W; p.Cin = Cin;
  p.bw = W < 128 ? W : 128;
  p.bh = H < 128 / p.bw ? H : 128 / p.bw;
  p.bd = D < 128 / (p.bw * p.bh) ? D : 128 / (p.bw * p.bh);
  p.bn = 128 / (p.bw * p.bh * p.bd);
  FEM_CHECK_ARG(p.bw * p.bh * p.bd * p.bn == 128 && W % p.bw == 0 && H % p.bh == 0 && D % p.bd == 0 &&
                N % p.bn == 0 && p.bw <= 256 && p.bh <= 256 && p.bd <= 256 && p.bn <= 256,
                "grid (N=%d, D=%d, H=%d, W=%d) does not tile into 128-voxel bricks", N, D, H, W);
  p.tw = W / p.bw; p.th = H / p.bh; p.td = D / p.bd;
  const int64_t tiles = int64_t(p.tw) * p.th * p.td * (N / p.bn);
  FEM_CHECK_ARG(tiles < (int64_t(1) << 31), "too many tiles");
  p.bias = d_bias;
  p.relu = relu;
  p.out = static_cast<__nv_bfloat16*>(d_out);
  p.err = err_flag_device();
  FEM_CHECK_ARG(p.err != nullptr, "error flag allocation failed");
  const int BK = bk_for(Cin);
  CUtensorMap ta, tb;
  int rc = make_map_5d(&ta, d_in, Cin, W, H, D, N, BK, p.bw, p.bh, p.bd, p.bn);
  if (rc) return rc;
  rc = make_map_2d(&tb, d_w, uint64_t(27) * Cin, Cout, BK, Cout);
  if (rc) return rc;
  return dispatch_tc<MODE_CONV>(Cout, BK, ta, tb, p, dim3(unsigned(tiles)), as_stream(stream));
}

extern "C" int fem_gemm_bf16_tn_f32(const void* d_a, const void* d_b, float* d_c, int M, int N, int K, int ldc,
                                    int split_k, void* stream) {
  FEM_CHECK_ARG(M > 0 && N > 0 && K > 0, "empty GEMM");
  FEM_CHECK_ARG(K % 16 == 0, "K must be a multiple of 16 (got %d)", K);
  FEM_CHECK_ARG(N == 16 || N == 32 || N == 64 || N % 128 == 0, "N must be 16/32/64 or a multiple of 128");
  FEM_CHECK_ARG(ldc >= N && split_k >= 1, "bad ldc/split_k");
  FEM_CHECK_ARG((reinterpret_cast<uintptr_t>(d_a) | reinterpret_cast<uintptr_t>(d_b)) % 16 == 0,
                "operands must be 16-byte aligned");
  const int BN = N < 128 ? N : 128;
  const int BK = bk_for(K);
  TcParams p{};
  p.M = M; p.Ng = N; p.K = K; p.ldc = ldc;
  const int kc = (K + BK - 1) / BK;
  p.kchunks_per_split = (kc + split_k - 1) / split_k;
  const int splits = (kc + p.kchunks_per_split - 1) / p.kchunks_per_split;
  p.C = d_c;
  p.err = err_flag_device();
  FEM_CHECK_ARG(p.err != nullptr, "error flag allocation failed");
  CUtensorMap ta, tb;
  int rc = make_map_2d(&ta, d_a, K, M, BK, 128);
  if (rc) return rc;
  rc = make_map_2d(&tb, d_b, K, N, BK, BN);
  if (rc) return rc;
  dim3 grid(unsigned((M + 127) / 128), unsigned(N / BN), unsigned(splits));
  return dispatch_tc<MODE_GEMM>(BN, BK, ta, tb, p, grid, as_stream(stream));
}

extern "C" int fem_tc_error(int* h_err, int reset) {
  int* e = err_flag_device();
  FEM_CHECK_ARG(e != nullptr && h_err != nullptr, "error flag unavailable");
  FEM_CUDA_TRY(cudaMemcpy(h_err, e, sizeof(int), cudaMemcpyDeviceToHost));
  if (reset) FEM_CUDA_TRY(cudaMemset(e, 0, sizeof(int)));
  return FEM_OK;
}

extern "C" int fem_conv3d_im2col_t_bf16(const void* d_x, void* d_col, int N, int D, int H, int W, int C,
                                        void* stream) {
  FEM_CHECK_ARG(N > 0 && D > 0 && H > 0 && W > 0 && C > 0, "empty tensor");
  const int64_t V = int64_t(N) * D * H * W;
  im2col_t_kernel<<<grid_for(27 * C * V), 256, 0, as_stream(stream)>>>(
      static_cast<const __nv_bfloat16*>(d_x), static_cast<__nv_bfloat16*>(d_col), N, D, H, W, C, V);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}

extern "C" int fem_transpose_bf16(const void* d_in, void* d_out, int64_t rows, int cols, void* stream) {
  FEM_CHECK_ARG(rows > 0 && cols > 0, "empty tensor");
  transpose_kernel<<<grid_for(rows * cols), 256, 0, as_stream(stream)>>>(
      static_cast<const __nv_bfloat16*>(d_in), static_cast<__nv_bfloat16*>(d_out), rows, cols);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}

extern "C" int fem_conv3d_flip_weights_bf16(const void* d_w, void* d_wt, int Cout, int Cin, void* stream) {
  FEM_CHECK_ARG(Cout > 0 && Cin > 0, "empty weights");
  flip_weights_kernel<<<grid_for(int64_t(Cout) * 27 * Cin), 256, 0, as_stream(stream)>>>(
      static_cast<const __nv_bfloat16*>(d_w), static_cast<__nv_bfloat16*>(d_wt), Cout, Cin);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}

extern "C" int fem_relu_mask_bf16(const void* d_dy, const void* d_y, void* d_dz, int64_t n, void* stream) {
  FEM_CHECK_ARG(n >= 0, "negative size");
  if (n == 0) return FEM_OK;
  relu_mask_kernel<<<grid_for(n), 256, 0, as_stream(stream)>>>(static_cast<const __nv_bfloat16*>(d_dy),
                                                              static_cast<const __nv_bfloat16*>(d_y),
                                                              static_cast<__nv_bfloat16*>(d_dz), n);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}
