// Block-CSR SpMV, mixed-precision refinement residual, dot product and the
// Newton right-hand side.  All HBM-streaming kernels.
#include <mutex>

#include "sparse.cuh"

namespace fem {
namespace {

template <int VEC, typename VT, typename XT, typename YT>
__global__ void __launch_bounds__(kRowThreads, kRowBlocksPerSM) spmv_kernel(int64_t n_brows, const int32_t* rp,
                                                          const int32_t* ci, const VT* vals,
                                                          const XT* __restrict__ x, YT* y) {
  using AT = typename std::conditional<(sizeof(VT) == 8 || sizeof(XT) == 8), double, float>::type;
  bsr_rows<VEC, VT, AT>(
      n_brows, rp, ci, vals, [&](int64_t i) { return x[i]; },
      [&](int64_t row, int c, AT val) {
        y[row * VEC + c] = YT(val);
      });
}

// r = b - A x (A f32, x/b/r f64, f64 accumulation)
template <int VEC>
__global__ void __launch_bounds__(kRowThreads, kRowBlocksPerSM) residual_mixed_kernel(int64_t n_brows, const int32_t* rp,
                                                                    const int32_t* ci, const float* vals,
                                                                    const double* __restrict__ x,
                                                                    const double* b, double* r) {
  bsr_rows<VEC, float, double>(
      n_brows, rp, ci, vals, [&](int64_t i) { return x[i]; },
      [&](int64_t row, int c, double val) {
        r[row * VEC + c] = b[row * VEC + c] - val;
      });
}

__global__ void dot_kernel(int64_t n, const double* x, const double* y, double* partials,
                           unsigned int* counter, double* out) {
  double v[1] = {0.0};
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    v[0] = fma(x[i], y[i], v[0]);
  double tot[1];
  if (last_block_reduce<1>(v, partials, counter, tot)) *out = tot[0];
}

__global__ void newton_rhs_kernel(int64_t n, const double* res, const double* fext,
                                  const double* lift, const uint8_t* bc, const double* u,
                                  const double* ubc, double* rbc, double* rhs, double* partials,
                                  unsigned int* counter, double* out) {
  double v[1] = {0.0};
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const double R = res[i] + (fext ? fext[i] : 0.0);
    double rb, rh;
    if (bc != nullptr && bc[i]) {
      rb = u[i] - ubc[i];
      rh = -rb;
    } else {
      rb = R;
      rh = -(R + (lift ? lift[i] : 0.0));
    }
    if (rbc) rbc[i] = rb;
    if (rhs) rhs[i] = rh;
    v[0] = fma(rb, rb, v[0]);
  }
  double tot[1];
  if (out != nullptr) {
    if (last_block_reduce<1>(v, partials, counter, tot)) *out = tot[0];
  }
}

}  // namespace
}  // namespace fem

using namespace fem;

extern "C" int fem_bsr_spmv_f64(int vec, int64_t n_brows, const int32_t* d_row_ptr,
                                const int32_t* d_col_idx, const double* d_vals, const double* d_x,
                                double* d_y, void* stream) {
  FEM_CHECK_ARG(vec == 1 || vec == 3, "vec must be 1 or 3");
  FEM_CHECK_ARG(n_brows >= 0, "negative size");
  FEM_CHECK_ARG(bsr_aligned(d_vals, d_col_idx), "vals and col_idx must be 16-byte aligned");
  if (n_brows == 0) return FEM_OK;
  auto st = as_stream(stream);
  int rc = ensure_smem_attr(vec == 3 ? spmv_kernel<3, double, double, double> : spmv_kernel<1, double, double, double>);
  if (rc != FEM_OK) return rc;
  if (vec == 3)
    spmv_kernel<3, double, double, double><<<row_grid<double>(n_brows), kRowThreads, bsr_rows_smem(), st>>>(n_brows, d_row_ptr, d_col_idx, d_vals, d_x, d_y);
  else
    spmv_kernel<1, double, double, double><<<row_grid<double>(n_brows), kRowThreads, bsr_rows_smem(), st>>>(n_brows, d_row_ptr, d_col_idx, d_vals, d_x, d_y);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}

extern "C" int fem_bsr_spmv_f32(int vec, int64_t n_brows, const int32_t* d_row_ptr,
                                const int32_t* d_col_idx, const float* d_vals, const float* d_x,
                                float* d_y, void* stream) {
  FEM_CHECK_ARG(vec == 1 || vec == 3, "vec must be 1 or 3");
  FEM_CHECK_ARG(n_brows >= 0, "negative size");
  FEM_CHECK_ARG(bsr_aligned(d_vals, d_col_idx), "vals and col_idx must be 16-byte aligned");
  if (n_brows == 0) return FEM_OK;
  auto st = as_stream(stream);
  int rc = ensure_smem_attr(vec == 3 ? spmv_kernel<3, float, float, float> : spmv_kernel<1, float, float, float>);
  if (rc != FEM_OK) return rc;
  if (vec == 3)
    spmv_kernel<3, float, float, float><<<row_grid<float>(n_brows), kRowThreads, bsr_rows_smem(), st>>>(n_brows, d_row_ptr, d_col_idx, d_vals, d_x, d_y);
  else
    spmv_kernel<1, float, float, float><<<row_grid<float>(n_brows), kRowThreads, bsr_rows_smem(), st>>>(n_brows, d_row_ptr, d_col_idx, d_vals, d_x, d_y);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}

extern "C" int fem_bsr_residual_mixed(int vec, int64_t n_brows, const int32_t* d_row_ptr,
                                      const int32_t* d_col_idx, const float* d_vals,
                                      const double* d_x, const double* d_b, double* d_r,
                                      void* stream) {
  FEM_CHECK_ARG(vec == 1 || vec == 3, "vec must be 1 or 3");
  FEM_CHECK_ARG(n_brows >= 0, "negative size");
  FEM_CHECK_ARG(bsr_aligned(d_vals, d_col_idx), "vals and col_idx must be 16-byte aligned");
  if (n_brows == 0) return FEM_OK;
  auto st = as_stream(stream);
  int rc = ensure_smem_attr(vec == 3 ? residual_mixed_kernel<3> : residual_mixed_kernel<1>);
  if (rc != FEM_OK) return rc;
  if (vec == 3)
    residual_mixed_kernel<3><<<row_grid<float>(n_brows), kRowThreads, bsr_rows_smem(), st>>>(n_brows, d_row_ptr, d_col_idx, d_vals, d_x, d_b, d_r);
  else
    residual_mixed_kernel<1><<<row_grid<float>(n_brows), kRowThreads, bsr_rows_smem(), st>>>(n_brows, d_row_ptr, d_col_idx, d_vals, d_x, d_b, d_r);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}

extern "C" size_t fem_dot_workspace_bytes(int64_t n) {
  // partials for vec_grid(n) blocks + counter + result slot, 256-B aligned pieces
  (void)n;
  return size_t(num_sms()) * 8 * sizeof(double) + 512;
}

namespace {
struct RedWork {
  double* partials;
  unsigned int* counter;
  double* result;
};
int carve_red(void* d_work, size_t work_bytes, RedWork* w) {
  const size_t need = fem_dot_workspace_bytes(0);
  FEM_CHECK_ARG(d_work != nullptr && work_bytes >= need, "workspace too small (%zu < %zu)",
                work_bytes, need);
  char* p = static_cast<char*>(d_work);
  w->counter = reinterpret_cast<unsigned int*>(p);
  w->result = reinterpret_cast<double*>(p + 256);
  w->partials = reinterpret_cast<double*>(p + 512);
  return FEM_OK;
}
}  // namespace

extern "C" int fem_dot_f64(int64_t n, const double* d_x, const double* d_y, double* h_out,
                           void* d_work, size_t work_bytes, void* stream) {
  FEM_CHECK_ARG(n >= 0 && h_out != nullptr, "bad arguments");
  RedWork w;
  int rc = carve_red(d_work, work_bytes, &w);
  if (rc) return rc;
  auto st = as_stream(stream);
  FEM_CUDA_TRY(cudaMemsetAsync(w.counter, 0, 256, st));
  FEM_CUDA_TRY(cudaMemsetAsync(w.result, 0, sizeof(double), st));
  dot_kernel<<<vec_grid(n), 256, 0, st>>>(n, d_x, d_y, w.partials, w.counter, w.result);
  FEM_LAUNCH_CHECK();
  double* mb = host_mailbox();
  FEM_CHECK_ARG(mb != nullptr, "pinned mailbox allocation failed");
  FEM_CUDA_TRY(cudaMemcpyAsync(mb, w.result, sizeof(double), cudaMemcpyDeviceToHost, st));
  FEM_CUDA_TRY(cudaStreamSynchronize(st));
  *h_out = mb[0];
  return FEM_OK;
}

extern "C" int fem_newton_rhs(int64_t ndofs, const double* d_res, const double* d_fext,
                              const double* d_lift, const uint8_t* d_bc_mask, const double* d_u,
                              const double* d_ubc, double* d_rbc, double* d_rhs, double* h_norm2,
                              void* d_work, size_t work_bytes, void* stream) {
  FEM_CHECK_ARG(ndofs >= 0 && d_res != nullptr, "bad arguments");
  FEM_CHECK_ARG(d_bc_mask == nullptr || (d_u != nullptr && d_ubc != nullptr),
                "BC mask needs u and ubc");
  auto st = as_stream(stream);
  RedWork w{nullptr, nullptr, nullptr};
  if (h_norm2 != nullptr) {
    int rc = carve_red(d_work, work_bytes, &w);
    if (rc) return rc;
    FEM_CUDA_TRY(cudaMemsetAsync(w.counter, 0, 256, st));
    FEM_CUDA_TRY(cudaMemsetAsync(w.result, 0, sizeof(double), st));
  }
  if (ndofs > 0) {
    newton_rhs_kernel<<<vec_grid(ndofs), 256, 0, st>>>(ndofs, d_res, d_fext, d_lift, d_bc_mask, d_u,
                                                       d_ubc, d_rbc, d_rhs, w.partials, w.counter,
                                                       w.result);
    FEM_LAUNCH_CHECK();
  }
  if (h_norm2 != nullptr) {
    double* mb = host_mailbox();
    FEM_CHECK_ARG(mb != nullptr, "pinned mailbox allocation failed");
    FEM_CUDA_TRY(cudaMemcpyAsync(mb, w.result, sizeof(double), cudaMemcpyDeviceToHost, st));
    FEM_CUDA_TRY(cudaStreamSynchronize(st));
    *h_norm2 = mb[0];
  }
  return FEM_OK;
}

// ---------------------------------------------------------------------------
// Dot product that allocates nothing.
//
// For callers that cannot allocate device memory themselves: code running
// under a host framework that owns every device allocation through its own
// pool and forbids raw cudaMalloc, or a real-time loop that must not allocate
// (or risk an allocation failure) once it is running.  Same reduction kernel
// as fem_dot_f64; its per-block partial sums, completion counter and result
// slot live in the file-scope array below instead of a caller workspace.
//
// Limits and sharing rules:
//  - n <= kNoAllocMaxN (16,777,216 elements): one partial sum per 4096
//    elements, at most 4096 partial sums (32 KB).  Larger n is rejected with
//    FEM_ERR_ARG.
//  - Every GPU that loads this library holds the array until the process
//    exits.  All calls share it: two calls whose kernels overlap on the GPU
//    (e.g. on different streams) race and give wrong results.  The counter
//    and the result slot are cleared at the start of every call, so a call
//    never sees the previous call's contents.
//  - The first call on a device resolves the array's device address with
//    cudaGetSymbolAddress (once per device, that device current).  Make that
//    first call before any stream capture.
//  - `stream` must belong to the device that is current on the calling
//    thread (the address is that device's); a stream of another device is
//    rejected with FEM_ERR_ARG.
//  - The result is written to the caller's device double *d_out; the call is
//    asynchronous on `stream` (no host synchronisation, no pinned buffer).
// ---------------------------------------------------------------------------
namespace fem {
namespace {
constexpr int64_t kNoAllocItemsPerBlock = 4096;  // 256 threads x 16 elements
constexpr int64_t kNoAllocMaxBlocks = 4096;
constexpr int64_t kNoAllocMaxN = kNoAllocItemsPerBlock * kNoAllocMaxBlocks;
// doubles [0, 8): completion counter (first 4 bytes); [8]: reduction result;
// [16, 16 + kNoAllocMaxBlocks): per-block partial sums
static __device__ __align__(256) double g_noalloc_scratch[16 + kNoAllocMaxBlocks];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {nullptr};

int noalloc_scratch(double** out) {
  int dev = 0;
  FEM_CUDA_TRY(cudaGetDevice(&dev));
  FEM_CHECK_ARG(dev >= 0 && dev < 64, "device index %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (g_noalloc_addr[dev] == nullptr) {
    void* p = nullptr;
    FEM_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_addr[dev] = p;
  }
  *out = static_cast<double*>(g_noalloc_addr[dev]);
  return FEM_OK;
}

__global__ void copy_scalar_kernel(const double* src, double* dst) { *dst = *src; }
}  // namespace
}  // namespace fem

extern "C" int fem_dot_f64_noalloc(int64_t n, const double* d_x, const double* d_y, double* d_out,
                                   void* stream) {
  FEM_CHECK_ARG(n >= 0, "negative size");
  FEM_CHECK_ARG(n <= fem::kNoAllocMaxN,
                "fem_dot_f64_noalloc: n = %lld exceeds the no-alloc maximum of %lld elements",
                (long long)n, (long long)fem::kNoAllocMaxN);
  FEM_CHECK_ARG(d_out != nullptr && (n == 0 || (d_x != nullptr && d_y != nullptr)),
                "NULL pointer argument");
  auto st = as_stream(stream);
  if (st != nullptr) {
    int cur = 0, sdev = 0;
    FEM_CUDA_TRY(cudaGetDevice(&cur));
    FEM_CUDA_TRY(cudaStreamGetDevice(st, &sdev));
    FEM_CHECK_ARG(sdev == cur, "fem_dot_f64_noalloc: the stream belongs to device %d, not the current device %d",
                  sdev, cur);
  }
  double* scratch = nullptr;
  int rc = fem::noalloc_scratch(&scratch);
  if (rc != FEM_OK) return rc;
  unsigned int* counter = reinterpret_cast<unsigned int*>(scratch);
  double* result = scratch + 8;
  double* partials = scratch + 16;
  FEM_CUDA_TRY(cudaMemsetAsync(scratch, 0, 16 * sizeof(double), st));
  const int64_t blocks = n == 0 ? 1 : (n + fem::kNoAllocItemsPerBlock - 1) / fem::kNoAllocItemsPerBlock;
  dot_kernel<<<unsigned(blocks), 256, 0, st>>>(n, d_x, d_y, partials, counter, result);
  FEM_LAUNCH_CHECK();
  fem::copy_scalar_kernel<<<1, 1, 0, st>>>(result, d_out);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}
