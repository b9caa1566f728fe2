// Preconditioned CG and BiCGSTAB on block-CSR matrices, iterating on the
// device.  Replaces jax_solve / linear_solver (solver.py:63-92, 261-284).
//
// Every scalar of the recurrences (alpha, beta, rho, omega, norms) lives in a
// device-side state record; each reduction finishes in the last block of the
// kernel that produced it (fixed summation order, so results are bitwise
// reproducible) and that block also updates the scalars and the status word.
// Kernels see a non-zero status and return at once, so the host only polls
// the status every `check_every` iterations and never stalls the pipeline.
//
// CG is the Chronopoulos-Gear formulation (one reduction phase per
// iteration): a vector kernel updates p, s = A p, x, r and applies the Jacobi
// / 3x3 block-Jacobi preconditioner u = M r while it reduces gamma = r.u and
// r.r; a pure SpMV w = A u reduces delta = w.u, and its last block forms
// alpha and beta for the next iteration.  Two kernels per iteration.
//
// The mixed-precision CG (fem_krylov_solve_mixed) runs those same FP32
// kernels on an FP32 matrix and keeps the solution in FP64 with reliable
// updates (Sleijpen & van der Vorst 1996; the form of Clark et al. 2010 for
// lattice QCD): whenever the recursive residual has dropped by a factor
// `delta` below its largest value since the last update, the FP32 increment
// is folded into the FP64 solution and the residual is replaced by the true
// one, r = b - A x computed with FP64 accumulation.  The search direction is
// kept, so the Krylov recurrence is not restarted and the iteration count
// stays close to that of FP64 CG, while the true residual drives
// convergence.
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

#include "sparse.cuh"

namespace fem {
namespace {

enum : int { ST_RUNNING = 0, ST_CONVERGED = 1, ST_REPLACE = 2 };

struct KState {
  double rz, rr, pq, alpha, beta, tol2, bnorm2;
  double rho, omega, rz_prev;
  double rmax2;   // largest r.r since the last residual replacement
  double delta2;  // replacement trigger (delta^2); 0 = never (plain CG)
  int iter, status, maxiter, first;
};

template <typename T>
struct KVecs {
  T *r, *z, *p0, *p1, *q;                 // CG
  T *rhat, *p, *phat, *v, *s, *shat, *t;  // BiCGSTAB (p/q/r reused where possible)
  T* minv;                                // preconditioner (n or n*VEC values)
};

__device__ __forceinline__ bool finite_d(double x) { return isfinite(x); }

// ---- preconditioner setup -------------------------------------------------
template <int VEC, typename T>
__global__ void precond_setup_kernel(int precond, int64_t n_brows, const int32_t* diag,
                                     const T* vals, T* minv) {
  const int64_t nd = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (nd >= n_brows) return;
  const T* B = vals + int64_t(diag[nd]) * VEC * VEC;
  if (precond == FEM_PRECOND_JACOBI || VEC == 1) {
#pragma unroll
    for (int i = 0; i < VEC; ++i) {
      const double d = double(B[i * VEC + i]);
      minv[nd * VEC + i] = T(d != 0.0 ? 1.0 / d : 1.0);
    }
  } else {
    // 3x3 inverse in f64
    double a[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) a[i][j] = double(B[i * 3 + j]);
    const double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
    const double c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
    const double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
    const double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
    const double id = 1.0 / det;
    T* o = minv + nd * 9;
    o[0] = T(c00 * id);
    o[3] = T(c01 * id);
    o[6] = T(c02 * id);
    o[1] = T((a[0][2] * a[2][1] - a[0][1] * a[2][2]) * id);
    o[4] = T((a[0][0] * a[2][2] - a[0][2] * a[2][0]) * id);
    o[7] = T((a[0][1] * a[2][0] - a[0][0] * a[2][1]) * id);
    o[2] = T((a[0][1] * a[1][2] - a[0][2] * a[1][1]) * id);
    o[5] = T((a[0][2] * a[1][0] - a[0][0] * a[1][2]) * id);
    o[8] = T((a[0][0] * a[1][1] - a[0][1] * a[1][0]) * id);
  }
}

// z_node = M^{-1} r_node
template <int VEC, typename T>
__device__ __forceinline__ void apply_precond(int precond, int64_t nd, const T* minv, const T r[VEC],
                                              T z[VEC]) {
  if (precond == FEM_PRECOND_NONE) {
#pragma unroll
    for (int i = 0; i < VEC; ++i) z[i] = r[i];
  } else if (precond == FEM_PRECOND_JACOBI || VEC == 1) {
#pragma unroll
    for (int i = 0; i < VEC; ++i) z[i] = minv[nd * VEC + i] * r[i];
  } else {
    const T* m = minv + nd * 9;
#pragma unroll
    for (int i = 0; i < 3; ++i) z[i] = m[i * 3] * r[0] + m[i * 3 + 1] * r[1] + m[i * 3 + 2] * r[2];
  }
}

// r = b - A x
template <int VEC, typename T>
__global__ void __launch_bounds__(kRowThreads, kRowBlocksPerSM) kr_residual_kernel(int64_t n_brows, const int32_t* rp,
                                                                 const int32_t* ci, const T* vals,
                                                                 const T* __restrict__ x,
                                                                 const T* b, T* r) {
  bsr_rows<VEC, T, double>(
      n_brows, rp, ci, vals, [&](int64_t i) { return x[i]; },
      [&](int64_t row, int c, double val) {
        r[row * VEC + c] = T(double(b[row * VEC + c]) - val);
      });
}

// z = M r; rz = r.z, rr = r.r, bb = b.b; initial status.  With `replace`
// the residual r has just been replaced by the true one: only rz, rr and the
// status are refreshed (b may be null), and the recurrence carries on.
template <int VEC, typename T, typename BT>
__global__ void cg_init_kernel(int precond, int64_t n_brows, const T* minv, const T* r, T* z,
                               const BT* b, double* partials, unsigned int* counter, KState* S,
                               double rtol, double atol, bool replace) {
  double v[3] = {0.0, 0.0, 0.0};
  for (int64_t nd = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; nd < n_brows;
       nd += int64_t(gridDim.x) * blockDim.x) {
    T rn[VEC], zn[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) rn[i] = r[nd * VEC + i];
    apply_precond<VEC, T>(precond, nd, minv, rn, zn);
#pragma unroll
    for (int i = 0; i < VEC; ++i) {
      if (z != r) z[nd * VEC + i] = zn[i];
      v[0] = fma(double(rn[i]), double(zn[i]), v[0]);
      v[1] = fma(double(rn[i]), double(rn[i]), v[1]);
      if (b != nullptr) {
        const double bi = double(b[nd * VEC + i]);
        v[2] = fma(bi, bi, v[2]);
      }
    }
  }
  double tot[3];
  if (last_block_reduce<3>(v, partials, counter, tot)) {
    S->rz = tot[0];
    S->rr = tot[1];
    S->rmax2 = tot[1];
    if (replace) {
      if (!finite_d(tot[0]) || !finite_d(tot[1]))
        S->status = FEM_ERR_NONFINITE;
      else if (tot[1] <= S->tol2)
        S->status = ST_CONVERGED;
      else if (tot[0] == 0.0)
        S->status = FEM_ERR_BREAKDOWN;
      else
        S->status = ST_RUNNING;
      return;
    }
    S->bnorm2 = tot[2];
    const double t1 = rtol * rtol * tot[2], t2 = atol * atol;
    S->tol2 = t1 > t2 ? t1 : t2;
    S->beta = 0.0;
    S->rho = tot[0];
    S->omega = 1.0;
    S->alpha = 1.0;
    S->iter = 0;
    S->first = 1;  // the next CG SpMV starts a fresh recurrence (also after a restart)
    if (!finite_d(tot[0]) || !finite_d(tot[1]) || !finite_d(tot[2]))
      S->status = FEM_ERR_NONFINITE;
    else if (tot[1] <= S->tol2)
      S->status = ST_CONVERGED;
    else if (S->maxiter <= 0)
      S->status = FEM_ERR_NOT_CONVERGED;
    else
      S->status = ST_RUNNING;
  }
}

// CG SpMV: w = A u, delta = w . u; last block forms alpha, beta.
template <int VEC, typename T>
__global__ void __launch_bounds__(kRowThreads, kRowBlocksPerSM) cg_spmv_kernel(int64_t n_brows, const int32_t* rp,
                                                             const int32_t* ci, const T* vals,
                                                             const T* __restrict__ u, T* w,
                                                             double* partials, unsigned int* counter,
                                                             KState* S) {
  if (S->status != ST_RUNNING) return;
  double v[1] = {0.0};
  bsr_rows<VEC, T, T>(
      n_brows, rp, ci, vals, [&](int64_t i) { return u[i]; },
      [&](int64_t row, int c, T wo) {
        const int64_t i = row * VEC + c;
        w[i] = wo;
        v[0] = fma(double(u[i]), double(wo), v[0]);
      });
  double tot[1];
  if (last_block_reduce<1>(v, partials, counter, tot)) {
    const double delta = tot[0], gamma = S->rz;
    S->pq = delta;
    double denom;
    if (S->first) {
      S->beta = 0.0;
      denom = delta;
      S->first = 0;
    } else {
      S->beta = gamma / S->rz_prev;
      denom = delta - S->beta * gamma / S->alpha;
    }
    S->rz_prev = gamma;
    if (!finite_d(delta))
      S->status = FEM_ERR_NONFINITE;
    else if (!(denom > 0.0))
      S->status = FEM_ERR_BREAKDOWN;
    else
      S->alpha = gamma / denom;
  }
}

// CG vector step: p = u + beta p; s = w + beta s; x += alpha p; r -= alpha s;
// u = M r; gamma = r.u, rr = r.r; convergence / iteration bookkeeping.
template <int VEC, typename T>
__global__ void cg_vec_kernel(int precond, int64_t n_brows, const T* minv, T* x, T* r, T* u, T* p,
                              T* sv, const T* w, double* partials, unsigned int* counter, KState* S) {
  if (S->status != ST_RUNNING) return;
  const T alpha = T(S->alpha), beta = T(S->beta);
  double v[2] = {0.0, 0.0};
  for (int64_t nd = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; nd < n_brows;
       nd += int64_t(gridDim.x) * blockDim.x) {
    T rn[VEC], un[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) {
      const int64_t k = nd * VEC + i;
      const T pk = u[k] + beta * p[k];
      const T sk = w[k] + beta * sv[k];
      p[k] = pk;
      sv[k] = sk;
      x[k] += alpha * pk;
      rn[i] = r[k] - alpha * sk;
      r[k] = rn[i];
    }
    apply_precond<VEC, T>(precond, nd, minv, rn, un);
#pragma unroll
    for (int i = 0; i < VEC; ++i) {
      if (u != r) u[nd * VEC + i] = un[i];
      v[0] = fma(double(rn[i]), double(un[i]), v[0]);
      v[1] = fma(double(rn[i]), double(rn[i]), v[1]);
    }
  }
  double tot[2];
  if (last_block_reduce<2>(v, partials, counter, tot)) {
    S->iter += 1;
    S->rr = tot[1];
    S->rz = tot[0];
    if (!finite_d(tot[0]) || !finite_d(tot[1])) {
      S->status = FEM_ERR_NONFINITE;
    } else if (tot[1] <= S->tol2) {
      S->status = ST_CONVERGED;
    } else if (S->iter >= S->maxiter) {
      S->status = FEM_ERR_NOT_CONVERGED;
    } else if (tot[0] == 0.0) {
      S->status = FEM_ERR_BREAKDOWN;
    } else if (S->delta2 > 0.0) {
      // reliable update due: the residual fell by delta below its peak
      if (tot[1] < S->delta2 * S->rmax2) S->status = ST_REPLACE;
      else if (tot[1] > S->rmax2) S->rmax2 = tot[1];
    }
  }
}

// ---- BiCGSTAB (right-looking, as scipy/JAX bicgstab) ----------------------
// B1: p = r + beta (p - omega v); phat = M p
template <int VEC, typename T>
__global__ void bicg_p_kernel(int precond, int64_t n_brows, const T* minv, const T* r, T* p,
                              const T* v, T* phat, KState* S) {
  if (S->status != ST_RUNNING) return;
  const T beta = T(S->beta), omega = T(S->omega);
  for (int64_t nd = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; nd < n_brows;
       nd += int64_t(gridDim.x) * blockDim.x) {
    T pn[VEC], ph[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) {
      const int64_t k = nd * VEC + i;
      pn[i] = r[k] + beta * (p[k] - omega * v[k]);
      p[k] = pn[i];
    }
    apply_precond<VEC, T>(precond, nd, minv, pn, ph);
#pragma unroll
    for (int i = 0; i < VEC; ++i) phat[nd * VEC + i] = ph[i];
  }
}

// y = A x with partial dot products of y against up to two vectors.
// mode 0: (rhat . v) -> alpha; mode 1: (t . s, t . t) -> omega
template <int VEC, typename T>
__global__ void __launch_bounds__(kRowThreads, kRowBlocksPerSM) bicg_spmv_kernel(int mode, int64_t n_brows, const int32_t* rp,
                                                               const int32_t* ci, const T* vals,
                                                               const T* __restrict__ x, T* y,
                                                               const T* w, double* partials,
                                                               unsigned int* counter, KState* S) {
  if (S->status != ST_RUNNING) return;
  double v[2] = {0.0, 0.0};
  bsr_rows<VEC, T, T>(
      n_brows, rp, ci, vals, [&](int64_t i) { return x[i]; },
      [&](int64_t row, int c, T yo) {
        const int64_t i = row * VEC + c;
        y[i] = yo;
        v[0] = fma(double(w[i]), double(yo), v[0]);
        v[1] = fma(double(yo), double(yo), v[1]);
      });
  double tot[2];
  if (last_block_reduce<2>(v, partials, counter, tot)) {
    if (mode == 0) {
      if (!finite_d(tot[0]))
        S->status = FEM_ERR_NONFINITE;
      else if (tot[0] == 0.0)
        S->status = FEM_ERR_BREAKDOWN;
      else
        S->alpha = S->rho / tot[0];
    } else {
      if (!finite_d(tot[0]) || !finite_d(tot[1]))
        S->status = FEM_ERR_NONFINITE;
      else
        S->omega = tot[1] > 0.0 ? tot[0] / tot[1] : 0.0;
    }
  }
}

// B3: s = r - alpha v; shat = M s
template <int VEC, typename T>
__global__ void bicg_s_kernel(int precond, int64_t n_brows, const T* minv, const T* r, const T* v,
                              T* s, T* shat, KState* S) {
  if (S->status != ST_RUNNING) return;
  const T alpha = T(S->alpha);
  for (int64_t nd = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; nd < n_brows;
       nd += int64_t(gridDim.x) * blockDim.x) {
    T sn[VEC], sh[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) {
      const int64_t k = nd * VEC + i;
      sn[i] = r[k] - alpha * v[k];
      s[k] = sn[i];
    }
    apply_precond<VEC, T>(precond, nd, minv, sn, sh);
#pragma unroll
    for (int i = 0; i < VEC; ++i) shat[nd * VEC + i] = sh[i];
  }
}

// B5: x += alpha phat + omega shat; r = s - omega t; rho_new = rhat.r, rr
template <int VEC, typename T>
__global__ void bicg_x_kernel(int64_t n, T* x, T* r, const T* rhat, const T* phat, const T* shat,
                              const T* s, const T* t, double* partials, unsigned int* counter,
                              KState* S) {
  if (S->status != ST_RUNNING) return;
  const T alpha = T(S->alpha), omega = T(S->omega);
  double v[2] = {0.0, 0.0};
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n;
       k += int64_t(gridDim.x) * blockDim.x) {
    x[k] += alpha * phat[k] + omega * shat[k];
    const T rn = s[k] - omega * t[k];
    r[k] = rn;
    v[0] = fma(double(rhat[k]), double(rn), v[0]);
    v[1] = fma(double(rn), double(rn), v[1]);
  }
  double tot[2];
  if (last_block_reduce<2>(v, partials, counter, tot)) {
    S->iter += 1;
    S->rr = tot[1];
    if (!finite_d(tot[0]) || !finite_d(tot[1])) {
      S->status = FEM_ERR_NONFINITE;
    } else if (tot[1] <= S->tol2) {
      S->status = ST_CONVERGED;
    } else if (S->iter >= S->maxiter) {
      S->status = FEM_ERR_NOT_CONVERGED;
    } else if (S->omega == 0.0 || S->rho == 0.0) {
      S->status = FEM_ERR_BREAKDOWN;
    } else {
      S->beta = (tot[0] / S->rho) * (S->alpha / S->omega);
      S->rho = tot[0];
    }
  }
}

template <typename T>
__global__ void copy_kernel(int64_t n, const T* a, T* b) {
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n;
       k += int64_t(gridDim.x) * blockDim.x)
    b[k] = a[k];
}

// ---- mixed-precision CG: FP64 solution, true residual with FP64 accumulation --
// x64 += x32; x32 = 0
__global__ void fold_kernel(int64_t n, double* x64, float* x32) {
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n;
       k += int64_t(gridDim.x) * blockDim.x) {
    x64[k] += double(x32[k]);
    x32[k] = 0.0f;
  }
}

// r32 = b - A x (A f32, x and b f64, f64 accumulation, rounded once)
template <int VEC>
__global__ void __launch_bounds__(kRowThreads, kRowBlocksPerSM) kr_true_residual_kernel(
    int64_t n_brows, const int32_t* rp, const int32_t* ci, const float* vals,
    const double* __restrict__ x, const double* b, float* r) {
  bsr_rows<VEC, float, double>(
      n_brows, rp, ci, vals, [&](int64_t i) { return x[i]; },
      [&](int64_t row, int c, double val) {
        r[row * VEC + c] = float(b[row * VEC + c] - val);
      });
}

// ---- cached CUDA graphs of CG / BiCGSTAB iteration chunks --------------------
struct GraphKey {
  int method, precond, vec, tsize, chunk;
  int64_t n;
  const void* ptrs[24];
  bool operator<(const GraphKey& o) const {
    if (method != o.method) return method < o.method;
    if (precond != o.precond) return precond < o.precond;
    if (vec != o.vec) return vec < o.vec;
    if (tsize != o.tsize) return tsize < o.tsize;
    if (chunk != o.chunk) return chunk < o.chunk;
    if (n != o.n) return n < o.n;
    return std::memcmp(ptrs, o.ptrs, sizeof(ptrs)) < 0;
  }
};
std::mutex g_graph_mu;
std::map<GraphKey, cudaGraphExec_t>& graph_cache() {
  static std::map<GraphKey, cudaGraphExec_t> m;
  return m;
}
cudaGraphExec_t graph_lookup(const GraphKey& k) {
  int dev = 0;
  cudaGetDevice(&dev);
  GraphKey kk = k;
  kk.ptrs[23] = reinterpret_cast<const void*>(intptr_t(dev));
  std::lock_guard<std::mutex> lock(g_graph_mu);
  auto it = graph_cache().find(kk);
  return it == graph_cache().end() ? nullptr : it->second;
}
void graph_store(const GraphKey& k, cudaGraphExec_t e) {
  int dev = 0;
  cudaGetDevice(&dev);
  GraphKey kk = k;
  kk.ptrs[23] = reinterpret_cast<const void*>(intptr_t(dev));
  std::lock_guard<std::mutex> lock(g_graph_mu);
  auto& m = graph_cache();
  if (m.size() >= 64) {  // bounded: drop everything (workspaces moved)
    for (auto& kv : m) cudaGraphExecDestroy(kv.second);
    m.clear();
  }
  m[kk] = e;
}
// FEM_KRYLOV_GRAPHS=0 in the environment launches every kernel directly.
bool graphs_enabled() {
  static int on = -1;
  if (on < 0) {
    const char* e = std::getenv("FEM_KRYLOV_GRAPHS");
    on = (e != nullptr && e[0] == '0') ? 0 : 1;
  }
  return on == 1;
}

cudaStream_t capture_stream() {
  static std::mutex mu;
  static cudaStream_t s[64] = {nullptr};
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (s[dev] == nullptr && cudaStreamCreateWithFlags(&s[dev], cudaStreamNonBlocking) != cudaSuccess)
    s[dev] = nullptr;
  return s[dev];
}

// Launch one chunk of iterations: replayed from a cached CUDA graph in the
// steady state (kernel arguments are fixed pointers, so one capture serves
// every replay), launched directly otherwise or when capture fails.
template <class LaunchChunk>
int run_chunk(const GraphKey& key, bool steady, int kernels_per_iter, LaunchChunk& launch_chunk,
              cudaStream_t st) {
  const int chunk = key.chunk;
  if (steady && graphs_enabled()) {
    cudaGraphExec_t exec = graph_lookup(key);
    if (exec == nullptr) {
      cudaStream_t cap = capture_stream();
      if (cap != nullptr && cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const int lrc = launch_chunk(cap, chunk);
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(cap, &g);
        if (lrc == FEM_OK && ec == cudaSuccess && g != nullptr &&
            cudaGraphInstantiate(&exec, g, 0) == cudaSuccess) {
          graph_store(key, exec);
        } else {
          exec = nullptr;
        }
        if (g != nullptr) cudaGraphDestroy(g);
        cudaGetLastError();  // a failed capture falls back to direct launches
      }
    }
    if (exec != nullptr) {
      FEM_CUDA_TRY(cudaGraphLaunch(exec, st));
      launch_counter().fetch_add(int64_t(chunk) * kernels_per_iter, std::memory_order_relaxed);
      return FEM_OK;
    }
  }
  return launch_chunk(st, chunk);
}

// ---- workspace ----------------------------------------------------------------
inline size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

size_t workspace_bytes(int method, int precond, int vec, int64_t n_brows, size_t elem) {
  const size_t n = size_t(n_brows) * vec;
  const size_t nvec = (method == FEM_KRYLOV_CG) ? 5 : 8;
  size_t bytes = 256 /*state*/ + 256 /*counter*/ + al256(size_t(num_sms()) * 8 * 4 * sizeof(double));
  bytes += nvec * al256(n * elem);
  const size_t pre = (precond == FEM_PRECOND_BLOCK_JACOBI && vec == 3) ? size_t(n_brows) * 9 : n;
  bytes += al256(pre * elem);
  return bytes;
}

template <int VEC, typename T>
int solve_impl(int method, int precond, int64_t n_brows, const int32_t* rp, const int32_t* ci,
               const int32_t* diag, const T* vals, const T* b, T* x, double rtol, double atol,
               int maxiter, int check_every, void* work, size_t work_bytes, int* h_iters,
               double* h_relres, cudaStream_t st) {
  const size_t need = workspace_bytes(method, precond, VEC, n_brows, sizeof(T));
  FEM_CHECK_ARG(work != nullptr && work_bytes >= need, "krylov workspace too small (%zu < %zu)",
                work_bytes, need);
  FEM_CHECK_ARG(precond == FEM_PRECOND_NONE || diag != nullptr, "preconditioner needs diag");
  if (check_every <= 0) check_every = 16;
  const int64_t n = n_brows * VEC;
  char* p = static_cast<char*>(work);
  KState* S = reinterpret_cast<KState*>(p);
  unsigned int* counter = reinterpret_cast<unsigned int*>(p + 256);
  double* partials = reinterpret_cast<double*>(p + 512);
  p += 512 + al256(size_t(num_sms()) * 8 * 4 * sizeof(double));
  auto take = [&](size_t cnt) {
    T* q = reinterpret_cast<T*>(p);
    p += al256(cnt * sizeof(T));
    return q;
  };
  const int nvec = (method == FEM_KRYLOV_CG) ? 5 : 8;
  T* V[8];
  for (int i = 0; i < nvec; ++i) V[i] = take(size_t(n));
  T* minv = take((precond == FEM_PRECOND_BLOCK_JACOBI && VEC == 3) ? size_t(n_brows) * 9 : size_t(n));

  FEM_CUDA_TRY(cudaMemsetAsync(work, 0, 512, st));
  KState init{};
  init.maxiter = maxiter;
  init.first = 1;
  FEM_CUDA_TRY(cudaMemcpyAsync(S, &init, sizeof(KState), cudaMemcpyHostToDevice, st));
  // cudaMemcpyAsync from pageable memory is synchronous w.r.t. the host copy,
  // so `init` may go out of scope after this point.
  if (precond != FEM_PRECOND_NONE) {
    precond_setup_kernel<VEC, T><<<unsigned((n_brows + 255) / 256), 256, 0, st>>>(precond, n_brows,
                                                                                diag, vals, minv);
    FEM_LAUNCH_CHECK();
  }
  const unsigned rg = row_grid<T>(n_brows), vg = vec_grid(n_brows), vgn = vec_grid(n);
  {
    int rc = FEM_OK;
    if ((rc = ensure_smem_attr(kr_residual_kernel<VEC, T>)) != FEM_OK) return rc;
    if ((rc = ensure_smem_attr(cg_spmv_kernel<VEC, T>)) != FEM_OK) return rc;
    if ((rc = ensure_smem_attr(bicg_spmv_kernel<VEC, T>)) != FEM_OK) return rc;
  }
  T* r = V[0];
  T *z = nullptr, *p0 = nullptr, *p1 = nullptr, *q = nullptr;
  T *rhat = nullptr, *pp = nullptr, *phat = nullptr, *vv = nullptr, *s = nullptr, *shat = nullptr,
    *t = nullptr;
  if (method == FEM_KRYLOV_CG) {
    z = (precond == FEM_PRECOND_NONE) ? r : V[1];  // u = M r
    p0 = V[2];                                      // p
    p1 = V[3];                                      // s = A p
    q = V[4];                                       // w = A u
  } else {
    rhat = V[1];
    pp = V[2];
    phat = V[3];
    vv = V[4];
    s = V[5];
    shat = V[6];
    t = V[7];
  }
  // (Re)start from the true residual r = b - A x: at the start, and whenever
  // the recursively updated residual claims a convergence that the true
  // residual does not confirm (round-off drift, notably in FP32).
  auto start = [&]() -> int {
    kr_residual_kernel<VEC, T><<<rg, kRowThreads, bsr_rows_smem(), st>>>(n_brows, rp, ci, vals, x, b, r);
    FEM_LAUNCH_CHECK();
    if (method == FEM_KRYLOV_CG) {
      FEM_CUDA_TRY(cudaMemsetAsync(p0, 0, sizeof(T) * n, st));
      FEM_CUDA_TRY(cudaMemsetAsync(p1, 0, sizeof(T) * n, st));
      cg_init_kernel<VEC, T, T><<<vg, 256, 0, st>>>(precond, n_brows, minv, r, z, b, partials, counter,
                                                    S, rtol, atol, false);
      FEM_LAUNCH_CHECK();
      cg_spmv_kernel<VEC, T><<<rg, kRowThreads, bsr_rows_smem(), st>>>(n_brows, rp, ci, vals, z, q,
                                                                      partials, counter, S);
      FEM_LAUNCH_CHECK();
    } else {
      FEM_CUDA_TRY(cudaMemsetAsync(pp, 0, sizeof(T) * n, st));
      FEM_CUDA_TRY(cudaMemsetAsync(vv, 0, sizeof(T) * n, st));
      copy_kernel<T><<<vgn, 256, 0, st>>>(n, r, rhat);
      FEM_LAUNCH_CHECK();
      // rho = rhat.r = r.r, r.r and b.b (no preconditioning in this reduction)
      cg_init_kernel<VEC, T, T><<<vg, 256, 0, st>>>(FEM_PRECOND_NONE, n_brows, minv, r, r, b, partials,
                                                    counter, S, rtol, atol, false);
      FEM_LAUNCH_CHECK();
    }
    return FEM_OK;
  };
  double* mb = host_mailbox();
  FEM_CHECK_ARG(mb != nullptr, "pinned mailbox allocation failed");
  const KState* hs = reinterpret_cast<const KState*>(mb);
  auto read_state = [&]() -> int {
    FEM_CUDA_TRY(cudaMemcpyAsync(mb, S, sizeof(KState), cudaMemcpyDeviceToHost, st));
    FEM_CUDA_TRY(cudaStreamSynchronize(st));
    return FEM_OK;
  };
  auto launch_chunk = [&](cudaStream_t ls, int chunk) -> int {
    for (int k = 0; k < chunk; ++k) {
      if (method == FEM_KRYLOV_CG) {
        cg_vec_kernel<VEC, T><<<vg, 256, 0, ls>>>(precond, n_brows, minv, x, r, z, p0, p1, q, partials,
                                                  counter, S);
        FEM_LAUNCH_CHECK();
        cg_spmv_kernel<VEC, T><<<rg, kRowThreads, bsr_rows_smem(), ls>>>(n_brows, rp, ci, vals, z, q,
                                                                        partials, counter, S);
        FEM_LAUNCH_CHECK();
      } else {
        bicg_p_kernel<VEC, T><<<vg, 256, 0, ls>>>(precond, n_brows, minv, r, pp, vv, phat, S);
        FEM_LAUNCH_CHECK();
        bicg_spmv_kernel<VEC, T><<<rg, kRowThreads, bsr_rows_smem(), ls>>>(
            0, n_brows, rp, ci, vals, phat, vv, rhat, partials, counter, S);
        FEM_LAUNCH_CHECK();
        bicg_s_kernel<VEC, T><<<vg, 256, 0, ls>>>(precond, n_brows, minv, r, vv, s, shat, S);
        FEM_LAUNCH_CHECK();
        bicg_spmv_kernel<VEC, T><<<rg, kRowThreads, bsr_rows_smem(), ls>>>(
            1, n_brows, rp, ci, vals, shat, t, s, partials, counter, S);
        FEM_LAUNCH_CHECK();
        bicg_x_kernel<VEC, T><<<vgn, 256, 0, ls>>>(n, x, r, rhat, phat, shat, s, t, partials,
                                                   counter, S);
        FEM_LAUNCH_CHECK();
      }
    }
    return FEM_OK;
  };
  {
    int rc = start();
    if (rc != FEM_OK) return rc;
  }
  int status = ST_RUNNING, iters = 0, iter_base = 0, restarts = 0;
  double rr = 0.0, bb = 0.0;
  int launched = 0;
  while (true) {
    int rc = read_state();
    if (rc != FEM_OK) return rc;
    status = hs->status;
    iters = iter_base + hs->iter;
    rr = hs->rr;
    bb = hs->bnorm2;
    if ((status == ST_CONVERGED && iters > iter_base) ||
        (status == FEM_ERR_BREAKDOWN && iters > iter_base)) {
      // Confirm a convergence with the true residual, and answer a breakdown
      // (a non-positive curvature or zero denominator from round-off, near
      // the attainable accuracy) the same way: restart from r = b - A x.
      iter_base = iters;
      if ((rc = start()) != FEM_OK) return rc;
      if ((rc = read_state()) != FEM_OK) return rc;
      status = hs->status;
      rr = hs->rr;
      if (status != ST_RUNNING) break;
      if (++restarts > 3 || launched >= maxiter) {
        status = FEM_ERR_NOT_CONVERGED;
        break;
      }
      continue;
    }
    if (status != ST_RUNNING || launched >= maxiter) break;
    const int chunk = check_every < (maxiter - launched) ? check_every : (maxiter - launched);
    GraphKey key{};
    key.method = method; key.precond = precond; key.vec = VEC; key.tsize = int(sizeof(T));
    key.n = n_brows; key.chunk = chunk;
    const void* kp[] = {rp, ci, vals, minv, x, r, z, p0, p1, q, rhat, pp, phat, vv, s, shat, t,
                        partials, counter, S, b};
    for (int i = 0; i < int(sizeof(kp) / sizeof(kp[0])); ++i) key.ptrs[i] = kp[i];
    if ((rc = run_chunk(key, chunk == check_every, method == FEM_KRYLOV_CG ? 2 : 5, launch_chunk, st)) != FEM_OK)
      return rc;
    launched += chunk;
  }
  if (h_iters) *h_iters = iters;
  if (h_relres) *h_relres = bb > 0 ? sqrt(rr / bb) : sqrt(rr);
  if (status == ST_CONVERGED) return FEM_OK;
  if (status == ST_RUNNING) status = FEM_ERR_NOT_CONVERGED;
  set_error("krylov: status %d after %d iterations (relres %.3e)", status, iters,
            bb > 0 ? sqrt(rr / bb) : sqrt(rr));
  return status;
}

// Mixed-precision CG with reliable updates: FP32 matrix and iteration
// vectors, FP64 right-hand side and solution (see the file comment).
template <int VEC>
int solve_mixed_impl(int precond, int64_t n_brows, const int32_t* rp, const int32_t* ci,
                     const int32_t* diag, const float* vals, const double* b, double* x,
                     double rtol, double atol, int maxiter, int check_every, double delta,
                     void* work, size_t work_bytes, int* h_iters, int* h_replacements,
                     double* h_relres, cudaStream_t st) {
  const int64_t n = n_brows * VEC;
  const size_t base = workspace_bytes(FEM_KRYLOV_CG, precond, VEC, n_brows, sizeof(float));
  const size_t need = base + al256(size_t(n) * sizeof(float));
  FEM_CHECK_ARG(work != nullptr && work_bytes >= need, "krylov workspace too small (%zu < %zu)",
                work_bytes, need);
  FEM_CHECK_ARG(precond == FEM_PRECOND_NONE || diag != nullptr, "preconditioner needs diag");
  FEM_CHECK_ARG(delta > 0.0 && delta < 1.0, "replacement factor delta must be in (0, 1), got %g", delta);
  if (check_every <= 0) check_every = 16;
  char* p = static_cast<char*>(work);
  KState* S = reinterpret_cast<KState*>(p);
  unsigned int* counter = reinterpret_cast<unsigned int*>(p + 256);
  double* partials = reinterpret_cast<double*>(p + 512);
  p += 512 + al256(size_t(num_sms()) * 8 * 4 * sizeof(double));
  auto take = [&](size_t cnt) {
    float* q = reinterpret_cast<float*>(p);
    p += al256(cnt * sizeof(float));
    return q;
  };
  float* r = take(size_t(n));
  float* zb = take(size_t(n));
  float* p0 = take(size_t(n));  // p
  float* p1 = take(size_t(n));  // s = A p
  float* q = take(size_t(n));   // w = A u
  float* minv = take((precond == FEM_PRECOND_BLOCK_JACOBI && VEC == 3) ? size_t(n_brows) * 9 : size_t(n));
  float* x32 = reinterpret_cast<float*>(static_cast<char*>(work) + base);
  float* z = (precond == FEM_PRECOND_NONE) ? r : zb;

  FEM_CUDA_TRY(cudaMemsetAsync(work, 0, 512, st));
  FEM_CUDA_TRY(cudaMemsetAsync(x32, 0, sizeof(float) * n, st));
  FEM_CUDA_TRY(cudaMemsetAsync(p0, 0, sizeof(float) * n, st));
  FEM_CUDA_TRY(cudaMemsetAsync(p1, 0, sizeof(float) * n, st));
  KState init{};
  init.maxiter = maxiter;
  init.first = 1;
  init.delta2 = delta * delta;
  FEM_CUDA_TRY(cudaMemcpyAsync(S, &init, sizeof(KState), cudaMemcpyHostToDevice, st));
  if (precond != FEM_PRECOND_NONE) {
    precond_setup_kernel<VEC, float><<<unsigned((n_brows + 255) / 256), 256, 0, st>>>(precond, n_brows,
                                                                                    diag, vals, minv);
    FEM_LAUNCH_CHECK();
  }
  const unsigned rg = row_grid<float>(n_brows), vg = vec_grid(n_brows), vgn = vec_grid(n);
  {
    int rc = FEM_OK;
    if ((rc = ensure_smem_attr(kr_true_residual_kernel<VEC>)) != FEM_OK) return rc;
    if ((rc = ensure_smem_attr(cg_spmv_kernel<VEC, float>)) != FEM_OK) return rc;
  }
  // true residual into r, then u = M r and the reductions; `fresh` starts a
  // new recurrence (first call, breakdown), otherwise the direction is kept
  auto replace = [&](bool fresh) -> int {
    fold_kernel<<<vgn, 256, 0, st>>>(n, x, x32);
    FEM_LAUNCH_CHECK();
    kr_true_residual_kernel<VEC><<<rg, kRowThreads, bsr_rows_smem(), st>>>(n_brows, rp, ci, vals, x, b, r);
    FEM_LAUNCH_CHECK();
    if (fresh) {
      FEM_CUDA_TRY(cudaMemsetAsync(p0, 0, sizeof(float) * n, st));
      FEM_CUDA_TRY(cudaMemsetAsync(p1, 0, sizeof(float) * n, st));
    }
    cg_init_kernel<VEC, float, double><<<vg, 256, 0, st>>>(precond, n_brows, minv, r, z, fresh ? b : nullptr,
                                                           partials, counter, S, rtol, atol, !fresh);
    FEM_LAUNCH_CHECK();
    cg_spmv_kernel<VEC, float><<<rg, kRowThreads, bsr_rows_smem(), st>>>(n_brows, rp, ci, vals, z, q,
                                                                        partials, counter, S);
    FEM_LAUNCH_CHECK();
    return FEM_OK;
  };
  double* mb = host_mailbox();
  FEM_CHECK_ARG(mb != nullptr, "pinned mailbox allocation failed");
  const KState* hs = reinterpret_cast<const KState*>(mb);
  auto read_state = [&]() -> int {
    FEM_CUDA_TRY(cudaMemcpyAsync(mb, S, sizeof(KState), cudaMemcpyDeviceToHost, st));
    FEM_CUDA_TRY(cudaStreamSynchronize(st));
    return FEM_OK;
  };
  auto launch_chunk = [&](cudaStream_t ls, int chunk) -> int {
    for (int k = 0; k < chunk; ++k) {
      cg_vec_kernel<VEC, float><<<vg, 256, 0, ls>>>(precond, n_brows, minv, x32, r, z, p0, p1, q, partials,
                                                    counter, S);
      FEM_LAUNCH_CHECK();
      cg_spmv_kernel<VEC, float><<<rg, kRowThreads, bsr_rows_smem(), ls>>>(n_brows, rp, ci, vals, z, q,
                                                                          partials, counter, S);
      FEM_LAUNCH_CHECK();
    }
    return FEM_OK;
  };
  int rc = replace(true);
  if (rc != FEM_OK) return rc;
  int status = ST_RUNNING, iters = 0, iter_base = 0, restarts = 0, replacements = 0;
  int launched = 0;
  // Replacements are bounded: each one follows at least one iteration, and
  // a long run of them without progress ends as "not converged".
  const int max_replacements = maxiter;
  while (true) {
    if ((rc = read_state()) != FEM_OK) return rc;
    status = hs->status;
    iters = iter_base + hs->iter;
    if (status == ST_REPLACE || (status == ST_CONVERGED && iters > iter_base)) {
      // reliable update; a convergence claimed by the recursive residual is
      // confirmed (or not) by the true one
      if (++replacements > max_replacements) {
        status = FEM_ERR_NOT_CONVERGED;
        break;
      }
      if ((rc = replace(false)) != FEM_OK) return rc;
      if ((rc = read_state()) != FEM_OK) return rc;
      if (hs->status == ST_CONVERGED) {  // confirmed by the true residual
        status = ST_CONVERGED;
        break;
      }
      continue;
    }
    if (status == FEM_ERR_BREAKDOWN && iters > iter_base && restarts < 3 && launched < maxiter) {
      // round-off breakdown near the attainable accuracy: fresh recurrence
      // from the true residual
      ++restarts;
      iter_base = iters;
      if ((rc = replace(true)) != FEM_OK) return rc;
      continue;
    }
    if (status != ST_RUNNING || launched >= maxiter) break;
    const int chunk = check_every < (maxiter - launched) ? check_every : (maxiter - launched);
    GraphKey key{};
    key.method = FEM_KRYLOV_CG + 100;  // distinct from the plain FP32 CG graphs
    key.precond = precond; key.vec = VEC; key.tsize = int(sizeof(float));
    key.n = n_brows; key.chunk = chunk;
    const void* kp[] = {rp, ci, vals, minv, x32, r, z, p0, p1, q, partials, counter, S};
    for (int i = 0; i < int(sizeof(kp) / sizeof(kp[0])); ++i) key.ptrs[i] = kp[i];
    if ((rc = run_chunk(key, chunk == check_every, 2, launch_chunk, st)) != FEM_OK) return rc;
    launched += chunk;
  }
  // the FP64 solution takes the last FP32 increment; the reported residual
  // is the true one unless convergence was just confirmed
  fold_kernel<<<vgn, 256, 0, st>>>(n, x, x32);
  FEM_LAUNCH_CHECK();
  if (status != ST_CONVERGED) {
    kr_true_residual_kernel<VEC><<<rg, kRowThreads, bsr_rows_smem(), st>>>(n_brows, rp, ci, vals, x, b, r);
    FEM_LAUNCH_CHECK();
    cg_init_kernel<VEC, float, double><<<vg, 256, 0, st>>>(precond, n_brows, minv, r, z, nullptr, partials,
                                                           counter, S, rtol, atol, true);
    FEM_LAUNCH_CHECK();
  }
  if ((rc = read_state()) != FEM_OK) return rc;
  const double rr = hs->rr, bb = hs->bnorm2;
  if (status != ST_CONVERGED && hs->status == ST_CONVERGED) status = ST_CONVERGED;
  if (h_iters) *h_iters = iters;
  if (h_replacements) *h_replacements = replacements;
  if (h_relres) *h_relres = bb > 0 ? sqrt(rr / bb) : sqrt(rr);
  if (status == ST_CONVERGED) return FEM_OK;
  if (status == ST_RUNNING || status == ST_REPLACE) status = FEM_ERR_NOT_CONVERGED;
  set_error("krylov (mixed): status %d after %d iterations, %d replacements (relres %.3e)", status, iters,
            replacements, bb > 0 ? sqrt(rr / bb) : sqrt(rr));
  return status;
}

template <typename T>
int solve_dispatch(int method, int precond, int vec, int64_t n_brows, const int32_t* rp,
                   const int32_t* ci, const int32_t* diag, const T* vals, const T* b, T* x,
                   double rtol, double atol, int maxiter, int check_every, void* work,
                   size_t work_bytes, int* h_iters, double* h_relres, void* stream) {
  FEM_CHECK_ARG(vec == 1 || vec == 3, "vec must be 1 or 3");
  FEM_CHECK_ARG(method == FEM_KRYLOV_CG || method == FEM_KRYLOV_BICGSTAB, "unknown method %d", method);
  FEM_CHECK_ARG(precond >= FEM_PRECOND_NONE && precond <= FEM_PRECOND_BLOCK_JACOBI,
                "unknown preconditioner %d", precond);
  FEM_CHECK_ARG(n_brows > 0, "empty system");
  FEM_CHECK_ARG(rtol >= 0 && atol >= 0, "negative tolerance");
  FEM_CHECK_ARG(bsr_aligned(vals, ci), "vals and col_idx must be 16-byte aligned");
  auto st = as_stream(stream);
  if (vec == 3)
    return solve_impl<3, T>(method, precond, n_brows, rp, ci, diag, vals, b, x, rtol, atol, maxiter,
                            check_every, work, work_bytes, h_iters, h_relres, st);
  return solve_impl<1, T>(method, precond, n_brows, rp, ci, diag, vals, b, x, rtol, atol, maxiter,
                          check_every, work, work_bytes, h_iters, h_relres, st);
}

}  // namespace
}  // namespace fem

extern "C" size_t fem_krylov_workspace_bytes(int method, int precond, int vec, int64_t n_brows,
                                             int fp32) {
  return fem::workspace_bytes(method, precond, vec, n_brows, fp32 ? 4 : 8);
}

extern "C" int fem_krylov_solve_f64(int method, int precond, int vec, int64_t n_brows,
                                    const int32_t* d_row_ptr, const int32_t* d_col_idx,
                                    const int32_t* d_diag, const double* d_vals, const double* d_b,
                                    double* d_x, double rtol, double atol, int maxiter,
                                    int check_every, void* d_work, size_t work_bytes, int* h_iters,
                                    double* h_relres, void* stream) {
  return fem::solve_dispatch<double>(method, precond, vec, n_brows, d_row_ptr, d_col_idx, d_diag,
                                     d_vals, d_b, d_x, rtol, atol, maxiter, check_every, d_work,
                                     work_bytes, h_iters, h_relres, stream);
}

extern "C" int fem_krylov_solve_f32(int method, int precond, int vec, int64_t n_brows,
                                    const int32_t* d_row_ptr, const int32_t* d_col_idx,
                                    const int32_t* d_diag, const float* d_vals, const float* d_b,
                                    float* d_x, double rtol, double atol, int maxiter,
                                    int check_every, void* d_work, size_t work_bytes, int* h_iters,
                                    double* h_relres, void* stream) {
  return fem::solve_dispatch<float>(method, precond, vec, n_brows, d_row_ptr, d_col_idx, d_diag,
                                    d_vals, d_b, d_x, rtol, atol, maxiter, check_every, d_work,
                                    work_bytes, h_iters, h_relres, stream);
}

extern "C" size_t fem_krylov_mixed_workspace_bytes(int precond, int vec, int64_t n_brows) {
  return fem::workspace_bytes(FEM_KRYLOV_CG, precond, vec, n_brows, 4) +
         fem::al256(size_t(n_brows) * vec * sizeof(float));
}

extern "C" int fem_krylov_solve_mixed(int precond, int vec, int64_t n_brows, const int32_t* d_row_ptr,
                                      const int32_t* d_col_idx, const int32_t* d_diag,
                                      const float* d_vals, const double* d_b, double* d_x, double rtol,
                                      double atol, int maxiter, int check_every, double delta,
                                      void* d_work, size_t work_bytes, int* h_iters,
                                      int* h_replacements, double* h_relres, void* stream) {
  FEM_CHECK_ARG(vec == 1 || vec == 3, "vec must be 1 or 3");
  FEM_CHECK_ARG(precond >= FEM_PRECOND_NONE && precond <= FEM_PRECOND_BLOCK_JACOBI,
                "unknown preconditioner %d", precond);
  FEM_CHECK_ARG(n_brows > 0, "empty system");
  FEM_CHECK_ARG(rtol >= 0 && atol >= 0, "negative tolerance");
  FEM_CHECK_ARG(fem::bsr_aligned(d_vals, d_col_idx), "vals and col_idx must be 16-byte aligned");
  auto st = fem::as_stream(stream);
  if (vec == 3)
    return fem::solve_mixed_impl<3>(precond, n_brows, d_row_ptr, d_col_idx, d_diag, d_vals, d_b, d_x, rtol,
                                    atol, maxiter, check_every, delta, d_work, work_bytes, h_iters,
                                    h_replacements, h_relres, st);
  return fem::solve_mixed_impl<1>(precond, n_brows, d_row_ptr, d_col_idx, d_diag, d_vals, d_b, d_x, rtol,
                                  atol, maxiter, check_every, delta, d_work, work_bytes, h_iters,
                                  h_replacements, h_relres, st);
}
