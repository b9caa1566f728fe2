// Geometric multigrid for box-lattice meshes: Galerkin coarse operators,
// trilinear transfer, Chebyshev-Jacobi smoothing, V-cycles and a
// V-cycle-preconditioned CG.  Replaces the reference's optional AMGX path
// (solver.py:136-259) on the meshes box_mesh builds (generate_mesh.py:151-189).
//
// Lattice: node (i, j, k) = (i*ny + j)*nz + k, nx, ny, nz nodes per direction.
// A coarse level keeps every second node per direction (and the last node);
// fine node i of a direction lies between coarse nodes ilo[i] and ilo[i]+1
// with weight whi[i] on the upper one, so prolongation P is trilinear
// interpolation and restriction is P^T.  Coarse operators are P^T (A P): a
// first pass forms B = A P per fine row (27 coarse columns at most), a second
// pass sums the <= 27 fine rows of each coarse block (one thread per block:
// fixed summation order, no atomics).
//
// Smoothing: Chebyshev iteration on D^-1 A over [lmax/ratio, lmax] with
// lmax the Gershgorin bound of D^-1 A (D = the diagonal), kept on the device:
// the kernels derive their Chebyshev coefficients from it, so setup and
// V-cycles never wait for the host.  Each step is one SpMV with its vector
// updates fused into the row epilogue.  Pre- and
// post-smoothing apply the same polynomial, the coarsest level a longer one,
// so a V-cycle is a fixed symmetric positive operator (a CG preconditioner).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "sparse.cuh"

namespace fem {
namespace {

struct Lat {
  int64_t n[3];
};

inline Lat lat_of(const FemMGLevel& L) { return Lat{{L.nodes[0], L.nodes[1], L.nodes[2]}}; }

// 1-D interpolation weight of coarse node I at fine node i
__device__ __forceinline__ double w1(const int32_t* ilo, const double* whi, int64_t i, int64_t I) {
  const int64_t lo = ilo[i];
  if (lo == I) return 1.0 - whi[i];
  if (lo + 1 == I) return whi[i];
  return 0.0;
}

// Fine lattice indices that interpolate from coarse node I along one
// direction: strictly between the neighbouring coarse nodes.
__device__ __forceinline__ void fine_range(const int32_t* cpos, int64_t I, int64_t nc, int64_t nf, int64_t* lo,
                                           int64_t* hi) {
  *lo = I > 0 ? int64_t(cpos[I - 1]) + 1 : 0;
  *hi = I < nc - 1 ? int64_t(cpos[I + 1]) - 1 : nf - 1;
}

// ---- Galerkin coarse operator ---------------------------------------------------
// Window of coarse columns of fine node i along one direction: A P (i, J) can
// be non-zero only for J in base .. base+2, base = ilo[max(i-1, 0)].
__device__ __forceinline__ int64_t col_base(const int32_t* ilo, int64_t i) { return ilo[i > 0 ? i - 1 : 0]; }

// B[i][t] = sum_j A_ij w(j, J_t), J_t = base(i) + (t/9, t/3%3, t%3): one warp
// per fine row.  Lane o stages the row's block of neighbour offset
// o = (a, b, c) in shared memory (the row's blocks are contiguous).  P is a
// tensor product, w(j, J) = wx wy wz, so the 27 x 27 block products factor
// into three contractions of 27 outputs by 3 terms, one direction each, lane
// l forming output l of each:
//   T1[a,b,tz] = sum_c A[a,b,c] wz[c][tz],  T2[a,ty,tz] = sum_b T1[a,b,tz] wy[b][ty],
//   B[tx,ty,tz] = sum_a T2[a,ty,tz] wx[a][tx]   (FP64 sums).
constexpr int kApWarps = 8;
template <int VEC, typename T>
struct ApStage {
  static constexpr int VV = VEC * VEC;
  // staged blocks padded to a 16-byte multiple, read back with 16-byte loads
  static constexpr int PER16 = 16 / int(sizeof(T));
  static constexpr int VVP = ((VV + PER16 - 1) / PER16) * PER16;
  static constexpr int kA = 27 * VVP * int(sizeof(T));  // the row's blocks
  static constexpr int kT = 27 * VV * 8;                 // one FP64 intermediate
  static constexpr int kX = kA > kT ? kA : kT;            // A, then T2
  // both parts start on 16-byte boundaries in every warp's stage (A is read
  // back with 16-byte loads)
  static constexpr int kXr = ((kX + 15) / 16) * 16;
  static constexpr int kWarp = kXr + ((kT + 15) / 16) * 16;
  static_assert(kWarp % 16 == 0 && (VVP * int(sizeof(T))) % 16 == 0, "ap stage alignment");
};
template <int VEC, typename T>
__global__ void __launch_bounds__(kApWarps * 32) ap_kernel(Lat F, const int32_t* __restrict__ fst,
                                                           const T* __restrict__ fv, Lat C, const int32_t* ilo,
                                                           const double* whi, T* B) {
  using S = ApStage<VEC, T>;
  constexpr int VV = S::VV, VVP = S::VVP, PER16 = S::PER16;
  __shared__ __align__(16) unsigned char stage[kApWarps * S::kWarp];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T (*sA)[VVP] = reinterpret_cast<T (*)[VVP]>(stage + wid * S::kWarp);
  double (*sT2)[VV] = reinterpret_cast<double (*)[VV]>(stage + wid * S::kWarp);
  double (*sT1)[VV] = reinterpret_cast<double (*)[VV]>(stage + wid * S::kWarp + S::kXr);
  const int32_t* il[3] = {ilo, ilo + F.n[0], ilo + F.n[0] + F.n[1]};
  const double* wh[3] = {whi, whi + F.n[0], whi + F.n[0] + F.n[1]};
  const int64_t Nf = F.n[0] * F.n[1] * F.n[2];
  const int64_t w0 = int64_t(blockIdx.x) * kApWarps + wid, nw = int64_t(gridDim.x) * kApWarps;
  const int l = lane < 27 ? lane : 26;  // lanes 27-31 mirror lane 26's work and store nothing
  const int td[3] = {l / 9, (l / 3) % 3, l % 3};
  for (int64_t i = w0; i < Nf; i += nw) {
    __syncwarp();  // the previous row's stages are no longer read
    if (lane < 27) {
      const int32_t blk = fst[i * 27 + lane];
#pragma unroll
      for (int e = 0; e < VV; ++e) sA[lane][e] = blk >= 0 ? fv[int64_t(blk) * VV + e] : T(0);
    }
    const int64_t ii[3] = {i / (F.n[1] * F.n[2]), (i / F.n[2]) % F.n[1], i % F.n[2]};
    double w[3][3];  // w[d][k]: weight of column J_d = base + td[d] at fine index ii[d] + k - 1
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int64_t J = col_base(il[d], ii[d]) + td[d];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int64_t j = ii[d] + k - 1;
        w[d][k] = (J < C.n[d] && j >= 0 && j < F.n[d]) ? w1(il[d], wh[d], j, J) : 0.0;
      }
    }
    __syncwarp();
    double acc[VV];
    // z: T1[l = (a, b, tz)] from A[(a, b, c)], c = 0..2
#pragma unroll
    for (int e = 0; e < VV; ++e) acc[e] = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (w[2][c] == 0.0) continue;
      T blk[VVP];
      const uint4* src = reinterpret_cast<const uint4*>(&sA[(l / 3) * 3 + c][0]);
#pragma unroll
      for (int v = 0; v < VVP / PER16; ++v) reinterpret_cast<uint4*>(blk)[v] = src[v];
#pragma unroll
      for (int e = 0; e < VV; ++e) acc[e] = fma(w[2][c], double(blk[e]), acc[e]);
    }
    if (lane < 27)
#pragma unroll
      for (int e = 0; e < VV; ++e) sT1[l][e] = acc[e];
    __syncwarp();
    // y: T2[l = (a, ty, tz)] from T1[(a, b, tz)], b = 0..2 (T2 over A's stage)
#pragma unroll
    for (int e = 0; e < VV; ++e) acc[e] = 0.0;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      if (w[1][b] == 0.0) continue;
      const double* src = sT1[(l / 9) * 9 + b * 3 + l % 3];
#pragma unroll
      for (int e = 0; e < VV; ++e) acc[e] = fma(w[1][b], src[e], acc[e]);
    }
    __syncwarp();  // every lane has read its A blocks before T2 overwrites them
    if (lane < 27)
#pragma unroll
      for (int e = 0; e < VV; ++e) sT2[l][e] = acc[e];
    __syncwarp();
    // x: B[l = (tx, ty, tz)] from T2[(a, ty, tz)], a = 0..2
#pragma unroll
    for (int e = 0; e < VV; ++e) acc[e] = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (w[0][a] == 0.0) continue;
      const double* src = sT2[a * 9 + l % 9];
#pragma unroll
      for (int e = 0; e < VV; ++e) acc[e] = fma(w[0][a], src[e], acc[e]);
    }
    if (lane < 27)
#pragma unroll
      for (int e = 0; e < VV; ++e) B[(i * 27 + lane) * VV + e] = T(acc[e]);
  }
}

// A_c(I, J) = sum_i w(i, I) B[i][J - base(i)]: one thread per coarse block.
template <int VEC, typename T>
__global__ void ptap_kernel(Lat F, Lat C, const int32_t* __restrict__ cst, const T* __restrict__ B, T* cv,
                            const int32_t* cpos, const int32_t* ilo, const double* whi) {
  constexpr int VV = VEC * VEC;
  const int32_t* cp[3] = {cpos, cpos + C.n[0], cpos + C.n[0] + C.n[1]};
  const int32_t* il[3] = {ilo, ilo + F.n[0], ilo + F.n[0] + F.n[1]};
  const double* wh[3] = {whi, whi + F.n[0], whi + F.n[0] + F.n[1]};
  const int64_t Nc = C.n[0] * C.n[1] * C.n[2];
  for (int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < Nc * 27; g += int64_t(gridDim.x) * blockDim.x) {
    const int64_t I = g / 27;
    const int s = int(g - I * 27);
    const int32_t cblk = cst[g];
    if (cblk < 0) continue;
    const int64_t Ic[3] = {I / (C.n[1] * C.n[2]), (I / C.n[2]) % C.n[1], I % C.n[2]};
    const int64_t J[3] = {Ic[0] + s / 9 - 1, Ic[1] + (s / 3) % 3 - 1, Ic[2] + s % 3 - 1};
    int64_t lo[3], hi[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) fine_range(cp[d], Ic[d], C.n[d], F.n[d], &lo[d], &hi[d]);
    double acc[VV];
#pragma unroll
    for (int e = 0; e < VV; ++e) acc[e] = 0.0;
    for (int64_t ix = lo[0]; ix <= hi[0]; ++ix) {
      const double wx = w1(il[0], wh[0], ix, Ic[0]);
      const int64_t tx = J[0] - col_base(il[0], ix);
      if (wx == 0.0 || tx < 0 || tx > 2) continue;
      for (int64_t iy = lo[1]; iy <= hi[1]; ++iy) {
        const double wy = w1(il[1], wh[1], iy, Ic[1]);
        const int64_t ty = J[1] - col_base(il[1], iy);
        if (wy == 0.0 || ty < 0 || ty > 2) continue;
        for (int64_t iz = lo[2]; iz <= hi[2]; ++iz) {
          const double wz = w1(il[2], wh[2], iz, Ic[2]);
          const int64_t tz = J[2] - col_base(il[2], iz);
          if (wz == 0.0 || tz < 0 || tz > 2) continue;
          const double wi = wx * wy * wz;
          const int64_t i = (ix * F.n[1] + iy) * F.n[2] + iz;
          const T* bv = B + ((i * 27) + tx * 9 + ty * 3 + tz) * VV;
#pragma unroll
          for (int e = 0; e < VV; ++e) acc[e] = fma(wi, double(bv[e]), acc[e]);
        }
      }
    }
#pragma unroll
    for (int e = 0; e < VV; ++e) cv[int64_t(cblk) * VV + e] = T(acc[e]);
  }
}

// Coefficients of step k (k >= 1) of Chebyshev iteration on D^-1 A over
// [lmax/ratio, lmax]: d_k = a d_{k-1} + c D^-1 r_k; step 0 is d_0 = D^-1 r_0 / theta.
struct ChebCoef {
  double inv_theta, a, c;
};
__device__ __forceinline__ ChebCoef cheb_coef(const void* lmax_bits, double ratio, int k) {
  const double lmax = __longlong_as_double(*static_cast<const long long*>(lmax_bits));
  const double lmin = lmax / ratio;
  const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin), sigma = theta / delta;
  double rho_prev = 1.0 / sigma, rho = rho_prev;
  for (int j = 1; j <= k; ++j) {
    rho_prev = rho;
    rho = 1.0 / (2.0 * sigma - rho_prev);
  }
  return ChebCoef{1.0 / theta, rho * rho_prev, 2.0 * rho / delta};
}

// ---- transfers ---------------------------------------------------------------
// bc[I] = sum_i w_iI rf[i]   (P^T, one thread per coarse node).  Along each
// direction at most 3 fine nodes lie strictly between the neighbouring coarse
// nodes, so the 27 candidates are unrolled with their weights formed first and
// the gathers issued together; lattice indices fit in 32 bits.
// With dinvc given, the kernel also takes the coarse level's first Chebyshev
// step from a zero start (as cheb_first_kernel: r = b, d0 = D^-1 b / theta,
// x = d0), node by node, so that step needs no launch of its own.
template <int VEC, typename T>
__device__ __forceinline__ void restrict_body(Lat F, Lat C, const int32_t* cpos, const int32_t* ilo,
                                              const double* whi, const T* rf, T* bc, const T* __restrict__ dinvc,
                                              T* rc, T* d0c, T* xc, double inv_theta) {
  const int nc[3] = {int(C.n[0]), int(C.n[1]), int(C.n[2])};
  const int nf[3] = {int(F.n[0]), int(F.n[1]), int(F.n[2])};
  const int32_t* cp[3] = {cpos, cpos + nc[0], cpos + nc[0] + nc[1]};
  const int32_t* il[3] = {ilo, ilo + nf[0], ilo + nf[0] + nf[1]};
  const double* wh[3] = {whi, whi + nf[0], whi + nf[0] + nf[1]};
  const int Nc = nc[0] * nc[1] * nc[2];
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < Nc; I += gridDim.x * blockDim.x) {
    const int Ic[3] = {I / (nc[1] * nc[2]), (I / nc[2]) % nc[1], I % nc[2]};
    int fi[3][3];
    double fw[3][3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int lo = Ic[d] > 0 ? cp[d][Ic[d] - 1] + 1 : 0;
      const int hi = Ic[d] < nc[d] - 1 ? cp[d][Ic[d] + 1] - 1 : nf[d] - 1;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int i = lo + k;
        fi[d][k] = i <= hi ? i : lo;
        fw[d][k] = i <= hi ? w1(il[d], wh[d], i, Ic[d]) : 0.0;
      }
    }
    double acc[VEC];
#pragma unroll
    for (int c = 0; c < VEC; ++c) acc[c] = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const double wab = fw[0][a] * fw[1][b];
        const int rowab = (fi[0][a] * nf[1] + fi[1][b]) * nf[2];
#pragma unroll
        for (int e = 0; e < 3; ++e) {
          const double w = wab * fw[2][e];
          const int i = rowab + fi[2][e];
#pragma unroll
          for (int c = 0; c < VEC; ++c) acc[c] = fma(w, double(rf[int64_t(i) * VEC + c]), acc[c]);
        }
      }
#pragma unroll
    for (int c = 0; c < VEC; ++c) bc[int64_t(I) * VEC + c] = T(acc[c]);
    if (dinvc != nullptr) {
#pragma unroll
      for (int c = 0; c < VEC; ++c) {
        const int64_t q = int64_t(I) * VEC + c;
        const T bq = T(acc[c]);
        rc[q] = bq;
        const T dq = T(double(dinvc[q]) * double(bq) * inv_theta);
        d0c[q] = dq;
        xc[q] = dq;
      }
    }
  }
}

template <int VEC, typename T>
__global__ void restrict_kernel(Lat F, Lat C, const int32_t* cpos, const int32_t* ilo, const double* whi,
                                const T* __restrict__ rf, T* bc, const T* __restrict__ dinvc, T* rc, T* d0c, T* xc,
                                const void* lmaxc, double ratio, int early) {
  pdl_wait();
  // early: the next kernel is coarse_tail_kernel, which reads what this one
  // writes through L2 and may start (and copy its constant data) right away
  if (early) pdl_trigger();
  restrict_body<VEC, T>(F, C, cpos, ilo, whi, rf, bc, dinvc, rc, d0c, xc,
                        dinvc != nullptr ? cheb_coef(lmaxc, ratio, 0).inv_theta : 0.0);
}

// xf[i] += sum_J w_iJ ec[J]   (P, one thread per fine node)
template <int VEC, typename T>
__device__ __forceinline__ void prolong_add_body(Lat F, Lat C, const int32_t* ilo, const double* whi, const T* ec,
                                                 T* xf) {
  const int nf[3] = {int(F.n[0]), int(F.n[1]), int(F.n[2])};
  const int nc1 = int(C.n[1]), nc2 = int(C.n[2]);
  const int32_t* il[3] = {ilo, ilo + nf[0], ilo + nf[0] + nf[1]};
  const double* wh[3] = {whi, whi + nf[0], whi + nf[0] + nf[1]};
  const int Nf = nf[0] * nf[1] * nf[2];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Nf; i += gridDim.x * blockDim.x) {
    const int ii[3] = {i / (nf[1] * nf[2]), (i / nf[2]) % nf[1], i % nf[2]};
    int lo[3];
    double wup[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      lo[d] = il[d][ii[d]];
      wup[d] = wh[d][ii[d]];
    }
    double acc[VEC];
#pragma unroll
    for (int c = 0; c < VEC; ++c) acc[c] = 0.0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int bx = m >> 2, by = (m >> 1) & 1, bz = m & 1;
      const double w = (bx ? wup[0] : 1.0 - wup[0]) * (by ? wup[1] : 1.0 - wup[1]) * (bz ? wup[2] : 1.0 - wup[2]);
      if (w == 0.0) continue;
      const int J = ((lo[0] + bx) * nc1 + (lo[1] + by)) * nc2 + (lo[2] + bz);
#pragma unroll
      for (int c = 0; c < VEC; ++c) acc[c] = fma(w, double(ec[int64_t(J) * VEC + c]), acc[c]);
    }
#pragma unroll
    for (int c = 0; c < VEC; ++c) xf[int64_t(i) * VEC + c] = T(double(xf[int64_t(i) * VEC + c]) + acc[c]);
  }
}

template <int VEC, typename T>
__global__ void prolong_add_kernel(Lat F, Lat C, const int32_t* ilo, const double* whi, const T* __restrict__ ec,
                                   T* xf) {
  pdl_wait();
  prolong_add_body<VEC, T>(F, C, ilo, whi, ec, xf);
}

// ---- Jacobi scaling and the Gershgorin bound of D^-1 A ----------------------
// With absmax_bits given it also finds max |a| over the values (the scale of
// the level's FP16 copy; non-negative floats order like their bit patterns).
template <int VEC, typename T>
__global__ void jacobi_setup_kernel(int64_t n_brows, const int32_t* __restrict__ st, const T* __restrict__ vals,
                                    T* dinv, unsigned long long* lmax_bits, unsigned* absmax_bits) {
  constexpr int VV = VEC * VEC;
  double local = 0.0;
  float amax = 0.0f;
  for (int64_t dof = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; dof < n_brows * VEC;
       dof += int64_t(gridDim.x) * blockDim.x) {
    const int64_t row = dof / VEC;
    const int c = int(dof - row * VEC);
    const int32_t db = st[row * 27 + 13];
    const double aii = db >= 0 ? double(vals[int64_t(db) * VV + c * VEC + c]) : 0.0;
    double rs = 0.0;
    for (int o = 0; o < 27; ++o) {
      const int32_t blk = st[row * 27 + o];
      if (blk < 0) continue;
#pragma unroll
      for (int k = 0; k < VEC; ++k) {
        const double a = fabs(double(vals[int64_t(blk) * VV + c * VEC + k]));
        rs += a;
        amax = fmaxf(amax, float(a));
      }
    }
    const double ad = fabs(aii);
    dinv[dof] = T(ad > 0.0 ? 1.0 / aii : 0.0);
    if (ad > 0.0) local = fmax(local, rs / ad);
  }
  local = fmax(local, __shfl_xor_sync(0xffffffffu, local, 16));
  local = fmax(local, __shfl_xor_sync(0xffffffffu, local, 8));
  local = fmax(local, __shfl_xor_sync(0xffffffffu, local, 4));
  local = fmax(local, __shfl_xor_sync(0xffffffffu, local, 2));
  local = fmax(local, __shfl_xor_sync(0xffffffffu, local, 1));
  // non-negative doubles order like their bit patterns
  if ((threadIdx.x & 31) == 0) atomicMax(lmax_bits, static_cast<unsigned long long>(__double_as_longlong(local)));
  if (absmax_bits != nullptr) {
    for (int o = 16; o >= 1; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    if ((threadIdx.x & 31) == 0) atomicMax(absmax_bits, __float_as_uint(amax));
  }
}

template <typename T>
__global__ void cast_kernel(int64_t n, const double* __restrict__ a, T* b) {
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += int64_t(gridDim.x) * blockDim.x)
    b[k] = T(a[k]);
}
// level 0 values rounded from FP64: the count nnzb*vv is read from row_ptr
template <typename T>
__global__ void cast_vals_kernel(const int32_t* rp, int64_t n_brows, int vv, const double* __restrict__ a, T* b) {
  const int64_t n = int64_t(rp[n_brows]) * vv;
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += int64_t(gridDim.x) * blockDim.x)
    b[k] = T(a[k]);
}

// ---- Chebyshev smoothing ------------------------------------------------------
// First step: (zero start) r = b, x = d; otherwise x += d; d = D^-1 r / theta.
template <typename T>
__global__ void cheb_first_kernel(int64_t n, const T* __restrict__ dinv, const T* b, T* r, T* d, T* x,
                                  const void* lmax, double ratio, int zero_start) {
  pdl_wait();
  const double inv_theta = cheb_coef(lmax, ratio, 0).inv_theta;
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += int64_t(gridDim.x) * blockDim.x) {
    const T rk = zero_start ? b[k] : r[k];
    if (zero_start) r[k] = rk;
    const T dk = T(double(dinv[k]) * double(rk) * inv_theta);
    d[k] = dk;
    x[k] = zero_start ? dk : T(x[k] + dk);
  }
}

// Value types of the row kernels: the level's own (VT = T), or for a level of
// an FP32 hierarchy an FP16 copy of its values scaled by a power of two s
// (VT = __half; the row sums are multiplied by vinv[0] = 1/s).
// q = A d_old; r -= q; d_new = a d_old + c D^-1 r; x += d_new (x += d_old + d_new with fold)
template <int VEC, typename VT, typename T>
__global__ void __launch_bounds__(kRowThreads, kRowBlocksPerSM)
    cheb_step_kernel(int64_t n_brows, const int32_t* rp, const int32_t* ci, const VT* vals, const T* __restrict__ dold,
                     T* dnew, T* r, T* x, const T* __restrict__ dinv, const void* lmax, double ratio, int step,
                     int fold, const double* vinv) {
  pdl_wait();
  const ChebCoef cf = cheb_coef(lmax, ratio, step);
  const double a = cf.a, c = cf.c;
  const double vs = vinv != nullptr ? vinv[0] : 1.0;
  bsr_rows<VEC, VT, T>(
      n_brows, rp, ci, vals, [&](int64_t i) { return dold[i]; },
      [&](int64_t row, int comp, T q) {
        const int64_t i = row * VEC + comp;
        const double rn = double(r[i]) - double(q) * vs;
        r[i] = T(rn);
        const T dn = T(a * double(dold[i]) + c * double(dinv[i]) * rn);
        dnew[i] = dn;
        // fold: the first step's x += d_old was left to this step
        x[i] = fold ? T(T(x[i] + dold[i]) + dn) : T(x[i] + dn);
      });
}

// r -= A d
template <int VEC, typename VT, typename T>
__global__ void __launch_bounds__(kRowThreads, kRowBlocksPerSM)
    cheb_resid_kernel(int64_t n_brows, const int32_t* rp, const int32_t* ci, const VT* vals, const T* __restrict__ d,
                      T* r, const double* vinv) {
  pdl_wait();
  const double vs = vinv != nullptr ? vinv[0] : 1.0;
  bsr_rows<VEC, VT, T>(
      n_brows, rp, ci, vals, [&](int64_t i) { return d[i]; },
      [&](int64_t row, int comp, T q) {
        const int64_t i = row * VEC + comp;
        r[i] = T(double(r[i]) - double(q) * vs);
      });
}

// r = b - A x (values VT, vectors and row sums T)
template <int VEC, typename VT, typename T>
__global__ void __launch_bounds__(kRowThreads, kRowBlocksPerSM)
    mg_residual_kernel(int64_t n_brows, const int32_t* rp, const int32_t* ci, const VT* vals, const T* __restrict__ x,
                       const T* b, T* r, const T* __restrict__ dinv, T* d0, const void* lmax, double ratio,
                       const double* vinv) {
  pdl_wait();
  const double vs = vinv != nullptr ? vinv[0] : 1.0;
  // with d0 given: also the first Chebyshev step's d0 = D^-1 r / theta (its
  // x += d0 is folded into the next step)
  const double inv_theta = d0 != nullptr ? cheb_coef(lmax, ratio, 0).inv_theta : 0.0;
  bsr_rows<VEC, VT, T>(
      n_brows, rp, ci, vals, [&](int64_t i) { return x[i]; },
      [&](int64_t row, int comp, T q) {
        const int64_t i = row * VEC + comp;
        const T ri = T(double(b[i]) - double(q) * vs);
        r[i] = ri;
        if (d0 != nullptr) d0[i] = T(double(dinv[i]) * double(ri) * inv_theta);
      });
}

// ---- exact solve of a small coarsest level -------------------------------------
// Gauss-Jordan inversion in FP64 (no pivoting: the Galerkin operator of an
// SPD operator is SPD, so every pivot is positive).  A pivot that is not
// positive leaves the Jacobi inverse instead.  One CTA of 1024 threads; the
// matrix is gathered into shared memory, then held in registers: thread
// (ty, tx) = (tid / 128, tid % 128) owns column j = tx, rows ty + 8 r
// (r < 16), so with n <= FEM_MG_DENSE_MAX = 128 every entry has an owner.
constexpr int kDenseThreads = 1024;
constexpr int kDenseCols = 128, kDenseRowStep = kDenseThreads / kDenseCols, kDenseRows = 16;
static_assert(FEM_MG_DENSE_MAX <= kDenseCols && FEM_MG_DENSE_MAX <= kDenseRowStep * kDenseRows,
              "dense inverse: one owner per entry");
inline size_t dense_inverse_smem(int n) { return (size_t(n) * n + 2 * n) * sizeof(double); }

template <int VEC, typename T>
__global__ void __launch_bounds__(kDenseThreads)
    dense_inverse_kernel(int n_brows, const int32_t* rp, const int32_t* ci, const T* vals, double* inv) {
  constexpr int VV = VEC * VEC;
  extern __shared__ __align__(16) double dsm[];
  const int n = n_brows * VEC;
  double* M = dsm;
  double* col = dsm + n * n;  // column k of the current pivot
  double* prow = col + n;     // row k
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i < n * n; i += nt) M[i] = 0.0;
  __syncthreads();
  // one thread per stored value (its block row by a scan of the <= 43 row
  // pointers), so the loads are issued together
  const int nvals = rp[n_brows] * VV;
  for (int idx = tid; idx < nvals; idx += nt) {
    const int k = idx / VV, e = idx - (idx / VV) * VV;
    int br = 0;
    while (br + 1 < n_brows && rp[br + 1] <= k) ++br;
    M[(br * VEC + e / VEC) * n + ci[k] * VEC + e % VEC] = double(vals[int64_t(k) * VV + e]);
  }
  __syncthreads();
  const int j = tid % kDenseCols, ty = tid / kDenseCols;
  const bool own = j < n;
  double m[kDenseRows];
#pragma unroll
  for (int r = 0; r < kDenseRows; ++r) {
    const int i = ty + kDenseRowStep * r;
    m[r] = own && i < n ? M[i * n + j] : 0.0;
  }
  // Per pivot k: the owners of row k and column k publish them (barrier);
  // with q_j = M_kj / piv (q_k = 1 / piv), row k becomes q_j and every other
  // row M_ij - M_ik q_j: one broadcast load and one FMA per entry (barrier
  // before the next pivot's row and column overwrite these).
  bool ok = true;
  for (int k = 0; k < n; ++k) {
    if (own) {
#pragma unroll
      for (int r = 0; r < kDenseRows; ++r) {
        const int i = ty + kDenseRowStep * r;
        if (i == k) prow[j] = m[r];
        if (j == k && i < n) col[i] = m[r];
      }
    }
    __syncthreads();
    const double piv = prow[k];  // same value in every thread
    if (!(piv > 0.0) || !isfinite(piv)) {  // uniform exit
      ok = false;
      break;
    }
    if (own) {
      const double ip = __drcp_rn(piv);  // 1 / piv, correctly rounded
      const double qj = j == k ? ip : prow[j] * ip;
      const bool jk = j == k;
#pragma unroll
      for (int r = 0; r < kDenseRows; ++r) {
        const int i = ty + kDenseRowStep * r;
        if (i < n) m[r] = i == k ? qj : fma(-col[i], qj, jk ? 0.0 : m[r]);
      }
    }
    __syncthreads();
  }
  if (ok) {
    if (own) {
#pragma unroll
      for (int r = 0; r < kDenseRows; ++r) {
        const int i = ty + kDenseRowStep * r;
        if (i < n) inv[i * n + j] = m[r];
      }
    }
  } else {
    for (int idx = tid; idx < n * n; idx += nt) inv[idx] = 0.0;
    __syncthreads();
    for (int br = tid; br < n_brows; br += nt)
      for (int k = rp[br]; k < rp[br + 1]; ++k)
        if (ci[k] == br)
          for (int c = 0; c < VEC; ++c) {
            const double a = double(vals[int64_t(k) * VV + c * VEC + c]);
            inv[(br * VEC + c) * n + br * VEC + c] = a > 0.0 ? 1.0 / a : 0.0;
          }
  }
}

// x = inv b (one warp per row)
template <typename T>
__device__ __forceinline__ void dense_apply_body(int n, const double* __restrict__ inv, const T* b, T* x) {
  const int lane = threadIdx.x & 31;
  for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n; row += (gridDim.x * blockDim.x) >> 5) {
    double acc = 0.0;
    for (int j = lane; j < n; j += 32) acc = fma(inv[int64_t(row) * n + j], double(b[j]), acc);
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) x[row] = T(acc);
  }
}

template <typename T>
__global__ void dense_apply_kernel(int n, const double* __restrict__ inv, const T* __restrict__ b, T* x) {
  pdl_wait();
  dense_apply_body<T>(n, inv, b, x);
}

// ---- the coarse end of a V-cycle in one CTA ------------------------------------
// The last levels of a hierarchy are small (the 50^3 lattice ends with 5^3
// and 3^3 nodes) and each of their steps as a launch costs its completion
// and the next launch's dependent loads, 3-5 us, for a few thousand FMAs.
// When their patterns, values, Jacobi scaling, vectors, Chebyshev
// coefficient tables, transfer arrays and (where it fits) the dense coarsest
// inverse fit in one CTA's shared memory, the V-cycle from such a level s
// down runs as one kernel.  The restriction into level s releases it early
// (pdl_trigger after its own wait), so the constant data are copied in while
// that restriction runs; level s's x, b, r and d0 are read after the wait,
// through L2.  The steps are those of vcycle_level and smooth (the same
// coefficients, transfers and dense coarsest solve), separated by
// __syncthreads; the row products take eight lanes per block row.  Level s's
// x goes back to global memory at the end.
constexpr int kTailThreads = 1024;
constexpr int kTailMaxLevels = 4;
constexpr int kTailMaxSteps = 33;  // Chebyshev coefficient tables: steps 0 .. max(nu, coarse_steps)
constexpr size_t kTailSmemMax = 226 * 1024;  // the opt-in limit of one CTA (227 KB) less static shared memory

template <typename T>
struct TailLevel {
  Lat lat;
  int n_brows, nnzb, nu;
  const int32_t* rp;
  const int32_t* ci;
  const T* vals;
  const T* dinv;
  const void* lmax;
  const int32_t* cpos;  // transfer from the finer level (levels after the first)
  const int32_t* ilo;
  const double* whi;
  const double* cinv;  // dense inverse of a coarsest level, or NULL
  // byte offsets of this level's arrays in shared memory (o_inv: its dense
  // inverse, or -1 to read it from global memory; o_cheb: its Chebyshev
  // coefficients, kTailMaxSteps entries; o_cpos, o_ilo, o_whi: the transfer
  // from the finer level, levels after the first)
  int o_vals, o_ci, o_rp, o_dinv, o_x, o_b, o_r, o_d0, o_d1, o_inv, o_cheb, o_cpos, o_ilo, o_whi;
  int n_cpos, n_fine;  // transfer lengths: sum of this level's / the finer level's nodes per direction
};
template <typename T>
struct TailArgs {
  TailLevel<T> lv[kTailMaxLevels];
  int nl;  // levels s .. s + nl - 1
  int nu, coarse_steps;
  int nsteps;  // Chebyshev coefficients per level: steps 0 .. nsteps-1 (<= kTailMaxSteps)
  int pre_done;  // the restriction into level s took its first step
  double ratio;
  T* x;  // level s in global memory: x (in and out), b, r, d0 (in)
  const T* b;
  const T* r;
  const T* d0;
};

// A level's arrays in shared memory (cpos, ilo, whi: levels after the
// first; inv: the global copy when the inverse is not staged)
template <typename T>
struct TailView {
  const T* vals;
  const int32_t* ci;
  const int32_t* rp;
  const T* dinv;
  T *x, *b, *r, *d0, *d1;
  const ChebCoef* cheb;
  const int32_t* cpos;
  const int32_t* ilo;
  const double* whi;
  const double* inv;
};
template <typename T>
__device__ __forceinline__ TailView<T> tail_view(const TailLevel<T>& L, unsigned char* sm) {
  TailView<T> v;
  v.vals = reinterpret_cast<const T*>(sm + L.o_vals);
  v.ci = reinterpret_cast<const int32_t*>(sm + L.o_ci);
  v.rp = reinterpret_cast<const int32_t*>(sm + L.o_rp);
  v.dinv = reinterpret_cast<const T*>(sm + L.o_dinv);
  v.x = reinterpret_cast<T*>(sm + L.o_x);
  v.b = reinterpret_cast<T*>(sm + L.o_b);
  v.r = reinterpret_cast<T*>(sm + L.o_r);
  v.d0 = reinterpret_cast<T*>(sm + L.o_d0);
  v.d1 = reinterpret_cast<T*>(sm + L.o_d1);
  v.cheb = reinterpret_cast<const ChebCoef*>(sm + L.o_cheb);
  v.cpos = L.o_cpos >= 0 ? reinterpret_cast<const int32_t*>(sm + L.o_cpos) : nullptr;
  v.ilo = L.o_ilo >= 0 ? reinterpret_cast<const int32_t*>(sm + L.o_ilo) : nullptr;
  v.whi = L.o_whi >= 0 ? reinterpret_cast<const double*>(sm + L.o_whi) : nullptr;
  v.inv = L.o_inv >= 0 ? reinterpret_cast<const double*>(sm + L.o_inv) : L.cinv;
  return v;
}

// q = (A v)_i for every unknown i of a level held in shared memory; epi(i, q).
// Eight lanes per block row: lane g takes the row's blocks g, g+8, ... for
// every component, and three xor-shuffles sum the eight partial rows (the
// loop runs the same number of times in every lane of the block, so the
// shuffles see full warps).  Pattern indices are clamped to the level's
// shared-memory arrays: a malformed pattern gives wrong values, never an
// access outside them.
constexpr int kTailRowLanes = 8;
template <int VEC, typename T, class EPI>
__device__ __forceinline__ void tail_rows(int n_brows, int nnzb, const TailView<T>& V, const T* v, EPI epi) {
  constexpr int VV = VEC * VEC;
  const int g = threadIdx.x & (kTailRowLanes - 1);
  const int rows_per_pass = blockDim.x / kTailRowLanes;
  for (int base = 0; base < n_brows; base += rows_per_pass) {
    const int row = base + threadIdx.x / kTailRowLanes;
    T acc[VEC];
#pragma unroll
    for (int c = 0; c < VEC; ++c) acc[c] = T(0);
    if (row < n_brows) {
      const int k0 = max(V.rp[row], 0), k1 = min(V.rp[row + 1], nnzb);
      for (int k = k0 + g; k < k1; k += kTailRowLanes) {
        const T* blk = V.vals + k * VV;
        const T* xv = v + min(max(V.ci[k], 0), n_brows - 1) * VEC;
        T xc[VEC];
#pragma unroll
        for (int c = 0; c < VEC; ++c) xc[c] = xv[c];
#pragma unroll
        for (int r = 0; r < VEC; ++r)
#pragma unroll
          for (int c = 0; c < VEC; ++c) acc[r] = fma(blk[r * VEC + c], xc[c], acc[r]);
      }
    }
#pragma unroll
    for (int c = 0; c < VEC; ++c)
#pragma unroll
      for (int o = kTailRowLanes / 2; o >= 1; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
    if (row < n_brows && g < VEC) {
      T q = acc[0];
#pragma unroll
      for (int c = 1; c < VEC; ++c)
        if (g == c) q = acc[c];
      epi(row * VEC + g, q);
    }
  }
}

// smooth() on a level in shared memory, __syncthreads after every step
template <int VEC, typename T>
__device__ void tail_smooth(const TailLevel<T>& L, const TailView<T>& V, int m, bool zero_start, bool want_residual,
                            bool first_done, bool fold) {
  const ChebCoef* cheb = V.cheb;
  const int n = L.n_brows * VEC;
  T* d[2] = {V.d0, V.d1};
  if (!first_done) {
    const double inv_theta = cheb[0].inv_theta;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const T ri = zero_start ? V.b[i] : V.r[i];
      if (zero_start) V.r[i] = ri;
      const T di = T(double(V.dinv[i]) * double(ri) * inv_theta);
      d[0][i] = di;
      V.x[i] = zero_start ? di : T(V.x[i] + di);
    }
    __syncthreads();
  }
  int cur = 0;
  for (int k = 1; k < m; ++k) {
    const ChebCoef cf = cheb[k];
    const T* dold = d[cur];
    T* dnew = d[cur ^ 1];
    const bool fk = fold && k == 1;
    tail_rows<VEC, T>(L.n_brows, L.nnzb, V, dold, [&](int i, T q) {
      const double rn = double(V.r[i]) - double(q);
      V.r[i] = T(rn);
      const T dn = T(cf.a * double(dold[i]) + cf.c * double(V.dinv[i]) * rn);
      dnew[i] = dn;
      V.x[i] = fk ? T(T(V.x[i] + dold[i]) + dn) : T(V.x[i] + dn);
    });
    __syncthreads();
    cur ^= 1;
  }
  if (want_residual) {
    const T* dc = d[cur];
    tail_rows<VEC, T>(L.n_brows, L.nnzb, V, dc, [&](int i, T q) { V.r[i] = T(double(V.r[i]) - double(q)); });
    __syncthreads();
  }
}

// bytes from global to shared memory (dst 16-byte aligned): 16-byte cp.async
// transfers, all in flight together, when src is 16-byte aligned too, else
// 4-byte copies (every array here holds 4- or 8-byte values)
__device__ __forceinline__ void tail_copy(unsigned char* dst, const void* src, int bytes) {
  const unsigned char* s = static_cast<const unsigned char*>(src);
  if ((reinterpret_cast<uintptr_t>(s) & 15u) == 0) {
    const int n16 = bytes >> 4;
    for (int c = threadIdx.x; c < n16; c += blockDim.x) cp_async16(dst + c * 16, s + c * 16);
    for (int w = n16 * 4 + threadIdx.x; w < bytes / 4; w += blockDim.x)
      reinterpret_cast<uint32_t*>(dst)[w] = reinterpret_cast<const uint32_t*>(s)[w];
  } else {
    for (int w = threadIdx.x; w < bytes / 4; w += blockDim.x)
      reinterpret_cast<uint32_t*>(dst)[w] = reinterpret_cast<const uint32_t*>(s)[w];
  }
}

template <int VEC, typename T>
__global__ void __launch_bounds__(kTailThreads, 1) coarse_tail_kernel(const __grid_constant__ TailArgs<T> a) {
  constexpr int VV = VEC * VEC;
  extern __shared__ __align__(16) unsigned char tsm[];
  __shared__ int s_nz[kTailMaxLevels];
  // Constant level data first (no V-cycle kernel writes it).  The stored
  // block counts (row_ptr[n]) are read while the fixed-size copies fly.
  if (threadIdx.x < a.nl) {
    const TailLevel<T>& L = a.lv[threadIdx.x];
    s_nz[threadIdx.x] = min(max(L.rp[L.n_brows], 0), L.nnzb);  // within the bound
  }
  for (int l = 0; l < a.nl; ++l) {
    const TailLevel<T>& L = a.lv[l];
    tail_copy(tsm + L.o_rp, L.rp, (L.n_brows + 1) * 4);
    tail_copy(tsm + L.o_dinv, L.dinv, L.n_brows * VEC * int(sizeof(T)));
    if (L.o_inv >= 0) {
      const int n = L.n_brows * VEC;
      tail_copy(tsm + L.o_inv, L.cinv, n * n * 8);
    }
    if (l > 0) {
      tail_copy(tsm + L.o_cpos, L.cpos, L.n_cpos * 4);
      tail_copy(tsm + L.o_ilo, L.ilo, L.n_fine * 4);
      tail_copy(tsm + L.o_whi, L.whi, L.n_fine * 8);
    }
    if ((threadIdx.x >> 5) == l) {  // warp l: level l's Chebyshev coefficients, one step per lane
      ChebCoef* cheb = reinterpret_cast<ChebCoef*>(tsm + L.o_cheb);
      for (int k = threadIdx.x & 31; k < a.nsteps; k += 32) cheb[k] = cheb_coef(L.lmax, a.ratio, k);
    }
  }
  __syncthreads();
  for (int l = 0; l < a.nl; ++l) {
    const TailLevel<T>& L = a.lv[l];
    tail_copy(tsm + L.o_vals, L.vals, s_nz[l] * VV * int(sizeof(T)));
    tail_copy(tsm + L.o_ci, L.ci, s_nz[l] * 4);
  }
  cp_async_wait_all();
  // Level s's vectors after the wait.  The restriction into level s lets this
  // kernel start early (it calls pdl_trigger after its own wait), so they are
  // read through L2: an L1 line its CTAs loaded on this SM is not refreshed
  // by the wait.
  pdl_wait();
  {
    const TailView<T> V = tail_view(a.lv[0], tsm);
    for (int i = threadIdx.x; i < a.lv[0].n_brows * VEC; i += blockDim.x) {
      V.x[i] = __ldcg(a.x + i);
      V.b[i] = __ldcg(a.b + i);
      V.r[i] = __ldcg(a.r + i);
      V.d0[i] = __ldcg(a.d0 + i);
    }
  }
  __syncthreads();
  const int last = a.nl - 1;
  for (int l = 0; l < last; ++l) {
    const TailLevel<T>& L = a.lv[l];
    const TailLevel<T>& C = a.lv[l + 1];
    const TailView<T> V = tail_view(L, tsm), W = tail_view(C, tsm);
    const int nul = L.nu > 0 ? L.nu : a.nu;
    tail_smooth<VEC, T>(L, V, nul, true, true, l > 0 || a.pre_done, false);
    const bool fuse_next = !(l + 1 == last && C.cinv != nullptr);
    restrict_body<VEC, T>(L.lat, C.lat, W.cpos, W.ilo, W.whi, V.r, W.b, fuse_next ? W.dinv : nullptr, W.r, W.d0, W.x,
                          W.cheb[0].inv_theta);
    __syncthreads();
  }
  {
    const TailLevel<T>& L = a.lv[last];
    const TailView<T> V = tail_view(L, tsm);
    if (L.cinv != nullptr) {
      dense_apply_body<T>(L.n_brows * VEC, V.inv, V.b, V.x);
      __syncthreads();
    } else {
      tail_smooth<VEC, T>(L, V, a.coarse_steps, true, false, last > 0 || a.pre_done, false);
    }
  }
  for (int l = last - 1; l >= 0; --l) {
    const TailLevel<T>& L = a.lv[l];
    const TailLevel<T>& C = a.lv[l + 1];
    const TailView<T> V = tail_view(L, tsm), W = tail_view(C, tsm);
    const int nul = L.nu > 0 ? L.nu : a.nu;
    prolong_add_body<VEC, T>(L.lat, C.lat, W.ilo, W.whi, W.x, V.x);
    __syncthreads();
    // post-smoothing with two or more steps: the residual forms the first
    // step's d0 and the second step adds its x += d0 (as vcycle_level)
    const bool fuse_post = nul >= 2;
    const double inv_theta = V.cheb[0].inv_theta;
    tail_rows<VEC, T>(L.n_brows, L.nnzb, V, V.x, [&](int i, T q) {
      const T ri = T(double(V.b[i]) - double(q));
      V.r[i] = ri;
      if (fuse_post) V.d0[i] = T(double(V.dinv[i]) * double(ri) * inv_theta);
    });
    __syncthreads();
    tail_smooth<VEC, T>(L, V, nul, false, false, fuse_post, fuse_post);
  }
  const TailView<T> V0 = tail_view(a.lv[0], tsm);
  for (int i = threadIdx.x; i < a.lv[0].n_brows * VEC; i += blockDim.x) a.x[i] = V0.x[i];
}

// ---- host side -------------------------------------------------------------------
inline unsigned vgrid(int64_t n) {
  const int64_t b = (n + 255) / 256;
  const int64_t cap = int64_t(num_sms()) * 8;
  return unsigned(b < 1 ? 1 : (b < cap ? b : cap));
}

template <int VEC, typename T>
int check_levels(int nlevels, const FemMGLevel* L) {
  FEM_CHECK_ARG(nlevels >= 1 && nlevels <= 16, "nlevels must be in [1, 16] (got %d)", nlevels);
  FEM_CHECK_ARG(L != nullptr, "levels is NULL");
  for (int l = 0; l < nlevels; ++l) {
    const FemMGLevel& v = L[l];
    FEM_CHECK_ARG(v.nodes[0] >= 2 && v.nodes[1] >= 2 && v.nodes[2] >= 2, "level %d: lattice needs >= 2 nodes per direction", l);
    FEM_CHECK_ARG(v.n_brows == v.nodes[0] * v.nodes[1] * v.nodes[2], "level %d: n_brows != nodes product", l);
    FEM_CHECK_ARG(v.row_ptr && v.col_idx && v.stencil && v.vals && v.dinv && v.r && v.d0 && v.d1 && v.lmax,
                  "level %d: NULL pattern, values, bound slot or work vector", l);
    FEM_CHECK_ARG(bsr_aligned(v.vals, v.col_idx), "level %d: vals and col_idx must be 16-byte aligned", l);
    FEM_CHECK_ARG(v.nu >= 0 && v.nu <= 16, "level %d: nu must be in [0, 16]", l);
    FEM_CHECK_ARG(v.vals_lo == nullptr || (sizeof(T) == 4 && v.lo_scale != nullptr &&
                                           (reinterpret_cast<uintptr_t>(v.vals_lo) & 15u) == 0),
                  "level %d: an FP16 value copy needs an FP32 hierarchy, 16-byte alignment and lo_scale", l);
    FEM_CHECK_ARG(v.cinv == nullptr || (l == nlevels - 1 && v.n_brows * VEC <= FEM_MG_DENSE_MAX),
                  "level %d: a dense inverse is for a coarsest level of at most %d unknowns", l, FEM_MG_DENSE_MAX);
    if (l >= 1) {
      FEM_CHECK_ARG(v.x && v.b && v.cpos && v.ilo && v.whi, "level %d: NULL transfer data or work vector", l);
      for (int d = 0; d < 3; ++d)
        FEM_CHECK_ARG(v.nodes[d] <= L[l - 1].nodes[d], "level %d: coarser than its finer level expected", l);
    }
  }
  return FEM_OK;
}

// The coarse tail (coarse_tail_kernel): FEM_MG_TAIL=0 in the environment
// turns it off.  A level's blocks are bounded by its lattice stencil,
// prod_d (3 n_d - 2) (every coarse level is a lattice operator).
bool mg_tail_enabled() {
  static int on = -1;
  if (on < 0) {
    const char* e = std::getenv("FEM_MG_TAIL");
    on = (e != nullptr && e[0] == '0') ? 0 : 1;
  }
  return on == 1;
}
inline size_t al16(size_t x) { return (x + 15) & ~size_t(15); }

// Fills a's levels s .. nlevels-1 with their shared-memory layout; returns
// the bytes it needs (0 when the levels cannot form a tail).
template <int VEC, typename T>
size_t tail_layout(int s, int nlevels, const FemMGLevel* L, TailArgs<T>* a) {
  const int nl = nlevels - s;
  if (s < 1 || nl < 2 || nl > kTailMaxLevels) return 0;
  size_t off = 0;
  for (int k = 0; k < nl; ++k) {
    const FemMGLevel& v = L[s + k];
    if (v.vals_lo != nullptr || v.n_brows * VEC > (int64_t(1) << 20)) return 0;
    const int64_t nb = (3 * v.nodes[0] - 2) * (3 * v.nodes[1] - 2) * (3 * v.nodes[2] - 2);
    const size_t n = size_t(v.n_brows) * VEC;
    TailLevel<T>& t = a->lv[k];
    t.lat = lat_of(v);
    t.n_brows = int(v.n_brows);
    t.nnzb = int(nb);
    t.nu = v.nu;
    t.rp = v.row_ptr;
    t.ci = v.col_idx;
    t.vals = static_cast<const T*>(v.vals);
    t.dinv = static_cast<const T*>(v.dinv);
    t.lmax = v.lmax;
    t.cpos = v.cpos;
    t.ilo = v.ilo;
    t.whi = v.whi;
    t.cinv = v.cinv;
    t.o_vals = int(off), off = al16(off + size_t(nb) * VEC * VEC * sizeof(T));
    t.o_ci = int(off), off = al16(off + size_t(nb) * 4);
    t.o_rp = int(off), off = al16(off + size_t(v.n_brows + 1) * 4);
    t.o_dinv = int(off), off = al16(off + n * sizeof(T));
    t.o_x = int(off), off = al16(off + n * sizeof(T));
    t.o_b = int(off), off = al16(off + n * sizeof(T));
    t.o_r = int(off), off = al16(off + n * sizeof(T));
    t.o_d0 = int(off), off = al16(off + n * sizeof(T));
    t.o_d1 = int(off), off = al16(off + n * sizeof(T));
    t.o_cheb = int(off), off = al16(off + kTailMaxSteps * sizeof(ChebCoef));
    t.o_inv = -1;
    t.o_cpos = t.o_ilo = t.o_whi = -1;
    t.n_cpos = t.n_fine = 0;
    if (k > 0) {
      const FemMGLevel& f = L[s + k - 1];
      t.n_cpos = int(v.nodes[0] + v.nodes[1] + v.nodes[2]);
      t.n_fine = int(f.nodes[0] + f.nodes[1] + f.nodes[2]);
      t.o_cpos = int(off), off = al16(off + size_t(t.n_cpos) * 4);
      t.o_ilo = int(off), off = al16(off + size_t(t.n_fine) * 4);
      t.o_whi = int(off), off = al16(off + size_t(t.n_fine) * 8);
    }
    if (off > kTailSmemMax) return 0;
  }
  // the dense inverse of the coarsest level too, where it still fits
  TailLevel<T>& c = a->lv[nl - 1];
  if (c.cinv != nullptr) {
    const size_t n = size_t(c.n_brows) * VEC;
    if (al16(off + n * n * 8) <= kTailSmemMax) {
      c.o_inv = int(off);
      off = al16(off + n * n * 8);
    }
  }
  a->nl = nl;
  return off;
}

// Chebyshev steps the tail from level s takes on one level, at most (its
// coefficient tables hold steps 0 .. that)
inline int tail_steps(int s, int nlevels, const FemMGLevel* L, int nu, int coarse_steps) {
  int m = 1;
  for (int l = s; l < nlevels - 1; ++l) m = std::max(m, L[l].nu > 0 ? L[l].nu : nu);
  if (L[nlevels - 1].cinv == nullptr) m = std::max(m, coarse_steps);
  return m;
}

// First level (>= 1) from which the V-cycle runs as one coarse_tail_kernel,
// or -1.
template <int VEC, typename T>
int tail_start(int nlevels, const FemMGLevel* L, int nu, int coarse_steps) {
  if (!mg_tail_enabled()) return -1;
  TailArgs<T> a{};
  for (int s = 1; s <= nlevels - 2; ++s)
    if (tail_steps(s, nlevels, L, nu, coarse_steps) < kTailMaxSteps && tail_layout<VEC, T>(s, nlevels, L, &a) > 0)
      return s;
  return -1;
}

template <int VEC, typename T>
int launch_tail(int s, int nlevels, const FemMGLevel* L, int nu, int coarse_steps, double ratio, bool pre_done,
                cudaStream_t st) {
  TailArgs<T> a{};
  const size_t bytes = tail_layout<VEC, T>(s, nlevels, L, &a);
  FEM_CHECK_ARG(bytes > 0, "coarse tail: levels %d.. do not fit", s);
  a.nu = nu;
  a.coarse_steps = coarse_steps;
  a.nsteps = tail_steps(s, nlevels, L, nu, coarse_steps) + 1;
  FEM_CHECK_ARG(a.nsteps <= kTailMaxSteps, "coarse tail: %d Chebyshev steps exceed its tables", a.nsteps - 1);
  a.pre_done = pre_done ? 1 : 0;
  a.ratio = ratio;
  a.x = static_cast<T*>(L[s].x);
  a.b = static_cast<const T*>(L[s].b);
  a.r = static_cast<const T*>(L[s].r);
  a.d0 = static_cast<const T*>(L[s].d0);
  FEM_CUDA_TRY(launch_pdl(coarse_tail_kernel<VEC, T>, 1, kTailThreads, bytes, st, a));
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}

template <int VEC, typename T>
int ensure_attrs() {
  int rc;
  {
    static std::mutex mu;  // per instantiation, once per device
    static std::set<int> done;
    int dev = 0;
    FEM_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (!done.count(dev)) {
      FEM_CUDA_TRY(cudaFuncSetAttribute(coarse_tail_kernel<VEC, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        int(kTailSmemMax)));
      done.insert(dev);
    }
  }
  if ((rc = ensure_smem_attr(cheb_step_kernel<VEC, T, T>)) != FEM_OK) return rc;
  if ((rc = ensure_smem_attr(cheb_resid_kernel<VEC, T, T>)) != FEM_OK) return rc;
  if ((rc = ensure_smem_attr(mg_residual_kernel<VEC, T, T>)) != FEM_OK) return rc;
  if constexpr (sizeof(T) == 4) {
    if ((rc = ensure_smem_attr(cheb_step_kernel<VEC, __half, T>)) != FEM_OK) return rc;
    if ((rc = ensure_smem_attr(cheb_resid_kernel<VEC, __half, T>)) != FEM_OK) return rc;
    if ((rc = ensure_smem_attr(mg_residual_kernel<VEC, __half, T>)) != FEM_OK) return rc;
  }
  return FEM_OK;
}

// ---- FP16 copy of a level's values (FP32 hierarchies) ---------------------------
// a16 = round(a s) with s = 2^e the largest power of two with max|a| s <=
// 2^14 (well inside FP16's range); scale[0] = 1/s for the row kernels.
__global__ void half_vals_kernel(const int32_t* rp, int64_t n_brows, int vv, const float* __restrict__ a,
                                 const unsigned* maxbits, __half* a16, double* scale) {
  const float m = __uint_as_float(*maxbits);
  const int e = m > 0.0f ? 14 - ilogbf(m) - 1 : 0;
  const float s = ldexpf(1.0f, e);
  if (blockIdx.x == 0 && threadIdx.x == 0) scale[0] = ldexp(1.0, -e);
  const int64_t n = int64_t(rp[n_brows]) * vv;
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += int64_t(gridDim.x) * blockDim.x)
    a16[k] = __float2half_rn(a[k] * s);
}

size_t setup_scratch_bytes(int vec, int64_t fine_n_brows, size_t elem) {
  return size_t(fine_n_brows) * 27 * vec * vec * elem;
}

template <int VEC, typename T>
int setup_impl(int nlevels, const FemMGLevel* L, const double* fine64, void* scratch, size_t scratch_bytes,
               cudaStream_t st) {
  int rc = check_levels<VEC, T>(nlevels, L);
  if (rc != FEM_OK) return rc;
  constexpr int VV = VEC * VEC;
  FEM_CHECK_ARG(nlevels == 1 || (scratch != nullptr && scratch_bytes >= setup_scratch_bytes(VEC, L[0].n_brows, sizeof(T))),
                "setup scratch too small (%zu < %zu)", scratch_bytes, setup_scratch_bytes(VEC, L[0].n_brows, sizeof(T)));
  T* B = static_cast<T*>(scratch);
  for (int l = 0; l < nlevels; ++l) {
    if (l == 0 && fine64 != nullptr) {
      cast_vals_kernel<T><<<unsigned(num_sms()) * 8, 256, 0, st>>>(L[0].row_ptr, L[0].n_brows, VV, fine64,
                                                                  static_cast<T*>(L[0].vals));
      FEM_LAUNCH_CHECK();
    }
    if (l >= 1) {
      const Lat F = lat_of(L[l - 1]), C = lat_of(L[l]);
      const int64_t apb = (L[l - 1].n_brows + kApWarps - 1) / kApWarps;
      const unsigned apg = unsigned(apb < int64_t(num_sms()) * 16 ? apb : int64_t(num_sms()) * 16);
      ap_kernel<VEC, T><<<apg, kApWarps * 32, 0, st>>>(F, L[l - 1].stencil,
                                                                     static_cast<const T*>(L[l - 1].vals), C, L[l].ilo,
                                                                     L[l].whi, B);
      FEM_LAUNCH_CHECK();
      ptap_kernel<VEC, T><<<vgrid(L[l].n_brows * 27), 256, 0, st>>>(F, C, L[l].stencil, B, static_cast<T*>(L[l].vals),
                                                                   L[l].cpos, L[l].ilo, L[l].whi);
      FEM_LAUNCH_CHECK();
    }
    // the level's FP16 copy (FP32 hierarchies): its scale comes from the
    // max |a| the Jacobi setup finds
    const bool lo = sizeof(T) == 4 && L[l].vals_lo != nullptr;
    unsigned* maxbits = lo ? reinterpret_cast<unsigned*>(L[l].lo_scale + 1) : nullptr;
    if (lo) FEM_CUDA_TRY(cudaMemsetAsync(maxbits, 0, sizeof(unsigned), st));
    FEM_CUDA_TRY(cudaMemsetAsync(L[l].lmax, 0, sizeof(unsigned long long), st));
    jacobi_setup_kernel<VEC, T><<<vgrid(L[l].n_brows * VEC), 256, 0, st>>>(
        L[l].n_brows, L[l].stencil, static_cast<const T*>(L[l].vals), static_cast<T*>(L[l].dinv),
        static_cast<unsigned long long*>(L[l].lmax), maxbits);
    FEM_LAUNCH_CHECK();
    if (lo) {
      half_vals_kernel<<<unsigned(num_sms()) * 8, 256, 0, st>>>(L[l].row_ptr, L[l].n_brows, VV,
                                                                reinterpret_cast<const float*>(L[l].vals), maxbits,
                                                                static_cast<__half*>(L[l].vals_lo), L[l].lo_scale);
      FEM_LAUNCH_CHECK();
    }
    if (L[l].cinv != nullptr) {
      const int n = int(L[l].n_brows) * VEC;
      const size_t sm = dense_inverse_smem(n);
      static std::mutex attr_mu;  // per instantiation, once per device
      static std::set<int> attr_done;
      int dev = 0;
      FEM_CUDA_TRY(cudaGetDevice(&dev));
      {
        std::lock_guard<std::mutex> lock(attr_mu);
        if (!attr_done.count(dev)) {
          FEM_CUDA_TRY(cudaFuncSetAttribute(dense_inverse_kernel<VEC, T>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            int(dense_inverse_smem(FEM_MG_DENSE_MAX))));
          attr_done.insert(dev);
        }
      }
      dense_inverse_kernel<VEC, T><<<1, kDenseThreads, sm, st>>>(int(L[l].n_brows), L[l].row_ptr, L[l].col_idx,
                                                                 static_cast<const T*>(L[l].vals), L[l].cinv);
      FEM_LAUNCH_CHECK();
    }
  }
  return ensure_attrs<VEC, T>();
}

// m Chebyshev steps on level l (x, r, d0/d1 of the level; b as rhs).  With
// want_residual the level's r ends as b - A x.  first_done: the first step
// was taken by the kernel before (restriction from a zero start, or the
// residual's d0 with fold, whose x += d0 the second step then adds).
template <int VEC, typename T>
int smooth(const FemMGLevel& L, const T* b, T* x, int m, double ratio, bool zero_start, bool want_residual,
           cudaStream_t st, bool first_done = false, bool fold = false) {
  const int64_t n = L.n_brows * VEC;
  T* r = static_cast<T*>(L.r);
  T* d[2] = {static_cast<T*>(L.d0), static_cast<T*>(L.d1)};
  const T* dinv = static_cast<const T*>(L.dinv);
  const T* vals = static_cast<const T*>(L.vals);
  const unsigned rg = row_grid<T>(L.n_brows);
  if (!first_done) {
    FEM_CUDA_TRY(launch_pdl(cheb_first_kernel<T>, vgrid(n), 256, 0, st, n, dinv, b, r, d[0], x, L.lmax, ratio,
                            zero_start ? 1 : 0));
    FEM_LAUNCH_CHECK();
  }
  const bool lo = sizeof(T) == 4 && L.vals_lo != nullptr;  // the level's FP16 value copy
  const __half* v16 = static_cast<const __half*>(L.vals_lo);
  const double* vinv = lo ? L.lo_scale : nullptr;
  int cur = 0;
  for (int k = 1; k < m; ++k) {
    if (lo)
      FEM_CUDA_TRY(launch_pdl(cheb_step_kernel<VEC, __half, T>, rg, kRowThreads, bsr_rows_smem(), st, L.n_brows,
                              L.row_ptr, L.col_idx, v16, static_cast<const T*>(d[cur]), d[cur ^ 1], r, x, dinv,
                              L.lmax, ratio, k, (fold && k == 1) ? 1 : 0, vinv));
    else
      FEM_CUDA_TRY(launch_pdl(cheb_step_kernel<VEC, T, T>, rg, kRowThreads, bsr_rows_smem(), st, L.n_brows,
                              L.row_ptr, L.col_idx, vals, static_cast<const T*>(d[cur]), d[cur ^ 1], r, x, dinv,
                              L.lmax, ratio, k, (fold && k == 1) ? 1 : 0, vinv));
    FEM_LAUNCH_CHECK();
    cur ^= 1;
  }
  if (want_residual) {
    if (lo)
      FEM_CUDA_TRY(launch_pdl(cheb_resid_kernel<VEC, __half, T>, rg, kRowThreads, bsr_rows_smem(), st, L.n_brows,
                              L.row_ptr, L.col_idx, v16, static_cast<const T*>(d[cur]), r, vinv));
    else
      FEM_CUDA_TRY(launch_pdl(cheb_resid_kernel<VEC, T, T>, rg, kRowThreads, bsr_rows_smem(), st, L.n_brows,
                              L.row_ptr, L.col_idx, vals, static_cast<const T*>(d[cur]), r, vinv));
    FEM_LAUNCH_CHECK();
  }
  return FEM_OK;
}

// pre_done: the restriction into this level already took its first
// smoothing step.
template <int VEC, typename T>
int vcycle_level(int l, int nlevels, const FemMGLevel* L, int nu, int coarse_steps, double ratio, const T* b, T* x,
                 cudaStream_t st, bool pre_done = false) {
  int rc;
  if (l >= 1 && static_cast<const void*>(b) == L[l].b && static_cast<const void*>(x) == L[l].x &&
      tail_start<VEC, T>(nlevels, L, nu, coarse_steps) == l)
    return launch_tail<VEC, T>(l, nlevels, L, nu, coarse_steps, ratio, pre_done, st);
  if (l == nlevels - 1) {
    if (L[l].cinv != nullptr) {
      const int n = int(L[l].n_brows) * VEC;
      FEM_CUDA_TRY(launch_pdl(dense_apply_kernel<T>, unsigned((n + 7) / 8), 256, 0, st, n,
                              static_cast<const double*>(L[l].cinv), b, x));
      FEM_LAUNCH_CHECK();
      return FEM_OK;
    }
    return smooth<VEC, T>(L[l], b, x, coarse_steps, ratio, true, false, st, pre_done);
  }
  const int nul = L[l].nu > 0 ? L[l].nu : nu;
  if ((rc = smooth<VEC, T>(L[l], b, x, nul, ratio, true, true, st, pre_done)) != FEM_OK) return rc;
  const FemMGLevel& C = L[l + 1];
  T* bc = static_cast<T*>(C.b);
  T* xc = static_cast<T*>(C.x);
  // the next level starts with a zero-start Chebyshev step unless it is a
  // coarsest level solved by its dense inverse: the restriction takes it
  const bool fuse_next = !(l + 1 == nlevels - 1 && C.cinv != nullptr);
  FEM_CUDA_TRY(launch_pdl(restrict_kernel<VEC, T>, vgrid(C.n_brows), 256, 0, st, lat_of(L[l]), lat_of(C), C.cpos,
                          C.ilo, C.whi, static_cast<const T*>(L[l].r), bc,
                          fuse_next ? static_cast<const T*>(C.dinv) : static_cast<const T*>(nullptr),
                          static_cast<T*>(C.r), static_cast<T*>(C.d0), xc, static_cast<const void*>(C.lmax), ratio,
                          tail_start<VEC, T>(nlevels, L, nu, coarse_steps) == l + 1 ? 1 : 0));
  FEM_LAUNCH_CHECK();
  if ((rc = vcycle_level<VEC, T>(l + 1, nlevels, L, nu, coarse_steps, ratio, bc, xc, st, fuse_next)) != FEM_OK)
    return rc;
  FEM_CUDA_TRY(launch_pdl(prolong_add_kernel<VEC, T>, vgrid(L[l].n_brows), 256, 0, st, lat_of(L[l]), lat_of(C), C.ilo,
                          C.whi, static_cast<const T*>(xc), x));
  FEM_LAUNCH_CHECK();
  // post-smoothing with two or more steps: the residual kernel forms the
  // first step's d0 and the second step adds its x += d0
  const bool fuse_post = nul >= 2;
  T* d0p = fuse_post ? static_cast<T*>(L[l].d0) : static_cast<T*>(nullptr);
  if (sizeof(T) == 4 && L[l].vals_lo != nullptr)
    FEM_CUDA_TRY(launch_pdl(mg_residual_kernel<VEC, __half, T>, row_grid<T>(L[l].n_brows), kRowThreads,
                            bsr_rows_smem(), st, L[l].n_brows, L[l].row_ptr, L[l].col_idx,
                            static_cast<const __half*>(L[l].vals_lo), static_cast<const T*>(x), b,
                            static_cast<T*>(L[l].r), static_cast<const T*>(L[l].dinv), d0p,
                            static_cast<const void*>(L[l].lmax), ratio, static_cast<const double*>(L[l].lo_scale)));
  else
    FEM_CUDA_TRY(launch_pdl(mg_residual_kernel<VEC, T, T>, row_grid<T>(L[l].n_brows), kRowThreads, bsr_rows_smem(),
                            st, L[l].n_brows, L[l].row_ptr, L[l].col_idx, static_cast<const T*>(L[l].vals),
                            static_cast<const T*>(x), b, static_cast<T*>(L[l].r), static_cast<const T*>(L[l].dinv),
                            d0p, static_cast<const void*>(L[l].lmax), ratio, static_cast<const double*>(nullptr)));
  FEM_LAUNCH_CHECK();
  return smooth<VEC, T>(L[l], b, x, nul, ratio, false, false, st, fuse_post, fuse_post);
}

template <int VEC, typename T>
int vcycle_impl(int nlevels, const FemMGLevel* L, int nu, int coarse_steps, double ratio, const T* rhs, T* z,
                cudaStream_t st) {
  FEM_CHECK_ARG(rhs != nullptr && z != nullptr, "rhs and z must not be NULL");
  FEM_CHECK_ARG(nu >= 1 && nu <= 16 && coarse_steps >= 1 && coarse_steps <= 512, "nu in [1,16], coarse_steps in [1,512]");
  FEM_CHECK_ARG(ratio > 1.0, "ratio must exceed 1");
  FEM_CHECK_ARG(L[0].n_brows < (int64_t(1) << 31), "lattice node indices must fit in 32 bits");
  return vcycle_level<VEC, T>(0, nlevels, L, nu, coarse_steps, ratio, rhs, z, st);
}

// ---- V-cycle preconditioned CG (FP64) -------------------------------------------
struct PState {
  double gamma, alpha, beta, rr, tol2, bb, pq;
  double true_rr;  // ||b - A x||^2 at exit
  int iter, status, maxiter, first;
  int loops;  // bodies run by the device-side loop (its own bound)
};
enum : int { PS_RUNNING = 0, PS_CONVERGED = 1 };

template <int VEC>
__global__ void pcg_init_kernel(int64_t n, const double* r, const double* b, double* partials, unsigned* counter,
                                PState* S, double rtol, double atol) {
  double v[2] = {0.0, 0.0};
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += int64_t(gridDim.x) * blockDim.x) {
    v[0] = fma(r[k], r[k], v[0]);
    v[1] = fma(b[k], b[k], v[1]);
  }
  double tot[2];
  if (last_block_reduce<2>(v, partials, counter, tot)) {
    S->rr = tot[0];
    S->bb = tot[1];
    S->tol2 = fmax(rtol * rtol * tot[1], atol * atol);
    S->iter = 0;
    S->first = 1;
    S->gamma = 0.0;
    S->beta = 0.0;
    if (!isfinite(tot[0]) || !isfinite(tot[1])) S->status = FEM_ERR_NONFINITE;
    else if (tot[0] <= S->tol2) S->status = PS_CONVERGED;
    else if (S->maxiter <= 0) S->status = FEM_ERR_NOT_CONVERGED;
    else S->status = PS_RUNNING;
  }
}

// ||q||^2 into S->true_rr (the exit check: q = b - A x)
__global__ void pcg_true_rr_kernel(int64_t n, const double* q, double* partials, unsigned* counter, PState* S) {
  double v[1] = {0.0};
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += int64_t(gridDim.x) * blockDim.x)
    v[0] = fma(q[k], q[k], v[0]);
  double tot[1];
  if (last_block_reduce<1>(v, partials, counter, tot)) S->true_rr = tot[0];
}

// Chronopoulos-Gear form of preconditioned CG: one product and one fused pair
// of reductions per iteration.  With z = M r (the V-cycle) and w = A z,
//   gamma = r.z, delta = z.w, beta = gamma / gamma_old,
//   alpha = gamma / (delta - beta gamma / alpha_old)   (= gamma / p.Ap),
//   p = z + beta p, q = w + beta q (= A p), x += alpha p, r -= alpha q.
// w = A z with gamma and delta; the last block forms beta and alpha.  z is
// read as ZT (FP32 when the hierarchy is FP32) and widened on the fly.
template <int VEC, typename VT, typename ZT>
__global__ void __launch_bounds__(kRowThreads, kRowBlocksPerSM)
    pcg_spmv_kernel(int64_t n_brows, const int32_t* rp, const int32_t* ci, const VT* vals, const ZT* __restrict__ z,
                    const double* __restrict__ r, double* w, double* partials, unsigned* counter, PState* S) {
  pdl_wait();
  if (S->status != PS_RUNNING) return;
  double v[2] = {0.0, 0.0};
  bsr_rows<VEC, VT, double>(
      n_brows, rp, ci, vals, [&](int64_t i) { return double(z[i]); },
      [&](int64_t row, int c, double wo) {
        const int64_t i = row * VEC + c;
        const double zi = double(z[i]);
        w[i] = wo;
        v[0] = fma(r[i], zi, v[0]);
        v[1] = fma(zi, wo, v[1]);
      });
  double tot[2];
  if (last_block_reduce<2>(v, partials, counter, tot)) {
    const double g = tot[0], dl = tot[1];
    if (!isfinite(g) || !isfinite(dl)) {
      S->status = FEM_ERR_NONFINITE;
    } else if (!(g > 0.0)) {
      S->status = FEM_ERR_BREAKDOWN;  // preconditioner lost definiteness (or r = 0)
    } else {
      const double beta = S->first ? 0.0 : g / S->gamma;
      const double pq = S->first ? dl : dl - beta * g / S->alpha;
      if (!(pq > 0.0)) {
        S->status = FEM_ERR_BREAKDOWN;  // operator not positive definite along p
      } else {
        S->beta = beta;
        S->gamma = g;
        S->pq = pq;
        S->alpha = g / pq;
        S->first = 0;
      }
    }
  }
}

// p = z + beta p; q = w + beta q; x += alpha p; r -= alpha q; rr = r.r;
// bookkeeping.  Also rounds r into the FP32 hierarchy's right-hand side when
// r32 is given.
template <typename ZT>
__global__ void pcg_update_kernel(int64_t n, const ZT* __restrict__ z, const double* __restrict__ w, double* x,
                                  double* r, double* p, double* q, float* r32, double* partials, unsigned* counter,
                                  PState* S) {
  pdl_wait();
  if (S->status != PS_RUNNING) return;
  const double alpha = S->alpha, beta = S->beta;
  double v[1] = {0.0};
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += int64_t(gridDim.x) * blockDim.x) {
    const double pk = fma(beta, p[k], double(z[k]));
    const double qk = fma(beta, q[k], w[k]);
    p[k] = pk;
    q[k] = qk;
    x[k] = fma(alpha, pk, x[k]);
    const double rk = fma(-alpha, qk, r[k]);
    r[k] = rk;
    if (r32 != nullptr) r32[k] = float(rk);
    v[0] = fma(rk, rk, v[0]);
  }
  double tot[1];
  if (last_block_reduce<1>(v, partials, counter, tot)) {
    S->iter += 1;
    S->rr = tot[0];
    if (!isfinite(tot[0])) S->status = FEM_ERR_NONFINITE;
    else if (tot[0] <= S->tol2) S->status = PS_CONVERGED;
    else if (S->iter >= S->maxiter) S->status = FEM_ERR_NOT_CONVERGED;
  }
}

// Condition of the device-side iteration loop (a WHILE node of the solve
// graph): continue while the state is RUNNING.  The loop keeps its own count
// of bodies run, so it ends after maxiter bodies whatever the state says.
__global__ void pcg_cond_kernel(PState* S, cudaGraphConditionalHandle h, int in_body) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (in_body) S->loops += 1;
  const bool go = S->status == PS_RUNNING && S->loops < S->maxiter;
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

inline size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

// Cached CUDA graphs of PCG iteration chunks (V-cycles included): the launch
// sequence depends only on the pointers and parameters in the key, so one
// capture serves every later solve on the same hierarchy and buffers.
// FEM_MG_GRAPHS=0 in the environment launches every kernel directly.
bool mg_graphs_enabled() {
  static int on = -1;
  if (on < 0) {
    const char* e = std::getenv("FEM_MG_GRAPHS");
    on = (e != nullptr && e[0] == '0') ? 0 : 1;
  }
  return on == 1;
}
std::mutex g_mg_mu;
struct MGGraph {
  cudaGraphExec_t exec;
  int64_t kernels;  // launches one replay stands for
};
std::map<std::string, MGGraph>& mg_graph_cache() {
  static std::map<std::string, MGGraph> m;
  return m;
}
cudaStream_t mg_capture_stream() {
  static std::mutex mu;
  static cudaStream_t s[64] = {nullptr};
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (s[dev] == nullptr && cudaStreamCreateWithFlags(&s[dev], cudaStreamNonBlocking) != cudaSuccess) s[dev] = nullptr;
  return s[dev];
}

// Graph: condition kernel -> WHILE node (body: one iteration, then the
// condition kernel).  Returns nullptr when any step fails (the caller then
// launches directly); *nbody = kernels per body.
template <typename F>
cudaGraphExec_t build_loop_graph(PState* S, F&& body_fn, int64_t* nbody) {
  cudaStream_t cap = mg_capture_stream();
  if (cap == nullptr) return nullptr;
  cudaGraph_t g = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) return nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphConditionalHandle h = 0;
  cudaGraphNode_t kn = nullptr, wn = nullptr;
  bool ok = cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault) == cudaSuccess;
  if (ok) {
    int first = 0;
    void* args[] = {&S, &h, &first};
    cudaKernelNodeParams kp{};
    kp.func = reinterpret_cast<void*>(pcg_cond_kernel);
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(32);
    kp.sharedMemBytes = 0;
    kp.kernelParams = args;
    kp.extra = nullptr;
    ok = cudaGraphAddKernelNode(&kn, g, nullptr, 0, &kp) == cudaSuccess;
  }
  cudaGraphNodeParams cp{};
  if (ok) {
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    ok = cudaGraphAddNode(&wn, g, &kn, 1, &cp) == cudaSuccess;
  }
  if (ok) {
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    ok = cudaStreamBeginCaptureToGraph(cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
         cudaSuccess;
    if (ok) {
      const int64_t c0 = launch_counter().load();
      int lrc = body_fn(cap);
      if (lrc == FEM_OK) {
        pcg_cond_kernel<<<1, 32, 0, cap>>>(S, h, 1);
        if (cudaGetLastError() != cudaSuccess) lrc = FEM_ERR_CUDA;
      }
      const int64_t nk = launch_counter().load() - c0;
      launch_counter().fetch_sub(nk, std::memory_order_relaxed);  // counted when run
      *nbody = nk + 1;
      cudaGraph_t out = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(cap, &out);
      ok = lrc == FEM_OK && ec == cudaSuccess;
    }
  }
  if (ok && cudaGraphInstantiate(&exec, g, 0) != cudaSuccess) exec = nullptr;
  cudaGraphDestroy(g);
  cudaGetLastError();  // a failed build falls back to direct launches
  return exec;
}

size_t pcg_workspace_bytes(int vec, int64_t n_brows) {
  const size_t n = size_t(n_brows) * vec;
  return 256 + 256 + al256(size_t(num_sms()) * 8 * 4 * sizeof(double)) + 5 * al256(n * sizeof(double));
}

template <int VEC, typename VT>
int pcg_impl(int64_t n_brows, const int32_t* rp, const int32_t* ci, const VT* vals, const double* b, double* x,
             double rtol, double atol, int maxiter, int check_every, int nlevels, const FemMGLevel* L, int fp32,
             int nu, int coarse_steps, double ratio, void* work, size_t work_bytes, int* h_iters, double* h_relres,
             cudaStream_t st) {
  const int64_t n = n_brows * VEC;
  const size_t need = pcg_workspace_bytes(VEC, n_brows);
  FEM_CHECK_ARG(work != nullptr && work_bytes >= need, "mg pcg workspace too small (%zu < %zu)", work_bytes, need);
  FEM_CHECK_ARG(rp && ci && vals && b && x, "NULL operator or vector");
  FEM_CHECK_ARG(bsr_aligned(vals, ci), "vals and col_idx must be 16-byte aligned");
  FEM_CHECK_ARG(nlevels >= 1 && L != nullptr && L[0].n_brows == n_brows, "level 0 must be the operator's lattice");
  FEM_CHECK_ARG(n_brows < (int64_t(1) << 31), "lattice node indices must fit in 32 bits");
  FEM_CHECK_ARG(!fp32 || (L[0].x != nullptr && L[0].b != nullptr), "FP32 hierarchy needs level 0 x and b");
  if (check_every <= 0) check_every = 4;
  char* p8 = static_cast<char*>(work);
  PState* S = reinterpret_cast<PState*>(p8);
  unsigned* counter = reinterpret_cast<unsigned*>(p8 + 256);
  double* partials = reinterpret_cast<double*>(p8 + 512);
  p8 += 512 + al256(size_t(num_sms()) * 8 * 4 * sizeof(double));
  double* r = reinterpret_cast<double*>(p8);
  double* z = reinterpret_cast<double*>(p8 + al256(n * sizeof(double)));
  double* pv = reinterpret_cast<double*>(p8 + 2 * al256(n * sizeof(double)));
  double* q = reinterpret_cast<double*>(p8 + 3 * al256(n * sizeof(double)));
  double* w = reinterpret_cast<double*>(p8 + 4 * al256(n * sizeof(double)));
  int rc;
  if ((rc = ensure_smem_attr(pcg_spmv_kernel<VEC, VT, float>)) != FEM_OK) return rc;
  if ((rc = ensure_smem_attr(pcg_spmv_kernel<VEC, VT, double>)) != FEM_OK) return rc;
  if ((rc = ensure_smem_attr(mg_residual_kernel<VEC, VT, double>)) != FEM_OK) return rc;
  if ((rc = (fp32 ? ensure_attrs<VEC, float>() : ensure_attrs<VEC, double>())) != FEM_OK) return rc;
  FEM_CUDA_TRY(cudaMemsetAsync(work, 0, 512, st));
  FEM_CUDA_TRY(cudaMemsetAsync(pv, 0, sizeof(double) * n, st));
  FEM_CUDA_TRY(cudaMemsetAsync(q, 0, sizeof(double) * n, st));
  PState init{};
  init.maxiter = maxiter;
  init.first = 1;
  FEM_CUDA_TRY(cudaMemcpyAsync(S, &init, sizeof(PState), cudaMemcpyHostToDevice, st));
  const unsigned rg = row_grid<double>(n_brows), vg = vgrid(n);
  float* r32 = fp32 ? static_cast<float*>(L[0].b) : nullptr;
  float* z32 = fp32 ? static_cast<float*>(L[0].x) : nullptr;
  // r = b - A x, the reductions and status
  mg_residual_kernel<VEC, VT, double><<<rg, kRowThreads, bsr_rows_smem(), st>>>(
      n_brows, rp, ci, vals, x, b, r, static_cast<const double*>(nullptr), static_cast<double*>(nullptr), nullptr, 0.0,
      static_cast<const double*>(nullptr));
  FEM_LAUNCH_CHECK();
  pcg_init_kernel<VEC><<<vg, 256, 0, st>>>(n, r, b, partials, counter, S, rtol, atol);
  FEM_LAUNCH_CHECK();
  if (fp32) {
    cast_kernel<float><<<vg, 256, 0, st>>>(n, r, r32);
    FEM_LAUNCH_CHECK();
  }
  double* mb = host_mailbox();
  FEM_CHECK_ARG(mb != nullptr, "pinned mailbox allocation failed");
  static_assert(sizeof(PState) <= 256, "PState must fit its slot and the mailbox");
  const PState* hs = reinterpret_cast<const PState*>(mb);
  auto read_state = [&]() -> int {
    FEM_CUDA_TRY(cudaMemcpyAsync(mb, S, sizeof(PState), cudaMemcpyDeviceToHost, st));
    FEM_CUDA_TRY(cudaStreamSynchronize(st));
    return FEM_OK;
  };
  // one PCG iteration: V-cycle, w = A z with r.z and z.w, update
  auto launch_iter = [&](cudaStream_t ls) -> int {
    int rc2;
    if (fp32) {
      if ((rc2 = vcycle_level<VEC, float>(0, nlevels, L, nu, coarse_steps, ratio, r32, z32, ls)) != FEM_OK) return rc2;
      FEM_CUDA_TRY(launch_pdl(pcg_spmv_kernel<VEC, VT, float>, rg, kRowThreads, bsr_rows_smem(), ls, n_brows, rp, ci,
                              vals, static_cast<const float*>(z32), static_cast<const double*>(r), w, partials,
                              counter, S));
      FEM_LAUNCH_CHECK();
      FEM_CUDA_TRY(launch_pdl(pcg_update_kernel<float>, vg, 256, 0, ls, n, static_cast<const float*>(z32),
                              static_cast<const double*>(w), x, r, pv, q, r32, partials, counter, S));
      FEM_LAUNCH_CHECK();
    } else {
      if ((rc2 = vcycle_level<VEC, double>(0, nlevels, L, nu, coarse_steps, ratio, r, z, ls)) != FEM_OK) return rc2;
      FEM_CUDA_TRY(launch_pdl(pcg_spmv_kernel<VEC, VT, double>, rg, kRowThreads, bsr_rows_smem(), ls, n_brows, rp, ci,
                              vals, static_cast<const double*>(z), static_cast<const double*>(r), w, partials,
                              counter, S));
      FEM_LAUNCH_CHECK();
      FEM_CUDA_TRY(launch_pdl(pcg_update_kernel<double>, vg, 256, 0, ls, n, static_cast<const double*>(z),
                              static_cast<const double*>(w), x, r, pv, q, static_cast<float*>(nullptr), partials,
                              counter, S));
      FEM_LAUNCH_CHECK();
    }
    return FEM_OK;
  };
  bool looped = false;
  int64_t nbody_run = 0;  // kernels per body of the graph launched
  if (mg_graphs_enabled()) {
    // The whole iteration loop as one graph: a WHILE node whose body is one
    // iteration and whose condition the device sets from the state, so the
    // host waits once per solve and no iteration runs after convergence.
    std::string key(reinterpret_cast<const char*>(L), sizeof(FemMGLevel) * size_t(nlevels));
    const void* ptrs[] = {rp, ci, vals, b, x, work};
    key.append(reinterpret_cast<const char*>(ptrs), sizeof(ptrs));
    const double params[] = {double(nlevels), double(fp32), double(nu), double(coarse_steps), ratio, double(n_brows),
                             double(VEC), double(sizeof(VT))};
    key.append(reinterpret_cast<const char*>(params), sizeof(params));
    int dev = 0;
    cudaGetDevice(&dev);
    key.append(reinterpret_cast<const char*>(&dev), sizeof(dev));
    cudaGraphExec_t exec = nullptr;
    int64_t nbody = 0;
    {
      std::lock_guard<std::mutex> lock(g_mg_mu);
      auto it = mg_graph_cache().find(key);
      if (it != mg_graph_cache().end()) {
        exec = it->second.exec;
        nbody = it->second.kernels;
      }
    }
    if (exec == nullptr && (exec = build_loop_graph(S, launch_iter, &nbody)) != nullptr) {
      std::lock_guard<std::mutex> lock(g_mg_mu);
      auto& m = mg_graph_cache();
      if (m.size() >= 32) {  // bounded: drop everything (hierarchies were rebuilt)
        for (auto& kv : m) cudaGraphExecDestroy(kv.second.exec);
        m.clear();
      }
      m[key] = MGGraph{exec, nbody};
    }
    if (exec != nullptr) {
      FEM_CUDA_TRY(cudaGraphLaunch(exec, st));
      looped = true;
      nbody_run = nbody;
    }
  }
  if (!looped) {
    // direct launches, the state read every check_every iterations
    int launched = 0;
    while (true) {
      if ((rc = read_state()) != FEM_OK) return rc;
      if (hs->status != PS_RUNNING || launched >= maxiter) break;
      const int chunk = check_every < maxiter - launched ? check_every : maxiter - launched;
      for (int k = 0; k < chunk; ++k)
        if ((rc = launch_iter(st)) != FEM_OK) return rc;
      launched += chunk;
    }
  }
  // the true residual ||b - A x||, queued behind the iterations: one host
  // wait per solve reads it with the loop's state
  mg_residual_kernel<VEC, VT, double><<<rg, kRowThreads, bsr_rows_smem(), st>>>(
      n_brows, rp, ci, vals, x, b, q, static_cast<const double*>(nullptr), static_cast<double*>(nullptr), nullptr, 0.0,
      static_cast<const double*>(nullptr));
  FEM_LAUNCH_CHECK();
  FEM_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned), st));
  pcg_true_rr_kernel<<<vg, 256, 0, st>>>(n, q, partials, counter, S);
  FEM_LAUNCH_CHECK();
  if ((rc = read_state()) != FEM_OK) return rc;
  if (looped) launch_counter().fetch_add(1 + int64_t(hs->loops) * nbody_run, std::memory_order_relaxed);
  const int status = hs->status;
  const int iters = hs->iter;
  const double bb = hs->bb;
  const double rr = hs->true_rr;
  if (h_iters) *h_iters = iters;
  if (h_relres) *h_relres = bb > 0 ? std::sqrt(rr / bb) : std::sqrt(rr);
  if (status == PS_CONVERGED) return FEM_OK;
  const int st_out = (status == PS_RUNNING) ? FEM_ERR_NOT_CONVERGED : status;
  set_error("mg pcg: status %d after %d iterations (relres %.3e)", st_out, iters, bb > 0 ? std::sqrt(rr / bb) : std::sqrt(rr));
  return st_out;
}

}  // namespace
}  // namespace fem

using namespace fem;

extern "C" size_t fem_mg_setup_scratch_bytes(int vec, int64_t fine_n_brows, int fp32) {
  return setup_scratch_bytes(vec, fine_n_brows, fp32 ? sizeof(float) : sizeof(double));
}

extern "C" int fem_mg_setup_f64(int vec, int nlevels, const FemMGLevel* levels, void* d_scratch, size_t scratch_bytes,
                                void* stream) {
  FEM_CHECK_ARG(vec == 1 || vec == 3, "vec must be 1 or 3");
  return vec == 3 ? setup_impl<3, double>(nlevels, levels, nullptr, d_scratch, scratch_bytes, as_stream(stream))
                  : setup_impl<1, double>(nlevels, levels, nullptr, d_scratch, scratch_bytes, as_stream(stream));
}

extern "C" int fem_mg_setup_f32(int vec, int nlevels, const FemMGLevel* levels, const double* d_fine_f64,
                                void* d_scratch, size_t scratch_bytes, void* stream) {
  FEM_CHECK_ARG(vec == 1 || vec == 3, "vec must be 1 or 3");
  return vec == 3 ? setup_impl<3, float>(nlevels, levels, d_fine_f64, d_scratch, scratch_bytes, as_stream(stream))
                  : setup_impl<1, float>(nlevels, levels, d_fine_f64, d_scratch, scratch_bytes, as_stream(stream));
}

extern "C" int fem_mg_vcycle_f64(int vec, int nlevels, const FemMGLevel* levels, int nu, int coarse_steps,
                                 double ratio, const double* d_rhs, double* d_z, void* stream) {
  FEM_CHECK_ARG(vec == 1 || vec == 3, "vec must be 1 or 3");
  int rc = vec == 3 ? check_levels<3, double>(nlevels, levels) : check_levels<1, double>(nlevels, levels);
  if (rc != FEM_OK) return rc;
  rc = vec == 3 ? ensure_attrs<3, double>() : ensure_attrs<1, double>();
  if (rc != FEM_OK) return rc;
  return vec == 3 ? vcycle_impl<3, double>(nlevels, levels, nu, coarse_steps, ratio, d_rhs, d_z, as_stream(stream))
                  : vcycle_impl<1, double>(nlevels, levels, nu, coarse_steps, ratio, d_rhs, d_z, as_stream(stream));
}

extern "C" int fem_mg_vcycle_f32(int vec, int nlevels, const FemMGLevel* levels, int nu, int coarse_steps,
                                 double ratio, const float* d_rhs, float* d_z, void* stream) {
  FEM_CHECK_ARG(vec == 1 || vec == 3, "vec must be 1 or 3");
  int rc = vec == 3 ? check_levels<3, float>(nlevels, levels) : check_levels<1, float>(nlevels, levels);
  if (rc != FEM_OK) return rc;
  rc = vec == 3 ? ensure_attrs<3, float>() : ensure_attrs<1, float>();
  if (rc != FEM_OK) return rc;
  return vec == 3 ? vcycle_impl<3, float>(nlevels, levels, nu, coarse_steps, ratio, d_rhs, d_z, as_stream(stream))
                  : vcycle_impl<1, float>(nlevels, levels, nu, coarse_steps, ratio, d_rhs, d_z, as_stream(stream));
}

extern "C" int fem_mg_tail_plan(int vec, int nlevels, const FemMGLevel* levels, int fp32, int nu, int coarse_steps,
                                int* start, size_t* smem_bytes) {
  FEM_CHECK_ARG(vec == 1 || vec == 3, "vec must be 1 or 3");
  FEM_CHECK_ARG(nlevels >= 1 && nlevels <= 16 && levels != nullptr, "nlevels must be in [1, 16] with levels given");
  FEM_CHECK_ARG(start != nullptr && smem_bytes != nullptr, "start and smem_bytes must not be NULL");
  FEM_CHECK_ARG(nu >= 1 && nu <= 16 && coarse_steps >= 1 && coarse_steps <= 512, "nu in [1,16], coarse_steps in [1,512]");
  int s = -1;
  size_t bytes = 0;
  auto plan = [&](auto tag) {
    using T = decltype(tag);
    s = vec == 3 ? tail_start<3, T>(nlevels, levels, nu, coarse_steps)
                 : tail_start<1, T>(nlevels, levels, nu, coarse_steps);
    if (s >= 0) {
      TailArgs<T> a{};
      bytes = vec == 3 ? tail_layout<3, T>(s, nlevels, levels, &a) : tail_layout<1, T>(s, nlevels, levels, &a);
    }
  };
  if (fp32) plan(float{});
  else plan(double{});
  *start = s;
  *smem_bytes = bytes;
  return FEM_OK;
}

extern "C" size_t fem_mg_pcg_workspace_bytes(int vec, int64_t n_brows) { return pcg_workspace_bytes(vec, n_brows); }

namespace fem {
namespace {
template <typename VT>
int pcg_entry(int vec, int64_t n_brows, const int32_t* d_row_ptr, const int32_t* d_col_idx, const VT* d_vals,
              const double* d_b, double* d_x, double rtol, double atol, int maxiter, int check_every, int nlevels,
              const FemMGLevel* levels, int levels_fp32, int nu, int coarse_steps, double ratio, void* d_work,
              size_t work_bytes, int* h_iters, double* h_relres, void* stream) {
  FEM_CHECK_ARG(vec == 1 || vec == 3, "vec must be 1 or 3");
  FEM_CHECK_ARG(rtol >= 0 && atol >= 0, "negative tolerance");
  int rc = levels_fp32 ? (vec == 3 ? check_levels<3, float>(nlevels, levels) : check_levels<1, float>(nlevels, levels))
                       : (vec == 3 ? check_levels<3, double>(nlevels, levels) : check_levels<1, double>(nlevels, levels));
  if (rc != FEM_OK) return rc;
  FEM_CHECK_ARG(nu >= 1 && nu <= 16 && coarse_steps >= 1 && coarse_steps <= 512 && ratio > 1.0,
                "nu in [1,16], coarse_steps in [1,512], ratio > 1");
  auto st = as_stream(stream);
  return vec == 3 ? pcg_impl<3, VT>(n_brows, d_row_ptr, d_col_idx, d_vals, d_b, d_x, rtol, atol, maxiter, check_every,
                                    nlevels, levels, levels_fp32, nu, coarse_steps, ratio, d_work, work_bytes, h_iters,
                                    h_relres, st)
                  : pcg_impl<1, VT>(n_brows, d_row_ptr, d_col_idx, d_vals, d_b, d_x, rtol, atol, maxiter, check_every,
                                    nlevels, levels, levels_fp32, nu, coarse_steps, ratio, d_work, work_bytes, h_iters,
                                    h_relres, st);
}
}  // namespace
}  // namespace fem

extern "C" int fem_mg_pcg_solve(int vec, int64_t n_brows, const int32_t* d_row_ptr, const int32_t* d_col_idx,
                                const double* d_vals, const double* d_b, double* d_x, double rtol, double atol,
                                int maxiter, int check_every, int nlevels, const FemMGLevel* levels, int levels_fp32,
                                int nu, int coarse_steps, double ratio, void* d_work, size_t work_bytes, int* h_iters,
                                double* h_relres, void* stream) {
  return pcg_entry<double>(vec, n_brows, d_row_ptr, d_col_idx, d_vals, d_b, d_x, rtol, atol, maxiter, check_every,
                           nlevels, levels, levels_fp32, nu, coarse_steps, ratio, d_work, work_bytes, h_iters, h_relres,
                           stream);
}

extern "C" int fem_mg_pcg_solve_mixed(int vec, int64_t n_brows, const int32_t* d_row_ptr, const int32_t* d_col_idx,
                                      const float* d_vals, const double* d_b, double* d_x, double rtol, double atol,
                                      int maxiter, int check_every, int nlevels, const FemMGLevel* levels,
                                      int levels_fp32, int nu, int coarse_steps, double ratio, void* d_work,
                                      size_t work_bytes, int* h_iters, double* h_relres, void* stream) {
  return pcg_entry<float>(vec, n_brows, d_row_ptr, d_col_idx, d_vals, d_b, d_x, rtol, atol, maxiter, check_every,
                          nlevels, levels, levels_fp32, nu, coarse_steps, ratio, d_work, work_bytes, h_iters, h_relres,
                          stream);
}
