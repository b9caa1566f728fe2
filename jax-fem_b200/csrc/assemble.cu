// HEX8 cell assembly: residual, BC-eliminated block-CSR tangent and Dirichlet
// lift in one pass over the cells.
//
// Replaces the reference's per-cell weak-form kernel + jacfwd
// (problem.py:189-214, 262-266, 299-301, 334-338), the residual scatter
// (problem.py:426-437) and the PETSc COO insertion + zeroRows of get_A
// (solver.py:485-491).  The reference differentiates the kernel with 24
// forward-mode JVPs per cell; here every law supplies its exact tangent in a
// rank-structured form (see law_quad below), so one evaluation per quadrature
// point yields residual and tangent together.
//
// Precision: geometry, the constitutive update and the residual are FP64 in
// every variant; the tangent (its per-quad factors in shared memory, the
// node-pair products and the stored values) is FP64 or FP32.
//
// Work split: 12 threads per cell, 8 cells (96 threads) per block.
//  phase 0  thread t < 8 loads node t of its cell (coords, u, Dirichlet data)
//  phase 1  thread t < 8 = quadrature point q: geometry (J, det, grad N),
//           grad u, the constitutive update; P*JxW (FP64) and the tangent
//           factors -> smem
//  phase 2  residual: thread t < 8 = node a, r_a = sum_q P_q g_a,q in FP64;
//           tangent: every element matrix here is symmetric, so only the 36
//           node pairs a <= b are formed, three per thread.  Each pair goes
//           to the block of the global upper triangle (row node < column
//           node), transposed when the local order is reversed, through the
//           precomputed cell->block map (no sort, no search), with Dirichlet
//           row/column elimination.  The lift K d of the eliminated columns
//           gathers per cell in shared memory.
//  mirror   a second kernel writes each lower block as the transpose of its
//           upper partner, so the stored matrix stays the full block CSR.
// A cell's threads span warps, so phases are separated by __syncthreads.
#include "common.cuh"
#include "tangent.cuh"

namespace fem {
namespace {

struct AsmArgs {
  int64_t num_cells;
  const int32_t* cells;
  const double* points;
  const double* u;
  const double* iv0;
  const double* iv1;
  const double* iv2;
  const int32_t* scatter;
  const uint8_t* bc;
  const double* dvec;
  double* res;
  double* lift;
  void* vals;
  double p[4];
};

constexpr int kCellsPerBlock = 8;
constexpr int kThreadsPerCell = 12;
constexpr int kAsmThreads = kCellsPerBlock * kThreadsPerCell;

template <int LAW>
struct LawTraits {
  static constexpr int NV = (LAW == FEM_LAW_NEO_HOOKEAN) ? 2 : ((LAW == FEM_LAW_J2) ? 1 : 0);
};

// Per-quad record in shared memory (type T, the tangent's type):
//   [0,24)            g_b  (physical shape gradients of the 8 nodes)
//   [24, 24+24 NV)    law vectors per node (NH: F g_b, F^-T g_b; J2: s g_b)
//   then 4            tangent coefficients * JxW
// The stress P * JxW (and, with an FP32 record, the shape gradients) go to a
// separate FP64 area, so the residual is FP64 whatever T is.
template <int VEC, int LAW>
struct QuadLayout {
  static constexpr int NV = LawTraits<LAW>::NV;
  static constexpr int G = 0;
  static constexpr int V1 = 24;
  static constexpr int V2 = 48;
  static constexpr int C = 24 + 24 * NV;
  static constexpr int QF = C + 4;
};

// Words per cell padded so that consecutive cells start 8 banks apart.
template <typename T>
__host__ __device__ constexpr int padded_cell_elems(int n) {
  // elements -> 4-byte words: n * sizeof(T)/4; want words % 32 == 8
  return (sizeof(T) == 8) ? (n + ((4 - n % 16) + 16) % 16) : (n + ((8 - n % 32) + 32) % 32);
}

template <int VEC>
struct NodeLayout {
  static constexpr int U = 3;
  static constexpr int D = 3 + VEC;
  static constexpr int NF = 3 + 2 * VEC;
};

// FP64 copies of the shape gradients for the residual, kept only when the
// tangent record is FP32 (an FP64 record already holds them).
template <typename T>
__host__ __device__ constexpr int residual_g_elems() {
  return sizeof(T) == 8 ? 0 : 24;
}

template <int VEC, int LAW, typename T>
__host__ __device__ constexpr size_t asm_smem_bytes() {
  return size_t(kCellsPerBlock) * padded_cell_elems<T>(8 * QuadLayout<VEC, LAW>::QF) * sizeof(T) +
         size_t(kCellsPerBlock) * 8 * (VEC * 3 + residual_g_elems<T>()) * sizeof(double) +  // P*JxW, g (FP64)
         size_t(kCellsPerBlock) * 8 * NodeLayout<VEC>::NF * sizeof(double) +              // node data
         size_t(kCellsPerBlock) * 8 * VEC * sizeof(double) +                              // lift accumulators
         size_t(kCellsPerBlock) * 8 * 2 * sizeof(int);                                    // BC bits, node ids
}

// Phase 1: constitutive update at one quadrature point, in FP64.
// ug = grad u (VEC x 3), g = physical shape gradients; returns P*JxW in P and
// writes the tangent coefficients*JxW and per-node law vectors (as T).
template <int VEC, int LAW, typename T>
__device__ __forceinline__ void law_quad(const AsmArgs& A, int64_t c, int q, const double ug[VEC][3],
                                         const double g[8][3], double jxw, T* qd, double* P) {
  using L = QuadLayout<VEC, LAW>;
  T* cf = qd + L::C;
  if constexpr (LAW == FEM_LAW_LAPLACE) {
#pragma unroll
    for (int i = 0; i < VEC; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) P[i * 3 + j] = ug[i][j] * jxw;
    cf[0] = T(jxw);
    cf[1] = cf[2] = cf[3] = T(0);
  } else if constexpr (LAW == FEM_LAW_LINEAR || LAW == FEM_LAW_SIMP) {
    double E, nu;
    if constexpr (LAW == FEM_LAW_LINEAR) {
      E = A.p[0];
      nu = A.p[1];
    } else {
      const double th = A.iv0[c * 8 + q];
      const double E0 = A.p[0], Emin = A.p[1], pen = A.p[3];
      nu = A.p[2];
      E = Emin + (E0 - Emin) * pow(th, pen);
    }
    const double mu = E / (2.0 * (1.0 + nu));
    const double lm = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    double eps[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) eps[i][j] = 0.5 * (ug[i][j] + ug[j][i]);
    const double tr = eps[0][0] + eps[1][1] + eps[2][2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) P[i * 3 + j] = jxw * (2.0 * mu * eps[i][j] + (i == j ? lm * tr : 0.0));
    cf[0] = T(lm * jxw);
    cf[1] = T(mu * jxw);
    cf[2] = cf[3] = T(0);
  } else if constexpr (LAW == FEM_LAW_NEO_HOOKEAN) {
    const double E = A.p[0], nu = A.p[1];
    const double mu = E / (2.0 * (1.0 + nu));
    const double kappa = E / (3.0 * (1.0 - 2.0 * nu));
    double F[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) F[i][j] = ug[i][j] + (i == j ? 1.0 : 0.0);
    double cof[3][3];
    cof[0][0] = F[1][1] * F[2][2] - F[1][2] * F[2][1];
    cof[0][1] = F[1][2] * F[2][0] - F[1][0] * F[2][2];
    cof[0][2] = F[1][0] * F[2][1] - F[1][1] * F[2][0];
    cof[1][0] = F[0][2] * F[2][1] - F[0][1] * F[2][2];
    cof[1][1] = F[0][0] * F[2][2] - F[0][2] * F[2][0];
    cof[1][2] = F[0][1] * F[2][0] - F[0][0] * F[2][1];
    cof[2][0] = F[0][1] * F[1][2] - F[0][2] * F[1][1];
    cof[2][1] = F[0][2] * F[1][0] - F[0][0] * F[1][2];
    cof[2][2] = F[0][0] * F[1][1] - F[0][1] * F[1][0];
    const double J = F[0][0] * cof[0][0] + F[0][1] * cof[0][1] + F[0][2] * cof[0][2];
    const double iJ = 1.0 / J;
    double H[3][3];  // F^{-T}
    double I1 = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        H[i][j] = cof[i][j] * iJ;
        I1 += F[i][j] * F[i][j];
      }
    const double cb = cbrt(J);
    const double m = mu / (cb * cb);  // mu J^{-2/3}
    double scale = jxw;
    if (A.iv0 != nullptr) scale *= A.iv0[c * 8 + q];
    const double kJ1 = kappa * J * (J - 1.0);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) P[i * 3 + j] = scale * (m * (F[i][j] - I1 * H[i][j] / 3.0) + kJ1 * H[i][j]);
    // K_ab = m (ga.gb) I - 2/3 m (f_a (x) h_b + h_a (x) f_b)
    //        + (2/9 m I1 + kappa (2J-1) J) h_a (x) h_b + (1/3 m I1 - kappa J (J-1)) h_b (x) h_a
    cf[0] = T(scale * m);
    cf[1] = T(scale * (-2.0 / 3.0) * m);
    cf[2] = T(scale * (2.0 / 9.0 * m * I1 + kappa * (2.0 * J - 1.0) * J));
    cf[3] = T(scale * (m * I1 / 3.0 - kJ1));
    T* v1 = qd + L::V1;
    T* v2 = qd + L::V2;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        v1[b * 3 + i] = T(F[i][0] * g[b][0] + F[i][1] * g[b][1] + F[i][2] * g[b][2]);
        v2[b * 3 + i] = T(H[i][0] * g[b][0] + H[i][1] * g[b][1] + H[i][2] * g[b][2]);
      }
    }
  } else if constexpr (LAW == FEM_LAW_J2) {
    const double E = A.p[0], nu = A.p[1], sy0 = A.p[2], Hh = A.p[3];
    const double mu = E / (2.0 * (1.0 + nu));
    const double lm = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double* so = A.iv0 + (c * 8 + q) * 9;
    const double* eo = A.iv1 + (c * 8 + q) * 9;
    const double alpha = A.iv2[c * 8 + q];
    double de[3][3], st[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) de[i][j] = 0.5 * (ug[i][j] + ug[j][i]) - eo[i * 3 + j];
    const double trd = de[0][0] + de[1][1] + de[2][2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) st[i][j] = 2.0 * mu * de[i][j] + (i == j ? lm * trd : 0.0) + so[i * 3 + j];
    const double trs = (st[0][0] + st[1][1] + st[2][2]) / 3.0;
    double s[3][3];
    double ss = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        s[i][j] = st[i][j] - (i == j ? trs : 0.0);
        ss += s[i][j] * s[i][j];
      }
    const double qv = ss > 0.0 ? sqrt(1.5 * ss) : 0.0;
    const double syc = sy0 + Hh * alpha;
    const double f = qv - syc;
    double beta = 0.0, gam2 = 0.0;
    if (f > 0.0) {
      const double dg = f / (3.0 * mu + Hh);
      beta = 3.0 * mu * dg / qv;
      gam2 = 9.0 * mu * mu * syc / ((3.0 * mu + Hh) * qv * qv * qv);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) P[i * 3 + j] = jxw * (st[i][j] - beta * s[i][j]);
    // K_ab = cII ga (x) gb + (csym/2) ((ga.gb) I + gb (x) ga) - gam2 (s ga) (x) (s gb)
    cf[0] = T(jxw * (lm + 2.0 * mu * beta / 3.0));
    cf[1] = T(jxw * mu * (1.0 - beta));
    cf[2] = T(jxw * gam2);
    cf[3] = T(0);
    T* v1 = qd + L::V1;
#pragma unroll
    for (int b = 0; b < 8; ++b)
#pragma unroll
      for (int i = 0; i < 3; ++i) v1[b * 3 + i] = T(s[i][0] * g[b][0] + s[i][1] * g[b][1] + s[i][2] * g[b][2]);
  }
}

template <int VEC, int LAW, typename T>
__device__ __forceinline__ void pair_block(const T* qd, int a, int b, T K[VEC][VEC]) {
  using L = QuadLayout<VEC, LAW>;
  const T* g = qd + L::G;
  const T* cf = qd + L::C;
  const T ga0 = g[a * 3], ga1 = g[a * 3 + 1], ga2 = g[a * 3 + 2];
  const T gb0 = g[b * 3], gb1 = g[b * 3 + 1], gb2 = g[b * 3 + 2];
  const T dot = ga0 * gb0 + ga1 * gb1 + ga2 * gb2;
  if constexpr (LAW == FEM_LAW_LAPLACE) {
    const T s = cf[0] * dot;
#pragma unroll
    for (int i = 0; i < VEC; ++i) K[i][i] += s;
  } else {
    const T ga[3] = {ga0, ga1, ga2};
    const T gb[3] = {gb0, gb1, gb2};
    if constexpr (LAW == FEM_LAW_LINEAR || LAW == FEM_LAW_SIMP) {
      const T lm = cf[0], mu = cf[1];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int k = 0; k < 3; ++k) K[i][k] += lm * ga[i] * gb[k] + mu * gb[i] * ga[k];
        K[i][i] += mu * dot;
      }
    } else if constexpr (LAW == FEM_LAW_NEO_HOOKEAN) {
      const T* f = qd + L::V1;
      const T* h = qd + L::V2;
      const T m = cf[0], c2 = cf[1], c4 = cf[2], c5 = cf[3];
      T fa[3], ha[3], fb[3], hb[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        fa[i] = f[a * 3 + i];
        ha[i] = h[a * 3 + i];
        fb[i] = f[b * 3 + i];
        hb[i] = h[b * 3 + i];
      }
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const T ua = c2 * fa[i] + c4 * ha[i];
        const T va = c2 * ha[i];
#pragma unroll
        for (int k = 0; k < 3; ++k) K[i][k] += ua * hb[k] + va * fb[k] + c5 * hb[i] * ha[k];
        K[i][i] += m * dot;
      }
    } else if constexpr (LAW == FEM_LAW_J2) {
      const T* sg = qd + L::V1;
      const T cII = cf[0], ch = cf[1], g2 = cf[2];
      T sa[3], sb[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        sa[i] = sg[a * 3 + i];
        sb[i] = sg[b * 3 + i];
      }
#pragma unroll
      for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int k = 0; k < 3; ++k) K[i][k] += cII * ga[i] * gb[k] + ch * gb[i] * ga[k] - g2 * sa[i] * sb[k];
        K[i][i] += ch * dot;
      }
    }
  }
}

// Local node pairs (a, b), a <= b, in row-major order of the upper triangle.
__constant__ unsigned char kPairA[36] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 2, 2, 2,
                                         2, 2, 2, 3, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 6, 6, 7};
__constant__ unsigned char kPairB[36] = {0, 1, 2, 3, 4, 5, 6, 7, 1, 2, 3, 4, 5, 6, 7, 2, 3, 4,
                                         5, 6, 7, 3, 4, 5, 6, 7, 4, 5, 6, 7, 5, 6, 7, 6, 7, 7};

template <int VEC, int LAW, typename T, bool WANT_K>
#ifndef FEM_ASM_MIN_BLOCKS_F32
#define FEM_ASM_MIN_BLOCKS_F32 5
#endif
#ifndef FEM_ASM_MIN_BLOCKS_F64
#define FEM_ASM_MIN_BLOCKS_F64 4
#endif
// Resident blocks per SM: shared memory allows about 5 (FP32 records) and 4
// (FP64 records); the register budget is held to match.
__global__ void __launch_bounds__(kAsmThreads, sizeof(T) == 4 ? FEM_ASM_MIN_BLOCKS_F32 : FEM_ASM_MIN_BLOCKS_F64)
    assemble_kernel(const AsmArgs A) {
  using L = QuadLayout<VEC, LAW>;
  using N = NodeLayout<VEC>;
  constexpr int CELLF = padded_cell_elems<T>(8 * L::QF);
  extern __shared__ __align__(16) unsigned char smem[];
  T* sq = reinterpret_cast<T*>(smem);
  constexpr int QD = VEC * 3 + residual_g_elems<T>();  // per-quad FP64 residual data: P*JxW, then g
  double* sP = reinterpret_cast<double*>(smem + size_t(kCellsPerBlock) * CELLF * sizeof(T));
  double* sn = sP + kCellsPerBlock * 8 * QD;
  double* slift = sn + kCellsPerBlock * 8 * N::NF;
  int* sbc = reinterpret_cast<int*>(slift + kCellsPerBlock * 8 * VEC);
  int* snode = sbc + kCellsPerBlock * 8;

  const int cl = threadIdx.x / kThreadsPerCell;
  const int t = threadIdx.x - cl * kThreadsPerCell;
  const int64_t c = int64_t(blockIdx.x) * kCellsPerBlock + cl;
  const bool valid = c < A.num_cells;

  // ---- phase 0: node data ----
  if (t < 8) {
    const int node = valid ? A.cells[c * 8 + t] : 0;
    double* nd = sn + (cl * 8 + t) * N::NF;
    if (valid) {
      nd[0] = A.points[int64_t(node) * 3 + 0];
      nd[1] = A.points[int64_t(node) * 3 + 1];
      nd[2] = A.points[int64_t(node) * 3 + 2];
    } else {  // unit cube keeps the tail math finite; its outputs are dropped
      nd[0] = vtk_xbit(t);
      nd[1] = vtk_ybit(t);
      nd[2] = vtk_zbit(t);
    }
    int bits = 0;
#pragma unroll
    for (int i = 0; i < VEC; ++i) {
      const int64_t dof = int64_t(node) * VEC + i;
      nd[N::U + i] = valid ? A.u[dof] : 0.0;
      nd[N::D + i] = (valid && A.dvec != nullptr) ? A.dvec[dof] : 0.0;
      if (valid && A.bc != nullptr && A.bc[dof]) bits |= 1 << i;
      if (nd[N::D + i] != 0.0) bits |= kLiftBit;
      slift[(cl * 8 + t) * VEC + i] = 0.0;
    }
    sbc[cl * 8 + t] = bits;
    snode[cl * 8 + t] = node;
  }
  __syncthreads();

  // ---- phase 1: quadrature point q = t ----
  T* cq = sq + cl * CELLF;
  const double* nb = sn + cl * 8 * N::NF;
  if (t < 8) {
    const int q = t;
    double X[8][3], g[8][3];
#pragma unroll
    for (int b = 0; b < 8; ++b)
#pragma unroll
      for (int i = 0; i < 3; ++i) X[b][i] = nb[b * N::NF + i];
    double jxw;
    if (!hex8_box_geometry(q, X, g, &jxw)) hex8_geometry(q, X, g, &jxw);
    double ug[VEC][3];
#pragma unroll
    for (int i = 0; i < VEC; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) ug[i][j] = 0.0;
#pragma unroll
    for (int b = 0; b < 8; ++b)
#pragma unroll
      for (int i = 0; i < VEC; ++i) {
        const double ub = nb[b * N::NF + N::U + i];
#pragma unroll
        for (int j = 0; j < 3; ++j) ug[i][j] = fma(ub, g[b][j], ug[i][j]);
      }
    T* qd = cq + q * L::QF;
#pragma unroll
    for (int b = 0; b < 8; ++b)
#pragma unroll
      for (int j = 0; j < 3; ++j) qd[L::G + b * 3 + j] = T(g[b][j]);
    double* pq = sP + (cl * 8 + q) * QD;
    law_quad<VEC, LAW, T>(A, valid ? c : 0, q, ug, g, jxw, qd, pq);
    if constexpr (residual_g_elems<T>() > 0) {
#pragma unroll
      for (int b = 0; b < 8; ++b)
#pragma unroll
        for (int j = 0; j < 3; ++j) pq[VEC * 3 + b * 3 + j] = g[b][j];
    }
  }
  __syncthreads();

  // ---- phase 2a: residual of node a = t, r_a = sum_q P_q g_a,q (FP64) ----
  if (valid && t < 8 && A.res != nullptr) {
    const int a = t;
    double r[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) r[i] = 0.0;
#pragma unroll 1
    for (int q = 0; q < 8; ++q) {
      const double* pq = sP + (cl * 8 + q) * QD;
      double ga[3];
#pragma unroll
      for (int j = 0; j < 3; ++j)
        ga[j] = residual_g_elems<T>() > 0 ? pq[VEC * 3 + a * 3 + j] : double(cq[q * L::QF + L::G + a * 3 + j]);
#pragma unroll
      for (int i = 0; i < VEC; ++i) r[i] += pq[i * 3] * ga[0] + pq[i * 3 + 1] * ga[1] + pq[i * 3 + 2] * ga[2];
    }
    const int64_t node = snode[cl * 8 + a];
#pragma unroll
    for (int i = 0; i < VEC; ++i) atomicAdd(A.res + node * VEC + i, r[i]);
  }
  if constexpr (WANT_K) {
    if (A.vals == nullptr && A.lift == nullptr) return;  // uniform over the block
    T* vals = reinterpret_cast<T*>(A.vals);
    // ---- phase 2b: node pairs p = t, t+12, t+24 ----
    if (valid) {
#pragma unroll 1
      for (int p = t; p < 36; p += kThreadsPerCell) {
        const int a = kPairA[p], b = kPairB[p];
        T K[VEC][VEC];
#pragma unroll
        for (int i = 0; i < VEC; ++i)
#pragma unroll
          for (int k = 0; k < VEC; ++k) K[i][k] = T(0);
#pragma unroll 2
        for (int q = 0; q < 8; ++q) pair_block<VEC, LAW, T>(cq + q * L::QF, a, b, K);
        const int abits = sbc[cl * 8 + a], bbits = sbc[cl * 8 + b];
        if (A.lift != nullptr && (bbits & kLiftBit)) {
          // row a: K_ab d_b (only a node with non-zero d contributes)
#pragma unroll
          for (int i = 0; i < VEC; ++i) {
            double la = 0.0;
#pragma unroll
            for (int k = 0; k < VEC; ++k) la += double(K[i][k]) * nb[b * N::NF + N::D + k];
            atomicAdd(slift + (cl * 8 + a) * VEC + i, la);
          }
        }
        if (A.lift != nullptr && a != b && (abits & kLiftBit)) {
          // row b: K_ab^T d_a
#pragma unroll
          for (int k = 0; k < VEC; ++k) {
            double lb = 0.0;
#pragma unroll
            for (int i = 0; i < VEC; ++i) lb += double(K[i][k]) * nb[a * N::NF + N::D + i];
            atomicAdd(slift + (cl * 8 + b) * VEC + k, lb);
          }
        }
        if (vals != nullptr) {
          const int na = snode[cl * 8 + a], nbn = snode[cl * 8 + b];
          const int* smap = A.scatter + c * 64;
          if (a == b || na < nbn) {
            T* blk = vals + int64_t(smap[a * 8 + b]) * (VEC * VEC);
#pragma unroll
            for (int i = 0; i < VEC; ++i)
#pragma unroll
              for (int k = 0; k < VEC; ++k)
                if (!(((abits >> i) | (bbits >> k)) & 1)) atomicAdd(blk + i * VEC + k, K[i][k]);
          }
          if (a != b && na >= nbn) {  // (na == nbn only in a degenerate cell: both orientations)
            T* blk = vals + int64_t(smap[b * 8 + a]) * (VEC * VEC);
#pragma unroll
            for (int k = 0; k < VEC; ++k)
#pragma unroll
              for (int i = 0; i < VEC; ++i)
                if (!(((bbits >> k) | (abits >> i)) & 1)) atomicAdd(blk + k * VEC + i, K[i][k]);
          }
        }
      }
    }
    if (A.lift != nullptr) {
      __syncthreads();
      // the cell's lift is non-zero only if one of its nodes has non-zero d
      int any = 0;
#pragma unroll
      for (int b = 0; b < 8; ++b) any |= sbc[cl * 8 + b];
      if (valid && t < 8 && (any & kLiftBit)) {
        const int abits = sbc[cl * 8 + t];
        const int64_t node = snode[cl * 8 + t];
#pragma unroll
        for (int i = 0; i < VEC; ++i)
          if (!((abits >> i) & 1)) atomicAdd(A.lift + node * VEC + i, slift[(cl * 8 + t) * VEC + i]);
      }
    }
  }
}

template <int VEC, int LAW, typename T>
int launch_law(const AsmArgs& A, bool want_k, cudaStream_t st) {
  const unsigned grid = unsigned((A.num_cells + kCellsPerBlock - 1) / kCellsPerBlock);
  const size_t sm = asm_smem_bytes<VEC, LAW, T>();
  if (want_k) {
    auto k = assemble_kernel<VEC, LAW, T, true>;
    static bool attr = false;
    if (!attr) {
      FEM_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
      attr = true;
    }
    k<<<grid, kAsmThreads, sm, st>>>(A);
  } else {
    auto k = assemble_kernel<VEC, LAW, T, false>;
    static bool attr = false;
    if (!attr) {
      FEM_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
      attr = true;
    }
    k<<<grid, kAsmThreads, sm, st>>>(A);
  }
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}

template <typename T>
int assemble_impl(int law, const double* h_params, int n_params, int vec, int64_t num_cells,
                  int64_t num_nodes, const int32_t* d_cells, const double* d_points,
                  const double* d_u, const double* iv0, const double* iv1, const double* iv2,
                  const int32_t* d_scatter, const int32_t* d_diag, const int32_t* d_transpose,
                  int64_t nnzb, const uint8_t* d_bc, const double* d_dvec,
                  double* d_res, double* d_lift, T* d_vals, void* stream) {
  FEM_CHECK_ARG(num_cells >= 0 && num_nodes >= 0, "negative sizes");
  FEM_CHECK_ARG(vec == 1 || vec == 3, "vec must be 1 or 3 (got %d)", vec);
  FEM_CHECK_ARG(law == FEM_LAW_LAPLACE || vec == 3, "law %d needs vec=3", law);
  FEM_CHECK_ARG(law >= 0 && law <= FEM_LAW_J2, "unknown law %d", law);
  static const int need[] = {0, 2, 4, 2, 4};
  FEM_CHECK_ARG(n_params >= need[law] && (need[law] == 0 || h_params != nullptr),
                "law %d needs %d parameters (got %d)", law, need[law], n_params);
  FEM_CHECK_ARG(law != FEM_LAW_SIMP || iv0 != nullptr, "SIMP needs theta (ivar0)");
  FEM_CHECK_ARG(law != FEM_LAW_J2 || (iv0 && iv1 && iv2), "J2 needs sigma_old, eps_old, alpha_old");
  FEM_CHECK_ARG(d_vals == nullptr || (d_scatter != nullptr && nnzb > 0), "tangent needs scatter map");
  FEM_CHECK_ARG(d_vals == nullptr || d_transpose != nullptr,
                "tangent needs the block transpose map for its lower triangle");
  FEM_CHECK_ARG(d_vals == nullptr || d_bc == nullptr || d_diag != nullptr, "BC elimination needs diag");
  FEM_CHECK_ARG(d_lift == nullptr || (d_dvec != nullptr && d_scatter != nullptr), "lift needs dvec");
  cudaStream_t st = as_stream(stream);
  const int64_t ndofs = num_nodes * vec;
  if (d_res) FEM_CUDA_TRY(cudaMemsetAsync(d_res, 0, sizeof(double) * ndofs, st));
  if (d_lift) FEM_CUDA_TRY(cudaMemsetAsync(d_lift, 0, sizeof(double) * ndofs, st));
  if (d_vals) FEM_CUDA_TRY(cudaMemsetAsync(d_vals, 0, sizeof(T) * nnzb * vec * vec, st));
  if (num_cells == 0) return FEM_OK;
  AsmArgs A{};
  A.num_cells = num_cells;
  A.cells = d_cells;
  A.points = d_points;
  A.u = d_u;
  A.iv0 = iv0;
  A.iv1 = iv1;
  A.iv2 = iv2;
  A.scatter = d_scatter;
  A.bc = d_bc;
  A.dvec = d_dvec;
  A.res = d_res;
  A.lift = d_lift;
  A.vals = d_vals;
  for (int i = 0; i < 4 && i < n_params; ++i) A.p[i] = h_params[i];
  const bool want_k = (d_vals != nullptr) || (d_lift != nullptr);
  int rc = FEM_ERR_ARG;
  if (vec == 1) {
    rc = launch_law<1, FEM_LAW_LAPLACE, T>(A, want_k, st);
  } else {
    switch (law) {
      case FEM_LAW_LAPLACE: rc = launch_law<3, FEM_LAW_LAPLACE, T>(A, want_k, st); break;
      case FEM_LAW_LINEAR: rc = launch_law<3, FEM_LAW_LINEAR, T>(A, want_k, st); break;
      case FEM_LAW_SIMP: rc = launch_law<3, FEM_LAW_SIMP, T>(A, want_k, st); break;
      case FEM_LAW_NEO_HOOKEAN: rc = launch_law<3, FEM_LAW_NEO_HOOKEAN, T>(A, want_k, st); break;
      case FEM_LAW_J2: rc = launch_law<3, FEM_LAW_J2, T>(A, want_k, st); break;
    }
  }
  if (rc != FEM_OK) return rc;
  if (d_vals != nullptr) return finish_tangent<T>(vec, nnzb, ndofs, d_transpose, d_bc, d_diag, d_vals, st);
  return FEM_OK;
}

}  // namespace
}  // namespace fem

extern "C" int fem_assemble_f64(int law, const double* h_params, int n_params, int vec,
                                int64_t num_cells, int64_t num_nodes, const int32_t* d_cells,
                                const double* d_points, const double* d_u, const double* d_ivar0,
                                const double* d_ivar1, const double* d_ivar2,
                                const int32_t* d_scatter, const int32_t* d_diag,
                                const int32_t* d_transpose, int64_t nnzb,
                                const uint8_t* d_bc_mask, const double* d_dvec, double* d_res,
                                double* d_lift, double* d_vals, void* stream) {
  return fem::assemble_impl<double>(law, h_params, n_params, vec, num_cells, num_nodes, d_cells,
                                    d_points, d_u, d_ivar0, d_ivar1, d_ivar2, d_scatter, d_diag,
                                    d_transpose, nnzb, d_bc_mask, d_dvec, d_res, d_lift,
                                    d_vals, stream);
}

extern "C" int fem_assemble_f32(int law, const double* h_params, int n_params, int vec,
                                int64_t num_cells, int64_t num_nodes, const int32_t* d_cells,
                                const double* d_points, const double* d_u, const double* d_ivar0,
                                const double* d_ivar1, const double* d_ivar2,
                                const int32_t* d_scatter, const int32_t* d_diag,
                                const int32_t* d_transpose, int64_t nnzb,
                                const uint8_t* d_bc_mask, const double* d_dvec, double* d_res,
                                double* d_lift, float* d_vals, void* stream) {
  return fem::assemble_impl<float>(law, h_params, n_params, vec, num_cells, num_nodes, d_cells,
                                   d_points, d_u, d_ivar0, d_ivar1, d_ivar2, d_scatter, d_diag,
                                   d_transpose, nnzb, d_bc_mask, d_dvec, d_res, d_lift,
                                   d_vals, stream);
}
