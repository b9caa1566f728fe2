// Cell assembly for the element types other than the HEX8 fast path:
// TET4, TET10, HEX20 and HEX27 (basis.py:19-114), and HEX8 itself through
// the same code (a cross-check of assemble.cu).
//
// Replaces the same reference functions as assemble.cu -- the per-cell
// weak-form kernel and its jacfwd (problem.py:189-214, 262-266, 299-301),
// the residual scatter (problem.py:426-437) and the COO insertion + zeroRows
// of get_A (solver.py:485-491) -- plus, per (cell, quadrature point), the
// J2 state commit (test_plasticity.py:67-78) and the adjoint parameter VJP
// (solver.py:1340-1356).  The element enters only through its tabulation:
// the reference shape gradients at the quadrature points (nq, nen, 3) and
// the weights (nq), in mesh node order (get_shape_vals_and_grads,
// basis.py:141-175, computed on the host).  Geometry follows
// get_shape_grads (fe.py:112-141): J_ij = sum_a X_a[i] dN_a/dxi_j,
// grad N_a = dN_a/dxi . J^-1, JxW = det(J) w_q.
//
// Precision: everything is FP64 except the stored tangent of the _f32 entry
// (accumulated in FP64, stored and added in FP32).
//
// Work split: TPC threads per cell, CPB cells per block (128 threads); the
// quadrature points go through shared memory in chunks of QC:
//   phase 1  one thread per (cell, quadrature point of the chunk): J, det,
//            J^-1, grad N, grad u and the constitutive update -> a per-quad
//            record (shape gradients, law vectors, tangent coefficients and
//            P*JxW) in shared memory.  For HEX20 / HEX27 it is split: 1a per
//            point forms J^-1, grad u and the law only; 1b, all threads, one
//            (cell, point, node) item each, forms the node's shape gradient
//            and law vectors
//   phase 2  each thread adds the chunk into the node pairs a <= b it owns
//            (FP64 registers, PPT pairs per thread); thread t < nen adds the
//            residual of node t
// After the last chunk the pairs go to the upper block triangle with
// Dirichlet row/column elimination and the lift, as in the HEX8 kernel, and
// the shared passes of tangent.cuh fill the lower triangle and the unit
// Dirichlet diagonal.
#include "common.cuh"
#include "tangent.cuh"

namespace fem {
namespace {

constexpr int kElemThreads = 128;
constexpr int kMaxQuads = 4096;

struct ElemArgs {
  int64_t num_cells;
  int nq;
  const double* gref;  // (nq, nen, 3)
  const double* wq;    // (nq)
  const int32_t* cells;
  const double* points;
  const double* u;
  const double* iv0;
  const double* iv1;
  const double* iv2;
  const int32_t* scatter;  // (num_cells, nen*nen)
  const uint8_t* bc;
  const double* dvec;
  double* res;
  double* lift;
  void* vals;
  double p[4];
};

// Threads per cell, cells per block, quadrature points per chunk, and
// whether phase 1 is split (1a per point, 1b per (point, node)): measured on
// B200, the split pays where a point's per-node work is long (20, 27 nodes:
// 6 % faster) and costs where it is short (4 nodes: 13 % slower; 10: even).
template <int NEN>
struct ElemShape;
template <>
struct ElemShape<4> {
  static constexpr int TPC = 8, CPB = 16, QC = 4;
  static constexpr bool SPLIT = false;
};
template <>
struct ElemShape<8> {
  static constexpr int TPC = 16, CPB = 8, QC = 8;
  static constexpr bool SPLIT = false;
};
template <>
struct ElemShape<10> {
  static constexpr int TPC = 32, CPB = 4, QC = 4;
  static constexpr bool SPLIT = false;
};
template <>
struct ElemShape<20> {
  static constexpr int TPC = 128, CPB = 1, QC = 8;
  static constexpr bool SPLIT = true;
};
template <>
struct ElemShape<27> {  // 216 points at the default order: 8 chunks with 27 threads in phase 1a
  static constexpr int TPC = 128, CPB = 1, QC = 27;
  static constexpr bool SPLIT = true;
};

template <int LAW>
__host__ __device__ constexpr int law_vectors() {
  return LAW == FEM_LAW_NEO_HOOKEAN ? 2 : (LAW == FEM_LAW_J2 ? 1 : 0);
}

// Per-quad record (doubles): shape gradients g (nen x 3), law vectors
// v1 = M1 g_b and v2 = M2 g_b per node (NH: F g_b, F^-T g_b; J2: s g_b),
// four tangent coefficients * JxW, P * JxW (VEC x 3), then (split phase 1
// only) J^-1 and the law's matrices M1, M2 (3 x 3 each), which phase 1b
// turns into the per-node vectors.
template <int NEN, int VEC, int LAW>
struct ElemLayout {
  static constexpr int NV = law_vectors<LAW>();
  static constexpr int G = 0;
  static constexpr int V1 = NEN * 3;
  static constexpr int V2 = NEN * 6;
  static constexpr int C = NEN * 3 * (1 + NV);
  static constexpr int PO = C + 4;
  static constexpr int SC = PO + VEC * 3;
  static constexpr int QF = SC + (ElemShape<NEN>::SPLIT ? 9 * (1 + NV) : 0);
};

// Node record: X (3), u (VEC), d (VEC).
template <int VEC>
__host__ __device__ constexpr int node_fields() {
  return 3 + 2 * VEC;
}

template <int NEN, int VEC, int LAW>
__host__ __device__ constexpr size_t elem_smem_bytes() {
  using S = ElemShape<NEN>;
  using L = ElemLayout<NEN, VEC, LAW>;
  return sizeof(double) * (size_t(S::CPB) * S::QC * L::QF + size_t(S::CPB) * NEN * node_fields<VEC>() +
                           size_t(S::CPB) * NEN * VEC) +
         sizeof(int) * 2 * size_t(S::CPB) * NEN;
}

// J^-1 of a 3x3 matrix by cofactors; returns det J.
__device__ __forceinline__ double invert3(const double J[3][3], double inv[3][3]) {
  const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  const double id = 1.0 / det;
  inv[0][0] = c00 * id;
  inv[1][0] = c01 * id;
  inv[2][0] = c02 * id;
  inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  return det;
}

// J at reference gradients gr (nen x 3) and node coordinates X (stride xs);
// returns det J and writes J^-1.
template <int NEN>
__device__ __forceinline__ double elem_jacobian(const double* __restrict__ gr, const double* X, int xs,
                                                double inv[3][3]) {
  double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll 4
  for (int a = 0; a < NEN; ++a) {
    const double d0 = __ldg(gr + a * 3), d1 = __ldg(gr + a * 3 + 1), d2 = __ldg(gr + a * 3 + 2);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double x = X[a * xs + i];
      J[i][0] = fma(x, d0, J[i][0]);
      J[i][1] = fma(x, d1, J[i][1]);
      J[i][2] = fma(x, d2, J[i][2]);
    }
  }
  return invert3(J, inv);
}

__device__ __forceinline__ void phys_grad(const double* __restrict__ gr, int a, const double inv[3][3],
                                          double g[3]) {
  const double d0 = __ldg(gr + a * 3), d1 = __ldg(gr + a * 3 + 1), d2 = __ldg(gr + a * 3 + 2);
#pragma unroll
  for (int k = 0; k < 3; ++k) g[k] = d0 * inv[0][k] + d1 * inv[1][k] + d2 * inv[2][k];
}

// ---- constitutive laws ---------------------------------------------------------
// Compressible Neo-Hookean (hyperelastic3d_common.py:152-169): psi =
// mu/2 (J^-2/3 I1 - 3) + kappa/2 (J-1)^2, P = dpsi/dF.  Returns P (unscaled)
// and the quantities of its tangent.
struct NHState {
  double F[3][3], H[3][3], J, I1, m;
};

__device__ __forceinline__ void nh_stress(const double ug[3][3], double E, double nu, NHState* s,
                                          double P[3][3]) {
  const double mu = E / (2.0 * (1.0 + nu));
  const double kappa = E / (3.0 * (1.0 - 2.0 * nu));
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) s->F[i][j] = ug[i][j] + (i == j ? 1.0 : 0.0);
  const double(*F)[3] = s->F;
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
  double I1 = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      s->H[i][j] = cof[i][j] * iJ;
      I1 += F[i][j] * F[i][j];
    }
  const double cb = cbrt(J);
  const double m = mu / (cb * cb);  // mu J^{-2/3}
  const double kJ1 = kappa * J * (J - 1.0);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) P[i][j] = m * (F[i][j] - I1 * s->H[i][j] / 3.0) + kJ1 * s->H[i][j];
  s->J = J;
  s->I1 = I1;
  s->m = m;
}

// Small-strain J2 radial return with linear isotropic hardening
// (test_plasticity.py:42-64 at H = 0).  Trial state from the committed
// sigma_old, eps_old, alpha_old; returns the deviatoric trial stress s, the
// plastic multiplier dgamma and the scaling beta = 3 mu dgamma / q.
struct J2State {
  double eps[3][3], st[3][3], s[3][3], q, syc, dg, beta;
};

__device__ __forceinline__ void j2_trial(const double ug[3][3], const double* so, const double* eo, double alpha,
                                         double mu, double lm, double sy0, double Hh, J2State* r) {
  double de[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      r->eps[i][j] = 0.5 * (ug[i][j] + ug[j][i]);
      de[i][j] = r->eps[i][j] - eo[i * 3 + j];
    }
  const double trd = de[0][0] + de[1][1] + de[2][2];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r->st[i][j] = 2.0 * mu * de[i][j] + (i == j ? lm * trd : 0.0) + so[i * 3 + j];
  const double tr3 = (r->st[0][0] + r->st[1][1] + r->st[2][2]) / 3.0;
  double ss = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      r->s[i][j] = r->st[i][j] - (i == j ? tr3 : 0.0);
      ss += r->s[i][j] * r->s[i][j];
    }
  r->q = ss > 0.0 ? sqrt(1.5 * ss) : 0.0;
  r->syc = sy0 + Hh * alpha;
  const double f = r->q - r->syc;
  r->dg = 0.0;
  r->beta = 0.0;
  if (f > 0.0) {
    r->dg = f / (3.0 * mu + Hh);
    r->beta = 3.0 * mu * r->dg / r->q;
  }
}

// The law at one quadrature point (k = cell * nq + q): P * JxW, the tangent
// coefficients * JxW and the matrices whose products with the shape
// gradients are the law vectors.  The element tangent of every law is
//   Laplace:  K_ab = c0 (ga.gb) I
//   linear:   K_ab = c0 ga (x) gb + c1 (gb (x) ga + (ga.gb) I)
//   NH:       K_ab = c0 (ga.gb) I + c1 (f_a (x) h_b + h_a (x) f_b) + c2 h_a (x) h_b + c3 h_b (x) h_a
//   J2:       K_ab = c0 ga (x) gb + c1 ((ga.gb) I + gb (x) ga) - c2 (s ga) (x) (s gb)
// with f = F g, h = F^-T g.
template <int VEC, int LAW>
__device__ __forceinline__ void elem_law(const ElemArgs& A, int64_t k, const double ug[VEC][3], double jxw,
                                         double* P, double* cf, double M1[3][3], double M2[3][3]) {
  cf[0] = cf[1] = cf[2] = cf[3] = 0.0;
  if constexpr (LAW == FEM_LAW_LAPLACE) {
#pragma unroll
    for (int i = 0; i < VEC; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) P[i * 3 + j] = ug[i][j] * jxw;
    cf[0] = jxw;
  } else if constexpr (LAW == FEM_LAW_LINEAR || LAW == FEM_LAW_SIMP) {
    double E, nu;
    if constexpr (LAW == FEM_LAW_LINEAR) {
      E = A.p[0];
      nu = A.p[1];
    } else {
      E = A.p[1] + (A.p[0] - A.p[1]) * pow(A.iv0[k], A.p[3]);
      nu = A.p[2];
    }
    const double mu = E / (2.0 * (1.0 + nu));
    const double lm = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double tr = ug[0][0] + ug[1][1] + ug[2][2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) P[i * 3 + j] = jxw * (mu * (ug[i][j] + ug[j][i]) + (i == j ? lm * tr : 0.0));
    cf[0] = lm * jxw;
    cf[1] = mu * jxw;
  } else if constexpr (LAW == FEM_LAW_NEO_HOOKEAN) {
    NHState s;
    double Pu[3][3];
    nh_stress(ug, A.p[0], A.p[1], &s, Pu);
    const double kappa = A.p[0] / (3.0 * (1.0 - 2.0 * A.p[1]));
    double scale = jxw;
    if (A.iv0 != nullptr) scale *= A.iv0[k];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        P[i * 3 + j] = scale * Pu[i][j];
        M1[i][j] = s.F[i][j];
        M2[i][j] = s.H[i][j];
      }
    cf[0] = scale * s.m;
    cf[1] = scale * (-2.0 / 3.0) * s.m;
    cf[2] = scale * (2.0 / 9.0 * s.m * s.I1 + kappa * (2.0 * s.J - 1.0) * s.J);
    cf[3] = scale * (s.m * s.I1 / 3.0 - kappa * s.J * (s.J - 1.0));
  } else if constexpr (LAW == FEM_LAW_J2) {
    const double E = A.p[0], nu = A.p[1], Hh = A.p[3];
    const double mu = E / (2.0 * (1.0 + nu));
    const double lm = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    J2State r;
    j2_trial(ug, A.iv0 + k * 9, A.iv1 + k * 9, A.iv2[k], mu, lm, A.p[2], Hh, &r);
    double gam2 = 0.0;
    if (r.dg > 0.0) gam2 = 9.0 * mu * mu * r.syc / ((3.0 * mu + Hh) * r.q * r.q * r.q);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        P[i * 3 + j] = jxw * (r.st[i][j] - r.beta * r.s[i][j]);
        M1[i][j] = r.s[i][j];
      }
    cf[0] = jxw * (lm + 2.0 * mu * r.beta / 3.0);
    cf[1] = jxw * mu * (1.0 - r.beta);
    cf[2] = jxw * gam2;
  }
}

// Phase 1 in one step (short per-node work): the record of quadrature point
// q of cell c (node record nd).
template <int NEN, int VEC, int LAW>
__device__ __forceinline__ void quad_record(const ElemArgs& A, int64_t c, int q, const double* nd, double* qd) {
  using L = ElemLayout<NEN, VEC, LAW>;
  constexpr int NF = node_fields<VEC>();
  const double* gr = A.gref + int64_t(q) * NEN * 3;
  double inv[3][3];
  const double det = elem_jacobian<NEN>(gr, nd, NF, inv);
  const double jxw = det * __ldg(A.wq + q);
  double ug[VEC][3];
#pragma unroll
  for (int i = 0; i < VEC; ++i) ug[i][0] = ug[i][1] = ug[i][2] = 0.0;
#pragma unroll 2
  for (int a = 0; a < NEN; ++a) {
    double g[3];
    phys_grad(gr, a, inv, g);
#pragma unroll
    for (int j = 0; j < 3; ++j) qd[L::G + a * 3 + j] = g[j];
#pragma unroll
    for (int i = 0; i < VEC; ++i) {
      const double ua = nd[a * NF + 3 + i];
#pragma unroll
      for (int j = 0; j < 3; ++j) ug[i][j] = fma(ua, g[j], ug[i][j]);
    }
  }
  double M1[3][3], M2[3][3];
  elem_law<VEC, LAW>(A, c * A.nq + q, ug, jxw, qd + L::PO, qd + L::C, M1, M2);
  if constexpr (L::NV >= 1) {
#pragma unroll 2
    for (int b = 0; b < NEN; ++b) {
      const double g0 = qd[L::G + b * 3], g1 = qd[L::G + b * 3 + 1], g2 = qd[L::G + b * 3 + 2];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        qd[L::V1 + b * 3 + i] = M1[i][0] * g0 + M1[i][1] * g1 + M1[i][2] * g2;
        if constexpr (L::NV == 2) qd[L::V2 + b * 3 + i] = M2[i][0] * g0 + M2[i][1] * g1 + M2[i][2] * g2;
      }
    }
  }
}

// Split phase 1a, per quadrature point q of cell c (node record nd): J and the
// reference gradient of u, sum_a u_a (x) dN_a/dxi, in one pass over the
// nodes; J^-1, JxW; grad u = (sum_a u_a (x) dN_a/dxi) J^-1; the law.  J^-1
// and the law's matrices go to the record's scratch for phase 1b.
template <int NEN, int VEC, int LAW>
__device__ __forceinline__ void quad_point(const ElemArgs& A, int64_t c, int q, const double* nd, double* qd) {
  using L = ElemLayout<NEN, VEC, LAW>;
  constexpr int NF = node_fields<VEC>();
  const double* gr = A.gref + int64_t(q) * NEN * 3;
  double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  double ur[VEC][3];
#pragma unroll
  for (int i = 0; i < VEC; ++i) ur[i][0] = ur[i][1] = ur[i][2] = 0.0;
#pragma unroll 4
  for (int a = 0; a < NEN; ++a) {
    const double d[3] = {__ldg(gr + a * 3), __ldg(gr + a * 3 + 1), __ldg(gr + a * 3 + 2)};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double x = nd[a * NF + i];
#pragma unroll
      for (int k = 0; k < 3; ++k) J[i][k] = fma(x, d[k], J[i][k]);
    }
#pragma unroll
    for (int i = 0; i < VEC; ++i) {
      const double ua = nd[a * NF + 3 + i];
#pragma unroll
      for (int k = 0; k < 3; ++k) ur[i][k] = fma(ua, d[k], ur[i][k]);
    }
  }
  double inv[3][3];
  const double det = invert3(J, inv);
  const double jxw = det * __ldg(A.wq + q);
  double ug[VEC][3];
#pragma unroll
  for (int i = 0; i < VEC; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) ug[i][k] = ur[i][0] * inv[0][k] + ur[i][1] * inv[1][k] + ur[i][2] * inv[2][k];
  double M1[3][3], M2[3][3];
  elem_law<VEC, LAW>(A, c * A.nq + q, ug, jxw, qd + L::PO, qd + L::C, M1, M2);
  double* sc = qd + L::SC;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      sc[i * 3 + k] = inv[i][k];
      if constexpr (L::NV >= 1) sc[9 + i * 3 + k] = M1[i][k];
      if constexpr (L::NV == 2) sc[18 + i * 3 + k] = M2[i][k];
    }
}

// Phase 1b, per (quadrature point q, node a): g_a = J^-T dN_a/dxi and the
// law vectors M1 g_a, M2 g_a, from the scratch phase 1a left in the record.
template <int NEN, int VEC, int LAW>
__device__ __forceinline__ void node_vectors(const ElemArgs& A, int q, int a, double* qd) {
  using L = ElemLayout<NEN, VEC, LAW>;
  const double* gr = A.gref + (int64_t(q) * NEN + a) * 3;
  const double d0 = __ldg(gr), d1 = __ldg(gr + 1), d2 = __ldg(gr + 2);
  const double* sc = qd + L::SC;
  double g[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    g[k] = d0 * sc[k] + d1 * sc[3 + k] + d2 * sc[6 + k];
    qd[L::G + a * 3 + k] = g[k];
  }
  if constexpr (L::NV >= 1) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      qd[L::V1 + a * 3 + i] = sc[9 + i * 3] * g[0] + sc[9 + i * 3 + 1] * g[1] + sc[9 + i * 3 + 2] * g[2];
      if constexpr (L::NV == 2)
        qd[L::V2 + a * 3 + i] = sc[18 + i * 3] * g[0] + sc[18 + i * 3 + 1] * g[1] + sc[18 + i * 3 + 2] * g[2];
    }
  }
}

// Phase 2: K_ab += the contribution of one quadrature record.
template <int NEN, int VEC, int LAW>
__device__ __forceinline__ void elem_pair(const double* qd, int a, int b, double K[VEC][VEC]) {
  using L = ElemLayout<NEN, VEC, LAW>;
  const double* g = qd + L::G;
  const double* cf = qd + L::C;
  const double ga[3] = {g[a * 3], g[a * 3 + 1], g[a * 3 + 2]};
  const double gb[3] = {g[b * 3], g[b * 3 + 1], g[b * 3 + 2]};
  const double dot = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
  if constexpr (LAW == FEM_LAW_LAPLACE) {
    const double s = cf[0] * dot;
#pragma unroll
    for (int i = 0; i < VEC; ++i) K[i][i] += s;
  } else if constexpr (LAW == FEM_LAW_LINEAR || LAW == FEM_LAW_SIMP) {
    const double lm = cf[0], mu = cf[1];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
      for (int k = 0; k < 3; ++k) K[i][k] += lm * ga[i] * gb[k] + mu * gb[i] * ga[k];
      K[i][i] += mu * dot;
    }
  } else if constexpr (LAW == FEM_LAW_NEO_HOOKEAN) {
    const double* f = qd + L::V1;
    const double* h = qd + L::V2;
    const double m = cf[0], c2 = cf[1], c4 = cf[2], c5 = cf[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double ua = c2 * f[a * 3 + i] + c4 * h[a * 3 + i];
      const double va = c2 * h[a * 3 + i];
#pragma unroll
      for (int k = 0; k < 3; ++k) K[i][k] += ua * h[b * 3 + k] + va * f[b * 3 + k] + c5 * h[b * 3 + i] * h[a * 3 + k];
      K[i][i] += m * dot;
    }
  } else if constexpr (LAW == FEM_LAW_J2) {
    const double* sg = qd + L::V1;
    const double cII = cf[0], ch = cf[1], g2 = cf[2];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
      for (int k = 0; k < 3; ++k) K[i][k] += cII * ga[i] * gb[k] + ch * gb[i] * ga[k] - g2 * sg[a * 3 + i] * sg[b * 3 + k];
      K[i][i] += ch * dot;
    }
  }
}

template <int NEN, int VEC, int LAW, typename T>
__global__ void __launch_bounds__(kElemThreads) elem_assemble_kernel(const ElemArgs A) {
  using S = ElemShape<NEN>;
  using L = ElemLayout<NEN, VEC, LAW>;
  constexpr int NF = node_fields<VEC>();
  constexpr int NP = NEN * (NEN + 1) / 2;
  constexpr int PPT = (NP + S::TPC - 1) / S::TPC;
  static_assert(S::TPC * S::CPB == kElemThreads && S::QC * S::CPB <= kElemThreads && NEN <= S::TPC,
                "element work split");
  extern __shared__ __align__(16) unsigned char smem[];
  double* sq = reinterpret_cast<double*>(smem);
  double* sn = sq + S::CPB * S::QC * L::QF;
  double* slift = sn + S::CPB * NEN * NF;
  int* sbc = reinterpret_cast<int*>(slift + S::CPB * NEN * VEC);
  int* snode = sbc + S::CPB * NEN;

  const int cl = threadIdx.x / S::TPC;
  const int t = threadIdx.x - cl * S::TPC;
  const int64_t c = int64_t(blockIdx.x) * S::CPB + cl;
  const bool valid = c < A.num_cells;

  // ---- phase 0: node data ----
  if (t < NEN) {
    const int node = valid ? A.cells[c * NEN + t] : 0;
    double* nd = sn + (cl * NEN + t) * NF;
    int bits = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) nd[i] = valid ? A.points[int64_t(node) * 3 + i] : 0.0;
#pragma unroll
    for (int i = 0; i < VEC; ++i) {
      const int64_t dof = int64_t(node) * VEC + i;
      nd[3 + i] = valid ? A.u[dof] : 0.0;
      nd[3 + VEC + i] = (valid && A.dvec != nullptr) ? A.dvec[dof] : 0.0;
      if (valid && A.bc != nullptr && A.bc[dof]) bits |= 1 << i;
      if (nd[3 + VEC + i] != 0.0) bits |= kLiftBit;
      slift[(cl * NEN + t) * VEC + i] = 0.0;
    }
    sbc[cl * NEN + t] = bits;
    snode[cl * NEN + t] = node;
  }

  // node pairs of this thread: p = t + k TPC, a <= b in row-major order of
  // the upper triangle
  int pa[PPT], pb[PPT];
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    int p = t + k * S::TPC;
    pa[k] = -1;
    pb[k] = 0;
    if (p < NP) {
      int a = 0;
      while (p >= NEN - a) {
        p -= NEN - a;
        ++a;
      }
      pa[k] = a;
      pb[k] = a + p;
    }
  }
  double K[PPT][VEC][VEC];
#pragma unroll
  for (int k = 0; k < PPT; ++k)
#pragma unroll
    for (int i = 0; i < VEC; ++i)
#pragma unroll
      for (int j = 0; j < VEC; ++j) K[k][i][j] = 0.0;
  double r[VEC];
#pragma unroll
  for (int i = 0; i < VEC; ++i) r[i] = 0.0;
  const bool want_k = A.vals != nullptr || A.lift != nullptr;
  __syncthreads();

  for (int q0 = 0; q0 < A.nq; q0 += S::QC) {
    // ---- phase 1 (1a): one thread per (cell, quadrature point of the chunk) ----
    if (threadIdx.x < S::CPB * S::QC) {
      const int wcl = threadIdx.x / S::QC;
      const int qi = threadIdx.x - wcl * S::QC;
      const int64_t wc = int64_t(blockIdx.x) * S::CPB + wcl;
      if (wc < A.num_cells && q0 + qi < A.nq) {
        if constexpr (S::SPLIT)
          quad_point<NEN, VEC, LAW>(A, wc, q0 + qi, sn + wcl * NEN * NF, sq + (wcl * S::QC + qi) * L::QF);
        else
          quad_record<NEN, VEC, LAW>(A, wc, q0 + qi, sn + wcl * NEN * NF, sq + (wcl * S::QC + qi) * L::QF);
      }
    }
    __syncthreads();
    if constexpr (S::SPLIT) {
      // ---- phase 1b: every thread, (cell, quadrature point, node) items ----
#pragma unroll 1
      for (int it = threadIdx.x; it < S::CPB * S::QC * NEN; it += kElemThreads) {
        const int wcl = it / (S::QC * NEN);
        const int rem = it - wcl * (S::QC * NEN);
        const int qi = rem / NEN;
        const int a = rem - qi * NEN;
        const int64_t wc = int64_t(blockIdx.x) * S::CPB + wcl;
        if (wc < A.num_cells && q0 + qi < A.nq)
          node_vectors<NEN, VEC, LAW>(A, q0 + qi, a, sq + (wcl * S::QC + qi) * L::QF);
      }
      __syncthreads();
    }
    // ---- phase 2: pairs and residual ----
    const int nqc = min(S::QC, A.nq - q0);
    if (valid) {
      const double* cq = sq + cl * S::QC * L::QF;
#pragma unroll 1
      for (int qi = 0; qi < nqc; ++qi) {
        const double* qd = cq + qi * L::QF;
        if (want_k) {
#pragma unroll
          for (int k = 0; k < PPT; ++k)
            if (pa[k] >= 0) elem_pair<NEN, VEC, LAW>(qd, pa[k], pb[k], K[k]);
        }
        if (t < NEN) {
          const double* P = qd + L::PO;
          const double g0 = qd[L::G + t * 3], g1 = qd[L::G + t * 3 + 1], g2 = qd[L::G + t * 3 + 2];
#pragma unroll
          for (int i = 0; i < VEC; ++i) r[i] += P[i * 3] * g0 + P[i * 3 + 1] * g1 + P[i * 3 + 2] * g2;
        }
      }
    }
    __syncthreads();
  }

  if (valid && t < NEN && A.res != nullptr) {
    const int64_t node = snode[cl * NEN + t];
#pragma unroll
    for (int i = 0; i < VEC; ++i) atomicAdd(A.res + node * VEC + i, r[i]);
  }
  if (!want_k) return;  // uniform over the block
  T* vals = reinterpret_cast<T*>(A.vals);
  const double* nb = sn + cl * NEN * NF;
  if (valid) {
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
      if (pa[k] < 0) continue;
      const int a = pa[k], b = pb[k];
      const int abits = sbc[cl * NEN + a], bbits = sbc[cl * NEN + b];
      if (A.lift != nullptr && (bbits & kLiftBit)) {
        // row a: K_ab d_b
#pragma unroll
        for (int i = 0; i < VEC; ++i) {
          double la = 0.0;
#pragma unroll
          for (int j = 0; j < VEC; ++j) la += K[k][i][j] * nb[b * NF + 3 + VEC + j];
          atomicAdd(slift + (cl * NEN + a) * VEC + i, la);
        }
      }
      if (A.lift != nullptr && a != b && (abits & kLiftBit)) {
        // row b: K_ab^T d_a
#pragma unroll
        for (int j = 0; j < VEC; ++j) {
          double lb = 0.0;
#pragma unroll
          for (int i = 0; i < VEC; ++i) lb += K[k][i][j] * nb[a * NF + 3 + VEC + i];
          atomicAdd(slift + (cl * NEN + b) * VEC + j, lb);
        }
      }
      if (vals != nullptr) {
        const int na = snode[cl * NEN + a], nbn = snode[cl * NEN + b];
        const int32_t* smap = A.scatter + c * (NEN * NEN);
        if (a == b || na < nbn) {
          T* blk = vals + int64_t(smap[a * NEN + b]) * (VEC * VEC);
#pragma unroll
          for (int i = 0; i < VEC; ++i)
#pragma unroll
            for (int j = 0; j < VEC; ++j)
              if (!(((abits >> i) | (bbits >> j)) & 1)) atomicAdd(blk + i * VEC + j, T(K[k][i][j]));
        }
        if (a != b && na >= nbn) {  // (na == nbn only in a degenerate cell: both orientations)
          T* blk = vals + int64_t(smap[b * NEN + a]) * (VEC * VEC);
#pragma unroll
          for (int j = 0; j < VEC; ++j)
#pragma unroll
            for (int i = 0; i < VEC; ++i)
              if (!(((bbits >> j) | (abits >> i)) & 1)) atomicAdd(blk + j * VEC + i, T(K[k][i][j]));
        }
      }
    }
  }
  if (A.lift != nullptr) {
    __syncthreads();
    int any = 0;
    for (int b = 0; b < NEN; ++b) any |= sbc[cl * NEN + b];
    if (valid && t < NEN && (any & kLiftBit)) {
      const int abits = sbc[cl * NEN + t];
      const int64_t node = snode[cl * NEN + t];
#pragma unroll
      for (int i = 0; i < VEC; ++i)
        if (!((abits >> i) & 1)) atomicAdd(A.lift + node * VEC + i, slift[(cl * NEN + t) * VEC + i]);
    }
  }
}

template <int NEN, int VEC, int LAW, typename T>
int launch_elem(const ElemArgs& A, cudaStream_t st) {
  using S = ElemShape<NEN>;
  const unsigned grid = unsigned((A.num_cells + S::CPB - 1) / S::CPB);
  constexpr size_t sm = elem_smem_bytes<NEN, VEC, LAW>();
  auto k = elem_assemble_kernel<NEN, VEC, LAW, T>;
  static bool attr = false;
  if (!attr) {
    FEM_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    attr = true;
  }
  k<<<grid, kElemThreads, sm, st>>>(A);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}

template <int NEN, typename T>
int dispatch_law(int law, int vec, const ElemArgs& A, cudaStream_t st) {
  if (vec == 1) return launch_elem<NEN, 1, FEM_LAW_LAPLACE, T>(A, st);
  switch (law) {
    case FEM_LAW_LAPLACE: return launch_elem<NEN, 3, FEM_LAW_LAPLACE, T>(A, st);
    case FEM_LAW_LINEAR: return launch_elem<NEN, 3, FEM_LAW_LINEAR, T>(A, st);
    case FEM_LAW_SIMP: return launch_elem<NEN, 3, FEM_LAW_SIMP, T>(A, st);
    case FEM_LAW_NEO_HOOKEAN: return launch_elem<NEN, 3, FEM_LAW_NEO_HOOKEAN, T>(A, st);
    case FEM_LAW_J2: return launch_elem<NEN, 3, FEM_LAW_J2, T>(A, st);
  }
  set_error("unknown law %d", law);
  return FEM_ERR_ARG;
}

bool supported_nen(int nen) { return nen == 4 || nen == 8 || nen == 10 || nen == 20 || nen == 27; }

template <typename T>
int elem_assemble_impl(int law, const double* h_params, int n_params, int vec, int nen, int nq,
                       const double* d_gref, const double* d_wq, int64_t num_cells, int64_t num_nodes,
                       const int32_t* d_cells, const double* d_points, const double* d_u, const double* iv0,
                       const double* iv1, const double* iv2, const int32_t* d_scatter, const int32_t* d_diag,
                       const int32_t* d_transpose, int64_t nnzb, const uint8_t* d_bc, const double* d_dvec,
                       double* d_res, double* d_lift, T* d_vals, void* stream) {
  FEM_CHECK_ARG(num_cells >= 0 && num_nodes >= 0, "negative sizes");
  FEM_CHECK_ARG(supported_nen(nen), "nodes per cell %d: supported are 4, 8, 10, 20, 27", nen);
  FEM_CHECK_ARG(nq >= 1 && nq <= kMaxQuads, "quadrature points %d outside [1, %d]", nq, kMaxQuads);
  FEM_CHECK_ARG(d_gref != nullptr && d_wq != nullptr, "element tables are NULL");
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
  FEM_CHECK_ARG(d_lift == nullptr || d_dvec != nullptr, "lift needs dvec");
  cudaStream_t st = as_stream(stream);
  const int64_t ndofs = num_nodes * vec;
  if (d_res) FEM_CUDA_TRY(cudaMemsetAsync(d_res, 0, sizeof(double) * ndofs, st));
  if (d_lift) FEM_CUDA_TRY(cudaMemsetAsync(d_lift, 0, sizeof(double) * ndofs, st));
  if (d_vals) FEM_CUDA_TRY(cudaMemsetAsync(d_vals, 0, sizeof(T) * nnzb * vec * vec, st));
  if (num_cells == 0) return d_vals ? finish_tangent<T>(vec, nnzb, ndofs, d_transpose, d_bc, d_diag, d_vals, st)
                                    : FEM_OK;
  ElemArgs A{};
  A.num_cells = num_cells;
  A.nq = nq;
  A.gref = d_gref;
  A.wq = d_wq;
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
  int rc = FEM_ERR_ARG;
  switch (nen) {
    case 4: rc = dispatch_law<4, T>(law, vec, A, st); break;
    case 8: rc = dispatch_law<8, T>(law, vec, A, st); break;
    case 10: rc = dispatch_law<10, T>(law, vec, A, st); break;
    case 20: rc = dispatch_law<20, T>(law, vec, A, st); break;
    case 27: rc = dispatch_law<27, T>(law, vec, A, st); break;
  }
  if (rc != FEM_OK) return rc;
  if (d_vals != nullptr) return finish_tangent<T>(vec, nnzb, ndofs, d_transpose, d_bc, d_diag, d_vals, st);
  return FEM_OK;
}

// ---- per (cell, quadrature point) passes ------------------------------------------
// One thread per (cell, quadrature point); a cell's node data is read from
// global memory by each of its threads (it stays in L1).

// grad of up to two nodal vector fields at quadrature point q of cell c;
// returns JxW.
template <int NEN>
__device__ __forceinline__ double point_grads(const int32_t* cells, const double* points, const double* gref,
                                              const double* wq, int64_t c, int q, const double* v0,
                                              const double* v1, double gu[3][3], double gl[3][3]) {
  const int32_t* cn = cells + c * NEN;
  const double* gr = gref + int64_t(q) * NEN * 3;
  double X[NEN * 3];
#pragma unroll
  for (int a = 0; a < NEN; ++a) {
    const int64_t n = cn[a];
#pragma unroll
    for (int i = 0; i < 3; ++i) X[a * 3 + i] = points[n * 3 + i];
  }
  double inv[3][3];
  const double det = elem_jacobian<NEN>(gr, X, 3, inv);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) gu[i][j] = gl[i][j] = 0.0;
#pragma unroll 1
  for (int a = 0; a < NEN; ++a) {
    const int64_t n = cn[a];
    double g[3];
    phys_grad(gr, a, inv, g);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double ua = v0 ? v0[n * 3 + i] : 0.0;
      const double la = v1 ? v1[n * 3 + i] : 0.0;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        gu[i][j] = fma(ua, g[j], gu[i][j]);
        gl[i][j] = fma(la, g[j], gl[i][j]);
      }
    }
  }
  return det * (wq ? wq[q] : 1.0);
}

template <int NEN>
__global__ void __launch_bounds__(128) elem_j2_commit_kernel(int64_t C, int nq, const double* gref,
                                                             const int32_t* cells, const double* points,
                                                             const double* u, double E, double nu, double sy0,
                                                             double Hh, const double* so, const double* eo,
                                                             const double* ao, double* sn, double* en,
                                                             double* an) {
  const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= C * nq) return;
  const int64_t c = k / nq;
  const int q = int(k - c * nq);
  double gu[3][3], gl[3][3];
  point_grads<NEN>(cells, points, gref, nullptr, c, q, u, nullptr, gu, gl);
  const double mu = E / (2.0 * (1.0 + nu));
  const double lm = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  J2State r;
  j2_trial(gu, so + k * 9, eo + k * 9, ao[k], mu, lm, sy0, Hh, &r);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      sn[k * 9 + i * 3 + j] = r.st[i][j] - r.beta * r.s[i][j];
      en[k * 9 + i * 3 + j] = r.eps[i][j];
    }
  an[k] = ao[k] + r.dg;
}

// grad[c,q] = -(dP/dtheta : grad lambda) JxW (SIMP: theta; NEO_HOOKEAN: the
// psi scale, dP/ds = P of the unscaled law).
template <int NEN>
__global__ void __launch_bounds__(128) elem_param_vjp_kernel(int law, int64_t C, int nq, const double* gref,
                                                             const double* wq, const int32_t* cells,
                                                             const double* points, const double* u,
                                                             const double* lam, const double* theta, double p0,
                                                             double p1, double p2, double p3, double* grad) {
  const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= C * nq) return;
  const int64_t c = k / nq;
  const int q = int(k - c * nq);
  double gu[3][3], gl[3][3];
  const double jxw = point_grads<NEN>(cells, points, gref, wq, c, q, u, lam, gu, gl);
  double dP[3][3];
  if (law == FEM_LAW_SIMP) {
    const double E0 = p0, Emin = p1, nu = p2, pen = p3;
    const double dE = (E0 - Emin) * pen * pow(theta[k], pen - 1.0);
    const double mu = 1.0 / (2.0 * (1.0 + nu));
    const double lm = nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double tr = gu[0][0] + gu[1][1] + gu[2][2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) dP[i][j] = dE * (mu * (gu[i][j] + gu[j][i]) + (i == j ? lm * tr : 0.0));
  } else {
    NHState s;
    nh_stress(gu, p0, p1, &s, dP);
  }
  double acc = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) acc = fma(dP[i][j], gl[i][j], acc);
  grad[k] = -acc * jxw;
}

}  // namespace
}  // namespace fem

using namespace fem;

extern "C" int fem_assemble_elem_f64(int law, const double* h_params, int n_params, int vec, int nen, int nq,
                                     const double* d_gref, const double* d_wq, int64_t num_cells,
                                     int64_t num_nodes, const int32_t* d_cells, const double* d_points,
                                     const double* d_u, const double* d_ivar0, const double* d_ivar1,
                                     const double* d_ivar2, const int32_t* d_scatter, const int32_t* d_diag,
                                     const int32_t* d_transpose, int64_t nnzb, const uint8_t* d_bc_mask,
                                     const double* d_dvec, double* d_res, double* d_lift, double* d_vals,
                                     void* stream) {
  return elem_assemble_impl<double>(law, h_params, n_params, vec, nen, nq, d_gref, d_wq, num_cells, num_nodes,
                                    d_cells, d_points, d_u, d_ivar0, d_ivar1, d_ivar2, d_scatter, d_diag,
                                    d_transpose, nnzb, d_bc_mask, d_dvec, d_res, d_lift, d_vals, stream);
}

extern "C" int fem_assemble_elem_f32(int law, const double* h_params, int n_params, int vec, int nen, int nq,
                                     const double* d_gref, const double* d_wq, int64_t num_cells,
                                     int64_t num_nodes, const int32_t* d_cells, const double* d_points,
                                     const double* d_u, const double* d_ivar0, const double* d_ivar1,
                                     const double* d_ivar2, const int32_t* d_scatter, const int32_t* d_diag,
                                     const int32_t* d_transpose, int64_t nnzb, const uint8_t* d_bc_mask,
                                     const double* d_dvec, double* d_res, double* d_lift, float* d_vals,
                                     void* stream) {
  return elem_assemble_impl<float>(law, h_params, n_params, vec, nen, nq, d_gref, d_wq, num_cells, num_nodes,
                                   d_cells, d_points, d_u, d_ivar0, d_ivar1, d_ivar2, d_scatter, d_diag,
                                   d_transpose, nnzb, d_bc_mask, d_dvec, d_res, d_lift, d_vals, stream);
}

extern "C" int fem_j2_commit_elem(const double* h_params, int n_params, int nen, int nq, const double* d_gref,
                                  int64_t num_cells, const int32_t* d_cells, const double* d_points,
                                  const double* d_u, const double* d_sigma_old, const double* d_eps_old,
                                  const double* d_alpha_old, double* d_sigma_new, double* d_eps_new,
                                  double* d_alpha_new, void* stream) {
  FEM_CHECK_ARG(h_params != nullptr && n_params >= 4, "J2 needs E, nu, sigma_y, H");
  FEM_CHECK_ARG(supported_nen(nen), "nodes per cell %d: supported are 4, 8, 10, 20, 27", nen);
  FEM_CHECK_ARG(nq >= 1 && nq <= kMaxQuads && d_gref != nullptr, "element tables");
  FEM_CHECK_ARG(num_cells >= 0, "negative size");
  FEM_CHECK_ARG(d_cells && d_points && d_u && d_sigma_old && d_eps_old && d_alpha_old && d_sigma_new &&
                    d_eps_new && d_alpha_new,
                "J2 state pointer is NULL");
  const int64_t n = num_cells * nq;
  if (n == 0) return FEM_OK;
  const unsigned grid = unsigned((n + 127) / 128);
  cudaStream_t st = as_stream(stream);
  const double E = h_params[0], nu = h_params[1], sy = h_params[2], H = h_params[3];
#define FEM_J2_ELEM(NEN_)                                                                              \
  elem_j2_commit_kernel<NEN_><<<grid, 128, 0, st>>>(num_cells, nq, d_gref, d_cells, d_points, d_u, E, nu, \
                                                    sy, H, d_sigma_old, d_eps_old, d_alpha_old,         \
                                                    d_sigma_new, d_eps_new, d_alpha_new)
  switch (nen) {
    case 4: FEM_J2_ELEM(4); break;
    case 8: FEM_J2_ELEM(8); break;
    case 10: FEM_J2_ELEM(10); break;
    case 20: FEM_J2_ELEM(20); break;
    case 27: FEM_J2_ELEM(27); break;
  }
#undef FEM_J2_ELEM
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}

extern "C" int fem_param_vjp_elem_f64(int law, const double* h_params, int n_params, int nen, int nq,
                                      const double* d_gref, const double* d_wq, int64_t num_cells,
                                      const int32_t* d_cells, const double* d_points, const double* d_u,
                                      const double* d_ivar0, const double* d_lambda, double* d_grad,
                                      void* stream) {
  FEM_CHECK_ARG(law == FEM_LAW_SIMP || law == FEM_LAW_NEO_HOOKEAN,
                "parameter VJP is defined for SIMP (theta) and NEO_HOOKEAN (psi scale), not law %d", law);
  FEM_CHECK_ARG(h_params != nullptr && n_params >= (law == FEM_LAW_SIMP ? 4 : 2), "law parameters");
  FEM_CHECK_ARG(law != FEM_LAW_SIMP || d_ivar0 != nullptr, "SIMP needs theta (ivar0)");
  FEM_CHECK_ARG(supported_nen(nen), "nodes per cell %d: supported are 4, 8, 10, 20, 27", nen);
  FEM_CHECK_ARG(nq >= 1 && nq <= kMaxQuads && d_gref != nullptr && d_wq != nullptr, "element tables");
  FEM_CHECK_ARG(num_cells >= 0, "negative size");
  FEM_CHECK_ARG(d_cells && d_points && d_u && d_lambda && d_grad, "param VJP: NULL pointer");
  const int64_t n = num_cells * nq;
  if (n == 0) return FEM_OK;
  const unsigned grid = unsigned((n + 127) / 128);
  cudaStream_t st = as_stream(stream);
  double p[4] = {0, 0, 0, 0};
  for (int i = 0; i < 4 && i < n_params; ++i) p[i] = h_params[i];
#define FEM_VJP_ELEM(NEN_)                                                                                   \
  elem_param_vjp_kernel<NEN_><<<grid, 128, 0, st>>>(law, num_cells, nq, d_gref, d_wq, d_cells, d_points, d_u, \
                                                    d_lambda, d_ivar0, p[0], p[1], p[2], p[3], d_grad)
  switch (nen) {
    case 4: FEM_VJP_ELEM(4); break;
    case 8: FEM_VJP_ELEM(8); break;
    case 10: FEM_VJP_ELEM(10); break;
    case 20: FEM_VJP_ELEM(20); break;
    case 27: FEM_VJP_ELEM(27); break;
  }
#undef FEM_VJP_ELEM
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}
