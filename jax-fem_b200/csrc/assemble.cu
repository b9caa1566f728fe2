// HEX8 cell assembly: residual, BC-eliminated block-CSR tangent and Dirichlet
// lift in one pass over the cells.
//
// Replaces the reference's per-cell weak-form kernel + jacfwd
// (problem.py:189-214, 262-266, 299-301, 334-338), the residual scatter
// (problem.py:426-437) and the PETSc COO insertion + zeroRows of get_A
// (solver.py:485-491).  The reference differentiates the kernel with 24
// forward-mode JVPs per cell; here every law supplies its exact tangent in a
// rank-structured form (law_quad / pair_row below), so one evaluation per
// quadrature point yields residual and tangent together.
//
// Precision: geometry, the constitutive update and the residual are FP64 in
// every variant; the tangent (its per-quad factors and node vectors in shared
// memory, the row products and the stored values) is FP64 or FP32.
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

// ---- work split --------------------------------------------------------------
// Each warp owns groups of kGroupCells = 4 consecutive cells and loops over
// them (grid-stride); warps share nothing, so only __syncwarp orders the
// phases.  For one group:
//  phase 0  lane = (cell, node): connectivity, coordinates, u, the prescribed
//           increment d and the Dirichlet bits of one node -> warp smem
//  phase 1  lane = (cell, quadrature point), all 32 lanes busy: FP64
//           geometry, grad u and the constitutive update; the per-node law
//           vectors and the tangent coefficients (type T) -> warp smem; the
//           residual contributions of the 8 nodes are summed over the cell's
//           8 lanes by a transposed shuffle reduction (each round halves the
//           values a lane holds, 21 FP64 shuffles), after which lane q holds
//           node q's residual and adds it to R with 3 atomics
//  phase 2  lane = element-matrix row (node a, component i); for VEC = 3 one
//           cell per pass (24 lanes), for VEC = 1 four cells per pass.  Every
//           element matrix here is symmetric, so of the 64 node blocks only
//           36 are formed: row a takes the blocks (a, a + j mod 8), j = 0..3,
//           and j = 4 for a < 4 (each unordered pair once; 5 or 4 blocks per
//           lane).  The lane keeps its own node's vectors in registers and
//           reads node b's from the record; as the lanes of a warp read one
//           record at 8 distinct nodes, whose rows are laid out bank-disjoint,
//           a 16-byte load is a single shared-memory wavefront.  The blocks go
//           to the global upper triangle (row node < column node), transposed
//           when the local order is reversed, through the cell -> block map,
//           with Dirichlet rows and columns left out; the lift K d of the
//           eliminated columns is gathered per cell in warp smem.
//  mirror   finish_tangent writes each lower block as the transpose of its
//           upper partner, and the unit diagonal at Dirichlet dofs.
constexpr int kGroupCells = 4;
constexpr int kAsmWarps = 4;
constexpr int kAsmThreads = 32 * kAsmWarps;

// Per-node vectors a law stores per quadrature point: g (physical shape
// gradient) for all; NH adds f = F g and h = F^-T g; J2 adds s g (deviatoric
// trial stress applied to g).
template <int LAW>
struct LawTraits {
  static constexpr int NV = (LAW == FEM_LAW_NEO_HOOKEAN) ? 3 : ((LAW == FEM_LAW_J2) ? 2 : 1);
};

// Record of one (cell, quadrature point) in warp smem, in units of T:
//   [0, 4)              tangent coefficients * JxW
//   [4 + b NS, ...)     node b's vectors g, (f, h | s), padded to NS
// NS keeps every node row 16-byte aligned and the 8 rows of a record in
// disjoint banks (float: 4 or 12 words; double: 6 or 10 doubles).
template <int LAW, typename T>
struct Rec {
  static constexpr int NV = LawTraits<LAW>::NV;
  static constexpr int NS = sizeof(T) == 4 ? (NV == 1 ? 4 : 12) : (NV == 3 ? 10 : 6);
  static constexpr int SIZE = 4 + 8 * NS;
};

// Per-node data of the group's 32 nodes (FP64): x, u, d.
template <int VEC>
struct NodeRec {
  static constexpr int X = 0;
  static constexpr int U = 3;
  static constexpr int D = 3 + VEC;
  static constexpr int NF = 3 + 2 * VEC;
};

template <int VEC, int LAW, typename T>
__host__ __device__ constexpr size_t warp_smem_bytes() {
  return size_t(kGroupCells) * 8 * Rec<LAW, T>::SIZE * sizeof(T) +     // records
         size_t(kGroupCells) * 8 * NodeRec<VEC>::NF * sizeof(double) +  // node data
         size_t(kGroupCells) * 8 * VEC * sizeof(double) +               // lift accumulators
         size_t(kGroupCells) * 8 * 2 * sizeof(int);                     // Dirichlet bits, node ids
}

// Phase 1 law update at one quadrature point (FP64): P*JxW and the record.
template <int VEC, int LAW, typename T>
__device__ __forceinline__ void law_quad(const AsmArgs& A, int64_t c, int q, const double ug[VEC][3],
                                         const double g[8][3], double jxw, T* rec, double P[VEC * 3]) {
  using R = Rec<LAW, T>;
  T* cf = rec;
  T* nd = rec + 4;
#pragma unroll
  for (int b = 0; b < 8; ++b)
#pragma unroll
    for (int j = 0; j < 3; ++j) nd[b * R::NS + j] = T(g[b][j]);
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
    const double tr = ug[0][0] + ug[1][1] + ug[2][2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) P[i * 3 + j] = jxw * (mu * (ug[i][j] + ug[j][i]) + (i == j ? lm * tr : 0.0));
    // K_ab = lm g_a (x) g_b + mu g_b (x) g_a + mu (g_a . g_b) I
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
#pragma unroll
    for (int b = 0; b < 8; ++b)
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        nd[b * R::NS + 3 + i] = T(F[i][0] * g[b][0] + F[i][1] * g[b][1] + F[i][2] * g[b][2]);
        nd[b * R::NS + 6 + i] = T(H[i][0] * g[b][0] + H[i][1] * g[b][1] + H[i][2] * g[b][2]);
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
#pragma unroll
    for (int b = 0; b < 8; ++b)
#pragma unroll
      for (int i = 0; i < 3; ++i)
        nd[b * R::NS + 3 + i] = T(s[i][0] * g[b][0] + s[i][1] * g[b][1] + s[i][2] * g[b][2]);
  }
}

// Select v[i] for a lane-dependent i in {0, 1, 2} without local memory.
template <typename T>
__device__ __forceinline__ T pick3(const T v[3], int i) {
  return i == 0 ? v[0] : (i == 1 ? v[1] : v[2]);
}

// Phase 2 update of one row (a, i) against node b at one quadrature point:
// K[k] += K_ab[i][k] except the (g_a . g_b) I term, whose coefficient times
// the dot product is returned (added to K[i] once, after the quadrature loop).
// ar: the lane's own node vectors premultiplied as each law needs (own_row);
// br: node b's vectors; cf: the record's coefficients.
template <int LAW, typename T>
__device__ __forceinline__ T pair_row(const T* ar, const T* br, const T* cf, int i, T K[3]) {
  const T dot = ar[0] * br[0] + ar[1] * br[1] + ar[2] * br[2];
  if constexpr (LAW == FEM_LAW_LAPLACE) {
    return cf[0] * dot;
  } else if constexpr (LAW == FEM_LAW_LINEAR || LAW == FEM_LAW_SIMP) {
    // ar[3] = lm g_a[i];  K[k] += lm ga_i gb_k + mu gb_i ga_k
    const T y = cf[1] * pick3(br, i);
#pragma unroll
    for (int k = 0; k < 3; ++k) K[k] += ar[3] * br[k] + y * ar[k];
    return cf[1] * dot;
  } else if constexpr (LAW == FEM_LAW_NEO_HOOKEAN) {
    // ar[3] = c2 f_a[i] + c4 h_a[i], ar[4] = c2 h_a[i], ar[5..8) = h_a
    // K[k] += ar3 hb_k + ar4 fb_k + c5 hb_i ha_k
    const T* fb = br + 3;
    const T* hb = br + 6;
    const T y = cf[3] * pick3(hb, i);
#pragma unroll
    for (int k = 0; k < 3; ++k) K[k] += ar[3] * hb[k] + ar[4] * fb[k] + y * ar[5 + k];
    return cf[0] * dot;
  } else {  // J2
    // ar[3] = cII g_a[i], ar[4] = -gam2 (s g)_a[i]
    // K[k] += cII ga_i gb_k + ch gb_i ga_k - gam2 sa_i sb_k
    const T* sb = br + 3;
    const T y = cf[1] * pick3(br, i);
#pragma unroll
    for (int k = 0; k < 3; ++k) K[k] += ar[3] * br[k] + y * ar[k] + ar[4] * sb[k];
    return cf[1] * dot;
  }
}

// The lane's own node vectors for pair_row (see there).
template <int LAW, typename T>
__device__ __forceinline__ void own_row(const T* na, const T* cf, int i, T ar[8]) {
  ar[0] = na[0], ar[1] = na[1], ar[2] = na[2];
  if constexpr (LAW == FEM_LAW_LINEAR || LAW == FEM_LAW_SIMP) {
    ar[3] = cf[0] * pick3(na, i);
  } else if constexpr (LAW == FEM_LAW_NEO_HOOKEAN) {
    const T fi = pick3(na + 3, i), hi = pick3(na + 6, i);
    ar[3] = cf[1] * fi + cf[2] * hi;
    ar[4] = cf[1] * hi;
    ar[5] = na[6], ar[6] = na[7], ar[7] = na[8];
  } else if constexpr (LAW == FEM_LAW_J2) {
    ar[3] = cf[0] * pick3(na, i);
    ar[4] = -cf[2] * pick3(na + 3, i);
  }
}

// Load a record node row (NV vectors of 3) into registers with 16-byte loads.
template <int LAW, typename T>
__device__ __forceinline__ void load_row(const T* src, T* dst) {
  constexpr int N = 3 * LawTraits<LAW>::NV;
  if constexpr (sizeof(T) == 4) {
    const float4* s4 = reinterpret_cast<const float4*>(src);
    float tmp[4 * ((N + 3) / 4)];
#pragma unroll
    for (int v = 0; v < (N + 3) / 4; ++v) {
      const float4 x = s4[v];
      tmp[4 * v] = x.x, tmp[4 * v + 1] = x.y, tmp[4 * v + 2] = x.z, tmp[4 * v + 3] = x.w;
    }
#pragma unroll
    for (int v = 0; v < N; ++v) dst[v] = tmp[v];
  } else {
    const double2* s2 = reinterpret_cast<const double2*>(src);
#pragma unroll
    for (int v = 0; v < (N + 1) / 2; ++v) {
      const double2 x = s2[v];
      dst[2 * v] = x.x;
      if (2 * v + 1 < N) dst[2 * v + 1] = x.y;
    }
  }
}

// Resident blocks per SM the register budget is held to: shared memory allows
// about 3 (FP32 records) and 2 (FP64 records) for the Neo-Hookean law.
template <int VEC, int LAW, typename T, bool WANT_K>
__global__ void __launch_bounds__(kAsmThreads, sizeof(T) == 4 ? 3 : 2) assemble_kernel(const AsmArgs A) {
  using R = Rec<LAW, T>;
  using N = NodeRec<VEC>;
  constexpr int NCV = 3 * LawTraits<LAW>::NV;
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* ws = smem + size_t(warp) * warp_smem_bytes<VEC, LAW, T>();
  T* srec = reinterpret_cast<T*>(ws);
  double* snode = reinterpret_cast<double*>(srec + kGroupCells * 8 * R::SIZE);
  double* slift = snode + kGroupCells * 8 * N::NF;
  int* sbits = reinterpret_cast<int*>(slift + kGroupCells * 8 * VEC);
  int* sid = sbits + kGroupCells * 8;
  T* vals = reinterpret_cast<T*>(A.vals);
  const bool want_k = WANT_K && (A.vals != nullptr || A.lift != nullptr);

  const int64_t groups = (A.num_cells + kGroupCells - 1) / kGroupCells;
  const int64_t wstride = int64_t(gridDim.x) * kAsmWarps;
  for (int64_t grp = int64_t(blockIdx.x) * kAsmWarps + warp; grp < groups; grp += wstride) {
    const int64_t c0 = grp * kGroupCells;
    // ---- phase 0: lane = (cell cl, node t) ----
    {
      const int cl = lane >> 3, t = lane & 7;
      const int64_t c = c0 + cl;
      const bool valid = c < A.num_cells;
      const int node = valid ? A.cells[c * 8 + t] : 0;
      double* nd = snode + lane * N::NF;
      if (valid) {
        nd[N::X + 0] = A.points[int64_t(node) * 3 + 0];
        nd[N::X + 1] = A.points[int64_t(node) * 3 + 1];
        nd[N::X + 2] = A.points[int64_t(node) * 3 + 2];
      } else {  // unit cube keeps the tail math finite; its outputs are dropped
        nd[N::X + 0] = vtk_xbit(t);
        nd[N::X + 1] = vtk_ybit(t);
        nd[N::X + 2] = vtk_zbit(t);
      }
      int bits = 0;
#pragma unroll
      for (int i = 0; i < VEC; ++i) {
        const int64_t dof = int64_t(node) * VEC + i;
        nd[N::U + i] = valid ? A.u[dof] : 0.0;
        const double d = (valid && A.dvec != nullptr) ? A.dvec[dof] : 0.0;
        nd[N::D + i] = d;
        if (valid && A.bc != nullptr && A.bc[dof]) bits |= 1 << i;
        if (d != 0.0) bits |= kLiftBit;
        slift[lane * VEC + i] = 0.0;
      }
      sbits[lane] = bits;
      sid[lane] = node;
    }
    __syncwarp();
    // ---- phase 1: lane = (cell cl, quadrature point q) ----
    {
      const int cl = lane >> 3, q = lane & 7;
      const int64_t c = c0 + cl;
      const bool valid = c < A.num_cells;
      const double* nb = snode + cl * 8 * N::NF;
      double X[8][3], g[8][3];
#pragma unroll
      for (int b = 0; b < 8; ++b)
#pragma unroll
        for (int i = 0; i < 3; ++i) X[b][i] = nb[b * N::NF + N::X + i];
      double jxw;
      hex8_geometry(q, X, g, &jxw);
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
      double P[VEC * 3];
      law_quad<VEC, LAW, T>(A, valid ? c : c0, q, ug, g, jxw, srec + lane * R::SIZE, P);
      if (A.res != nullptr) {
        // r_b = P g_b for the 8 nodes, summed over the cell's 8 lanes: round
        // r keeps the half of the nodes selected by bit (2 - r) of q.
        double r[8 * VEC];
#pragma unroll
        for (int b = 0; b < 8; ++b)
#pragma unroll
          for (int i = 0; i < VEC; ++i)
            r[b * VEC + i] = P[i * 3] * g[b][0] + P[i * 3 + 1] * g[b][1] + P[i * 3 + 2] * g[b][2];
        const bool h4 = q & 4, h2 = q & 2, h1 = q & 1;
#pragma unroll
        for (int v = 0; v < 4 * VEC; ++v) {
          const double send = h4 ? r[v] : r[4 * VEC + v];
          const double keep = h4 ? r[4 * VEC + v] : r[v];
          r[v] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
        }
#pragma unroll
        for (int v = 0; v < 2 * VEC; ++v) {
          const double send = h2 ? r[v] : r[2 * VEC + v];
          const double keep = h2 ? r[2 * VEC + v] : r[v];
          r[v] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
        }
#pragma unroll
        for (int v = 0; v < VEC; ++v) {
          const double send = h1 ? r[v] : r[VEC + v];
          const double keep = h1 ? r[VEC + v] : r[v];
          r[v] = keep + __shfl_xor_sync(0xffffffffu, send, 1);
        }
        if (valid) {
          const int64_t node = sid[lane];  // lane (cl, q) now holds node q of cell cl
#pragma unroll
          for (int i = 0; i < VEC; ++i) atomicAdd(A.res + node * VEC + i, r[i]);
        }
      }
    }
    __syncwarp();
    if (!want_k) continue;
    // ---- phase 2: lane = row (node a, component i) ----
    constexpr int ROWS = 8 * VEC;                    // rows per cell
    constexpr int CPP = VEC == 1 ? kGroupCells : 1;  // cells per pass
    for (int pass = 0; pass < kGroupCells / CPP; ++pass) {
      const int cl = VEC == 1 ? (lane >> 3) : pass;
      const int rl = VEC == 1 ? (lane & 7) : lane;
      const int64_t c = c0 + cl;
      const bool active = rl < ROWS && c < A.num_cells;
      const int a = rl / VEC, i = rl - (rl / VEC) * VEC;
      const T* rec0 = srec + (cl * 8) * R::SIZE;
      const int nblk = a < 4 ? 5 : 4;
      T K[5][3];
      T Kd[5];
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        Kd[j] = T(0);
#pragma unroll
        for (int k = 0; k < 3; ++k) K[j][k] = T(0);
      }
      if (active) {
#pragma unroll 1
        for (int q = 0; q < 8; ++q) {
          const T* rec = rec0 + q * R::SIZE;
          const T cf[4] = {rec[0], rec[1], rec[2], rec[3]};
          T na[NCV], ar[8];
          load_row<LAW, T>(rec + 4 + a * R::NS, na);
          own_row<LAW, T>(na, cf, i, ar);
#pragma unroll
          for (int j = 0; j < 5; ++j) {
            if (j < nblk) {
              const int b = (a + j) & 7;
              T br[NCV];
              load_row<LAW, T>(rec + 4 + b * R::NS, br);
              Kd[j] += pair_row<LAW, T>(ar, br, cf, i, K[j]);
            }
          }
        }
      }
      // the (g_a . g_b) I term on the row's own component
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        if constexpr (VEC == 1) {
          K[j][0] += Kd[j];
        } else {
          K[j][0] += i == 0 ? Kd[j] : T(0);
          K[j][1] += i == 1 ? Kd[j] : T(0);
          K[j][2] += i == 2 ? Kd[j] : T(0);
        }
      }
      const int ca = cl * 8;  // the cell's first node slot
      const bool lift_cell =
          A.lift != nullptr && (__reduce_or_sync(0xffffffffu, active ? (sbits[ca + a] & kLiftBit) : 0) != 0);
      if (active) {
        const int abits = sbits[ca + a];
        const int na_id = sid[ca + a];
        const bool arow_bc = (abits >> i) & 1;
        double lrow = 0.0;
#pragma unroll
        for (int j = 0; j < 5; ++j) {
          if (j >= nblk) continue;
          const int b = (a + j) & 7;
          const int bbits = sbits[ca + b];
          if (lift_cell) {
            // row (a, i): K_ab[i][:] d_b; row (b, k): K_ab[i][k] d_a[i]
            const double* db = snode + (ca + b) * N::NF + N::D;
            if (bbits & kLiftBit)
#pragma unroll
              for (int k = 0; k < VEC; ++k) lrow += double(K[j][k]) * db[k];
            if (b != a && (abits & kLiftBit)) {
              const double dai = snode[(ca + a) * N::NF + N::D + i];
#pragma unroll
              for (int k = 0; k < VEC; ++k) atomicAdd(slift + (ca + b) * VEC + k, double(K[j][k]) * dai);
            }
          }
          if (vals != nullptr && !arow_bc) {
            const int nb_id = sid[ca + b];
            const int* smap = A.scatter + c * 64;
            if (a == b || na_id < nb_id) {
              T* blk = vals + int64_t(smap[a * 8 + b]) * (VEC * VEC) + i * VEC;
#pragma unroll
              for (int k = 0; k < VEC; ++k)
                if (!((bbits >> k) & 1)) atomicAdd(blk + k, K[j][k]);
            } else {
              T* blk = vals + int64_t(smap[b * 8 + a]) * (VEC * VEC) + i;
#pragma unroll
              for (int k = 0; k < VEC; ++k)
                if (!((bbits >> k) & 1)) atomicAdd(blk + k * VEC, K[j][k]);
            }
          }
        }
        if (lift_cell) atomicAdd(slift + (ca + a) * VEC + i, lrow);
      }
      if (lift_cell) {
        __syncwarp();
        if (active && !((sbits[ca + a] >> i) & 1))
          atomicAdd(A.lift + int64_t(sid[ca + a]) * VEC + i, slift[(ca + a) * VEC + i]);
      }
    }
    __syncwarp();
  }
}

template <int VEC, int LAW, typename T, bool WANT_K>
int launch_variant(const AsmArgs& A, cudaStream_t st) {
  auto k = assemble_kernel<VEC, LAW, T, WANT_K>;
  const size_t sm = size_t(kAsmWarps) * warp_smem_bytes<VEC, LAW, T>();
  static int blocks_per_sm = 0;
  if (blocks_per_sm == 0) {
    FEM_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    FEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k, kAsmThreads, sm));
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  const int64_t groups = (A.num_cells + kGroupCells - 1) / kGroupCells;
  const int64_t need = (groups + kAsmWarps - 1) / kAsmWarps;
  const int64_t cap = int64_t(num_sms()) * blocks_per_sm;
  const unsigned grid = unsigned(need < cap ? need : cap);
  k<<<grid, kAsmThreads, sm, st>>>(A);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}

template <int VEC, int LAW, typename T>
int launch_law(const AsmArgs& A, bool want_k, cudaStream_t st) {
  return want_k ? launch_variant<VEC, LAW, T, true>(A, st) : launch_variant<VEC, LAW, T, false>(A, st);
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
