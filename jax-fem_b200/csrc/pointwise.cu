// Quadrature-point kernels outside assembly: the J2 state commit and the
// adjoint parameter VJP.  One thread per (cell, quadrature point); the 8
// threads of a cell stage its node data in shared memory once.
#include "common.cuh"

namespace fem {
namespace {

constexpr int kCellsPB = 16;

// Stage coords and up to two nodal vectors of the cell, then compute the
// physical gradients at quadrature point q = threadIdx.x & 7.
struct CellQuad {
  double g[8][3];
  double jxw;
};

__device__ __forceinline__ void load_cell(int64_t c, bool valid, const int32_t* cells,
                                          const double* points, const double* v0, const double* v1,
                                          double (*s)[8][9]) {
  const int cl = threadIdx.x >> 3, t = threadIdx.x & 7;
  const int node = valid ? cells[c * 8 + t] : 0;
  double* d = s[cl][t];
  for (int i = 0; i < 3; ++i) {
    d[i] = valid ? points[int64_t(node) * 3 + i] : double((i == 0) ? vtk_xbit(t) : (i == 1) ? vtk_ybit(t) : vtk_zbit(t));
    d[3 + i] = (valid && v0) ? v0[int64_t(node) * 3 + i] : 0.0;
    d[6 + i] = (valid && v1) ? v1[int64_t(node) * 3 + i] : 0.0;
  }
}

__device__ __forceinline__ void quad_grads(const double (*cellnodes)[9], int q, double g[8][3],
                                           double* jxw, double gu[3][3], double gl[3][3]) {
  double X[8][3];
#pragma unroll
  for (int b = 0; b < 8; ++b)
#pragma unroll
    for (int i = 0; i < 3; ++i) X[b][i] = cellnodes[b][i];
  hex8_geometry(q, X, g, jxw);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double su = 0.0, sl = 0.0;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        su = fma(cellnodes[b][3 + i], g[b][j], su);
        sl = fma(cellnodes[b][6 + i], g[b][j], sl);
      }
      gu[i][j] = su;
      gl[i][j] = sl;
    }
}

__global__ void __launch_bounds__(128) j2_commit_kernel(int64_t C, const int32_t* cells,
                                                        const double* points, const double* u,
                                                        double E, double nu, double sy0, double Hh,
                                                        const double* so, const double* eo,
                                                        const double* ao, double* sn, double* en,
                                                        double* an) {
  __shared__ double s[kCellsPB][8][9];
  const int cl = threadIdx.x >> 3, q = threadIdx.x & 7;
  const int64_t c = int64_t(blockIdx.x) * kCellsPB + cl;
  const bool valid = c < C;
  load_cell(c, valid, cells, points, u, nullptr, s);
  __syncwarp();
  if (!valid) return;
  double g[8][3], jxw, gu[3][3], gl[3][3];
  quad_grads(s[cl], q, g, &jxw, gu, gl);
  const double mu = E / (2.0 * (1.0 + nu));
  const double lm = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  const int64_t k = c * 8 + q;
  double eps[3][3], de[3][3], st[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      eps[i][j] = 0.5 * (gu[i][j] + gu[j][i]);
      de[i][j] = eps[i][j] - eo[k * 9 + i * 3 + j];
    }
  const double trd = de[0][0] + de[1][1] + de[2][2];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) st[i][j] = 2.0 * mu * de[i][j] + (i == j ? lm * trd : 0.0) + so[k * 9 + i * 3 + j];
  const double tr3 = (st[0][0] + st[1][1] + st[2][2]) / 3.0;
  double sdev[3][3], ss = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      sdev[i][j] = st[i][j] - (i == j ? tr3 : 0.0);
      ss += sdev[i][j] * sdev[i][j];
    }
  const double qv = ss > 0.0 ? sqrt(1.5 * ss) : 0.0;
  const double alpha = ao[k];
  const double f = qv - (sy0 + Hh * alpha);
  double beta = 0.0, dg = 0.0;
  if (f > 0.0) {
    dg = f / (3.0 * mu + Hh);
    beta = 3.0 * mu * dg / qv;
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      sn[k * 9 + i * 3 + j] = st[i][j] - beta * sdev[i][j];
      en[k * 9 + i * 3 + j] = eps[i][j];
    }
  an[k] = alpha + dg;
}

// grad[c,q] = -(dP/dtheta : grad lambda) JxW at (c,q).
__global__ void __launch_bounds__(128) param_vjp_kernel(int law, int64_t C, const int32_t* cells,
                                                        const double* points, const double* u,
                                                        const double* lam, const double* theta,
                                                        double p0, double p1, double p2, double p3,
                                                        double* grad) {
  __shared__ double s[kCellsPB][8][9];
  const int cl = threadIdx.x >> 3, q = threadIdx.x & 7;
  const int64_t c = int64_t(blockIdx.x) * kCellsPB + cl;
  const bool valid = c < C;
  load_cell(c, valid, cells, points, u, lam, s);
  __syncwarp();
  if (!valid) return;
  double g[8][3], jxw, gu[3][3], gl[3][3];
  quad_grads(s[cl], q, g, &jxw, gu, gl);
  const int64_t k = c * 8 + q;
  double dP[3][3];
  if (law == FEM_LAW_SIMP) {
    // P = E(theta) Phat, Phat the unit-modulus stress; dE/dtheta = (E0-Emin) p theta^(p-1)
    const double E0 = p0, Emin = p1, nu = p2, pen = p3;
    const double th = theta[k];
    const double dE = (E0 - Emin) * pen * pow(th, pen - 1.0);
    const double mu = 1.0 / (2.0 * (1.0 + nu));
    const double lm = nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double tr = gu[0][0] + gu[1][1] + gu[2][2];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        dP[i][j] = dE * (mu * (gu[i][j] + gu[j][i]) + (i == j ? lm * tr : 0.0));
  } else {
    // Neo-Hookean psi scale: dP/ds = P of the unscaled law
    const double E = p0, nu = p1;
    const double mu = E / (2.0 * (1.0 + nu));
    const double kappa = E / (3.0 * (1.0 - 2.0 * nu));
    double F[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) F[i][j] = gu[i][j] + (i == j ? 1.0 : 0.0);
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
    double I1 = 0.0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) I1 += F[i][j] * F[i][j];
    const double cb = cbrt(J);
    const double m = mu / (cb * cb);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        const double H = cof[i][j] / J;
        dP[i][j] = m * (F[i][j] - I1 * H / 3.0) + kappa * J * (J - 1.0) * H;
      }
  }
  double acc = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) acc = fma(dP[i][j], gl[i][j], acc);
  grad[k] = -acc * jxw;
}

}  // namespace
}  // namespace fem

using namespace fem;

extern "C" int fem_j2_commit(const double* h_params, int n_params, int64_t num_cells,
                             const int32_t* d_cells, const double* d_points, const double* d_u,
                             const double* d_sigma_old, const double* d_eps_old,
                             const double* d_alpha_old, double* d_sigma_new, double* d_eps_new,
                             double* d_alpha_new, void* stream) {
  FEM_CHECK_ARG(h_params != nullptr && n_params >= 4, "J2 needs E, nu, sigma_y, H");
  FEM_CHECK_ARG(num_cells >= 0, "negative size");
  FEM_CHECK_ARG(d_sigma_old && d_eps_old && d_alpha_old && d_sigma_new && d_eps_new && d_alpha_new,
                "J2 state pointer is NULL");
  if (num_cells == 0) return FEM_OK;
  j2_commit_kernel<<<unsigned((num_cells + kCellsPB - 1) / kCellsPB), 128, 0, as_stream(stream)>>>(
      num_cells, d_cells, d_points, d_u, h_params[0], h_params[1], h_params[2], h_params[3],
      d_sigma_old, d_eps_old, d_alpha_old, d_sigma_new, d_eps_new, d_alpha_new);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}

extern "C" int fem_param_vjp_f64(int law, const double* h_params, int n_params, int64_t num_cells,
                                 const int32_t* d_cells, const double* d_points, const double* d_u,
                                 const double* d_ivar0, const double* d_lambda, double* d_grad,
                                 void* stream) {
  FEM_CHECK_ARG(law == FEM_LAW_SIMP || law == FEM_LAW_NEO_HOOKEAN,
                "parameter VJP is defined for SIMP (theta) and NEO_HOOKEAN (scale), got law %d", law);
  FEM_CHECK_ARG(h_params != nullptr && n_params >= (law == FEM_LAW_SIMP ? 4 : 2), "missing params");
  FEM_CHECK_ARG(law != FEM_LAW_SIMP || d_ivar0 != nullptr, "SIMP VJP needs theta");
  FEM_CHECK_ARG(num_cells >= 0, "negative size");
  if (num_cells == 0) return FEM_OK;
  const double p2 = n_params > 2 ? h_params[2] : 0.0, p3 = n_params > 3 ? h_params[3] : 0.0;
  param_vjp_kernel<<<unsigned((num_cells + kCellsPB - 1) / kCellsPB), 128, 0, as_stream(stream)>>>(
      law, num_cells, d_cells, d_points, d_u, d_lambda, d_ivar0, h_params[0], h_params[1], p2, p3,
      d_grad);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}
