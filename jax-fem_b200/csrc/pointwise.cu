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

// Derivative of the J2 return map (the commit above) with respect to the
// initial yield stress sigma_y, given the derivatives of its inputs: u' (the
// nodal displacement sensitivity; null = 0, which gives the explicit part
// used as the right-hand side of the sensitivity solve) and the committed
// state's sensitivities sigma_old', eps_old', alpha_old' (null = 0, the first
// increment).  Writes sigma', eps' = sym grad u' (if den) and alpha'.
//   trial:   sigma_tr' = sigma_old' + C : (eps(u') - eps_old'),  s' = dev sigma_tr'
//   elastic: sigma' = sigma_tr',  alpha' = alpha_old'
//   plastic: q' = 3/2 (s : s') / q,  f' = q' - 1 - H alpha_old',
//            dgamma' = f' / (3 mu + H),  beta' = 3 mu (dgamma' q - dgamma q') / q^2,
//            sigma' = sigma_tr' - beta' s - beta s',  alpha' = alpha_old' + dgamma'
__global__ void __launch_bounds__(128) j2_sens_kernel(int64_t C, const int32_t* cells,
                                                      const double* points, const double* u,
                                                      const double* du, double E, double nu,
                                                      double sy0, double Hh, const double* so,
                                                      const double* eo, const double* ao,
                                                      const double* dso, const double* deo,
                                                      const double* dao, double* dsn, double* den,
                                                      double* dan) {
  __shared__ double s[kCellsPB][8][9];
  const int cl = threadIdx.x >> 3, q = threadIdx.x & 7;
  const int64_t c = int64_t(blockIdx.x) * kCellsPB + cl;
  const bool valid = c < C;
  load_cell(c, valid, cells, points, u, du, s);
  __syncwarp();
  if (!valid) return;
  double g[8][3], jxw, gu[3][3], gd[3][3];
  quad_grads(s[cl], q, g, &jxw, gu, gd);
  const double mu = E / (2.0 * (1.0 + nu));
  const double lm = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  const int64_t k = c * 8 + q;
  double de[3][3], dde[3][3], deps[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      de[i][j] = 0.5 * (gu[i][j] + gu[j][i]) - eo[k * 9 + i * 3 + j];
      deps[i][j] = 0.5 * (gd[i][j] + gd[j][i]);
      dde[i][j] = deps[i][j] - (deo ? deo[k * 9 + i * 3 + j] : 0.0);
    }
  const double trd = de[0][0] + de[1][1] + de[2][2];
  const double trdd = dde[0][0] + dde[1][1] + dde[2][2];
  double st[3][3], dst[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      st[i][j] = 2.0 * mu * de[i][j] + (i == j ? lm * trd : 0.0) + so[k * 9 + i * 3 + j];
      dst[i][j] = 2.0 * mu * dde[i][j] + (i == j ? lm * trdd : 0.0) + (dso ? dso[k * 9 + i * 3 + j] : 0.0);
    }
  const double tr3 = (st[0][0] + st[1][1] + st[2][2]) / 3.0;
  const double dtr3 = (dst[0][0] + dst[1][1] + dst[2][2]) / 3.0;
  double sd[3][3], dsd[3][3], ss = 0.0, sds = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      sd[i][j] = st[i][j] - (i == j ? tr3 : 0.0);
      dsd[i][j] = dst[i][j] - (i == j ? dtr3 : 0.0);
      ss += sd[i][j] * sd[i][j];
      sds += sd[i][j] * dsd[i][j];
    }
  const double qv = ss > 0.0 ? sqrt(1.5 * ss) : 0.0;
  const double dalpha_old = dao ? dao[k] : 0.0;
  const double f = qv - (sy0 + Hh * ao[k]);
  double beta = 0.0, dbeta = 0.0, ddg = 0.0;
  if (f > 0.0) {
    const double dg = f / (3.0 * mu + Hh);
    const double dq = 1.5 * sds / qv;
    const double df = dq - 1.0 - Hh * dalpha_old;
    ddg = df / (3.0 * mu + Hh);
    beta = 3.0 * mu * dg / qv;
    dbeta = 3.0 * mu * (ddg * qv - dg * dq) / (qv * qv);
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      dsn[k * 9 + i * 3 + j] = dst[i][j] - dbeta * sd[i][j] - beta * dsd[i][j];
      if (den) den[k * 9 + i * 3 + j] = deps[i][j];
    }
  dan[k] = dalpha_old + ddg;
}

// out[node, i] += sum_q sum_j stress[c,q,i,j] dN_node/dx_j JxW  (the internal
// force of a given quadrature-point stress field, problem.py:189-214 with P
// supplied).  The 8 quadrature threads of a cell sum by warp shuffles; lane t
// then adds node t's three components.
__global__ void __launch_bounds__(128) stress_div_kernel(int64_t C, const int32_t* cells,
                                                         const double* points, const double* stress,
                                                         double* out) {
  __shared__ double s[kCellsPB][8][9];
  const int cl = threadIdx.x >> 3, q = threadIdx.x & 7;
  const int64_t c = int64_t(blockIdx.x) * kCellsPB + cl;
  const bool valid = c < C;
  load_cell(c, valid, cells, points, nullptr, nullptr, s);
  __syncwarp();
  double g[8][3], jxw = 0.0, gu[3][3], gl[3][3];
  if (valid) quad_grads(s[cl], q, g, &jxw, gu, gl);
  double sig[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) sig[i][j] = valid ? stress[(c * 8 + q) * 9 + i * 3 + j] : 0.0;
  double mine[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int b = 0; b < 8; ++b) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      double v = valid ? (sig[i][0] * g[b][0] + sig[i][1] * g[b][1] + sig[i][2] * g[b][2]) * jxw : 0.0;
      v += __shfl_xor_sync(0xffffffffu, v, 1);
      v += __shfl_xor_sync(0xffffffffu, v, 2);
      v += __shfl_xor_sync(0xffffffffu, v, 4);
      if (q == b) mine[i] = v;
    }
  }
  if (!valid) return;
  const int64_t node = cells[c * 8 + q];
  for (int i = 0; i < 3; ++i) atomicAdd(out + node * 3 + i, mine[i]);
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

extern "C" int fem_j2_sensitivity(const double* h_params, int n_params, int64_t num_cells,
                                  const int32_t* d_cells, const double* d_points, const double* d_u,
                                  const double* d_du, const double* d_sigma_old,
                                  const double* d_eps_old, const double* d_alpha_old,
                                  const double* d_dsigma_old, const double* d_deps_old,
                                  const double* d_dalpha_old, double* d_dsigma, double* d_deps,
                                  double* d_dalpha, void* stream) {
  FEM_CHECK_ARG(h_params != nullptr && n_params >= 4, "J2 needs E, nu, sigma_y, H");
  FEM_CHECK_ARG(num_cells >= 0, "negative size");
  FEM_CHECK_ARG(d_u && d_sigma_old && d_eps_old && d_alpha_old && d_dsigma && d_dalpha,
                "J2 sensitivity: state or output pointer is NULL");
  if (num_cells == 0) return FEM_OK;
  j2_sens_kernel<<<unsigned((num_cells + kCellsPB - 1) / kCellsPB), 128, 0, as_stream(stream)>>>(
      num_cells, d_cells, d_points, d_u, d_du, h_params[0], h_params[1], h_params[2], h_params[3],
      d_sigma_old, d_eps_old, d_alpha_old, d_dsigma_old, d_deps_old, d_dalpha_old, d_dsigma, d_deps,
      d_dalpha);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}

extern "C" int fem_stress_divergence(int64_t num_cells, const int32_t* d_cells, const double* d_points,
                                     const double* d_stress, double* d_out, void* stream) {
  FEM_CHECK_ARG(num_cells >= 0, "negative size");
  FEM_CHECK_ARG(d_cells && d_points && d_stress && d_out, "stress divergence: NULL pointer");
  if (num_cells == 0) return FEM_OK;
  stress_div_kernel<<<unsigned((num_cells + kCellsPB - 1) / kCellsPB), 128, 0, as_stream(stream)>>>(
      num_cells, d_cells, d_points, d_stress, d_out);
  FEM_LAUNCH_CHECK();
  return FEM_OK;
}
