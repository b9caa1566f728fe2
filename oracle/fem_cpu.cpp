// CPU restatement of the reference's HEX8 assemble-and-solve path, in C++
// with OpenMP.  TEST INFRASTRUCTURE: the timed CPU baseline of bench.py
// (``--impl reference`` and the ``cpu_baseline`` leg); the product never
// links, loads or calls it.
//
// It restates, for structured HEX8 boxes, what one Newton solve of the
// reference does on its CPU path (jax_fem/solver.py, problem.py, fe.py):
//
//  * setup (outside the timed solve, as in the reference): box_mesh numbering
//    (generate_mesh.py:151-189), physical shape gradients and JxW per
//    (cell, quadrature point) stored once (fe.py:112-141,
//    problem.py:130-151), the COO pattern of every cell's 24 x 24 block and
//    its summation map into CSR (problem.py:94-107; PETSc
//    setPreallocationCOO, solver.py:466-478);
//  * per Newton iteration: the cell residuals and their Jacobians by
//    forward-mode differentiation along the 24 cell dofs (the reference's
//    value_and_jacfwd of the laplace kernel, problem.py:189-214,262-266,
//    334-338), here as one pass of 24-component dual numbers; the residual
//    scatter (problem.py:426-437); the COO sum into CSR and zeroRows on the
//    Dirichlet rows, diagonal 1, columns kept (solver.py:480-491); the
//    Dirichlet rows of the residual set to u - u_D (solver.py:290-304);
//  * the linear solve: BiCGSTAB with the Jacobi preconditioner x / diag(A),
//    stopping when the recursive residual satisfies
//    ||r|| <= max(tol ||b||, atol), tol = atol = 1e-10, maxiter 10000, from
//    x0 = u_D - u on Dirichlet rows and 0 elsewhere (jax_solve,
//    solver.py:63-92, and its x0, solver.py:400-409; the iteration is
//    jax.scipy.sparse.linalg.bicgstab's right-preconditioned van der Vorst
//    recurrence with its early exit on s), or CG with the Jacobi
//    preconditioner and PETSc's test, the preconditioned residual norm below
//    rtol times its initial value (petsc_solve, solver.py:108-133, with
//    -ksp_rtol; see cg_jacobi for its initial guess);
//  * the Newton loop: stop when ||R||/||R0|| <= rel_tol or ||R|| <= tol
//    (solver.py:1232-1318).
//
// Laws: linear elasticity, sigma = lambda tr(eps) I + 2 mu eps
// (tests/benchmarks/linear_elasticity_cube/test_linear_elasticity_cube.py:
// 16-25) and the compressible Neo-Hookean first Piola stress, the gradient
// of psi = mu/2 (J^-2/3 I1 - 3) + kappa/2 (J - 1)^2
// (applications/scalability/hyperelastic3d_common.py:18-35), written here in
// closed form: P = mu J^-2/3 (F - I1/3 F^-T) + kappa (J - 1) J F^-T.
//
// Reductions are OpenMP reductions: their summation order, and so the last
// bits of a dot product and the Krylov iteration count, may vary from run to
// run.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr int ND = 24;  // dofs of a HEX8 cell with vec = 3

// Forward-mode number: a value and its derivatives along the 24 cell dofs.
struct Dual {
  double v;
  double d[ND];
};

inline Dual dconst(double c) {
  Dual r;
  r.v = c;
  for (int k = 0; k < ND; ++k) r.d[k] = 0.0;
  return r;
}
inline Dual operator+(const Dual& a, const Dual& b) {
  Dual r;
  r.v = a.v + b.v;
  for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
inline Dual operator-(const Dual& a, const Dual& b) {
  Dual r;
  r.v = a.v - b.v;
  for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
inline Dual operator*(const Dual& a, const Dual& b) {
  Dual r;
  r.v = a.v * b.v;
  for (int k = 0; k < ND; ++k) r.d[k] = a.v * b.d[k] + b.v * a.d[k];
  return r;
}
inline Dual operator*(double s, const Dual& a) {
  Dual r;
  r.v = s * a.v;
  for (int k = 0; k < ND; ++k) r.d[k] = s * a.d[k];
  return r;
}
inline Dual operator*(const Dual& a, double s) { return s * a; }
inline Dual operator+(const Dual& a, double s) {
  Dual r = a;
  r.v += s;
  return r;
}
inline Dual operator-(const Dual& a, double s) {
  Dual r = a;
  r.v -= s;
  return r;
}
inline Dual inv(const Dual& a) {  // 1 / a
  Dual r;
  r.v = 1.0 / a.v;
  const double g = -r.v * r.v;
  for (int k = 0; k < ND; ++k) r.d[k] = g * a.d[k];
  return r;
}
inline Dual powd(const Dual& a, double e) {  // a^e, a > 0
  Dual r;
  r.v = std::pow(a.v, e);
  const double g = e * r.v / a.v;
  for (int k = 0; k < ND; ++k) r.d[k] = g * a.d[k];
  return r;
}
inline double val(double a) { return a; }
inline double val(const Dual& a) { return a.v; }
inline double inv(double a) { return 1.0 / a; }
inline double powd(double a, double e) { return std::pow(a, e); }
template <class T>
inline T cst(double c);
template <>
inline double cst<double>(double c) {
  return c;
}
template <>
inline Dual cst<Dual>(double c) {
  return dconst(c);
}

enum Law { LAW_LINEAR = 0, LAW_NEO_HOOKEAN = 1 };

// First Piola stress (or Cauchy stress of linear elasticity) of u_grad.
template <class T>
void stress(int law, double mu, double lam_or_kappa, const T ug[3][3], T P[3][3]) {
  if (law == LAW_LINEAR) {
    const double lam = lam_or_kappa;
    T tr = ug[0][0] + ug[1][1] + ug[2][2];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        P[i][j] = mu * (ug[i][j] + ug[j][i]);
        if (i == j) P[i][j] = P[i][j] + lam * tr;
      }
    return;
  }
  const double kappa = lam_or_kappa;
  T F[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) F[i][j] = (i == j) ? ug[i][j] + 1.0 : ug[i][j];
  // cofactor matrix: cof = J F^-T
  T C[3][3];
  C[0][0] = F[1][1] * F[2][2] - F[1][2] * F[2][1];
  C[0][1] = F[1][2] * F[2][0] - F[1][0] * F[2][2];
  C[0][2] = F[1][0] * F[2][1] - F[1][1] * F[2][0];
  C[1][0] = F[0][2] * F[2][1] - F[0][1] * F[2][2];
  C[1][1] = F[0][0] * F[2][2] - F[0][2] * F[2][0];
  C[1][2] = F[0][1] * F[2][0] - F[0][0] * F[2][1];
  C[2][0] = F[0][1] * F[1][2] - F[0][2] * F[1][1];
  C[2][1] = F[0][2] * F[1][0] - F[0][0] * F[1][2];
  C[2][2] = F[0][0] * F[1][1] - F[0][1] * F[1][0];
  T J = F[0][0] * C[0][0] + F[0][1] * C[0][1] + F[0][2] * C[0][2];
  T I1 = cst<T>(0.0);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) I1 = I1 + F[i][j] * F[i][j];
  T Jm23 = powd(J, -2.0 / 3.0);
  T Jinv = inv(J);
  T a = mu * Jm23;                                  // mu J^-2/3
  T b = (a * I1) * (1.0 / 3.0);                     // mu J^-2/3 I1 / 3
  T c = kappa * (J - 1.0);                          // kappa (J - 1): coefficient of cof
  T bc = b * Jinv;                                  // F^-T = cof / J
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) P[i][j] = a * F[i][j] + (c - bc) * C[i][j];
}

// The reference's laplace kernel for one cell: r[a*3+i] = sum_q sum_j
// P_q[i][j] dN_a/dx_j JxW_q, with u_grad = sum_a u_a (x) grad N_a.
template <class T>
void cell_residual(int law, double mu, double lk, const double* sg /* 8 x 8 x 3 */, const double* jxw /* 8 */,
                   const T* ue, T* re) {
  for (int r = 0; r < ND; ++r) re[r] = cst<T>(0.0);
  for (int q = 0; q < 8; ++q) {
    const double* g = sg + q * 24;
    T ug[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) ug[i][j] = cst<T>(0.0);
    for (int a = 0; a < 8; ++a)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) ug[i][j] = ug[i][j] + g[a * 3 + j] * ue[a * 3 + i];
    T P[3][3];
    stress<T>(law, mu, lk, ug, P);
    const double w = jxw[q];
    for (int a = 0; a < 8; ++a)
      for (int i = 0; i < 3; ++i) {
        T s = P[i][0] * (g[a * 3 + 0] * w) + P[i][1] * (g[a * 3 + 1] * w);
        s = s + P[i][2] * (g[a * 3 + 2] * w);
        re[a * 3 + i] = re[a * 3 + i] + s;
      }
  }
}

struct Problem {
  int nx, ny, nz, law, nthreads;
  double mu, lk;
  int64_t n_nodes, n_cells, ndofs, nnz;
  std::vector<int32_t> cells;   // (C, 8), VTK order
  std::vector<double> sg, jxw;  // (C, 8, 8, 3), (C, 8)
  std::vector<int64_t> row_ptr;
  std::vector<int32_t> col, diag;
  std::vector<int64_t> jmap;    // (nnz + 1): COO entries summed into each CSR entry
  std::vector<int32_t> perm;    // (C * 576): COO entry index, grouped by CSR entry
  std::vector<double> V;        // (C, 24, 24): cell Jacobians (the reference's problem.V)
  std::vector<double> vals;     // CSR values
  std::vector<double> res;      // global residual
  std::vector<int64_t> bc_dofs;
  std::vector<double> bc_vals;
  // statistics of the last solve
  int newton = 0, krylov = 0;
  double t_assembly = 0.0, t_linear = 0.0;
};

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// HEX8 reference gradients at the 2x2x2 Gauss points of [0,1]^3, VTK node order.
void hex8_ref_grads(double G[8][8][3], double W[8]) {
  const double g0 = 0.5 - 0.5 / std::sqrt(3.0), g1 = 0.5 + 0.5 / std::sqrt(3.0);
  const double gp[2] = {g0, g1};
  const int vx[8] = {0, 1, 1, 0, 0, 1, 1, 0}, vy[8] = {0, 0, 1, 1, 0, 0, 1, 1}, vz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
  int q = 0;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j)
      for (int k = 0; k < 2; ++k, ++q) {
        const double xi[3] = {gp[i], gp[j], gp[k]};
        W[q] = 0.125;
        for (int a = 0; a < 8; ++a) {
          const int v[3] = {vx[a], vy[a], vz[a]};
          double f[3], df[3];
          for (int d = 0; d < 3; ++d) {
            f[d] = v[d] ? xi[d] : 1.0 - xi[d];
            df[d] = v[d] ? 1.0 : -1.0;
          }
          G[q][a][0] = df[0] * f[1] * f[2];
          G[q][a][1] = f[0] * df[1] * f[2];
          G[q][a][2] = f[0] * f[1] * df[2];
        }
      }
}

}  // namespace

extern "C" {

// Setup of an nx x ny x nz HEX8 box of size Lx x Ly x Lz (box_mesh
// numbering), law 0 (linear) / 1 (Neo-Hookean) with Young's modulus E and
// Poisson ratio nu, on nthreads OpenMP threads (<= 0: the default).
// Returns a handle, or nullptr.
void* fcpu_create(int nx, int ny, int nz, double Lx, double Ly, double Lz, int law, double E, double nu,
                  int nthreads) {
  if (nx < 1 || ny < 1 || nz < 1 || (law != LAW_LINEAR && law != LAW_NEO_HOOKEAN)) return nullptr;
  Problem* p = new Problem();
  p->nx = nx, p->ny = ny, p->nz = nz, p->law = law;
  p->nthreads = nthreads > 0 ? nthreads : omp_get_max_threads();
  p->mu = E / (2.0 * (1.0 + nu));
  p->lk = law == LAW_LINEAR ? E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)) : E / (3.0 * (1.0 - 2.0 * nu));
  const int64_t NX = nx + 1, NY = ny + 1, NZ = nz + 1;
  p->n_nodes = NX * NY * NZ;
  p->n_cells = (int64_t)nx * ny * nz;
  p->ndofs = 3 * p->n_nodes;
  auto nid = [&](int64_t i, int64_t j, int64_t k) { return (int32_t)((i * NY + j) * NZ + k); };
  p->cells.resize(p->n_cells * 8);
  {
    int64_t c = 0;
    for (int64_t i = 0; i < nx; ++i)
      for (int64_t j = 0; j < ny; ++j)
        for (int64_t k = 0; k < nz; ++k, ++c) {
          int32_t* v = &p->cells[c * 8];
          v[0] = nid(i, j, k), v[1] = nid(i + 1, j, k), v[2] = nid(i + 1, j + 1, k), v[3] = nid(i, j + 1, k);
          v[4] = nid(i, j, k + 1), v[5] = nid(i + 1, j, k + 1), v[6] = nid(i + 1, j + 1, k + 1);
          v[7] = nid(i, j + 1, k + 1);
        }
  }
  // physical shape gradients and JxW per (cell, quad), from node coordinates
  double G[8][8][3], W[8];
  hex8_ref_grads(G, W);
  p->sg.resize(p->n_cells * 192);
  p->jxw.resize(p->n_cells * 8);
  const double hx = Lx / nx, hy = Ly / ny, hz = Lz / nz;
#pragma omp parallel for schedule(static) num_threads(p->nthreads)
  for (int64_t c = 0; c < p->n_cells; ++c) {
    double X[8][3];
    for (int a = 0; a < 8; ++a) {
      const int64_t n = p->cells[c * 8 + a];
      X[a][0] = (double)(n / (NY * NZ)) * hx;
      X[a][1] = (double)((n / NZ) % NY) * hy;
      X[a][2] = (double)(n % NZ) * hz;
    }
    for (int q = 0; q < 8; ++q) {
      double J[3][3] = {};
      for (int a = 0; a < 8; ++a)
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) J[i][j] += X[a][i] * G[q][a][j];
      const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                         J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                         J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
      double Ji[3][3];
      Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
      Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
      Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
      Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
      Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
      Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
      Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
      Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
      Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
      p->jxw[c * 8 + q] = det * W[q];
      for (int a = 0; a < 8; ++a)
        for (int j = 0; j < 3; ++j) {
          double s = 0.0;
          for (int i = 0; i < 3; ++i) s += G[q][a][i] * Ji[i][j];
          p->sg[c * 192 + q * 24 + a * 3 + j] = s;
        }
    }
  }
  // scalar CSR pattern: node neighbours on the lattice (|di|,|dj|,|dk| <= 1)
  p->row_ptr.assign(p->ndofs + 1, 0);
  std::vector<int64_t> nb_count(p->n_nodes);
  for (int64_t n = 0; n < p->n_nodes; ++n) {
    const int64_t i = n / (NY * NZ), j = (n / NZ) % NY, k = n % NZ;
    const int64_t ci = 1 + (i > 0) + (i < NX - 1), cj = 1 + (j > 0) + (j < NY - 1), ck = 1 + (k > 0) + (k < NZ - 1);
    nb_count[n] = ci * cj * ck;
  }
  for (int64_t n = 0; n < p->n_nodes; ++n)
    for (int c = 0; c < 3; ++c) p->row_ptr[3 * n + c + 1] = 3 * nb_count[n];
  for (int64_t r = 0; r < p->ndofs; ++r) p->row_ptr[r + 1] += p->row_ptr[r];
  p->nnz = p->row_ptr[p->ndofs];
  p->col.resize(p->nnz);
  p->diag.resize(p->ndofs);
#pragma omp parallel for schedule(static) num_threads(p->nthreads)
  for (int64_t n = 0; n < p->n_nodes; ++n) {
    const int64_t i = n / (NY * NZ), j = (n / NZ) % NY, k = n % NZ;
    std::vector<int32_t> nb;
    for (int64_t a = std::max<int64_t>(i - 1, 0); a <= std::min<int64_t>(i + 1, NX - 1); ++a)
      for (int64_t b = std::max<int64_t>(j - 1, 0); b <= std::min<int64_t>(j + 1, NY - 1); ++b)
        for (int64_t c = std::max<int64_t>(k - 1, 0); c <= std::min<int64_t>(k + 1, NZ - 1); ++c)
          nb.push_back(nid(a, b, c));  // ascending: lattice order
    for (int cc = 0; cc < 3; ++cc) {
      const int64_t r = 3 * n + cc;
      int64_t pos = p->row_ptr[r];
      for (int32_t m : nb)
        for (int d = 0; d < 3; ++d) {
          if (m == n && d == cc) p->diag[r] = (int32_t)(pos - p->row_ptr[r]);
          p->col[pos++] = 3 * m + d;
        }
    }
  }
  // COO -> CSR summation map (PETSc's setPreallocationCOO: per CSR entry, the
  // COO entries that add into it)
  const int64_t ncoo = p->n_cells * ND * ND;
  std::vector<int64_t> target(ncoo);
#pragma omp parallel for schedule(static) num_threads(p->nthreads)
  for (int64_t c = 0; c < p->n_cells; ++c) {
    const int32_t* v = &p->cells[c * 8];
    for (int a = 0; a < 8; ++a)
      for (int i = 0; i < 3; ++i) {
        const int64_t r = 3 * (int64_t)v[a] + i;
        const int32_t* cb = &p->col[p->row_ptr[r]];
        const int64_t len = p->row_ptr[r + 1] - p->row_ptr[r];
        for (int b = 0; b < 8; ++b)
          for (int k = 0; k < 3; ++k) {
            const int32_t cl = 3 * v[b] + k;
            const int64_t off = std::lower_bound(cb, cb + len, cl) - cb;
            target[c * 576 + (a * 3 + i) * ND + b * 3 + k] = p->row_ptr[r] + off;
          }
      }
  }
  p->jmap.assign(p->nnz + 1, 0);
  for (int64_t e = 0; e < ncoo; ++e) p->jmap[target[e] + 1]++;
  for (int64_t k = 0; k < p->nnz; ++k) p->jmap[k + 1] += p->jmap[k];
  p->perm.resize(ncoo);
  {
    std::vector<int64_t> fill(p->jmap.begin(), p->jmap.end() - 1);
    for (int64_t e = 0; e < ncoo; ++e) p->perm[fill[target[e]]++] = (int32_t)e;
  }
  p->V.resize(ncoo);
  p->vals.resize(p->nnz);
  p->res.resize(p->ndofs);
  return p;
}

void fcpu_destroy(void* h) { delete static_cast<Problem*>(h); }

int64_t fcpu_ndofs(void* h) { return static_cast<Problem*>(h)->ndofs; }
int64_t fcpu_nnz(void* h) { return static_cast<Problem*>(h)->nnz; }
int fcpu_threads(void* h) { return static_cast<Problem*>(h)->nthreads; }

// Dirichlet dofs and values of the current load step (the reference's
// node_inds_list / vec_inds_list / vals_list, flattened to dof indices).
int fcpu_set_dirichlet(void* h, int64_t n, const int64_t* dofs, const double* vals) {
  Problem* p = static_cast<Problem*>(h);
  p->bc_dofs.assign(dofs, dofs + n);
  p->bc_vals.assign(vals, vals + n);
  for (int64_t d : p->bc_dofs)
    if (d < 0 || d >= p->ndofs) return -1;
  return 0;
}

}  // extern "C"

namespace {

// newton_update + get_A: residual (with Dirichlet rows u - u_D) and the
// row-zeroed CSR Jacobian at u.  Returns ||R||.
double update(Problem* p, const double* u) {
  const double t0 = now();
  std::fill(p->res.begin(), p->res.end(), 0.0);
  const int64_t C = p->n_cells;
  // cell residuals and Jacobians (vmap of value_and_jacfwd over the cells);
  // the residual scatter needs no atomics: cells are grouped in 8 colours of
  // the lattice so that cells of one colour share no node
  std::vector<double> rcell(C * ND);
#pragma omp parallel for schedule(static) num_threads(p->nthreads)
  for (int64_t c = 0; c < C; ++c) {
    const int32_t* v = &p->cells[c * 8];
    Dual ue[ND], re[ND];
    for (int a = 0; a < 8; ++a)
      for (int i = 0; i < 3; ++i) {
        Dual& x = ue[a * 3 + i];
        x = dconst(u[3 * (int64_t)v[a] + i]);
        x.d[a * 3 + i] = 1.0;
      }
    cell_residual<Dual>(p->law, p->mu, p->lk, &p->sg[c * 192], &p->jxw[c * 8], ue, re);
    double* Vc = &p->V[c * 576];
    for (int r = 0; r < ND; ++r) {
      rcell[c * ND + r] = re[r].v;
      for (int k = 0; k < ND; ++k) Vc[r * ND + k] = re[r].d[k];
    }
  }
  // res.at[cells].add(r_e): node-owned gather of the cells around each node
  const int64_t NY = p->ny + 1, NZ = p->nz + 1, NX = p->nx + 1;
#pragma omp parallel for schedule(static) num_threads(p->nthreads)
  for (int64_t n = 0; n < p->n_nodes; ++n) {
    const int64_t i = n / (NY * NZ), j = (n / NZ) % NY, k = n % NZ;
    double s[3] = {0.0, 0.0, 0.0};
    for (int64_t a = std::max<int64_t>(i - 1, 0); a <= std::min<int64_t>(i, NX - 2); ++a)
      for (int64_t b = std::max<int64_t>(j - 1, 0); b <= std::min<int64_t>(j, NY - 2); ++b)
        for (int64_t c = std::max<int64_t>(k - 1, 0); c <= std::min<int64_t>(k, NZ - 2); ++c) {
          const int64_t cell = (a * p->ny + b) * p->nz + c;
          const int32_t* v = &p->cells[cell * 8];
          for (int l = 0; l < 8; ++l)
            if (v[l] == n)
              for (int d = 0; d < 3; ++d) s[d] += rcell[cell * ND + l * 3 + d];
        }
    for (int d = 0; d < 3; ++d) p->res[3 * n + d] = s[d];
  }
  // setValuesCOO: sum the COO entries into the CSR values
#pragma omp parallel for schedule(static) num_threads(p->nthreads)
  for (int64_t e = 0; e < p->nnz; ++e) {
    double s = 0.0;
    for (int64_t j = p->jmap[e]; j < p->jmap[e + 1]; ++j) s += p->V[p->perm[j]];
    p->vals[e] = s;
  }
  // zeroRows (diagonal 1, columns untouched) and the residual's Dirichlet rows
  for (size_t m = 0; m < p->bc_dofs.size(); ++m) {
    const int64_t r = p->bc_dofs[m];
    for (int64_t e = p->row_ptr[r]; e < p->row_ptr[r + 1]; ++e) p->vals[e] = 0.0;
    p->vals[p->row_ptr[r] + p->diag[r]] = 1.0;
  }
  for (size_t m = 0; m < p->bc_dofs.size(); ++m) p->res[p->bc_dofs[m]] = u[p->bc_dofs[m]] - p->bc_vals[m];
  double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s) num_threads(p->nthreads)
  for (int64_t r = 0; r < p->ndofs; ++r) s += p->res[r] * p->res[r];
  p->t_assembly += now() - t0;
  return std::sqrt(s);
}

void spmv(const Problem* p, const double* x, double* y) {
#pragma omp parallel for schedule(static) num_threads(p->nthreads)
  for (int64_t r = 0; r < p->ndofs; ++r) {
    double s = 0.0;
    for (int64_t e = p->row_ptr[r]; e < p->row_ptr[r + 1]; ++e) s += p->vals[e] * x[p->col[e]];
    y[r] = s;
  }
}

double dot(const Problem* p, const double* a, const double* b) {
  double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s) num_threads(p->nthreads)
  for (int64_t r = 0; r < p->ndofs; ++r) s += a[r] * b[r];
  return s;
}

// jax.scipy.sparse.linalg.bicgstab(A, b, x0, M=x/diag(A), tol, atol, maxiter):
// right-preconditioned BiCGSTAB; returns iterations (negative on breakdown).
int bicgstab(Problem* p, const double* b, double* x, double tol, double atol, int maxiter) {
  const int64_t n = p->ndofs;
  std::vector<double> dinv(n), r(n), rhat(n), pv(n, 0.0), q(n, 0.0), phat(n), s(n), shat(n), t(n);
  for (int64_t i = 0; i < n; ++i) dinv[i] = 1.0 / p->vals[p->row_ptr[i] + p->diag[i]];
  const double atol2 = std::max(tol * tol * dot(p, b, b), atol * atol);
  spmv(p, x, t.data());
#pragma omp parallel for schedule(static) num_threads(p->nthreads)
  for (int64_t i = 0; i < n; ++i) r[i] = rhat[i] = pv[i] = q[i] = b[i] - t[i];
  double rho = 1.0, alpha = 1.0, omega = 1.0;
  int k = 0;
  while (dot(p, r.data(), r.data()) > atol2 && k < maxiter) {
    const double rho_ = dot(p, rhat.data(), r.data());
    if (rho_ == 0.0) return -10;
    const double beta = rho_ / rho * alpha / omega;
#pragma omp parallel for schedule(static) num_threads(p->nthreads)
    for (int64_t i = 0; i < n; ++i) {
      pv[i] = r[i] + beta * (pv[i] - omega * q[i]);
      phat[i] = dinv[i] * pv[i];
    }
    spmv(p, phat.data(), q.data());
    const double alpha_ = rho_ / dot(p, rhat.data(), q.data());
#pragma omp parallel for schedule(static) num_threads(p->nthreads)
    for (int64_t i = 0; i < n; ++i) s[i] = r[i] - alpha_ * q[i];
    const bool exit_early = dot(p, s.data(), s.data()) < atol2;
    double omega_ = 0.0;
    if (!exit_early) {
#pragma omp parallel for schedule(static) num_threads(p->nthreads)
      for (int64_t i = 0; i < n; ++i) shat[i] = dinv[i] * s[i];
      spmv(p, shat.data(), t.data());
      omega_ = dot(p, t.data(), s.data()) / dot(p, t.data(), t.data());
    }
#pragma omp parallel for schedule(static) num_threads(p->nthreads)
    for (int64_t i = 0; i < n; ++i) {
      if (exit_early) {
        x[i] += alpha_ * phat[i];
        r[i] = s[i];
      } else {
        x[i] += alpha_ * phat[i] + omega_ * shat[i];
        r[i] = s[i] - omega_ * t[i];
      }
    }
    ++k;
    if (exit_early) break;
    if (omega_ == 0.0 || alpha_ == 0.0) return -11;
    rho = rho_, alpha = alpha_, omega = omega_;
  }
  return k;
}

// KSPCG + PCJACOBI with PETSc's preconditioned-norm test
// ||M^-1 r|| <= rtol ||M^-1 r0||, from x0 = u_D - u on Dirichlet rows (the
// guess jax_solve gets).  petsc_solve starts from zero instead; on the
// row-zeroed matrix, which is not symmetric, CG from zero diverges (the 20^3
// stretch: ||Ax - b|| ~ 1e24 after 10000 iterations), while from x0 the
// Dirichlet rows of r stay zero and CG runs on the symmetric free block.
int cg_jacobi(Problem* p, const double* b, double* x, double rtol, int maxiter) {
  const int64_t n = p->ndofs;
  std::vector<double> dinv(n), r(n), z(n), pv(n), q(n);
  for (int64_t i = 0; i < n; ++i) dinv[i] = 1.0 / p->vals[p->row_ptr[i] + p->diag[i]];
  spmv(p, x, q.data());
  for (int64_t i = 0; i < n; ++i) {
    r[i] = b[i] - q[i];
    pv[i] = z[i] = dinv[i] * r[i];
  }
  double rz = dot(p, r.data(), z.data());
  const double zn0 = std::sqrt(dot(p, z.data(), z.data()));
  int k = 0;
  while (k < maxiter) {
    if (std::sqrt(dot(p, z.data(), z.data())) <= rtol * zn0) break;
    spmv(p, pv.data(), q.data());
    const double alpha = rz / dot(p, pv.data(), q.data());
#pragma omp parallel for schedule(static) num_threads(p->nthreads)
    for (int64_t i = 0; i < n; ++i) {
      x[i] += alpha * pv[i];
      r[i] -= alpha * q[i];
      z[i] = dinv[i] * r[i];
    }
    const double rz_new = dot(p, r.data(), z.data());
    const double beta = rz_new / rz;
    rz = rz_new;
#pragma omp parallel for schedule(static) num_threads(p->nthreads)
    for (int64_t i = 0; i < n; ++i) pv[i] = z[i] + beta * pv[i];
    ++k;
  }
  return k;
}

}  // namespace

extern "C" {

// The Newton solve of the current load step, u (ndofs) in/out holding the
// initial guess.  method 0: jax_solve's BiCGSTAB (lin_tol, lin_atol);
// method 1: PETSc CG + Jacobi (lin_tol as rtol).  Returns 0, -1 (Newton did
// not converge in max_iter), -2 (linear solver breakdown or residual check
// ||A x - b|| >= 0.1 failed), -3 (non-finite values).
int fcpu_newton(void* h, double* u, double rel_tol, double tol, int method, double lin_tol, double lin_atol,
                int lin_maxiter, int max_iter) {
  Problem* p = static_cast<Problem*>(h);
  p->newton = p->krylov = 0;
  p->t_assembly = p->t_linear = 0.0;
  const int64_t n = p->ndofs;
  std::vector<double> b(n), x(n), y(n);
  double res = update(p, u);
  const double res0 = res;
  double rel = res0 > 0 ? res / res0 : 0.0;
  while (rel > rel_tol && res > tol) {
    if (p->newton >= max_iter) return -1;
    p->newton++;
    const double t0 = now();
    for (int64_t i = 0; i < n; ++i) b[i] = -p->res[i];
    std::fill(x.begin(), x.end(), 0.0);
    for (size_t m = 0; m < p->bc_dofs.size(); ++m) x[p->bc_dofs[m]] = p->bc_vals[m] - u[p->bc_dofs[m]];
    const int k = method == 0 ? bicgstab(p, b.data(), x.data(), lin_tol, lin_atol, lin_maxiter)
                              : cg_jacobi(p, b.data(), x.data(), lin_tol, lin_maxiter);
    if (k < 0) return -2;
    p->krylov += k;
    spmv(p, x.data(), y.data());  // the solvers' residual check (err < 0.1)
    double e2 = 0.0;
    for (int64_t i = 0; i < n; ++i) e2 += (y[i] - b[i]) * (y[i] - b[i]);
    if (!(std::sqrt(e2) < 0.1)) return -2;
    for (int64_t i = 0; i < n; ++i) u[i] += x[i];
    p->t_linear += now() - t0;
    res = update(p, u);
    rel = res / res0;
    if (!std::isfinite(res)) return -3;
  }
  return 0;
}

// Statistics of the last fcpu_newton: Newton and Krylov iterations and the
// assembly / linear-solve seconds.
void fcpu_stats(void* h, int* newton, int* krylov, double* t_assembly, double* t_linear) {
  const Problem* p = static_cast<const Problem*>(h);
  *newton = p->newton, *krylov = p->krylov, *t_assembly = p->t_assembly, *t_linear = p->t_linear;
}

// The residual (Dirichlet rows u - u_D) and the row-zeroed CSR Jacobian at u,
// for checks against the Python oracle.  res: ndofs; row_ptr: ndofs + 1;
// col, vals: nnz.
double fcpu_residual_tangent(void* h, const double* u, double* res, int64_t* row_ptr, int32_t* col, double* vals) {
  Problem* p = static_cast<Problem*>(h);
  const double r = update(p, u);
  std::memcpy(res, p->res.data(), sizeof(double) * p->ndofs);
  std::memcpy(row_ptr, p->row_ptr.data(), sizeof(int64_t) * (p->ndofs + 1));
  std::memcpy(col, p->col.data(), sizeof(int32_t) * p->nnz);
  std::memcpy(vals, p->vals.data(), sizeof(double) * p->nnz);
  return r;
}

}  // extern "C"
