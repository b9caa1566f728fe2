// Shared helpers of the jaxfem_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdio>
#include <string>

#include "jaxfem_b200.h"

namespace fem {

// ---- error reporting across the C ABI --------------------------------------
void set_error(const char* fmt, ...);
std::atomic<int64_t>& launch_counter();
// Pinned host buffer (64 doubles) for synchronous scalar read-backs.
double* host_mailbox();

#define FEM_CHECK_ARG(cond, ...)            \
  do {                                      \
    if (!(cond)) {                          \
      ::fem::set_error(__VA_ARGS__);        \
      return FEM_ERR_ARG;                   \
    }                                       \
  } while (0)

#define FEM_CUDA_TRY(call)                                                        \
  do {                                                                            \
    cudaError_t _e = (call);                                                      \
    if (_e != cudaSuccess) {                                                      \
      ::fem::set_error("%s:%d %s -> %s", __FILE__, __LINE__, #call,               \
                       cudaGetErrorString(_e));                                   \
      return FEM_ERR_CUDA;                                                        \
    }                                                                             \
  } while (0)

// Check the launch that was just made; count it.
#define FEM_LAUNCH_CHECK()                                                        \
  do {                                                                            \
    ::fem::launch_counter().fetch_add(1, std::memory_order_relaxed);              \
    cudaError_t _e = cudaGetLastError();                                          \
    if (_e != cudaSuccess) {                                                      \
      ::fem::set_error("%s:%d kernel launch -> %s", __FILE__, __LINE__,           \
                       cudaGetErrorString(_e));                                   \
      return FEM_ERR_CUDA;                                                        \
    }                                                                             \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ---- programmatic dependent launch --------------------------------------------
// A kernel launched with launch_pdl may be scheduled while its predecessor in
// the stream is still finishing (its launch and block set-up overlap the
// predecessor's tail).  Such a kernel calls pdl_wait() before it touches any
// memory its predecessor reads or writes: the wait returns once the
// predecessor has completed and its writes are visible.  Outside such a
// launch pdl_wait() returns at once.  FEM_PDL=0 in the environment launches
// normally.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// Lets the next kernel in the stream (launched with launch_pdl) be scheduled
// once every CTA of this one has called it or exited, instead of at its end.
// Called only after this kernel's own pdl_wait(), so the kernel before it
// has completed and the successor overlaps this kernel alone.  pdl_wait()
// in the successor orders this kernel's writes before its reads, but an L1
// line that this kernel's CTAs loaded on the successor's SM after the
// successor started is not refreshed: the successor reads what this kernel
// writes through L2 (ld.global.cg).
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

bool pdl_enabled();

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

inline int num_sms() {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

// ---- HEX8 reference element -------------------------------------------------
// Trilinear HEX8 on [0,1]^3 with VTK/meshio node order (basix P1 hexahedron
// re-ordered by [0,1,3,2,4,5,7,6]); 2x2x2 Gauss-Legendre points at
// 1/2 -+ 1/(2 sqrt 3) per axis, quadrature point q = 4 ix + 2 iy + iz
// (x slowest), every weight 1/8.
constexpr double kGaussOff = 0.28867513459481288225457439025098;  // 1/(2 sqrt 3)
constexpr double kQuadWeight = 0.125;

__host__ __device__ __forceinline__ int vtk_xbit(int a) { return ((a + 1) >> 1) & 1; }
__host__ __device__ __forceinline__ int vtk_ybit(int a) { return (a >> 1) & 1; }
__host__ __device__ __forceinline__ int vtk_zbit(int a) { return a >> 2; }

// Reference coordinates of quadrature point q.
__host__ __device__ __forceinline__ void quad_point(int q, double xi[3]) {
  xi[0] = ((q >> 2) & 1) ? 0.5 + kGaussOff : 0.5 - kGaussOff;
  xi[1] = ((q >> 1) & 1) ? 0.5 + kGaussOff : 0.5 - kGaussOff;
  xi[2] = (q & 1) ? 0.5 + kGaussOff : 0.5 - kGaussOff;
}

// Reference gradient of shape function a at reference point xi.
__host__ __device__ __forceinline__ void shape_grad_ref(int a, const double xi[3], double dn[3]) {
  const int bx = vtk_xbit(a), by = vtk_ybit(a), bz = vtk_zbit(a);
  const double fx = bx ? xi[0] : 1.0 - xi[0];
  const double fy = by ? xi[1] : 1.0 - xi[1];
  const double fz = bz ? xi[2] : 1.0 - xi[2];
  const double sx = bx ? 1.0 : -1.0, sy = by ? 1.0 : -1.0, sz = bz ? 1.0 : -1.0;
  dn[0] = sx * fy * fz;
  dn[1] = fx * sy * fz;
  dn[2] = fx * fy * sz;
}

// Physical shape gradients and JxW at quadrature point q from 8 node coords.
// Matches fe.py get_shape_grads: J_ij = sum_a X_a[i] dN_a/dxi_j,
// grad N_a = dN_a/dxi . J^{-1}, JxW = det(J) w_q.  Returns det(J).
__device__ __forceinline__ double hex8_geometry(int q, const double X[8][3], double g[8][3],
                                                double* jxw) {
  double xi[3];
  quad_point(q, xi);
  double dn[8][3];
  double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    shape_grad_ref(a, xi, dn[a]);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) J[i][j] = fma(X[a][i], dn[a][j], J[i][j]);
  }
  const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  const double id = 1.0 / det;
  double inv[3][3];
  inv[0][0] = c00 * id;
  inv[1][0] = c01 * id;
  inv[2][0] = c02 * id;
  inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int k = 0; k < 3; ++k)
      g[a][k] = dn[a][0] * inv[0][k] + dn[a][1] * inv[1][k] + dn[a][2] * inv[2][k];
  *jxw = det * kQuadWeight;
  return det;
}

// The same for a cell that is an axis-aligned box (as every cell of a
// box_mesh lattice is): J = diag(h), so grad N_a = dN_a/dxi / h and
// JxW = hx hy hz w.  The test is exact: along each axis every node takes the
// coordinate of node 0 or of the node one step along that axis (VTK nodes 1,
// 3, 4), as its reference bit says.  Returns false (nothing written) for any
// other cell.
__device__ __forceinline__ bool hex8_box_geometry(int q, const double X[8][3], double g[8][3], double* jxw) {
  const int corner[3] = {1, 3, 4};
  double h[3];
  bool box = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double lo = X[0][d], hi = X[corner[d]][d];
    h[d] = hi - lo;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const int bit = d == 0 ? vtk_xbit(a) : (d == 1 ? vtk_ybit(a) : vtk_zbit(a));
      box = box && (X[a][d] == (bit ? hi : lo));
    }
  }
  box = box && h[0] != 0.0 && h[1] != 0.0 && h[2] != 0.0;
  if (!box) return false;
  double xi[3];
  quad_point(q, xi);
  const double ih[3] = {1.0 / h[0], 1.0 / h[1], 1.0 / h[2]};
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    double dn[3];
    shape_grad_ref(a, xi, dn);
#pragma unroll
    for (int k = 0; k < 3; ++k) g[a][k] = dn[k] * ih[k];
  }
  *jxw = h[0] * h[1] * h[2] * kQuadWeight;
  return true;
}

// ---- reductions ----------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace fem
