// Error reporting, launch accounting and version of the jaxfem_b200 library.
#include <cstdarg>
#include <mutex>
#include <set>
#include <utility>

#include "sparse.cuh"

namespace fem {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

std::atomic<int64_t>& launch_counter() {
  static std::atomic<int64_t> n{0};
  return n;
}

bool pdl_enabled() {
  static int on = -1;
  if (on < 0) {
    const char* e = std::getenv("FEM_PDL");
    on = (e != nullptr && e[0] == '0') ? 0 : 1;
  }
  return on == 1;
}

double* host_mailbox() {
  static double* p = nullptr;
  if (p == nullptr) {
    if (cudaMallocHost(&p, 64 * sizeof(double)) != cudaSuccess) p = nullptr;
  }
  return p;
}

int ensure_smem_attr_ptr(const void* kernel) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({kernel, dev})) return FEM_OK;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(bsr_rows_smem()));
  // the row kernels are sized for kRowBlocksPerSM resident blocks: ask for
  // the largest shared-memory carve-out
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                             int(cudaSharedmemCarveoutMaxShared));
  if (e != cudaSuccess) {
    set_error("cudaFuncSetAttribute(bsr smem) -> %s", cudaGetErrorString(e));
    return FEM_ERR_CUDA;
  }
  done.insert({kernel, dev});
  return FEM_OK;
}

}  // namespace fem

extern "C" const char* fem_version(void) { return "jaxfem_b200 0.1 (sm_100a)"; }
extern "C" const char* fem_last_error(void) { return fem::g_err; }
extern "C" int64_t fem_launch_count(void) { return fem::launch_counter().load(); }
