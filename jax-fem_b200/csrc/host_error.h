// Error reporting for host-only translation units of the jaxfem_b200 library.
#pragma once
#include "jaxfem_b200.h"

namespace fem {
void set_error(const char* fmt, ...);
}  // namespace fem

#define FEM_CHECK_ARG(cond, ...)     \
  do {                               \
    if (!(cond)) {                   \
      ::fem::set_error(__VA_ARGS__); \
      return FEM_ERR_ARG;            \
    }                                \
  } while (0)
