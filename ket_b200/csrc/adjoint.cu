// adjoint.cu -- reverse-sweep (adjoint) gradients of <psi(theta)|H|psi(theta)>.
#include <cuda_runtime.h>

#include "internal.h"

#define KB_API extern "C" __attribute__((visibility("default")))

KB_API int ketgpu_adjoint(int32_t, const ketgpu_op*, uint64_t, const int32_t*, const double*, uint64_t, uint64_t,
                          const double*, const char* const*, uint64_t, int32_t, int32_t, double*, double*) {
  return KETGPU_ERR_LOGIC;
}
