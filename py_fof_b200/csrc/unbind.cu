// Gravitational unbinding (bound_fortran.f90) -- placeholder until the
// solver kernels land.
#include "context.cuh"
#include "unbind.cuh"

namespace pyfof {

int32_t unbind_stage(Context &ctx, const FofArgs &a, FofState &st) {
  (void)ctx; (void)a; (void)st;
  set_error("bound_check is not available in this build");
  return kInvalid;
}

}  // namespace pyfof
