// Particle-mesh unbinding (bound_fortran.f90:2206-2735, :3125-3552).
#include "context.cuh"
#include "unbind_internal.cuh"

namespace pyfof {

int32_t unbind_pm(Context &ctx, const FofArgs &a, const GridRules &rules, const Members &m,
                  const std::vector<HaloTask> &tasks, const std::vector<int32_t> &list,
                  HaloResult *res, uint8_t *keep, float *phi_out) {
  (void)ctx; (void)a; (void)rules; (void)m; (void)tasks; (void)list; (void)res; (void)keep;
  (void)phi_out;
  set_error("particle-mesh unbinding (candidates above 1000 members) is not available yet");
  return kInvalid;
}

}  // namespace pyfof
