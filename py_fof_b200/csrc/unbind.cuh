// Gravitational unbinding of FoF candidates on the device.
#pragma once

#include "fof_internal.cuh"

namespace pyfof {

// Runs the bound_check=True branch of fof_fortran (fof_fortran.f90:252-360)
// for the candidates found by the FoF stages and writes in_halo, halo_id and
// ang_mom.
int32_t unbind_stage(Context &ctx, const FofArgs &a, FofState &st);

}  // namespace pyfof
