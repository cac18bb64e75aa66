// Halo catalogue of fof_with_info on the device.
#pragma once

#include "context.cuh"

namespace pyfof {

// From the device halo ids of a finished call: members (host, capacity n)
// receives the particle indices of all valid halos, ascending per halo,
// halos in id order; offsets (host, offsets_cap >= halos + 1) the start of
// every halo and the total; nfound the number of halos.  Enqueued on the
// context's stream; members is complete after the stream is synchronised.
int32_t build_catalogue(Context &ctx, const int32_t *d_halo_id, int64_t n, int32_t *members,
                        int64_t *offsets, int64_t offsets_cap, int32_t *nfound);

}  // namespace pyfof
