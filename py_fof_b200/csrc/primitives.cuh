// Device-wide primitives: exclusive scan and stable LSD radix sort.
#pragma once

#include "common.cuh"

namespace pyfof {

// out[i] = sum(in[0:i]) (u32, wrap-around); in may alias out.  If total is
// non-null the grand total is written there (device pointer).
int32_t exclusive_scan_u32(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *total,
                           Arena &scratch, cudaStream_t s);

// Stable sort of (key, value) pairs by the low `bits` bits of key.  vals_in
// may be null, meaning value = position.  The sorted pairs end up in
// (*keys_out, *vals_out), which point either at the alt buffers or at the
// caller's out buffers.
int32_t radix_sort_pairs(const uint32_t *keys_in, const uint32_t *vals_in, int64_t n, int bits,
                         uint32_t *keys_a, uint32_t *vals_a, uint32_t *keys_b, uint32_t *vals_b,
                         uint32_t **keys_out, uint32_t **vals_out, Arena &scratch,
                         cudaStream_t s);

}  // namespace pyfof
