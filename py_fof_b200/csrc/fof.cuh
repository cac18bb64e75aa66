// Friends-of-friends pipeline on one device.
#pragma once

#include "common.cuh"

namespace pyfof {

// Launch shapes that never change a result (set from the tile table the
// autotuner writes; pyfof_set_tile).  Index of a grid size n in the
// per-grid arrays: kGridIndex(n).
struct TileTable {
  // threads per block of the direct-summation removal loop for halos of at
  // most 32, 64, 128, 256, 512, 1000 members
  int direct_threads[6] = {64, 64, 128, 128, 256, 256};
  // halos per particle-mesh convolution batch for n = 48, 64, 128, 216,
  // 256 (0: as many as the batch memory budget allows)
  int pm_batch[5] = {0, 0, 0, 0, 0};
  // the fused z pass of the convolution splits a batch so that its grid
  // covers at least this many full waves of the GPU
  int conv_waves[5] = {4, 4, 4, 4, 4};
};
inline int kGridIndex(int n) { return n == 48 ? 0 : n == 64 ? 1 : n == 128 ? 2 : n == 216 ? 3 : n == 256 ? 4 : -1; }
constexpr int kDirectBucketEdge[6] = {32, 64, 128, 256, 512, 1000};

// Arguments of one fof_fortran-equivalent call (fof_fortran.f90:10-58).
// All particle arrays are device pointers.
struct FofArgs {
  const double *xp = nullptr;  // (3,N): soa ? x[d*N+i] : x[3i+d]
  const double *vp = nullptr;  // same layout; null means all velocities are zero
  const double *mp = nullptr;  // (N); null means unit masses
  int32_t soa = 1;
  const int32_t *np_halo = nullptr;  // host array (nhalo)
  int32_t nhalo = 0;
  int64_t total_np = 0;
  double L_Box = 512.0, link = 0.2;
  int32_t np_halo_min = 10, bound_check = 0, verbose = 0;
  double softening = 0.1, a_val = 1.0, b_val = 0.0, s15 = 15.0 * 0.67 * 512.0 / 300.0;
  int32_t n_threads = 0;
  int64_t ng = 256;
  double ng_global = 512.0;
  int32_t bound_fp64 = 0;  // 1: plain FP64 unbinding path instead of the FP32 product path
  int32_t bound_per_halo = 0;  // 1: FP64, one halo per launch sequence (the plain baseline)
  int64_t big_np = 0;          // PM halos above this many members use the chunked removal loop (0: default)
  int32_t cell_order = 0;      // 0: by key width, 1: per-cell sorts where cells allow, 2: radix sort
  TileTable tiles;
  // masses are divided by m_div right after their check (code units); only
  // with mp in the library's own scratch, which the check then rewrites
  double m_div = 1.0;
  // host-memory calls: masses_ready is recorded on `input_stream` when mp
  // is on the device, inputs_ready when vp is too (they copy while the
  // linking runs; the velocities arrive last and are packed for the
  // unbinding on that stream, see unbind_stage); null when the inputs are
  // already on the device
  cudaEvent_t masses_ready = nullptr, inputs_ready = nullptr;
  cudaStream_t input_stream = nullptr;
  // outputs (device): in_halo, halo_id (N int32); ang_mom host (3,nhalo) F-order
  int32_t *in_halo = nullptr, *halo_id = nullptr;
  double *ang_mom = nullptr;
};

struct Context;

// In-place conversions of device arrays to code units, ordered on stream s:
// x[i] / d, x[i] * f, and x[i] = v.  IEEE double operations, so the results
// equal the host's.
int32_t divide_inplace(double *x, int64_t n, double d, cudaStream_t s);
int32_t multiply_inplace(double *x, int64_t n, double f, cudaStream_t s);
int32_t fill_value(double *x, int64_t n, double v, cudaStream_t s);
// mask[i] = (halo_id[i] > 0) as 0/1 bytes; halo_id 16-byte aligned, mask
// 4-byte aligned
int32_t member_mask(const int32_t *halo_id, int64_t n, uint8_t *mask, cudaStream_t s);

// Runs the whole call on ctx's stream; returns a reference ierr code (or
// kCuda).  Synchronises the stream before returning.
int32_t fof_run(Context &ctx, const FofArgs &a);

}  // namespace pyfof
