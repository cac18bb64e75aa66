// Halo catalogue of fof_with_info on the device (py_fof/__init__.py:481-518):
// the member indices of every valid halo, ascending, halos in halo-id order,
// and the offsets of the halos in that list.  A stable radix sort of the
// particle indices by halo id gives exactly that order (ids are 1..nfound,
// non-members have id 0 and sort first).
#include <algorithm>

#include "catalogue.cuh"
#include "fof_internal.cuh"
#include "primitives.cuh"

namespace pyfof {

namespace {

constexpr int CB = 256;

__global__ void cat_max_kernel(const int32_t *__restrict__ hid, int64_t n, int32_t *__restrict__ out) {
  int m = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    m = max(m, hid[i]);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0) atomicMax(out, m);
}

// start[id] = first sorted position of halo id (positions of a run's first key)
__global__ void cat_start_kernel(const uint32_t *__restrict__ key, int64_t n, int64_t *__restrict__ start) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t k = key[i];
    if (k != 0 && (i == 0 || key[i - 1] != k)) start[k] = i;
  }
}

}  // namespace

int32_t build_catalogue(Context &ctx, const int32_t *d_halo_id, int64_t n, int32_t *members,
                        int64_t *offsets, int64_t offsets_cap, int32_t *nfound) {
  cudaStream_t s = ctx.stream;
  Arena &W = ctx.work;
  *nfound = 0;
  int32_t *dmax = ctx.d_flags + FLAG_COUNT_C;
  PYFOF_CUDA(cudaMemsetAsync(dmax, 0, sizeof(int32_t), s));
  const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(std::max<int64_t>(n, 1), CB), (int64_t)kNumSMs * 16);
  if (n > 0) {
    cat_max_kernel<<<grid, CB, 0, s>>>(d_halo_id, n, dmax);
    PYFOF_CHECK_LAUNCH();
  }
  PYFOF_CUDA(cudaMemcpyAsync(ctx.h_flags + FLAG_COUNT_C, dmax, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  const int32_t maxid = ctx.h_flags[FLAG_COUNT_C];
  if (maxid <= 0) {
    if (offsets_cap >= 1) offsets[0] = 0;
    return kOk;
  }
  if (offsets_cap < (int64_t)maxid + 1) {
    set_error("catalogue: %d halos need %d offsets, capacity %lld", maxid, maxid + 1, (long long)offsets_cap);
    *nfound = maxid;
    return kInvalid;
  }
  uint32_t *ka = W.carve<uint32_t>(n), *va = W.carve<uint32_t>(n), *kb = W.carve<uint32_t>(n),
           *vb = W.carve<uint32_t>(n);
  int64_t *start = W.carve<int64_t>((size_t)maxid + 2);
  if (!ka || !va || !kb || !vb || !start) {
    set_error("workspace exhausted (catalogue)");
    return kAlloc;
  }
  int bits = 0;
  while (bits < 32 && ((uint64_t)maxid >> bits) != 0) ++bits;
  uint32_t *sk, *sv;
  PYFOF_TRY(radix_sort_pairs(reinterpret_cast<const uint32_t *>(d_halo_id), nullptr, n, bits, ka, va, kb, vb,
                             &sk, &sv, W, s));
  PYFOF_CUDA(cudaMemsetAsync(start, 0xff, sizeof(int64_t) * ((size_t)maxid + 2), s));
  cat_start_kernel<<<grid, CB, 0, s>>>(sk, n, start);
  PYFOF_CHECK_LAUNCH();
  std::vector<int64_t> hstart((size_t)maxid + 2);
  PYFOF_CUDA(cudaMemcpyAsync(hstart.data() + 1, start + 1, sizeof(int64_t) * maxid, cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  hstart[(size_t)maxid + 1] = n;
  for (int32_t h = maxid; h >= 1; --h)  // an id without members starts where the next one does
    if (hstart[h] < 0) hstart[h] = hstart[h + 1];
  const int64_t z0 = hstart[1];
  const int64_t m = n - z0;
  PYFOF_CUDA(cudaMemcpyAsync(members, sv + z0, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, s));
  for (int32_t h = 0; h < maxid; ++h) offsets[h] = hstart[h + 1] - z0;
  offsets[maxid] = m;
  *nfound = maxid;
  return kOk;
}

}  // namespace pyfof
