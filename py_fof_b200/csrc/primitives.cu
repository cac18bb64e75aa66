// Exclusive scan and stable LSD radix sort for 32-bit keys/values.
//
// Scan: three-phase (tile reduce, recursive scan of tile sums, tile scan +
// offset).  Radix sort: 8-bit digits; per-tile digit histograms, a scan of
// the digit-major histogram table, then a stable scatter in which every warp
// ranks its elements in input order with __match_any_sync.
#include "primitives.cuh"

namespace pyfof {

namespace {

constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;  // 4096

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread; returns the block total
// through *total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *total) {
  __shared__ uint32_t warp_sums[SCAN_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = warp_incl_scan(v);
  if (lane == 31) warp_sums[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < SCAN_THREADS / 32 ? warp_sums[lane] : 0;
    uint32_t wi = warp_incl_scan(w);
    if (lane < SCAN_THREADS / 32) warp_sums[lane] = wi - w;
    if (lane == SCAN_THREADS / 32 - 1) *total = wi;
  }
  __syncthreads();
  uint32_t res = warp_sums[warp] + inc - v;
  __syncthreads();
  return res;
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_reduce_kernel(const uint32_t *__restrict__ in,
                                                                   int64_t n,
                                                                   uint32_t *__restrict__ sums) {
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
  uint32_t acc = 0;
#pragma unroll
  for (int j = 0; j < SCAN_ITEMS; ++j) {
    int64_t i = base + (int64_t)j * SCAN_THREADS + threadIdx.x;
    if (i < n) acc += in[i];
  }
  __shared__ uint32_t red[SCAN_THREADS / 32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    uint32_t v = threadIdx.x < SCAN_THREADS / 32 ? red[threadIdx.x] : 0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) sums[blockIdx.x] = v;
  }
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_apply_kernel(const uint32_t *in, uint32_t *out,
                                                                  int64_t n,
                                                                  const uint32_t *__restrict__ offs,
                                                                  uint32_t *total) {
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
  uint32_t v[SCAN_ITEMS];
  uint32_t sum = 0;
#pragma unroll
  for (int j = 0; j < SCAN_ITEMS; ++j) {
    int64_t i = base + j;
    v[j] = i < n ? in[i] : 0u;
    sum += v[j];
  }
  __shared__ uint32_t btot;
  uint32_t run = block_excl_scan(sum, &btot);
  if (offs) run += offs[blockIdx.x];
#pragma unroll
  for (int j = 0; j < SCAN_ITEMS; ++j) {
    int64_t i = base + j;
    if (i < n) out[i] = run;
    run += v[j];
  }
  if (total && threadIdx.x == SCAN_THREADS - 1 && blockIdx.x == gridDim.x - 1) *total = run;
}

// ------------------------------------------------------------ radix sort

// exclusive scan over the 256 threads of a block (one value each)
__device__ __forceinline__ uint32_t block_excl_scan_256(uint32_t v, uint32_t *total) {
  __shared__ uint32_t ws[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t inc = warp_incl_scan(v);
  if (lane == 31) ws[warp] = inc;
  __syncthreads();
  uint32_t before = 0, all = 0;
#pragma unroll
  for (int w = 0; w < 8; ++w) {
    const uint32_t s = ws[w];
    before += w < warp ? s : 0u;
    all += s;
  }
  *total = all;
  return before + inc - v;
}

constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ROUNDS = 16;                          // items per lane
constexpr int RS_TILE = RS_THREADS * RS_ROUNDS;        // 4096
constexpr int RS_BINS = 256;

__global__ void __launch_bounds__(RS_THREADS) rs_upsweep(const uint32_t *__restrict__ keys,
                                                         int64_t n, int shift,
                                                         uint32_t *__restrict__ hist,
                                                         int64_t ntiles) {
  __shared__ uint32_t h[RS_BINS];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * RS_TILE;
#pragma unroll 4
  for (int j = 0; j < RS_ROUNDS; ++j) {
    int64_t i = base + (int64_t)j * RS_THREADS + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 0xffu], 1u);
  }
  __syncthreads();
  hist[(int64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one tile: warp ranks by digit (__match_any_sync, in
// input order), then the tile is reordered by digit in shared memory and
// written out in that order, so consecutive threads store consecutive
// positions of the same digit run.
__global__ void __launch_bounds__(RS_THREADS) rs_downsweep(const uint32_t *__restrict__ kin,
                                                           const uint32_t *__restrict__ vin,
                                                           uint32_t *__restrict__ kout,
                                                           uint32_t *__restrict__ vout, int64_t n,
                                                           int shift,
                                                           const uint32_t *__restrict__ offs,
                                                           int64_t ntiles) {
  __shared__ uint32_t wh[RS_WARPS][RS_BINS];
  __shared__ uint32_t tstart[RS_BINS], glob[RS_BINS];
  __shared__ uint32_t sk[RS_TILE], sv[RS_TILE];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int d = lane; d < RS_BINS; d += 32) wh[warp][d] = 0;
  __syncwarp();
  const int64_t tbase = (int64_t)blockIdx.x * RS_TILE;
  const int64_t wbase = tbase + (int64_t)warp * (32 * RS_ROUNDS);
  uint32_t key[RS_ROUNDS], val[RS_ROUNDS], rank[RS_ROUNDS];
  const unsigned lt = lanemask_lt();
#pragma unroll
  for (int r = 0; r < RS_ROUNDS; ++r) {
    int64_t i = wbase + r * 32 + lane;
    bool ok = i < n;
    key[r] = ok ? kin[i] : 0xffffffffu;
    val[r] = ok ? (vin ? vin[i] : (uint32_t)i) : 0u;
    uint32_t d = ok ? ((key[r] >> shift) & 0xffu) : RS_BINS;  // 256 = padding
    unsigned peers = __match_any_sync(0xffffffffu, d);
    uint32_t base = d < RS_BINS ? wh[warp][d] : 0u;
    rank[r] = base + __popc(peers & lt);
    __syncwarp();
    int leader = 31 - __clz(peers);
    if (lane == leader && d < RS_BINS) wh[warp][d] = base + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {
    // per digit: offsets of the warps inside the tile's run, the run's
    // start in the tile (block scan) and its global start
    const int d = threadIdx.x;  // RS_THREADS == RS_BINS
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) {
      const uint32_t c = wh[w][d];
      wh[w][d] = run;
      run += c;
    }
    uint32_t tot;
    tstart[d] = block_excl_scan_256(run, &tot);
    glob[d] = offs[(int64_t)d * ntiles + blockIdx.x];
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RS_ROUNDS; ++r) {
    int64_t i = wbase + r * 32 + lane;
    if (i < n) {
      const uint32_t d = (key[r] >> shift) & 0xffu;
      const uint32_t loc = tstart[d] + wh[warp][d] + rank[r];
      sk[loc] = key[r];
      sv[loc] = val[r];
    }
  }
  __syncthreads();
  const int tn = (int)min((int64_t)RS_TILE, n - tbase);
  for (int i = threadIdx.x; i < tn; i += RS_THREADS) {
    const uint32_t k = sk[i];
    const uint32_t d = (k >> shift) & 0xffu;
    const uint32_t pos = glob[d] + ((uint32_t)i - tstart[d]);
    kout[pos] = k;
    vout[pos] = sv[i];
  }
}

__global__ void iota_copy_kernel(const uint32_t *kin, const uint32_t *vin, uint32_t *kout,
                                 uint32_t *vout, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    kout[i] = kin[i];
    vout[i] = vin ? vin[i] : (uint32_t)i;
  }
}

}  // namespace

int32_t exclusive_scan_u32(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *total,
                           Arena &scratch, cudaStream_t s) {
  if (n <= 0) {
    if (total) PYFOF_CUDA(cudaMemsetAsync(total, 0, sizeof(uint32_t), s));
    return kOk;
  }
  int64_t nb = ceil_div(n, SCAN_TILE);
  if (nb == 1) {
    scan_apply_kernel<<<1, SCAN_THREADS, 0, s>>>(in, out, n, nullptr, total);
    PYFOF_CHECK_LAUNCH();
    return kOk;
  }
  uint32_t *sums = scratch.carve<uint32_t>((size_t)nb);
  uint32_t *offs = scratch.carve<uint32_t>((size_t)nb);
  if (!sums || !offs) {
    set_error("scan scratch exhausted");
    return kAlloc;
  }
  scan_reduce_kernel<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, sums);
  PYFOF_CHECK_LAUNCH();
  PYFOF_TRY(exclusive_scan_u32(sums, offs, nb, nullptr, scratch, s));
  scan_apply_kernel<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, out, n, offs, total);
  PYFOF_CHECK_LAUNCH();
  return kOk;
}

int32_t radix_sort_pairs(const uint32_t *keys_in, const uint32_t *vals_in, int64_t n, int bits,
                         uint32_t *keys_a, uint32_t *vals_a, uint32_t *keys_b, uint32_t *vals_b,
                         uint32_t **keys_out, uint32_t **vals_out, Arena &scratch,
                         cudaStream_t s) {
  *keys_out = keys_a;
  *vals_out = vals_a;
  if (n <= 0) return kOk;
  const int passes = bits <= 0 ? 0 : (bits + 7) / 8;
  if (passes == 0) {
    iota_copy_kernel<<<4 * kNumSMs, 256, 0, s>>>(keys_in, vals_in, keys_a, vals_a, n);
    PYFOF_CHECK_LAUNCH();
    return kOk;
  }
  const int64_t ntiles = ceil_div(n, RS_TILE);
  uint32_t *hist = scratch.carve<uint32_t>((size_t)(ntiles * RS_BINS));
  uint32_t *offs = scratch.carve<uint32_t>((size_t)(ntiles * RS_BINS));
  if (!hist || !offs) {
    set_error("radix scratch exhausted");
    return kAlloc;
  }
  const uint32_t *kin = keys_in, *vin = vals_in;
  uint32_t *ko = keys_a, *vo = vals_a;
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    rs_upsweep<<<(unsigned)ntiles, RS_THREADS, 0, s>>>(kin, n, shift, hist, ntiles);
    PYFOF_CHECK_LAUNCH();
    PYFOF_TRY(exclusive_scan_u32(hist, offs, ntiles * RS_BINS, nullptr, scratch, s));
    rs_downsweep<<<(unsigned)ntiles, RS_THREADS, 0, s>>>(kin, vin, ko, vo, n, shift, offs, ntiles);
    PYFOF_CHECK_LAUNCH();
    kin = ko;
    vin = vo;
    *keys_out = ko;
    *vals_out = vo;
    ko = (ko == keys_a) ? keys_b : keys_a;
    vo = (vo == vals_a) ? vals_b : vals_a;
  }
  return kOk;
}

}  // namespace pyfof
