// Particle-mesh unbinding of candidates with more than 1000 members
// (bound_check_grid for gid >= 1, bound_fortran.f90:2436-2864).
//
// Per halo: TSC weights and self-potential of every member (:2558-2602),
// then up to 20 passes of
//   C1: TSC deposit of the kept members on the zero-padded n^3 grid, FFT,
//       multiplication by the optimal Green's function, inverse FFT, TSC
//       gather, self term and the far-field constant (:2657-2703);
//   C2: short-range residual between the spline-softened kernel and the C1
//       split kernel for pairs closer than 3.5 grid cells (:3403-3552),
//       evaluated over 3.5-cell neighbour lists, recomputed over the kept set
//       each pass (the reference updates it incrementally; the sum is the
//       same set of pair terms);
//   removal: the inner loop of the direct path, with the top-2% selection
//       done by an in-block radix select (only the deleted set matters here).
// Halos of one grid class are batched: one launch deposits, transforms and
// gathers all of them.  R = float is the product path, R = double the plain
// FP64 path.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>

#include "context.cuh"
#include "fft.cuh"
#include "primitives.cuh"
#include "unbind_internal.cuh"

namespace pyfof {

namespace {

constexpr int BLK = 256;
constexpr int IBLK = 1024;  // inner-loop block
constexpr double kPi = 3.141592653589793238462643383279502884197;

// ---------------------------------------------------------------- Green

// bound_fft_wave_number (bound_fortran.f90:3563-3569)
__device__ __forceinline__ double wave_number(int i0, int n) {
  const int mode = ((i0 + n / 2) % n) - n / 2;
  return 2.0 * kPi * (double)mode / (double)n;
}

// bound_assignment_window_sq with assignment order 2 (:3571-3583)
__device__ __forceinline__ double window_sq(double k0, double k1, double k2) {
  double s = 1.0;
  double x = 0.5 * k0;
  if (x != 0.0) s = s * sin(x) / x;
  x = 0.5 * k1;
  if (x != 0.0) s = s * sin(x) / x;
  x = 0.5 * k2;
  if (x != 0.0) s = s * sin(x) / x;
  const double s2 = s * s, s3 = s2 * s;
  return s3 * s3;
}

// Alias-summed optimal Green's function (bound_calc_green_and_self,
// :2300-2371), one thread per half-spectrum point.
template <typename R>
__global__ void green_kernel(R *__restrict__ g, int n, double soft, double range, int truncated,
                             int32_t *flags) {
  const int nh = n / 2 + 1;
  const int64_t total = (int64_t)nh * n * n;
  const double radius = 0.5 * (double)n;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % nh);
    const int j = (int)((t / nh) % n);
    const int k = (int)(t / ((int64_t)nh * n));
    const double kv0 = wave_number(i, n), kv1 = wave_number(j, n), kv2 = wave_number(k, n);
    double asum = 0.0, bsum = 0.0;
    for (int ka = -2; ka <= 2; ++ka)
      for (int ja = -2; ja <= 2; ++ja)
        for (int ia = -2; ia <= 2; ++ia) {
          const double k0 = kv0 + 2.0 * kPi * (double)ia;
          const double k1 = kv1 + 2.0 * kPi * (double)ja;
          const double k2 = kv2 + 2.0 * kPi * (double)ka;
          const double kmag = sqrt(k0 * k0 + k1 * k1 + k2 * k2);
          const double uk2 = window_sq(k0, k1, k2);
          asum += uk2;
          double target;
          if (kmag == 0.0) {
            if (range == 0.0) target = -4.0 * kPi * radius * radius / 6.0;
            else if (truncated) target = 0.0;
            else target = -2.0 * kPi * (range * range - soft * soft) / 15.0;
          } else {
            double y = soft * kmag / 2.0;
            double y2 = y * y;
            const double ss = 12.0 * (1.0 / (y2 * y2)) * (2.0 - 2.0 * cos(y) - y * sin(y));
            double sr = 0.0;
            if (range != 0.0) {
              y = range * kmag / 2.0;
              y2 = y * y;
              sr = 12.0 * (1.0 / (y2 * y2)) * (2.0 - 2.0 * cos(y) - y * sin(y));
            }
            double cut = 1.0;
            if (truncated) {
              const double kr = kmag * radius;
              cut = 1.0 - sin(kr) / kr;
            }
            target = -4.0 * kPi * (ss * ss - sr * sr) * cut / (kmag * kmag);
          }
          bsum += uk2 * target;
        }
    if (!(asum > 2.2250738585072014e-308)) {
      atomicCAS(&flags[FLAG_ERR], 0, kInvalid);
      continue;
    }
    const double v = bsum / (asum * asum);
    g[t] = (R)v;  // FP32 path: the reference's complex(4) table
  }
}

template <typename R>
__global__ void self_extract_kernel(const R *__restrict__ grid, int n, R *__restrict__ self) {
  const int t = threadIdx.x;
  if (t >= 125) return;
  const int ox = t % 5 - 2, oy = (t / 5) % 5 - 2, oz = t / 25 - 2;
  const int x = (ox + n) % n, y = (oy + n) % n, z = (oz + n) % n;
  const R n3 = (R)((double)n * n * n);
  self[t] = grid[((int64_t)z * n + y) * n + x] / n3;
}

}  // namespace

struct GreenTable {
  int n = 0;
  void *g = nullptr;     // half-spectrum table (R)
  void *self = nullptr;  // 125 self-kernel values (R), device
  bool fp64 = false;
  ~GreenTable() {
    if (g) cudaFree(g);
    if (self) cudaFree(self);
  }
};

namespace {

// Green table of grid n for (soft, range, truncated), cached per context.
template <typename R>
int32_t get_green(Context &ctx, int n, double soft, double range, int truncated,
                  std::shared_ptr<GreenTable> *out) {
  const int kind = range == 0.0 ? 0 : (range < 10.0 ? 1 : 2);
  const int64_t key = ((int64_t)n << 8) | (kind << 1) | (sizeof(R) == 8 ? 1 : 0);
  std::lock_guard<std::mutex> lk(ctx.green->mu);
  auto it = ctx.green->tables.find(key);
  if (it != ctx.green->tables.end()) { *out = it->second; return kOk; }
  auto t = std::make_shared<GreenTable>();
  t->n = n;
  t->fp64 = sizeof(R) == 8;
  const int nh = n / 2 + 1;
  const int64_t cnt = (int64_t)nh * n * n;
  cudaStream_t s = ctx.stream;
  PYFOF_CUDA(cudaMalloc(&t->g, sizeof(R) * cnt));
  PYFOF_CUDA(cudaMalloc(&t->self, sizeof(R) * 125));
  PYFOF_CUDA(cudaMemsetAsync(ctx.d_flags, 0, sizeof(int32_t), s));
  green_kernel<R><<<(unsigned)std::min<int64_t>(ceil_div(cnt, 128), 148 * 64), 128, 0, s>>>(
      (R *)t->g, n, soft, range, truncated, ctx.d_flags);
  PYFOF_CHECK_LAUNCH();
  R *grid = nullptr;
  cplx_t<R> *spec = nullptr;
  PYFOF_CUDA(cudaMallocAsync(&grid, sizeof(R) * (size_t)n * n * n, s));
  PYFOF_CUDA(cudaMallocAsync(&spec, sizeof(cplx_t<R>) * spec_elems<R>(n), s));
  int32_t r = c2r_full<R>((const R *)t->g, spec, grid, n, s);
  if (r == kOk) {
    self_extract_kernel<R><<<1, 128, 0, s>>>(grid, n, (R *)t->self);
    PYFOF_CHECK_LAUNCH();
  }
  cudaFreeAsync(grid, s);
  cudaFreeAsync(spec, s);
  PYFOF_CUDA(cudaMemcpyAsync(ctx.h_flags, ctx.d_flags, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  if (r != kOk) return r;
  if (ctx.h_flags[FLAG_ERR]) {
    set_error("Green's function: zero assignment response");
    return kInvalid;
  }
  ctx.green->tables[key] = t;
  *out = t;
  return kOk;
}

// ---------------------------------------------------------------- setup

struct PmHalo {      // device copy of one PM halo's parameters
  int64_t off;       // first member
  int32_t np;
  int32_t n, sup;    // grid size and support side (n/2+1)
  float spacing;
  float origin[3];
  int64_t cell_off;  // first C2 cell
  int32_t nc[3];     // C2 cells per axis
  double u_min[3];   // C2 cell origin (q/spacing units)
  double mkeep;      // kept mass at the start of the pass (FP64)
  double cw_u;       // short-range cell width (grid units): 3.5, or 3.5/r_max two-level
  int32_t np_bound, status, pending;
  int32_t two_level; // dense regions refined on 128^3 / 216^3 inner grids
  int32_t r_max;     // largest refinement ratio of the halo's members
  int32_t pad;
};

// One refined region of a two-level halo (bound_fortran.f90:614-823)
struct TlRegion {
  int32_t h, b, r, n_in;
  float lo[3], hi[3];  // region bounds (grid units)
  float bo;            // source margin 3.5 + 3/r
  float u0[3];         // inner grid origin
};

// TSC weights and self potential (bound_fortran.f90:2562-2602).  FP32
// weights as in the reference; the self term accumulates in FP64.
template <typename R>
__global__ void pm_setup_kernel(const Members m, const PmHalo *__restrict__ H,
                                const int32_t *__restrict__ mhalo, int64_t M,
                                const R *const *__restrict__ selfs, int3 *__restrict__ first,
                                float *__restrict__ wt, R *__restrict__ selfv, int32_t *flags) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < M;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int h = mhalo[k];
    if (h < 0) continue;
    const PmHalo &p = H[h];
    float w9[9];
    int f[3];
    bool bad = false;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float t = __fdiv_rn(__fsub_rn(m.q[d][k], p.origin[d]), p.spacing);
      if (!isfinite(t)) bad = true;
      if (!(t >= 0.0f) || t >= (float)(p.n / 2 - 1)) bad = true;
      const int nearest = (int)lroundf(t);
      const float dl = __fsub_rn(t, (float)nearest);
      const float a = __fsub_rn(0.5f, dl), b = __fadd_rn(0.5f, dl);
      w9[3 * d + 0] = __fmul_rn(0.5f, __fmul_rn(a, a));
      w9[3 * d + 1] = __fsub_rn(0.75f, __fmul_rn(dl, dl));
      w9[3 * d + 2] = __fmul_rn(0.5f, __fmul_rn(b, b));
      f[d] = nearest;
    }
    if (bad) {
      atomicCAS(&flags[FLAG_ERR], 0, kInvalid);
      continue;
    }
    const R *sp = selfs[h];
    double acc = 0.0;
    for (int sz = 0; sz < 3; ++sz)
      for (int sy = 0; sy < 3; ++sy)
        for (int sx = 0; sx < 3; ++sx) {
          const float sw = __fmul_rn(__fmul_rn(w9[sx], w9[3 + sy]), w9[6 + sz]);
          for (int tz = 0; tz < 3; ++tz)
            for (int ty = 0; ty < 3; ++ty)
              for (int tx = 0; tx < 3; ++tx) {
                const float tw = __fmul_rn(__fmul_rn(w9[tx], w9[3 + ty]), w9[6 + tz]);
                acc += (double)__fmul_rn(sw, tw) *
                       (double)sp[((tz - sz + 2) * 5 + (ty - sy + 2)) * 5 + (tx - sx + 2)];
              }
        }
    selfv[k] = (R)acc;
    first[k] = make_int3(f[0], f[1], f[2]);
#pragma unroll
    for (int j = 0; j < 9; ++j) wt[9 * k + j] = w9[j];
  }
}

// u = q/spacing extent of every PM halo (bound_build_cells :3134-3138).
// Division by the positive spacing is monotone and correctly rounded, so
// min_k (q_k / s) = (min_k q_k) / s exactly: the members' FP32 extremes are
// found first (order-free integer atomics on the ordered images of the
// floats, many blocks per halo), then divided once.
__device__ __forceinline__ uint32_t flt_to_ord(float v) {
  const uint32_t b = __float_as_uint(v);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord_to_flt(uint32_t o) {
  return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

constexpr int64_t kExtentChunk = 16384;  // members per block

// One block per (halo, chunk of kExtentChunk members) of `work`; omin/omax
// (3 nh) start at 0xffffffff / 0
__global__ void __launch_bounds__(BLK) pm_extent_kernel(const Members m, const PmHalo *__restrict__ H,
                                                        const int2 *__restrict__ work,
                                                        uint32_t *__restrict__ omin, uint32_t *__restrict__ omax) {
  const int h = work[blockIdx.x].x;
  const PmHalo &p = H[h];
  const int64_t k0 = (int64_t)work[blockIdx.x].y * kExtentChunk;
  if (k0 >= p.np) return;
  const int64_t k1 = min((int64_t)p.np, k0 + kExtentChunk);
  uint32_t lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0u, 0u, 0u};
  for (int64_t k = p.off + k0 + threadIdx.x; k < p.off + k1; k += BLK)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const uint32_t o = flt_to_ord(m.q[d][k]);
      lo[d] = min(lo[d], o);
      hi[d] = max(hi[d], o);
    }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    lo[d] = __reduce_min_sync(0xffffffffu, lo[d]);
    hi[d] = __reduce_max_sync(0xffffffffu, hi[d]);
  }
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      atomicMin(&omin[3 * h + d], lo[d]);
      atomicMax(&omax[3 * h + d], hi[d]);
    }
}

__global__ void pm_extent_final_kernel(const PmHalo *__restrict__ H, int nh, const uint32_t *__restrict__ omin,
                                       const uint32_t *__restrict__ omax, double *__restrict__ ext) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * nh) return;
  const int h = i / 3, d = i % 3;
  const PmHalo &p = H[h];
  if (p.np <= 0) {
    ext[6 * h + d] = 1e30;
    ext[6 * h + 3 + d] = -1e30;
    return;
  }
  const double sp = (double)p.spacing;
  ext[6 * h + d] = (double)ord_to_flt(omin[i]) / sp;
  ext[6 * h + 3 + d] = (double)ord_to_flt(omax[i]) / sp;
}

// C2 cell key of every PM member (bound_build_cells :3166-3172), and a sort
// key that orders the members of a cell along a Morton curve of its
// (2^(sb/3))^3 sub-cells.
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
  uint32_t r = 0;
  for (int b = 0; b < 3; ++b) r |= ((v >> b) & 1u) << (3 * b);
  return r;
}

__global__ void pm_cellkey_kernel(const Members m, const PmHalo *__restrict__ H,
                                  const int32_t *__restrict__ mhalo, int64_t M,
                                  uint32_t *__restrict__ key, uint32_t sentinel, int sb,
                                  uint32_t *__restrict__ skey) {
  const int sub = 1 << (sb / 3);
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < M;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int h = mhalo[k];
    if (h < 0) {
      key[k] = sentinel;
      skey[k] = sentinel << sb;
      continue;
    }
    const PmHalo &p = H[h];
    int64_t c[3];
    uint32_t f[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double u = (double)m.q[d][k] / (double)p.spacing;
      const double g = (u - p.u_min[d]) / p.cw_u;
      double v = floor(g) + 1.0;
      if (!(v >= 1.0)) v = 1.0;
      if (v > (double)p.nc[d]) v = (double)p.nc[d];
      c[d] = (int64_t)v - 1;
      double fr = (g - (double)c[d]) * (double)sub;
      fr = fr < 0.0 ? 0.0 : (fr > (double)(sub - 1) ? (double)(sub - 1) : fr);
      f[d] = (uint32_t)fr;
    }
    const uint32_t cell = (uint32_t)(p.cell_off + c[0] + (int64_t)p.nc[0] * (c[1] + (int64_t)p.nc[1] * c[2]));
    key[k] = cell;
    skey[k] = (cell << sb) | (spread3(f[0]) | (spread3(f[1]) << 1) | (spread3(f[2]) << 2));
  }
}

__global__ void pm_cellcount_kernel(const uint32_t *__restrict__ key, int64_t M,
                                    uint32_t sentinel, uint32_t *__restrict__ cnt) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < M;
       k += (int64_t)gridDim.x * blockDim.x)
    if (key[k] != sentinel) atomicAdd(&cnt[key[k]], 1u);
}

// ---------------------------------------------------------------- passes

// Deterministic deposit.  The TSC contributions (the reference's FP32
// products w*wx*wy*wz, bound_fortran.f90:2657-2672) are added as 64-bit
// fixed-point integers: integer addition is associative, so the deposited
// grid does not depend on the order in which threads add, and every run
// gives the same bits.  The scale 2^(61 - e), e = ilogb(kept mass), keeps
// the sum of a halo's contributions below 2^62 (TSC weights sum to one per
// member); one unit is 2^-61 of the kept mass, far below FP32 rounding.
__device__ __forceinline__ int fx_exp(double mass) {
  return (mass > 0.0 && isfinite(mass)) ? ilogb(mass) : 0;
}

__device__ __forceinline__ unsigned long long fx_quantum(float v, double scale) {
  return __double2ull_rn((double)v * scale);
}

// Inverse scale of every grid of a batch: inv[j] = 2^(e - 61) of the halo
// that owns grid j (its region's halo for refined regions, A != nullptr).
__global__ void pm_batch_scale_kernel(const PmHalo *__restrict__ H, const int32_t *__restrict__ batch, int nb,
                                      const TlRegion *__restrict__ A, double *__restrict__ inv) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nb; j += gridDim.x * blockDim.x) {
    const int h = A ? A[batch[j]].h : batch[j];
    inv[j] = scalbn(1.0, fx_exp(H[h].mkeep) - 61);
  }
}

// Last entry e0 of the ascending array off[0..n] with off[e0] <= idx.
__device__ __forceinline__ int seg_of(const uint32_t *__restrict__ off, int n, uint32_t idx) {
  int lo = 0, hi = n;  // off[lo] <= idx < off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= idx) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Deposit of the kept members of a batch of halos (batch[j] = halo of
// grid j, bpre = prefix of their member counts), flat over the batch's
// members in their stored order (coalesced member reads).  Each of a
// member's 27 contributions is one 64-bit integer atomic add.
__global__ void __launch_bounds__(BLK) pm_deposit_kernel(const Members m, const PmHalo *__restrict__ H,
                                                         const int32_t *__restrict__ batch,
                                                         const uint32_t *__restrict__ bpre, int nb,
                                                         const uint8_t *__restrict__ keep,
                                                         const int3 *__restrict__ first,
                                                         const float *__restrict__ wt, int sup,
                                                         unsigned long long *__restrict__ acc) {
  const uint32_t total = bpre[nb];
  const int64_t sup3 = (int64_t)sup * sup * sup;
  for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    const int j = seg_of(bpre, nb, idx);
    const PmHalo &p = H[batch[j]];
    const int64_t k = p.off + (idx - bpre[j]);
    if (!keep[k]) continue;
    const double sc = scalbn(1.0, 61 - fx_exp(p.mkeep));
    const int3 f = first[k];
    const float *w9 = wt + 9 * k;
    const float wk = m.w[k];
    unsigned long long *g = acc + (int64_t)j * sup3;
    for (int sz = 0; sz < 3; ++sz)
      for (int sy = 0; sy < 3; ++sy)
        for (int sx = 0; sx < 3; ++sx) {
          const float v = __fmul_rn(__fmul_rn(__fmul_rn(wk, w9[sx]), w9[3 + sy]), w9[6 + sz]);
          atomicAdd(&g[((int64_t)(f.z + sz - 1) * sup + (f.y + sy - 1)) * sup + (f.x + sx - 1)],
                    fx_quantum(v, sc));
        }
  }
}

// TSC gather and the C1 potential (bound_fortran.f90:2681-2703) at the kept
// members of a batch; grid j holds the potential of halo batch[j].
template <typename R>
__global__ void pm_gather_kernel(const Members m, const PmHalo *__restrict__ H,
                                 const int32_t *__restrict__ batch, const uint32_t *__restrict__ bpre, int nb,
                                 const uint8_t *__restrict__ keep, const int3 *__restrict__ first,
                                 const float *__restrict__ wt, const R *__restrict__ selfv, int sup,
                                 const R *__restrict__ rho, double a_val, R *__restrict__ phi_c1) {
  const uint32_t total = bpre[nb];
  for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    const int j = seg_of(bpre, nb, idx);
    const PmHalo &p = H[batch[j]];
    const int64_t k = p.off + (idx - bpre[j]);
    if (!keep[k]) continue;
    const R *g = rho + (int64_t)j * sup * sup * sup;
    const int3 f = first[k];
    const float *w9 = wt + 9 * k;
    R raw = 0;
    for (int sz = 0; sz < 3; ++sz) {
      const int z = f.z + sz - 1;
      for (int sy = 0; sy < 3; ++sy) {
        const int y = f.y + sy - 1;
        for (int sx = 0; sx < 3; ++sx) {
          const int x = f.x + sx - 1;
          raw += g[((int64_t)z * sup + y) * sup + x] * (R)w9[sx] * (R)w9[3 + sy] * (R)w9[6 + sz];
        }
      }
    }
    const R wk = (R)m.w[k];
    const double rest = p.mkeep - (double)m.w[k];
    const R radius = (R)p.n / (R)2;
    const R dz0 = (R)(rest > 0.0 ? rest : 0.0) / radius;
    const R pref = (R)(a_val / (6.0 * kPi * (double)p.spacing));
    phi_c1[k] = pref * ((raw - wk * selfv[k]) - dz0);
  }
}

// bound_depth_continuous / bound_c2_delta_depth (:3080-3117)
template <typename T>
__device__ __forceinline__ T depth_c(T r, T h) {
  if (r <= (T)0) return (T)208 / ((T)70 * h);
  if (r >= h) return (T)1 / r;
  const T e = (T)2 * r / h;
  if (e <= (T)1) {
    const T prim = e * e * ((T)112 + e * e * ((T)-56 + e * ((T)14 + e * ((T)8 - (T)3 * e))));
    return ((T)208 - prim) / ((T)70 * h);
  }
  const T prim = e * e * ((T)448 + e * ((T)-280 + e * ((T)56 + e * ((T)14 + e * ((T)-8 + e))))) -
                 (T)224 * e - (T)12 / e;
  return ((T)128 - prim) / ((T)70 * h);
}

template <typename T>
__device__ __forceinline__ T c2_delta(T r, T ht, T hs) {
  if (r <= (T)0) return ((T)208 / (T)70) * ((T)1 / ht - (T)1 / hs);
  if (r >= ht && r >= hs) return (T)0;
  return depth_c<T>(r, ht) - depth_c<T>(r, hs);
}

// Short-range residual of every kept member: the spline-softened kernel
// minus the split kernel its potential already contains, over the kept
// members within the member's own cutoff a_i = 3.5 spacing / r_i, where
// r_i = 1 for plain C2 halos (bound_c2_calc_cells, :3403-3483; in grid
// units there) and the region refinement ratio for two-level halos
// (bound_two_level_pp_full, :1088-1343).  Both are
//     phi_i += w_j * -(a/(6 pi)) * (D(d, eps) - D(d, a_i)),  d < a_i.
// After a refresh the members removed since the previous pass take their
// terms back out (bound_c2_update_incremental_cells :3490-3552,
// bound_two_level_pp_update :1345-1498): UPDATE sums over those sources only
// and subtracts.
//
// Work is organised by target chunks: a warp takes up to 32 members of one
// C2 cell, in cell order (within a cell sorted by a Morton sub-key, so a
// chunk is spatially compact).  Sources are scanned cell by cell in
// coalesced batches of 32; a source enters the pair loop only if it lies
// within the chunk's largest cutoff of the chunk's bounding box, so the
// divergent pair arithmetic runs almost only on pairs that interact.  FP32
// sums are compensated (Kahan); FP64 sums are plain, which keeps the
// dependent chain per pair to one add.
// FP32 product path of the short-range kernel: the spline-softened 1/r of
// depth_c with its divisions replaced by products with per-h reciprocals and
// 1/r from rsqrtf (a few ulps; the FP64 path keeps the divisions).
struct DepthConst {
  float h, two_over_h, inv70h, six_h;
};
__device__ __forceinline__ DepthConst depth_const(float h) {
  return DepthConst{h, 2.0f / h, 1.0f / (70.0f * h), 6.0f * h};
}
__device__ __forceinline__ float depth_fast(float r, float rinv, const DepthConst &c) {
  if (r >= c.h) return rinv;
  const float e = r * c.two_over_h;
  if (e <= 1.0f) {
    const float prim = e * e * (112.0f + e * e * (-56.0f + e * (14.0f + e * (8.0f - 3.0f * e))));
    return (208.0f - prim) * c.inv70h;
  }
  // 12/e = 6 h / r
  const float prim = e * e * (448.0f + e * (-280.0f + e * (56.0f + e * (14.0f + e * (-8.0f + e))))) -
                     224.0f * e - c.six_h * rinv;
  return (128.0f - prim) * c.inv70h;
}

// FP64 path of the same kernel without divisions: 1/r from an FP32
// reciprocal square root seed refined by two Newton-Raphson steps in FP64,
// y <- y (3/2 - r2 y^2 / 2), which square the relative error each time
// (2^-22 -> ~1e-13 -> a few FP64 ulps); the per-h constants are FP64
// reciprocals.  For r2 outside the FP32 normal range the caller keeps the
// plain sqrt/division form.
struct DepthConst64 {
  double h, two_over_h, inv70h, six_h;
};
__device__ __forceinline__ DepthConst64 depth_const64(double h) {
  return DepthConst64{h, 2.0 / h, 1.0 / (70.0 * h), 6.0 * h};
}
__device__ __forceinline__ double rsqrt_nr64(double r2) {
  double y = (double)rsqrtf((float)r2);
  const double hr2 = 0.5 * r2;
  y = y * (1.5 - hr2 * y * y);
  y = y * (1.5 - hr2 * y * y);
  return y;
}
__device__ __forceinline__ double depth_fast64(double r, double rinv, const DepthConst64 &c) {
  if (r >= c.h) return rinv;
  const double e = r * c.two_over_h;
  if (e <= 1.0) {
    const double prim = e * e * (112.0 + e * e * (-56.0 + e * (14.0 + e * (8.0 - 3.0 * e))));
    return (208.0 - prim) * c.inv70h;
  }
  const double prim = e * e * (448.0 + e * (-280.0 + e * (56.0 + e * (14.0 + e * (-8.0 + e))))) -
                      224.0 * e - c.six_h * rinv;
  return (128.0 - prim) * c.inv70h;
}

struct SrChunk {
  uint32_t cell, e0;
};

template <typename R, bool UPDATE>
__global__ void __launch_bounds__(256, 4) sr_gather_kernel(
    const PmHalo *__restrict__ H, const int32_t *__restrict__ mhalo, const uint8_t *__restrict__ keep,
    const uint8_t *__restrict__ pr, const SrChunk *__restrict__ chunks, int64_t nchunks,
    const uint32_t *__restrict__ cstart, const uint32_t *__restrict__ cmem, const float4 *__restrict__ src4,
    const uint32_t *__restrict__ rpos, const uint32_t *__restrict__ rsrc, double a_val, double app,
    R *__restrict__ phi_sr, unsigned *__restrict__ next) {
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  // chunks come heaviest first; each warp takes the next one when it is
  // free (the sums of a chunk do not depend on which warp runs it)
  auto fetch = [&]() -> int64_t {
    unsigned v = 0;
    if (lane == 0) v = atomicAdd(next, 1u);
    return (int64_t)__shfl_sync(FULL, v, 0);
  };
  for (int64_t ch = fetch(); ch < nchunks; ch = fetch()) {
    const SrChunk C = chunks[ch];
    const uint32_t cend = cstart[C.cell + 1];
    const uint32_t e = C.e0 + lane;
    const bool valid = e < cend;
    const int64_t k = valid ? (int64_t)cmem[e] : -1;
    const int h = mhalo[cmem[C.e0]];
    const PmHalo &p = H[h];
    if (!p.pending) continue;
    const bool active = valid && keep[k] != 0;
    if (!__any_sync(FULL, active)) continue;
    float4 me = make_float4(0.f, 0.f, 0.f, 0.f);
    if (valid) me = src4[e];
    const double sp = (double)p.spacing;
    const int ri = active ? (int)pr[k] : 64;
    const R ai = (R)(3.5 * sp / (double)ri);
    const R a2 = ai * ai;
    // chunk bounding box of the active targets and its largest cutoff
    float lo[3] = {active ? me.x : 3e38f, active ? me.y : 3e38f, active ? me.z : 3e38f};
    float hi[3] = {active ? me.x : -3e38f, active ? me.y : -3e38f, active ? me.z : -3e38f};
    int rmin = ri;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        lo[d] = fminf(lo[d], __shfl_xor_sync(FULL, lo[d], o));
        hi[d] = fmaxf(hi[d], __shfl_xor_sync(FULL, hi[d], o));
      }
      rmin = min(rmin, __shfl_xor_sync(FULL, rmin, o));
    }
    // conservative filter radius (a little above every lane's cutoff)
    const float amax = (float)(3.5 * sp / (double)rmin) * 1.0001f + 1e-30f;
    const float amax2 = amax * amax;
    int kk = (int)ceil((3.5 / (double)rmin) / p.cw_u - 1e-9);
    kk = kk < 1 ? 1 : (kk > 4 ? 4 : kk);
    const int64_t local = (int64_t)C.cell - p.cell_off;
    const int64_t n0 = p.nc[0], n1 = p.nc[1], n2 = p.nc[2];
    const int64_t cx = local % n0, cy = (local / n0) % n1, cz = local / (n0 * n1);
    const R eps = (R)(double)(float)app;
    const R fac = (R)(a_val / (6.0 * kPi));
    const bool tl = p.two_level != 0;
    const DepthConst k_eps = depth_const((float)eps), k_ai = depth_const((float)ai);
    const DepthConst64 k64_eps = depth_const64((double)eps), k64_ai = depth_const64((double)ai);
    R acc = 0, comp = 0;
    // The (2kk+1)^3 neighbour cells, 32 at a time: a lane loads one cell's
    // source range, the ranges are concatenated by a warp prefix sum and
    // streamed in batches of 32 (a lane finds its source's cell by a binary
    // search over the prefix), so small cells share batches.
    const int wd = 2 * kk + 1, ncell = wd * wd * wd;
    for (int cb0 = 0; cb0 < ncell; cb0 += 32) {
      const int j = cb0 + lane;
      uint32_t s0 = 0, cnt = 0;
      if (j < ncell) {
        const int64_t x = cx + j % wd - kk, y = cy + (j / wd) % wd - kk, z = cz + j / (wd * wd) - kk;
        if (x >= 0 && x < n0 && y >= 0 && y < n1 && z >= 0 && z < n2) {
          const int64_t c = p.cell_off + x + n0 * (y + n1 * z);
          uint32_t a = cstart[c], b = cstart[c + 1];
          if (UPDATE) {
            a = rpos[a];
            b = rpos[b];
          }
          s0 = a;
          cnt = b - a;
        }
      }
      uint32_t incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += v;
      }
      const uint32_t excl = incl - cnt;
      const uint32_t T = __shfl_sync(FULL, incl, 31);
      for (uint32_t g0 = 0; g0 < T; g0 += 32) {
        const uint32_t g = g0 + (uint32_t)lane;
        int owner = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const uint32_t v = __shfl_sync(FULL, incl, owner + step - 1);
          if (v <= g) owner += step;
        }
        owner &= 31;
        const uint32_t os0 = __shfl_sync(FULL, s0, owner);
        const uint32_t oex = __shfl_sync(FULL, excl, owner);
        uint32_t se = 0;
        float4 sv = make_float4(0.f, 0.f, 0.f, 0.f);
        bool cand = false;
        if (g < T) {
          const uint32_t t = os0 + (g - oex);
          se = UPDATE ? rsrc[t] : t;
          sv = src4[se];
          cand = UPDATE || keep[cmem[se]] != 0;
          const float bx = fmaxf(fmaxf(lo[0] - sv.x, sv.x - hi[0]), 0.f);
          const float by = fmaxf(fmaxf(lo[1] - sv.y, sv.y - hi[1]), 0.f);
          const float bz = fmaxf(fmaxf(lo[2] - sv.z, sv.z - hi[2]), 0.f);
          cand = cand && (bx * bx + by * by + bz * bz <= amax2);
        }
        unsigned mask = __ballot_sync(FULL, cand);
        while (mask) {
          const int bl = __ffs(mask) - 1;
          mask &= mask - 1;
          const float jx = __shfl_sync(FULL, sv.x, bl), jy = __shfl_sync(FULL, sv.y, bl);
          const float jz = __shfl_sync(FULL, sv.z, bl), jw = __shfl_sync(FULL, sv.w, bl);
          const uint32_t je = __shfl_sync(FULL, se, bl);
          if (active && je != e) {
            R dx, dy, dz;
            if (tl) {
              dx = (R)jx - (R)me.x; dy = (R)jy - (R)me.y; dz = (R)jz - (R)me.z;
            } else {
              dx = (R)__fsub_rn(jx, me.x); dy = (R)__fsub_rn(jy, me.y); dz = (R)__fsub_rn(jz, me.z);
            }
            const R r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < a2) {
              R dphi;
              if constexpr (sizeof(R) == 4) {
                const float rinv = rsqrtf(r2), d = r2 * rinv;
                dphi = -(fac * (depth_fast(d, rinv, k_eps) - depth_fast(d, rinv, k_ai)));
              } else if (r2 > 1e-30 && r2 < 1e30) {
                const double rinv = rsqrt_nr64(r2), d = r2 * rinv;
                dphi = -(fac * (depth_fast64(d, rinv, k64_eps) - depth_fast64(d, rinv, k64_ai)));
              } else {
                const R d = sqrt(r2);
                dphi = -(fac * (depth_c<R>(d, eps) - depth_c<R>(d, ai)));
              }
              if constexpr (sizeof(R) == 4) {  // FP32: compensated sum
                const R yv = (R)jw * dphi - comp;
                const R tt = acc + yv;
                comp = (tt - acc) - yv;
                acc = tt;
              } else {  // FP64: a plain sum (one dependent add per pair)
                acc += (R)jw * dphi;
              }
            }
          }
        }
      }
    }
    if (active) {
      if (UPDATE) phi_sr[k] -= acc;
      else phi_sr[k] = acc;
    }
  }
}

// Cell-ordered copy of the members' positions and weights.
__global__ void sr_pack_kernel(const Members m, const uint32_t *__restrict__ cmem, int64_t n,
                               float4 *__restrict__ src4) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t k = cmem[e];
    src4[e] = make_float4(m.q[0][k], m.q[1][k], m.q[2][k], m.w[k]);
  }
}

// Target chunks: ceil(members / 32) per cell.
__global__ void sr_chunk_count_kernel(const uint32_t *__restrict__ cstart, int64_t ncell,
                                      uint32_t *__restrict__ cnt) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell;
       c += (int64_t)gridDim.x * blockDim.x)
    cnt[c] = (cstart[c + 1] - cstart[c] + 31u) / 32u;
}

__global__ void sr_chunk_fill_kernel(const uint32_t *__restrict__ cstart, const uint32_t *__restrict__ coff,
                                     int64_t ncell, SrChunk *__restrict__ chunks) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell;
       c += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t n = (cstart[c + 1] - cstart[c] + 31u) / 32u;
    for (uint32_t i = 0; i < n; ++i) chunks[coff[c] + i] = SrChunk{(uint32_t)c, cstart[c] + 32u * i};
  }
}

// Work order of the target chunks: heaviest first, the weight being the
// occupancy of the chunk's cell (the density its targets' cutoff spheres
// sample), so the dynamically fetched chunks end together.
__global__ void sr_chunk_key_kernel(const SrChunk *__restrict__ chunks, int64_t n,
                                    const uint32_t *__restrict__ cstart, uint32_t *__restrict__ key) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t c = chunks[i].cell;
    key[i] = 65535u - min(cstart[c + 1] - cstart[c], 65535u);
  }
}

__global__ void sr_chunk_order_kernel(const SrChunk *__restrict__ chunks, const uint32_t *__restrict__ idx,
                                      int64_t n, SrChunk *__restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = chunks[idx[i]];
}

// Members removed since the previous pass, in cell order: flag (and clear
// the removal mark) per cell-ordered position.
__global__ void sr_removed_flag_kernel(const uint32_t *__restrict__ cmem, int64_t n, uint8_t *__restrict__ jd,
                                       uint32_t *__restrict__ flag) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t k = cmem[e];
    flag[e] = jd[k];
    jd[k] = 0;
  }
}

__global__ void sr_removed_fill_kernel(const uint32_t *__restrict__ flag, const uint32_t *__restrict__ rpos,
                                       int64_t n, uint32_t *__restrict__ rsrc) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x)
    if (flag[e]) rsrc[rpos[e]] = (uint32_t)e;
}

// ---------------------------------------------------------------- two-level

// One refined region: halo h, region b (8x8x8 regions of 16 grid cells),
// ratio r, inner grid n_in (bound_two_level_build_halo, :614-823).
__device__ __forceinline__ void tl_t(const Members &m, const PmHalo &p, int64_t k, float *t) {
#pragma unroll
  for (int d = 0; d < 3; ++d)
    t[d] = (float)(((double)m.q[d][k] - (double)p.origin[d]) / (double)p.spacing);
}

__device__ __forceinline__ int tl_region(const float *t, int *bxyz) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int c = (int)floor((double)t[d]) / 16;
    bxyz[d] = c < 0 ? 0 : (c > 7 ? 7 : c);
  }
  return bxyz[0] + 8 * bxyz[1] + 64 * bxyz[2];
}

// fine-grid TSC of a coordinate relative to region R; false if the nodes
// leave the first half of the inner grid
__device__ __forceinline__ bool tl_tsc(const TlRegion &R, const float *t, int *f, float *w9) {
  bool ok = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float tf = __fmul_rn(__fsub_rn(t[d], R.u0[d]), (float)R.r);
    const int nearest = (int)lroundf(tf);
    const float dl = __fsub_rn(tf, (float)nearest);
    const float a = __fsub_rn(0.5f, dl), b = __fadd_rn(0.5f, dl);
    w9[3 * d + 0] = __fmul_rn(0.5f, __fmul_rn(a, a));
    w9[3 * d + 1] = __fsub_rn(0.75f, __fmul_rn(dl, dl));
    w9[3 * d + 2] = __fmul_rn(0.5f, __fmul_rn(b, b));
    f[d] = nearest;
    if (nearest < 1 || nearest + 2 > R.n_in / 2) ok = false;
  }
  return ok;
}

__global__ void tl_particle_kernel(const Members m, const PmHalo *__restrict__ H,
                                   const int32_t *__restrict__ mhalo, int64_t M,
                                   const uint8_t *__restrict__ region_r,
                                   const int32_t *__restrict__ act_of, uint8_t *__restrict__ pr,
                                   int32_t *__restrict__ preg) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < M;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int h = mhalo[k];
    if (h < 0) continue;
    const PmHalo &p = H[h];
    if (!p.two_level) { pr[k] = 1; preg[k] = -1; continue; }
    float t[3];
    int bx[3];
    tl_t(m, p, k, t);
    const int b = tl_region(t, bx);
    pr[k] = region_r[(int64_t)h * 512 + b];
    preg[k] = act_of[(int64_t)h * 512 + b];
  }
}

// Sources of every refined region: members inside the region box widened
// by 3.5 + 3/r grid cells (:685-745).  pass 0 counts, pass 1 fills.
__global__ void tl_source_kernel(const Members m, const PmHalo *__restrict__ H,
                                 const int32_t *__restrict__ mhalo, int64_t M,
                                 const int32_t *__restrict__ act_of, const TlRegion *__restrict__ A,
                                 uint32_t *__restrict__ cnt, uint32_t *__restrict__ src, int fill) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < M;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int h = mhalo[k];
    if (h < 0 || !H[h].two_level) continue;
    float t[3];
    int bx[3];
    tl_t(m, H[h], k, t);
    tl_region(t, bx);
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int x = bx[0] + dx, y = bx[1] + dy, z = bx[2] + dz;
          if (x < 0 || x > 7 || y < 0 || y > 7 || z < 0 || z > 7) continue;
          const int a = act_of[(int64_t)h * 512 + x + 8 * y + 64 * z];
          if (a < 0) continue;
          const TlRegion &R = A[a];
          bool in = true;
#pragma unroll
          for (int d = 0; d < 3; ++d)
            in = in && t[d] >= __fsub_rn(R.lo[d], R.bo) && t[d] <= __fadd_rn(R.hi[d], R.bo);
          if (!in) continue;
          const uint32_t pos = atomicAdd(&cnt[a], 1u);
          if (fill) src[pos] = (uint32_t)k;
        }
  }
}

// Targets of every refined region: its own members (pass 0 counts, 1 fills)
__global__ void tl_target_kernel(const int32_t *__restrict__ preg, int64_t M,
                                 uint32_t *__restrict__ cnt, uint32_t *__restrict__ tgt, int fill) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < M;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int a = preg[k];
    if (a < 0) continue;
    const uint32_t pos = atomicAdd(&cnt[a], 1u);
    if (fill) tgt[pos] = (uint32_t)k;
  }
}

// Node range checks of sources and targets, and the inner self term of
// every target (:729-800).
// Set-up of the refined regions, flat over all their sources and targets:
// every source must fall inside its region's inner grid, and every target
// gets its inner self term.
__global__ void tl_check_kernel(const Members m, const PmHalo *__restrict__ H,
                                const TlRegion *__restrict__ A, int na,
                                const uint32_t *__restrict__ src_start, const uint32_t *__restrict__ src,
                                int32_t *flags) {
  const uint32_t total = src_start[na];
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int a = seg_of(src_start, na, e);
    const TlRegion &Rg = A[a];
    float t[3], w9[9];
    int f[3];
    tl_t(m, H[Rg.h], src[e], t);
    if (!tl_tsc(Rg, t, f, w9)) atomicCAS(&flags[FLAG_ERR], 0, kInvalid);
  }
}

template <typename R>
__global__ void tl_self_kernel(const Members m, const PmHalo *__restrict__ H,
                               const TlRegion *__restrict__ A, int na,
                               const uint32_t *__restrict__ tgt_start, const uint32_t *__restrict__ tgt,
                               const R *__restrict__ self2, const R *__restrict__ self4,
                               R *__restrict__ self_in, int32_t *flags) {
  const uint32_t total = tgt_start[na];
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int a = seg_of(tgt_start, na, e);
    const TlRegion &Rg = A[a];
    const R *sp = Rg.r == 2 ? self2 : self4;
    const int64_t k = tgt[e];
    float t[3], w9[9];
    int f[3];
    tl_t(m, H[Rg.h], k, t);
    if (!tl_tsc(Rg, t, f, w9)) { atomicCAS(&flags[FLAG_ERR], 0, kInvalid); continue; }
    double acc = 0.0;
    for (int sz = 0; sz < 3; ++sz)
      for (int sy = 0; sy < 3; ++sy)
        for (int sx = 0; sx < 3; ++sx) {
          const float sw = __fmul_rn(__fmul_rn(w9[sx], w9[3 + sy]), w9[6 + sz]);
          for (int tz = 0; tz < 3; ++tz)
            for (int ty = 0; ty < 3; ++ty)
              for (int tx = 0; tx < 3; ++tx) {
                const float tw = __fmul_rn(__fmul_rn(w9[tx], w9[3 + ty]), w9[6 + tz]);
                acc += (double)__fmul_rn(sw, tw) *
                       (double)sp[((tz - sz + 2) * 5 + (ty - sy + 2)) * 5 + (tx - sx + 2)];
              }
        }
    self_in[k] = (R)acc;
  }
}

// Inner PM of a batch of refined regions of one inner grid size
// (bound_two_level_run_pm, :825-942): deposit of the kept sources ...
__global__ void tl_deposit_kernel(const Members m, const PmHalo *__restrict__ H,
                                  const TlRegion *__restrict__ A, const int32_t *__restrict__ batch,
                                  const uint32_t *__restrict__ bpre, int nb,
                                  const uint32_t *__restrict__ src_start, const uint32_t *__restrict__ src,
                                  const uint8_t *__restrict__ keep, int sup,
                                  unsigned long long *__restrict__ acc) {
  // flat over the sources of the batch: bpre[j] = first index of region j;
  // fixed-point integer adds as pm_deposit_kernel (order-independent)
  const uint32_t total = bpre[nb];
  for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    const int j = seg_of(bpre, nb, idx);
    const int a = batch[j];
    const TlRegion &Rg = A[a];
    const PmHalo &p = H[Rg.h];
    const int64_t k = src[src_start[a] + (idx - bpre[j])];
    if (!keep[k]) continue;
    unsigned long long *g = acc + (int64_t)j * sup * sup * sup;
    const double sc = scalbn(1.0, 61 - fx_exp(p.mkeep));
    float t[3], w9[9];
    int f[3];
    tl_t(m, p, k, t);
    tl_tsc(Rg, t, f, w9);
    const float wk = m.w[k];
    for (int sz = 0; sz < 3; ++sz)
      for (int sy = 0; sy < 3; ++sy)
        for (int sx = 0; sx < 3; ++sx) {
          const float v = __fmul_rn(__fmul_rn(__fmul_rn(wk, w9[sx]), w9[3 + sy]), w9[6 + sz]);
          atomicAdd(&g[((int64_t)(f[2] + sz - 1) * sup + (f[1] + sy - 1)) * sup + (f[0] + sx - 1)],
                    fx_quantum(v, sc));
        }
  }
}

// ... and gather at the kept targets: phi_in = a r/(6 pi sp) (raw - w self_in)
template <typename R>
__global__ void tl_gather_kernel(const Members m, const PmHalo *__restrict__ H,
                                 const TlRegion *__restrict__ A, const int32_t *__restrict__ batch,
                                 const uint32_t *__restrict__ bpre, int nb,
                                 const uint32_t *__restrict__ tgt_start, const uint32_t *__restrict__ tgt,
                                 const uint8_t *__restrict__ keep, const R *__restrict__ self_in, int sup,
                                 const R *__restrict__ rho, double a_val, R *__restrict__ phi_in) {
  const uint32_t total = bpre[nb];
  for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    const int j = seg_of(bpre, nb, idx);
    const int a = batch[j];
    const TlRegion &Rg = A[a];
    const PmHalo &p = H[Rg.h];
    const int64_t k = tgt[tgt_start[a] + (idx - bpre[j])];
    if (!keep[k]) continue;
    const R *g = rho + (int64_t)j * sup * sup * sup;
    const R pref = (R)(a_val * (double)Rg.r / (6.0 * kPi * (double)p.spacing));
    float t[3], w9[9];
    int f[3];
    tl_t(m, p, k, t);
    tl_tsc(Rg, t, f, w9);
    R raw = 0;
    for (int sz = 0; sz < 3; ++sz)
      for (int sy = 0; sy < 3; ++sy)
        for (int sx = 0; sx < 3; ++sx)
          raw += g[((int64_t)(f[2] + sz - 1) * sup + (f[1] + sy - 1)) * sup + (f[0] + sx - 1)] *
                 (R)w9[sx] * (R)w9[3 + sy] * (R)w9[6 + sz];
    phi_in[k] = pref * (raw - (R)m.w[k] * self_in[k]);
  }
}

// ---------------------------------------------------------------- removal

__device__ __forceinline__ double bsum_d(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  __syncthreads();
  return t;
}

__device__ __forceinline__ int bsum_i(int v, int *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  int t = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  __syncthreads();
  return t;
}

// Seven block sums at once: each value is reduced in the same order as by
// bsum_d (warp butterfly, then the warp partials in warp order), so the
// results are bit-identical, with 2 barriers instead of 21.
__device__ __forceinline__ void bsum7_d(double *v, double *red) {
  constexpr int NW = IBLK / 32;
#pragma unroll
  for (int j = 0; j < 7; ++j)
    for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_xor_sync(0xffffffffu, v[j], o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int j = 0; j < 7; ++j) red[j * NW + (threadIdx.x >> 5)] = v[j];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[j * NW + w];
    v[j] = t;
  }
}

// One block per pending halo: combine the potential, then the inner
// removal loop of bound_check_grid (:2739-2855).  Leaves status -1 when the
// potential must be refreshed (next pass).
template <typename R>
__global__ void __launch_bounds__(IBLK) pm_inner_kernel(const Members m, PmHalo *__restrict__ H,
                                                        const int32_t *__restrict__ list, int nlist,
                                                        uint8_t *__restrict__ keep,
                                                        uint8_t *__restrict__ jd,
                                                        const R *__restrict__ phi_c1,
                                                        const R *__restrict__ phi_in,
                                                        const R *__restrict__ phi_c2,
                                                        float *__restrict__ phi,
                                                        float *__restrict__ en, float b_val, int nmin,
                                                        int phi_only, int32_t *flags) {
  const int h = list[blockIdx.x];
  PmHalo &p = H[h];
  if (!p.pending) return;
  __shared__ double red7[7 * (IBLK / 32)];
  __shared__ int red_i[IBLK / 32];
  __shared__ unsigned hist[256];
  __shared__ int s_err;
  const int64_t b0 = p.off, np = p.np;
  if (threadIdx.x == 0) s_err = 0;
  int np_bound = p.np_bound;
  const int n_source = np_bound;
  for (int64_t i = threadIdx.x; i < np; i += IBLK) {
    const int64_t k = b0 + i;
    if (!keep[k]) continue;
    float v = (float)((phi_c1[k] + phi_in[k]) + phi_c2[k]);
    if (np_bound == 1 || n_source == 1) v = 0.0f;
    if (!isfinite(v)) s_err = kNonFinite;
    phi[k] = v;
  }
  __syncthreads();
  if (s_err) {
    if (threadIdx.x == 0) atomicCAS(&flags[FLAG_ERR], 0, s_err);
    return;
  }
  if (phi_only) {
    if (threadIdx.x == 0) { p.status = 0; p.pending = 0; }
    return;
  }
  int deleted = 0, status = -1;
  for (;;) {
    double a7[7] = {0, 0, 0, 0, 0, 0, 0};
    // top-digit histogram of the energies, filled by the energy sweep below
    for (int t = threadIdx.x; t < 256; t += IBLK) hist[t] = 0;
    for (int64_t i = threadIdx.x; i < np; i += IBLK) {
      const int64_t k = b0 + i;
      if (!keep[k]) continue;
      const double wi = (double)m.w[k];
      a7[0] += wi;
      for (int d = 0; d < 3; ++d) { a7[1 + d] += wi * (double)m.q[d][k]; a7[4 + d] += wi * (double)m.v[d][k]; }
    }
    bsum7_d(a7, red7);
    float qc[3], vc[3];
    for (int d = 0; d < 3; ++d) {
      qc[d] = __double2float_rn(a7[1 + d] / a7[0]);
      vc[d] = __double2float_rn(a7[4 + d] / a7[0]);
    }
    int nu = 0;
    for (int64_t i = threadIdx.x; i < np; i += IBLK) {
      const int64_t k = b0 + i;
      if (!keep[k]) continue;
      float s = 0.f;
      for (int d = 0; d < 3; ++d) {
        const float dv = __fadd_rn(__fsub_rn(m.v[d][k], vc[d]), __fmul_rn(b_val, __fsub_rn(m.q[d][k], qc[d])));
        s = d == 0 ? __fmul_rn(dv, dv) : __fadd_rn(s, __fmul_rn(dv, dv));
      }
      const float e = __fadd_rn(__fdiv_rn(s, 2.0f), phi[k]);
      if (!isfinite(e)) s_err = kInvalid;
      en[k] = e;
      nu += e >= 0.0f;
      if (e >= 0.0f) atomicAdd(&hist[__float_as_uint(e + 0.0f) >> 24], 1u);
    }
    nu = bsum_i(nu, red_i);
    if (s_err) break;
    if (nu == 0) {
      if (deleted == 0) status = 0;
      break;
    }
    int nb = max(1, (int)ceil(0.02 * (double)np_bound));
    nb = min(nu, nb);
    // radix select of the nb largest energies among the unbound members:
    // key = bits of (E + 0) (E >= 0, so the bits order like the values)
    unsigned prefix = 0, mask = 0;
    int need = nb, n_eq = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
      if (shift != 24) {  // the top digit's histogram came with the energies
        for (int t = threadIdx.x; t < 256; t += IBLK) hist[t] = 0;
        __syncthreads();
        for (int64_t i = threadIdx.x; i < np; i += IBLK) {
          const int64_t k = b0 + i;
          if (!keep[k]) continue;
          const float e = en[k];
          if (!(e >= 0.0f)) continue;
          const unsigned key = __float_as_uint(e + 0.0f);
          if ((key & mask) != prefix) continue;
          atomicAdd(&hist[(key >> shift) & 255u], 1u);
        }
        __syncthreads();
      }
      // digit holding the need-th largest key
      int digit = 255, above = 0;
      for (; digit >= 0; --digit) {
        const int c = (int)hist[digit];
        if (above + c >= need) {
          n_eq = c;  // at shift 0: the members whose key equals the threshold
          break;
        }
        above += c;
      }
      __syncthreads();
      need -= above;
      prefix |= (unsigned)digit << shift;
      mask |= 255u << shift;
    }
    // delete every key > threshold and the `need` lowest indices among
    // key == threshold (equal energies: lower index first)
    const unsigned thr = prefix;
    if (need == n_eq) {
      // every member at the threshold goes: no index order needed
      for (int64_t i = threadIdx.x; i < np; i += IBLK) {
        const int64_t k = b0 + i;
        if (!keep[k]) continue;
        const float e = en[k];
        if (e >= 0.0f && __float_as_uint(e + 0.0f) >= thr) {
          keep[k] = 0;
          jd[k] = 1;
        }
      }
      __syncthreads();
    }
    int taken_eq = 0;
    for (int64_t base = 0; base < (need == n_eq ? 0 : np); base += IBLK) {
      const int64_t i = base + threadIdx.x;
      int64_t k = b0 + i;
      bool del_gt = false, is_eq = false;
      if (i < np && keep[k]) {
        const float e = en[k];
        if (e >= 0.0f) {
          const unsigned key = __float_as_uint(e + 0.0f);
          del_gt = key > thr;
          is_eq = key == thr;
        }
      }
      // ordered rank of is_eq within this chunk
      const unsigned bal = __ballot_sync(0xffffffffu, is_eq);
      const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
      __syncthreads();
      if (lane == 0) red_i[warp] = __popc(bal);
      __syncthreads();
      int before = taken_eq;
      for (int w = 0; w < warp; ++w) before += red_i[w];
      before += __popc(bal & ((1u << lane) - 1u));
      int chunk_eq = 0;
      for (int w = 0; w < IBLK / 32; ++w) chunk_eq += red_i[w];
      if (i < np && (del_gt || (is_eq && before < need))) {
        keep[k] = 0;
        jd[k] = 1;
      }
      taken_eq += chunk_eq;
      __syncthreads();
    }
    np_bound -= nb;
    deleted += nb;
    if (np_bound < nmin) { status = 1; break; }
    if ((double)deleted >= 0.2 * (double)np_bound) break;
  }
  __syncthreads();
  if (s_err) {
    if (threadIdx.x == 0) atomicCAS(&flags[FLAG_ERR], 0, s_err);
    return;
  }
  if (threadIdx.x == 0) {
    p.np_bound = np_bound;
    p.status = status;
    if (status >= 0) p.pending = 0;
  }
}

// ------------------------------------------------- removal of large halos
// Halos above kBigNp members run the same removal loop as pm_inner_kernel,
// but spread over the whole GPU: their members are cut into chunks of
// kChunk, every sweep is a grid of chunk blocks, and the per-halo decisions
// (centre, selection, stop conditions) are small kernels between sweeps,
// driven by a host loop.  The unbound members of an iteration are compacted
// into a per-halo list, so the radix select runs over that list only.

constexpr int64_t kBigNp = 32768;  // default; option "unbind_big_np" overrides
constexpr int kChunk = 8192;

struct BigHalo {
  int32_t h;          // index into the PM halo table
  int32_t active;     // still in this pass's inner loop
  int64_t off, np;    // members
  int64_t uoff;       // first slot of the halo's unbound list
  int32_t chunk0, nchunk;
  int32_t np_bound, deleted, n_source, status;
  int32_t nu, nb;
  float qc[3], vc[3];
};

struct BigChunk {
  int32_t b;          // big halo
  int64_t start, end; // member range
};

// phi = (c1 + in) + c2 of the kept members at the start of a pass
template <typename R>
__global__ void big_phi_kernel(const BigChunk *__restrict__ ch, int nch, const BigHalo *__restrict__ B,
                               const uint8_t *__restrict__ keep, const R *__restrict__ c1,
                               const R *__restrict__ in, const R *__restrict__ c2, float *__restrict__ phi,
                               int32_t *flags) {
  const BigChunk c = ch[blockIdx.x];
  const BigHalo &bh = B[c.b];
  if (!bh.active) return;
  bool bad = false;
  for (int64_t k = c.start + threadIdx.x; k < c.end; k += blockDim.x) {
    if (!keep[k]) continue;
    float v = (float)((c1[k] + in[k]) + c2[k]);
    if (bh.np_bound == 1 || bh.n_source == 1) v = 0.0f;
    bad |= !isfinite(v);
    phi[k] = v;
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicCAS(&flags[FLAG_ERR], 0, kNonFinite);
}

// per-chunk sums of w, w q, w v over the kept members
__global__ void big_com_kernel(const Members m, const BigChunk *__restrict__ ch, const BigHalo *__restrict__ B,
                               const uint8_t *__restrict__ keep, double *__restrict__ part) {
  const BigChunk c = ch[blockIdx.x];
  if (!B[c.b].active) return;
  double a7[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int64_t k = c.start + threadIdx.x; k < c.end; k += blockDim.x) {
    if (!keep[k]) continue;
    const double wi = (double)m.w[k];
    a7[0] += wi;
    for (int d = 0; d < 3; ++d) { a7[1 + d] += wi * (double)m.q[d][k]; a7[4 + d] += wi * (double)m.v[d][k]; }
  }
  __shared__ double red[32];
  for (int j = 0; j < 7; ++j) {
    const double t = bsum_d(a7[j], red);
    if (threadIdx.x == 0) part[7 * (int64_t)blockIdx.x + j] = t;
  }
}

// per big halo: centre from the chunk sums (in chunk order)
__global__ void big_center_kernel(BigHalo *__restrict__ B, int nbig, const double *__restrict__ part,
                                  int32_t *__restrict__ ucount) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbig) return;
  BigHalo &bh = B[b];
  ucount[b] = 0;
  if (!bh.active) return;
  double a7[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int c = bh.chunk0; c < bh.chunk0 + bh.nchunk; ++c)
    for (int j = 0; j < 7; ++j) a7[j] += part[7 * (int64_t)c + j];
  for (int d = 0; d < 3; ++d) {
    bh.qc[d] = __double2float_rn(a7[1 + d] / a7[0]);
    bh.vc[d] = __double2float_rn(a7[4 + d] / a7[0]);
  }
}

// energies of the kept members; the unbound ones join the halo's list
__global__ void big_energy_kernel(const Members m, const BigChunk *__restrict__ ch, const BigHalo *__restrict__ B,
                                  const uint8_t *__restrict__ keep, const float *__restrict__ phi,
                                  float *__restrict__ en, float b_val, int32_t *__restrict__ ucount,
                                  uint32_t *__restrict__ ulist, int32_t *flags) {
  const BigChunk c = ch[blockIdx.x];
  const BigHalo &bh = B[c.b];
  if (!bh.active) return;
  bool bad = false;
  const int lane = threadIdx.x & 31;
  for (int64_t base = c.start; base < c.end; base += blockDim.x) {
    const int64_t k = base + threadIdx.x;
    bool unb = false;
    if (k < c.end && keep[k]) {
      float s = 0.f;
      for (int d = 0; d < 3; ++d) {
        const float dv = __fadd_rn(__fsub_rn(m.v[d][k], bh.vc[d]), __fmul_rn(b_val, __fsub_rn(m.q[d][k], bh.qc[d])));
        s = d == 0 ? __fmul_rn(dv, dv) : __fadd_rn(s, __fmul_rn(dv, dv));
      }
      const float e = __fadd_rn(__fdiv_rn(s, 2.0f), phi[k]);
      bad |= !isfinite(e);
      en[k] = e;
      unb = e >= 0.0f;
    }
    // warp-aggregated append
    const unsigned bal = __ballot_sync(0xffffffffu, unb);
    int basepos = 0;
    if (lane == 0 && bal) basepos = atomicAdd(&ucount[c.b], __popc(bal));
    basepos = __shfl_sync(0xffffffffu, basepos, 0);
    if (unb) ulist[bh.uoff + basepos + __popc(bal & ((1u << lane) - 1u))] = (uint32_t)(k - bh.off);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicCAS(&flags[FLAG_ERR], 0, kInvalid);
}

// per big halo, one block: the nb most unbound members leave (radix select
// over the compact list; equal energies: lower index first), then the stop
// conditions of the inner loop
__global__ void __launch_bounds__(IBLK) big_select_kernel(BigHalo *__restrict__ B, const int32_t *__restrict__ ucount,
                                                          const uint32_t *__restrict__ ulist,
                                                          uint32_t *__restrict__ eqbuf,
                                                          const float *__restrict__ en,
                                                          uint8_t *__restrict__ keep, uint8_t *__restrict__ jd,
                                                          int nmin, int32_t *__restrict__ nactive,
                                                          const int32_t *flags) {
  BigHalo &bh = B[blockIdx.x];
  if (!bh.active) return;
  __shared__ unsigned hist[IBLK / 32][64];  // per-warp 6-bit digit histograms
  __shared__ unsigned tot[64];
  __shared__ int s_digit, s_above, s_neq;
  if (flags[FLAG_ERR]) {  // a sweep failed: stop, the host reports it
    if (threadIdx.x == 0) { bh.active = 0; atomicSub(nactive, 1); }
    return;
  }
  const int nu = ucount[blockIdx.x];
  if (nu == 0) {
    if (threadIdx.x == 0) {
      if (bh.deleted == 0) bh.status = 0;
      bh.active = 0;
      atomicSub(nactive, 1);
    }
    return;
  }
  const int nb = min(nu, max(1, (int)ceil(0.02 * (double)bh.np_bound)));
  const uint32_t *L = ulist + bh.uoff;
  const float *E = en + bh.off;
  const int warp = threadIdx.x >> 5;
  unsigned prefix = 0, mask = 0;
  int need = nb;
  // 32-bit keys in digits of 6 bits from the top: 2 + 5 x 6
  for (int shift = 30; shift >= 0; shift -= 6) {
    const int bits = shift == 30 ? 2 : 6;
    const unsigned dm = (1u << bits) - 1u;
    for (int t = threadIdx.x; t < (IBLK / 32) * 64; t += IBLK) (&hist[0][0])[t] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < nu; i += IBLK) {
      const unsigned key = __float_as_uint(E[L[i]] + 0.0f);
      if ((key & mask) != prefix) continue;
      atomicAdd(&hist[warp][(key >> shift) & dm], 1u);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 64; t += IBLK) {
      unsigned s = 0;
      for (int w = 0; w < IBLK / 32; ++w) s += hist[w][t];
      tot[t] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int digit = (int)dm, above = 0;
      for (; digit >= 0; --digit) {
        const int c = (int)tot[digit];
        if (above + c >= need) break;
        above += c;
      }
      s_digit = digit;
      s_above = above;
    }
    __syncthreads();
    need -= s_above;
    prefix |= (unsigned)s_digit << shift;
    mask |= dm << shift;
    __syncthreads();
  }
  const unsigned thr = prefix;
  if (threadIdx.x == 0) s_neq = 0;
  __syncthreads();
  uint32_t *EQ = eqbuf + bh.uoff;
  for (int i = threadIdx.x; i < nu; i += IBLK) {
    const uint32_t li = L[i];
    const unsigned key = __float_as_uint(E[li] + 0.0f);
    if (key > thr) {
      keep[bh.off + li] = 0;
      jd[bh.off + li] = 1;
    } else if (key == thr) {
      EQ[atomicAdd(&s_neq, 1)] = li;
    }
  }
  __syncthreads();
  const int neq = s_neq;
  for (int i = threadIdx.x; i < neq; i += IBLK) {
    const uint32_t li = EQ[i];
    int rank = 0;
    for (int j = 0; j < neq; ++j) rank += EQ[j] < li;
    if (rank < need) {
      keep[bh.off + li] = 0;
      jd[bh.off + li] = 1;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    bh.np_bound -= nb;
    bh.deleted += nb;
    if (bh.np_bound < nmin) {
      bh.status = 1;
      bh.active = 0;
      atomicSub(nactive, 1);
    } else if ((double)bh.deleted >= 0.2 * (double)bh.np_bound) {
      bh.active = 0;
      atomicSub(nactive, 1);
    }
  }
}

// the pass's outcome back into the PM halo table
__global__ void big_finish_kernel(const BigHalo *__restrict__ B, int nbig, PmHalo *__restrict__ H) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbig) return;
  const BigHalo &bh = B[b];
  PmHalo &p = H[bh.h];
  if (!p.pending) return;
  p.np_bound = bh.np_bound;
  p.status = bh.status;
  if (bh.status >= 0) p.pending = 0;
}

// start of a pass: the pending big halos enter the inner loop
__global__ void big_start_kernel(BigHalo *__restrict__ B, int nbig, const PmHalo *__restrict__ H, int phi_only,
                                 int32_t *__restrict__ nactive) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbig) return;
  BigHalo &bh = B[b];
  const PmHalo &p = H[bh.h];
  bh.active = p.pending ? 1 : 0;
  bh.np_bound = p.np_bound;
  bh.n_source = p.np_bound;
  bh.deleted = 0;
  bh.status = -1;
  if (bh.active) atomicAdd(nactive, 1);
  (void)phi_only;
}

__global__ void big_phi_only_kernel(BigHalo *__restrict__ B, int nbig) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbig || !B[b].active) return;
  B[b].status = 0;
  B[b].active = 0;
}

// pm_mkeep_kernel of the big halos: chunk sums of the kept mass, then the
// ordered sum per halo
__global__ void big_mass_kernel(const Members m, const BigChunk *__restrict__ ch, const BigHalo *__restrict__ B,
                                const PmHalo *__restrict__ H, const uint8_t *__restrict__ keep,
                                double *__restrict__ part) {
  const BigChunk c = ch[blockIdx.x];
  if (!H[B[c.b].h].pending) return;
  double s = 0.0;
  for (int64_t k = c.start + threadIdx.x; k < c.end; k += blockDim.x)
    if (keep[k]) s += (double)m.w[k];
  __shared__ double red[32];
  s = bsum_d(s, red);
  if (threadIdx.x == 0) part[7 * (int64_t)blockIdx.x] = s;
}

__global__ void big_mass_sum_kernel(const BigHalo *__restrict__ B, int nbig, const double *__restrict__ part,
                                    PmHalo *__restrict__ H) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbig) return;
  const BigHalo &bh = B[b];
  PmHalo &p = H[bh.h];
  if (!p.pending) return;
  double s = 0.0;
  for (int c = bh.chunk0; c < bh.chunk0 + bh.nchunk; ++c) s += part[7 * (int64_t)c];
  p.mkeep = s;
}

__global__ void pm_mkeep_kernel(const Members m, PmHalo *__restrict__ H, const int32_t *list, int nlist,
                                const uint8_t *__restrict__ keep) {
  const int h = list[blockIdx.x];
  PmHalo &p = H[h];
  if (!p.pending) return;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < p.np; i += blockDim.x) {
    const int64_t k = p.off + i;
    if (keep[k]) s += (double)m.w[k];
  }
  __shared__ double red[32];
  s = bsum_d(s, red);
  if (threadIdx.x == 0) p.mkeep = s;
}

__global__ void pm_mark_halo_kernel(const PmHalo *__restrict__ H, int nh, int32_t *__restrict__ mhalo) {
  const int h = blockIdx.x;
  if (h >= nh) return;
  for (int64_t i = threadIdx.x; i < H[h].np; i += blockDim.x) mhalo[H[h].off + i] = h;
}

__global__ void pm_fill_i32(int32_t *a, int64_t n, int32_t v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    a[i] = v;
}

__global__ void pm_fill_u8(uint8_t *a, int64_t n, uint8_t v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    a[i] = v;
}

// Members per 16-cell region of every 256-grid halo
// (bound_two_level_setup_ratios, bound_fortran.f90:551-568).
__global__ void pm_region_count_kernel(const Members m, const PmHalo *__restrict__ H,
                                       const int32_t *__restrict__ mhalo, int64_t M,
                                       uint32_t *__restrict__ cnt) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < M;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int h = mhalo[k];
    if (h < 0 || H[h].n != 256) continue;
    const PmHalo &p = H[h];
    int b[3];
    for (int d = 0; d < 3; ++d) {
      const float t = (float)(((double)m.q[d][k] - (double)p.origin[d]) / (double)p.spacing);
      const int c = (int)floor((double)t) / 16;
      b[d] = c < 0 ? 0 : (c > 7 ? 7 : c);
    }
    atomicAdd(&cnt[(int64_t)h * 512 + b[0] + 8 * b[1] + 64 * b[2]], 1u);
  }
}

int bits_for(uint64_t v) {
  int b = 0;
  while (b < 64 && (v >> b) != 0) ++b;
  return b;
}

// One pass of the removal loop of the large halos (see BigHalo).
template <typename R>
int32_t big_removal(Context &ctx, const Members &m, BigHalo *dB, int nbig, const BigChunk *dCh, int nchb,
                    PmHalo *dH, uint8_t *keep, uint8_t *jd, const R *c1, const R *phi_in, const R *c2,
                    float *phi, float *en, double *part, int32_t *ucount, uint32_t *ulist, uint32_t *eqbuf,
                    int32_t *nactive, float b_val, int nmin, int phi_only) {
  cudaStream_t s = ctx.stream;
  const unsigned gb = (unsigned)ceil_div(nbig, 128);
  PYFOF_CUDA(cudaMemsetAsync(nactive, 0, sizeof(int32_t), s));
  big_start_kernel<<<gb, 128, 0, s>>>(dB, nbig, dH, phi_only, nactive);
  PYFOF_CHECK_LAUNCH();
  big_phi_kernel<R><<<nchb, 256, 0, s>>>(dCh, nchb, dB, keep, c1, phi_in, c2, phi, ctx.d_flags);
  PYFOF_CHECK_LAUNCH();
  if (phi_only) {
    big_phi_only_kernel<<<gb, 128, 0, s>>>(dB, nbig);
    PYFOF_CHECK_LAUNCH();
  } else {
    // iterations until every big halo left the inner loop; the host looks
    // every few iterations (an iteration removes >= 2 % of a halo, and a pass
    // ends after 20 %)
    PYFOF_CUDA(wait_velocities(ctx, s));
    for (int it = 0; it < 1 << 20; it += 4) {
      for (int j = 0; j < 4; ++j) {
        big_com_kernel<<<nchb, 256, 0, s>>>(m, dCh, dB, keep, part);
        PYFOF_CHECK_LAUNCH();
        big_center_kernel<<<gb, 128, 0, s>>>(dB, nbig, part, ucount);
        PYFOF_CHECK_LAUNCH();
        big_energy_kernel<<<nchb, 256, 0, s>>>(m, dCh, dB, keep, phi, en, b_val, ucount, ulist, ctx.d_flags);
        PYFOF_CHECK_LAUNCH();
        big_select_kernel<<<nbig, IBLK, 0, s>>>(dB, ucount, ulist, eqbuf, en, keep, jd, nmin, nactive,
                                                ctx.d_flags);
        PYFOF_CHECK_LAUNCH();
      }
      PYFOF_CUDA(cudaMemcpyAsync(ctx.h_flags + FLAG_COUNT_B, nactive, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      PYFOF_CUDA(cudaStreamSynchronize(s));
      if (ctx.h_flags[FLAG_COUNT_B] <= 0) break;
    }
  }
  big_finish_kernel<<<gb, 128, 0, s>>>(dB, nbig, dH);
  PYFOF_CHECK_LAUNCH();
  return kOk;
}

template <typename R>
int32_t run_pm(Context &ctx, const FofArgs &a, const GridRules &rules, const Members &m,
               const std::vector<HaloTask> &tasks, const std::vector<int32_t> &list,
               HaloResult *res, uint8_t *keep, float *phi_out, int phi_only) {
  (void)rules;
  cudaStream_t s = ctx.stream;
  Arena &W = ctx.work;
  const int nh = (int)list.size();
  const int64_t M = tasks.back().off + tasks.back().np;  // all packed members
  // Green tables of the grid classes in use
  std::shared_ptr<GreenTable> green_of[257];
  std::vector<PmHalo> H(nh);
  std::vector<const R *> selfs(nh);
  for (int h = 0; h < nh; ++h) {
    const HaloTask &t = tasks[list[h]];
    PmHalo &p = H[h];
    std::memset(&p, 0, sizeof(p));
    p.off = t.off;
    p.np = t.np;
    p.n = t.n;
    p.sup = t.n / 2 + 1;
    p.spacing = t.spacing;
    for (int d = 0; d < 3; ++d) p.origin[d] = t.origin[d];
    p.np_bound = t.np;
    p.status = -1;
    p.pending = 1;
    if (!green_of[t.n]) PYFOF_TRY(get_green<R>(ctx, t.n, 3.5, 0.0, 1, &green_of[t.n]));
    selfs[h] = (const R *)green_of[t.n]->self;
  }
  PmHalo *dH = W.carve<PmHalo>(nh);
  int32_t *dlist = W.carve<int32_t>(nh);
  const R **dselfs = W.carve<const R *>(nh);
  int32_t *mhalo = W.carve<int32_t>(M);
  int3 *first = W.carve<int3>(M);
  float *wt = W.carve<float>(9 * (size_t)M);
  R *selfv = W.carve<R>(M), *c1 = W.carve<R>(M), *c2 = W.carve<R>(M);
  float *phi = W.carve<float>(M), *en = W.carve<float>(M);
  R *tl_self_in = nullptr;
  uint8_t *jd = W.carve<uint8_t>(M);  // removed since the previous pass
  if (!jd) { set_error("workspace exhausted (removal marks)"); return kAlloc; }
  PYFOF_CUDA(cudaMemsetAsync(jd, 0, M, s));
  double *ext = W.carve<double>(6 * (size_t)nh);
  if (!dH || !dlist || !dselfs || !mhalo || !first || !wt || !selfv || !c1 || !c2 || !phi || !en || !ext) {
    set_error("workspace exhausted (PM members)");
    return kAlloc;
  }
  std::vector<int32_t> hl(nh);
  for (int h = 0; h < nh; ++h) hl[h] = h;
  PYFOF_TRY(upload(ctx, dH, H.data(), sizeof(PmHalo) * nh, s));
  PYFOF_TRY(upload(ctx, dlist, hl.data(), sizeof(int32_t) * nh, s));
  PYFOF_TRY(upload(ctx, dselfs, selfs.data(), sizeof(R *) * nh, s));
  const unsigned gM = (unsigned)std::min<int64_t>(ceil_div(M, BLK), (int64_t)kNumSMs * 16);
  pm_fill_i32<<<gM, BLK, 0, s>>>(mhalo, M, -1);
  PYFOF_CHECK_LAUNCH();
  pm_mark_halo_kernel<<<nh, BLK, 0, s>>>(dH, nh, mhalo);
  PYFOF_CHECK_LAUNCH();
  pm_setup_kernel<R><<<gM, BLK, 0, s>>>(m, dH, mhalo, M, dselfs, first, wt, selfv, ctx.d_flags);
  PYFOF_CHECK_LAUNCH();
  // mark PM members kept
  for (int h = 0; h < nh; ++h) {
    PYFOF_CUDA(cudaMemsetAsync(keep + H[h].off, 1, (size_t)H[h].np, s));
  }
  // two-level refinement of dense 16-cell regions of 256-grid halos
  // (bound_two_level_setup_ratios / build_halo, bound_fortran.f90:551-823)
  std::vector<TlRegion> act;
  std::vector<int32_t> act_of((size_t)nh * 512, -1);
  std::vector<uint8_t> region_r((size_t)nh * 512, 1);
  {
    uint32_t *rc = W.carve<uint32_t>((size_t)nh * 512);
    if (!rc) { set_error("workspace exhausted (regions)"); return kAlloc; }
    PYFOF_CUDA(cudaMemsetAsync(rc, 0, sizeof(uint32_t) * nh * 512, s));
    pm_region_count_kernel<<<gM, BLK, 0, s>>>(m, dH, mhalo, M, rc);
    PYFOF_CHECK_LAUNCH();
    std::vector<uint32_t> hrc((size_t)nh * 512);
    PYFOF_CUDA(cudaMemcpyAsync(hrc.data(), rc, sizeof(uint32_t) * nh * 512, cudaMemcpyDeviceToHost, s));
    PYFOF_CUDA(cudaStreamSynchronize(s));
    const double app_f = (double)(float)a.softening;
    for (int h = 0; h < nh; ++h) {
      if (H[h].n != 256) continue;
      const double sp = (double)H[h].spacing;
      int rmax = 1;
      for (int b = 0; b < 512; ++b) {
        const uint32_t c = hrc[(size_t)h * 512 + b];
        int r = c < 3926u ? 1 : (c < 14688u ? 2 : 4);
        if (r == 4 && 3.5 * (sp / 4.0) < app_f) r = 2;
        if (r == 2 && 3.5 * (sp / 2.0) < app_f) r = 1;
        region_r[(size_t)h * 512 + b] = (uint8_t)r;
        if (c > 0 && r > rmax) rmax = r;
      }
      if (rmax == 1) continue;
      H[h].two_level = 1;
      H[h].r_max = rmax;
      for (int b = 0; b < 512; ++b) {
        const uint32_t c = hrc[(size_t)h * 512 + b];
        const int r = region_r[(size_t)h * 512 + b];
        if (c == 0 || r == 1) continue;
        TlRegion Rg;
        Rg.h = h;
        Rg.b = b;
        Rg.r = r;
        Rg.n_in = r == 2 ? 128 : 216;
        const int bb[3] = {b % 8, (b / 8) % 8, b / 64};
        Rg.bo = 3.5f + 3.0f / (float)r;
        for (int d = 0; d < 3; ++d) {
          Rg.lo[d] = (float)(bb[d] * 16);
          Rg.hi[d] = std::min(Rg.lo[d] + 16.0f, 127.0f);
          Rg.u0[d] = ((Rg.lo[d] - Rg.bo) - (1.0f / (float)r)) + (0.0f / (float)r);
        }
        act_of[(size_t)h * 512 + b] = (int32_t)act.size();
        act.push_back(Rg);
      }
    }
    ctx.last_tl_regions = (int64_t)act.size();
  }
  // C2 cells (3.5 grid cells)
  {
    uint32_t *omin = W.carve<uint32_t>(3 * (size_t)nh), *omax = W.carve<uint32_t>(3 * (size_t)nh);
    if (!omin || !omax) { set_error("workspace exhausted (extents)"); return kAlloc; }
    std::vector<int2> work;
    for (int h = 0; h < nh; ++h)
      for (int64_t c = 0; c * kExtentChunk < std::max<int64_t>(H[h].np, 1); ++c) work.push_back(make_int2(h, (int)c));
    int2 *dwork = W.carve<int2>(work.size());
    if (!dwork) { set_error("workspace exhausted (extents)"); return kAlloc; }
    PYFOF_TRY(upload(ctx, dwork, work.data(), sizeof(int2) * work.size(), s));
    PYFOF_CUDA(cudaMemsetAsync(omin, 0xff, sizeof(uint32_t) * 3 * nh, s));
    PYFOF_CUDA(cudaMemsetAsync(omax, 0, sizeof(uint32_t) * 3 * nh, s));
    if (!work.empty()) {
      pm_extent_kernel<<<(unsigned)work.size(), BLK, 0, s>>>(m, dH, dwork, omin, omax);
      PYFOF_CHECK_LAUNCH();
    }
    pm_extent_final_kernel<<<(unsigned)ceil_div(3 * (int64_t)nh, 128), 128, 0, s>>>(dH, nh, omin, omax, ext);
    PYFOF_CHECK_LAUNCH();
  }
  std::vector<double> hext(6 * (size_t)nh);
  PYFOF_CUDA(cudaMemcpyAsync(hext.data(), ext, sizeof(double) * 6 * nh, cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  int64_t ncell = 0;
  for (int h = 0; h < nh; ++h) {
    PmHalo &p = H[h];
    p.cell_off = ncell;
    p.cw_u = p.two_level ? 3.5 / (double)p.r_max : 3.5;
    int64_t c = 1;
    for (int d = 0; d < 3; ++d) {
      p.u_min[d] = hext[6 * h + d];
      const double span = hext[6 * h + 3 + d] - hext[6 * h + d];
      p.nc[d] = std::max(1, (int)std::floor(span / p.cw_u) + 1);
      c *= p.nc[d];
    }
    ncell += c;
  }
  if (ncell >= 0xffffffffll) { set_error("too many C2 cells"); return kAlloc; }
  PYFOF_TRY(upload(ctx, dH, H.data(), sizeof(PmHalo) * nh, s));
  uint32_t *ckey = W.carve<uint32_t>(M), *cstart = W.carve<uint32_t>(ncell + 2);
  uint32_t *ka = W.carve<uint32_t>(M), *va = W.carve<uint32_t>(M), *kb = W.carve<uint32_t>(M),
           *vb = W.carve<uint32_t>(M);
  if (!ckey || !cstart || !ka || !va || !kb || !vb) { set_error("workspace exhausted (C2 cells)"); return kAlloc; }
  const uint32_t sentinel = (uint32_t)ncell;
  // Morton sub-key bits inside a cell (a multiple of 3, the key within 32 bits)
  const int sb = std::max(0, std::min(9, 32 - bits_for((uint64_t)ncell))) / 3 * 3;
  uint32_t *skey = W.carve<uint32_t>(M);
  if (!skey) { set_error("workspace exhausted (C2 cells)"); return kAlloc; }
  pm_cellkey_kernel<<<gM, BLK, 0, s>>>(m, dH, mhalo, M, ckey, sentinel, sb, skey);
  PYFOF_CHECK_LAUNCH();
  PYFOF_CUDA(cudaMemsetAsync(cstart, 0, sizeof(uint32_t) * (ncell + 2), s));
  pm_cellcount_kernel<<<gM, BLK, 0, s>>>(ckey, M, sentinel, cstart);
  PYFOF_CHECK_LAUNCH();
  PYFOF_TRY(exclusive_scan_u32(cstart, cstart, ncell + 1, nullptr, W, s));
  uint32_t *sk, *cmem;
  PYFOF_TRY(radix_sort_pairs(skey, nullptr, M, bits_for((uint64_t)sentinel << sb), ka, va, kb, vb, &sk, &cmem,
                             W, s));
  // cell-ordered positions and weights, target chunks, removal lists
  uint32_t npm = 0;
  PYFOF_CUDA(cudaMemcpyAsync(&npm, cstart + ncell, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  uint32_t *chcnt = W.carve<uint32_t>(ncell + 1);
  if (!chcnt) { set_error("workspace exhausted (C2 chunks)"); return kAlloc; }
  PYFOF_CUDA(cudaMemsetAsync(chcnt, 0, sizeof(uint32_t) * (ncell + 1), s));
  const unsigned gC = (unsigned)std::min<int64_t>(ceil_div(std::max<int64_t>(ncell, 1), BLK), 148 * 16);
  sr_chunk_count_kernel<<<gC, BLK, 0, s>>>(cstart, ncell, chcnt);
  PYFOF_CHECK_LAUNCH();
  PYFOF_TRY(exclusive_scan_u32(chcnt, chcnt, ncell + 1, nullptr, W, s));
  uint32_t nchunk = 0;
  PYFOF_CUDA(cudaMemcpyAsync(&nchunk, chcnt + ncell, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  float4 *src4 = W.carve<float4>(std::max<uint32_t>(npm, 1));
  SrChunk *chunks = W.carve<SrChunk>(std::max<uint32_t>(nchunk, 1));
  uint32_t *rflag = W.carve<uint32_t>((size_t)npm + 1), *rpos = W.carve<uint32_t>((size_t)npm + 1);
  uint32_t *rsrc = W.carve<uint32_t>(std::max<uint32_t>(npm, 1));
  if (!src4 || !chunks || !rflag || !rpos || !rsrc) { set_error("workspace exhausted (C2 sources)"); return kAlloc; }
  PYFOF_CUDA(cudaMemsetAsync(rflag, 0, sizeof(uint32_t) * ((size_t)npm + 1), s));
  const unsigned gP = (unsigned)std::min<int64_t>(ceil_div(std::max<uint32_t>(npm, 1), BLK), 148 * 16);
  sr_pack_kernel<<<gP, BLK, 0, s>>>(m, cmem, npm, src4);
  PYFOF_CHECK_LAUNCH();
  sr_chunk_fill_kernel<<<gC, BLK, 0, s>>>(cstart, chcnt, ncell, chunks);
  PYFOF_CHECK_LAUNCH();
  {
    // heaviest chunks first (a stable sort on the 16-bit weight key)
    const int64_t nc = std::max<uint32_t>(nchunk, 1);
    uint32_t *ck = W.carve<uint32_t>(nc), *c1k = W.carve<uint32_t>(nc), *c1v = W.carve<uint32_t>(nc),
             *c2k = W.carve<uint32_t>(nc), *c2v = W.carve<uint32_t>(nc);
    SrChunk *sorted = W.carve<SrChunk>(nc);
    if (!ck || !c1k || !c1v || !c2k || !c2v || !sorted) { set_error("workspace exhausted (C2 chunks)"); return kAlloc; }
    const unsigned gK = (unsigned)std::min<int64_t>(ceil_div(nc, BLK), 148 * 16);
    sr_chunk_key_kernel<<<gK, BLK, 0, s>>>(chunks, nchunk, cstart, ck);
    PYFOF_CHECK_LAUNCH();
    uint32_t *sk2, *order;
    PYFOF_TRY(radix_sort_pairs(ck, nullptr, nchunk, 16, c1k, c1v, c2k, c2v, &sk2, &order, W, s));
    sr_chunk_order_kernel<<<gK, BLK, 0, s>>>(chunks, order, nchunk, sorted);
    PYFOF_CHECK_LAUNCH();
    chunks = sorted;
  }
  unsigned *sr_next = W.carve<unsigned>(1);
  if (!sr_next) { set_error("workspace exhausted (C2 chunks)"); return kAlloc; }
  // persistent warps: the blocks that fit on the GPU at once (4 per SM)
  const unsigned gS = (unsigned)std::min<int64_t>(ceil_div((int64_t)std::max<uint32_t>(nchunk, 1) * 32, 256),
                                                  148 * 4);
  // per-member refinement ratio, refined-region sources and targets
  const int na = (int)act.size();
  uint8_t *pr = W.carve<uint8_t>(M);
  int32_t *preg = W.carve<int32_t>(M);
  R *phi_in = W.carve<R>(M);
  if (!pr || !preg || !phi_in) { set_error("workspace exhausted (two-level)"); return kAlloc; }
  PYFOF_CUDA(cudaMemsetAsync(phi_in, 0, sizeof(R) * M, s));
  PYFOF_CUDA(cudaMemsetAsync(pr, 1, M, s));
  PYFOF_CUDA(cudaMemsetAsync(preg, 0xff, sizeof(int32_t) * M, s));  // -1: no refined region
  TlRegion *dA = nullptr;
  uint32_t *src_start = nullptr, *src = nullptr, *tgt_start = nullptr, *tgt = nullptr;
  std::vector<uint32_t> hsrc, htgt;
  std::shared_ptr<GreenTable> g_r2, g_r4;
  {
    uint8_t *dregr = W.carve<uint8_t>((size_t)nh * 512);
    int32_t *dact_of = W.carve<int32_t>((size_t)nh * 512);
    if (!dregr || !dact_of) { set_error("workspace exhausted (two-level)"); return kAlloc; }
    PYFOF_TRY(upload(ctx, dregr, region_r.data(), (size_t)nh * 512, s));
    PYFOF_TRY(upload(ctx, dact_of, act_of.data(), sizeof(int32_t) * nh * 512, s));
    tl_particle_kernel<<<gM, BLK, 0, s>>>(m, dH, mhalo, M, dregr, dact_of, pr, preg);
    PYFOF_CHECK_LAUNCH();
    if (na > 0) {
      dA = W.carve<TlRegion>(na);
      uint32_t *cnt = W.carve<uint32_t>(na + 1);
      src_start = W.carve<uint32_t>(na + 1);
      tgt_start = W.carve<uint32_t>(na + 1);
      if (!dA || !cnt || !src_start || !tgt_start) { set_error("workspace exhausted (two-level)"); return kAlloc; }
      PYFOF_TRY(upload(ctx, dA, act.data(), sizeof(TlRegion) * na, s));
      // sources
      PYFOF_CUDA(cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * (na + 1), s));
      tl_source_kernel<<<gM, BLK, 0, s>>>(m, dH, mhalo, M, dact_of, dA, cnt, nullptr, 0);
      PYFOF_CHECK_LAUNCH();
      PYFOF_TRY(exclusive_scan_u32(cnt, src_start, na + 1, nullptr, W, s));
      hsrc.resize(na + 1);
      PYFOF_CUDA(cudaMemcpyAsync(hsrc.data(), src_start, sizeof(uint32_t) * (na + 1), cudaMemcpyDeviceToHost, s));
      PYFOF_CUDA(cudaStreamSynchronize(s));
      src = W.carve<uint32_t>(std::max<uint32_t>(hsrc[na], 1));
      if (!src) { set_error("workspace exhausted (two-level sources)"); return kAlloc; }
      PYFOF_CUDA(cudaMemcpyAsync(cnt, src_start, sizeof(uint32_t) * (na + 1), cudaMemcpyDeviceToDevice, s));
      tl_source_kernel<<<gM, BLK, 0, s>>>(m, dH, mhalo, M, dact_of, dA, cnt, src, 1);
      PYFOF_CHECK_LAUNCH();
      // targets
      PYFOF_CUDA(cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * (na + 1), s));
      tl_target_kernel<<<gM, BLK, 0, s>>>(preg, M, cnt, nullptr, 0);
      PYFOF_CHECK_LAUNCH();
      PYFOF_TRY(exclusive_scan_u32(cnt, tgt_start, na + 1, nullptr, W, s));
      htgt.resize(na + 1);
      PYFOF_CUDA(cudaMemcpyAsync(htgt.data(), tgt_start, sizeof(uint32_t) * (na + 1), cudaMemcpyDeviceToHost, s));
      PYFOF_CUDA(cudaStreamSynchronize(s));
      tgt = W.carve<uint32_t>(std::max<uint32_t>(htgt[na], 1));
      if (!tgt) { set_error("workspace exhausted (two-level targets)"); return kAlloc; }
      PYFOF_CUDA(cudaMemcpyAsync(cnt, tgt_start, sizeof(uint32_t) * (na + 1), cudaMemcpyDeviceToDevice, s));
      tl_target_kernel<<<gM, BLK, 0, s>>>(preg, M, cnt, tgt, 1);
      PYFOF_CHECK_LAUNCH();
      bool need2 = false, need4 = false;
      for (auto &Rg : act) { need2 |= Rg.r == 2; need4 |= Rg.r == 4; }
      if (need2) PYFOF_TRY(get_green<R>(ctx, 128, 3.5, 7.0, 0, &g_r2));
      if (need4) PYFOF_TRY(get_green<R>(ctx, 216, 3.5, 14.0, 0, &g_r4));
      R *self_in = c1;  // reuse: c1 is rewritten every pass, self_in must persist -> own array
      self_in = W.carve<R>(M);
      if (!self_in) { set_error("workspace exhausted (two-level self)"); return kAlloc; }
      const unsigned gs = (unsigned)std::min<int64_t>(ceil_div(std::max<uint32_t>(hsrc[na], 1), BLK), 148 * 16);
      tl_check_kernel<<<gs, BLK, 0, s>>>(m, dH, dA, na, src_start, src, ctx.d_flags);
      PYFOF_CHECK_LAUNCH();
      const unsigned gt = (unsigned)std::min<int64_t>(ceil_div(std::max<uint32_t>(htgt[na], 1), BLK), 148 * 16);
      tl_self_kernel<R><<<gt, BLK, 0, s>>>(m, dH, dA, na, tgt_start, tgt,
                                           g_r2 ? (const R *)g_r2->self : nullptr,
                                           g_r4 ? (const R *)g_r4->self : nullptr, self_in, ctx.d_flags);
      PYFOF_CHECK_LAUNCH();
      tl_self_in = self_in;
    }
  }
  PYFOF_CUDA(cudaMemcpyAsync(ctx.h_flags, ctx.d_flags, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  if (ctx.h_flags[FLAG_ERR]) {
    set_error("particle outside the PM source domain or non-finite grid coordinate");
    return ctx.h_flags[FLAG_ERR];
  }

  // grid batches per class, bounded by a spectrum budget; one scratch area,
  // sized for the largest batch, serves every batch of every pass
  const size_t budget = ctx.pm_budget;
  auto round256 = [](size_t b) { return (b + 255) & ~(size_t)255; };
  // per grid: the fixed-point deposit grid (8 B a node; the convolved
  // potential, R, is written back over it) and the half spectrum
  auto batch_bytes = [&](int n, int nb) {
    const size_t sup = n / 2 + 1;
    return round256(sizeof(unsigned long long) * nb * sup * sup * sup) +
           sizeof(cplx_t<R>) * (size_t)nb * spec_elems<R>(n);
  };
  auto max_batch = [&](int n) {
    const int by_budget = (int)std::max<size_t>(1, budget / batch_bytes(n, 1));
    const int cap = a.tiles.pm_batch[kGridIndex(n)];
    return cap > 0 ? std::min(cap, by_budget) : by_budget;
  };
  auto waves = [&](int n) { return a.tiles.conv_waves[kGridIndex(n)]; };
  size_t scratch_bytes = 256;
  for (int n : {48, 64, 128, 256}) {
    int cnt = 0;
    for (int h = 0; h < nh; ++h) cnt += H[h].n == n;
    if (cnt) scratch_bytes = std::max(scratch_bytes, batch_bytes(n, std::min(cnt, max_batch(n))));
  }
  for (int r : {2, 4}) {
    int cnt = 0;
    for (int ia = 0; ia < na; ++ia) cnt += act[ia].r == r;
    const int nin = r == 2 ? 128 : 216;
    if (cnt) scratch_bytes = std::max(scratch_bytes, batch_bytes(nin, std::min(cnt, max_batch(nin))));
  }
  unsigned char *scratch = W.carve<unsigned char>(scratch_bytes);
  int32_t *dpend = W.carve<int32_t>(nh);
  const int nbat = std::max(std::max(na, nh), 1);
  int32_t *dbatch = W.carve<int32_t>(nbat);
  uint32_t *dbpre = W.carve<uint32_t>(2 * (size_t)(nbat + 1));
  double *dinv = W.carve<double>(nbat);
  if (!scratch || !dpend || !dbatch || !dbpre || !dinv) {
    set_error("workspace exhausted (PM grids)");
    return kAlloc;
  }
  // halos above kBigNp members: chunked removal loop
  std::vector<BigHalo> hbig;
  std::vector<BigChunk> hch;
  std::vector<char> is_big(nh, 0);
  int64_t ubig = 0;
  for (int h = 0; h < nh; ++h) {
    if (H[h].np <= (a.big_np > 0 ? a.big_np : kBigNp)) continue;
    is_big[h] = 1;
    BigHalo bh{};
    bh.h = h;
    bh.off = H[h].off;
    bh.np = H[h].np;
    bh.uoff = ubig;
    bh.chunk0 = (int32_t)hch.size();
    for (int64_t st0 = 0; st0 < bh.np; st0 += kChunk)
      hch.push_back(BigChunk{(int32_t)hbig.size(), bh.off + st0, bh.off + std::min<int64_t>(bh.np, st0 + kChunk)});
    bh.nchunk = (int32_t)hch.size() - bh.chunk0;
    ubig += bh.np;
    hbig.push_back(bh);
  }
  const int nbig = (int)hbig.size(), nchb = (int)hch.size();
  BigHalo *dB = nullptr;
  BigChunk *dCh = nullptr;
  double *bpart = nullptr;
  int32_t *bucount = nullptr;
  uint32_t *bulist = nullptr, *beq = nullptr;
  int32_t *nactive = ctx.d_flags + FLAG_COUNT_B;
  if (nbig) {
    dB = W.carve<BigHalo>(nbig);
    dCh = W.carve<BigChunk>(nchb);
    bpart = W.carve<double>(7 * (size_t)nchb);
    bucount = W.carve<int32_t>(nbig);
    bulist = W.carve<uint32_t>(ubig);
    beq = W.carve<uint32_t>(ubig);
    if (!dB || !dCh || !bpart || !bucount || !bulist || !beq) {
      set_error("workspace exhausted (large halos)");
      return kAlloc;
    }
    PYFOF_TRY(upload(ctx, dB, hbig.data(), sizeof(BigHalo) * nbig, s));
    PYFOF_TRY(upload(ctx, dCh, hch.data(), sizeof(BigChunk) * nchb, s));
  }
  for (int pass = 1; pass <= kMaxPasses; ++pass) {
    std::vector<int32_t> pend;
    for (int h = 0; h < nh; ++h) if (H[h].pending) pend.push_back(h);
    if (pend.empty()) break;
    std::vector<int32_t> pend_small;
    for (int h : pend) if (!is_big[h]) pend_small.push_back(h);
    ++ctx.last_pm_passes;
    if (ctx.timing && pass > 1) ctx.gap_timer.end(s);
    if (!pend_small.empty()) {
      PYFOF_TRY(upload(ctx, dpend, pend_small.data(), sizeof(int32_t) * pend_small.size(), s));
      pm_mkeep_kernel<<<(unsigned)pend_small.size(), 256, 0, s>>>(m, dH, dpend, (int)pend_small.size(), keep);
      PYFOF_CHECK_LAUNCH();
    }
    if (nbig) {
      big_mass_kernel<<<nchb, 256, 0, s>>>(m, dCh, dB, dH, keep, bpart);
      PYFOF_CHECK_LAUNCH();
      big_mass_sum_kernel<<<(unsigned)ceil_div(nbig, 128), 128, 0, s>>>(dB, nbig, bpart, dH);
      PYFOF_CHECK_LAUNCH();
    }
    for (int n : {48, 64, 128, 256}) {
      std::vector<int32_t> grp;
      for (int h : pend) if (H[h].n == n) grp.push_back(h);
      if (grp.empty()) continue;
      const int sup = n / 2 + 1;
      const int maxb = max_batch(n);
      for (size_t g0 = 0; g0 < grp.size(); g0 += maxb) {
        const int nb = (int)std::min<size_t>(maxb, grp.size() - g0);
        // the batch's halos, their member prefix and their first cmem position
        std::vector<uint32_t> bp((size_t)nb + 1, 0);
        for (int j = 0; j < nb; ++j) bp[j + 1] = bp[j] + (uint32_t)H[grp[g0 + j]].np;
        PYFOF_TRY(upload(ctx, dbatch, grp.data() + g0, sizeof(int32_t) * nb, s));
        PYFOF_TRY(upload(ctx, dbpre, bp.data(), sizeof(uint32_t) * (nb + 1), s));
        unsigned long long *acc = reinterpret_cast<unsigned long long *>(scratch);
        R *rho = reinterpret_cast<R *>(scratch);  // the convolved grids overwrite acc
        cplx_t<R> *spec = reinterpret_cast<cplx_t<R> *>(
            scratch + round256(sizeof(unsigned long long) * (size_t)nb * sup * sup * sup));
        const int64_t ng = (int64_t)nb * sup * sup * sup;
        PYFOF_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * ng, s));
        pm_batch_scale_kernel<<<(unsigned)ceil_div(nb, 128), 128, 0, s>>>(dH, dbatch, nb, nullptr, dinv);
        PYFOF_CHECK_LAUNCH();
        const unsigned gb = (unsigned)std::min<int64_t>(ceil_div(std::max<uint32_t>(bp[nb], 1), BLK), 148 * 16);
        pm_deposit_kernel<<<gb, BLK, 0, s>>>(m, dH, dbatch, dbpre, nb, keep, first, wt, sup, acc);
        PYFOF_CHECK_LAUNCH();
        if (ctx.timing) ctx.conv_timer.begin(s);
        PYFOF_TRY(pm_convolve_batch<R>(rho, spec, (const R *)green_of[n]->g, n, sup, nb, s, acc, dinv, waves(n)));
        if (ctx.timing) ctx.conv_timer.end(s);
        ctx.last_pm_solves += nb;
        ctx.last_pm_fft_bytes += 4.0 * sizeof(R) * nb * (n + 2.0) * n * n;
        pm_gather_kernel<R><<<gb, BLK, 0, s>>>(m, dH, dbatch, dbpre, nb, keep, first, wt, selfv, sup, rho,
                                               a.a_val, c1);
        PYFOF_CHECK_LAUNCH();
      }
    }
    // refined regions of pending halos, batched per inner grid size
    for (int r : {2, 4}) {
      std::vector<int32_t> regs;
      for (int ia = 0; ia < na; ++ia)
        if (act[ia].r == r && H[act[ia].h].pending) regs.push_back(ia);
      if (regs.empty()) continue;
      const int nin = r == 2 ? 128 : 216;
      const int sup = nin / 2 + 1;
      const int maxb = max_batch(nin);
      const R *gin = (const R *)(r == 2 ? g_r2 : g_r4)->g;
      for (size_t g0 = 0; g0 < regs.size(); g0 += maxb) {
        const int nb = (int)std::min<size_t>(maxb, regs.size() - g0);
        unsigned long long *acc = reinterpret_cast<unsigned long long *>(scratch);
        R *rho = reinterpret_cast<R *>(scratch);  // the convolved grids overwrite acc
        cplx_t<R> *spec = reinterpret_cast<cplx_t<R> *>(
            scratch + round256(sizeof(unsigned long long) * (size_t)nb * sup * sup * sup));
        // prefix counts of the batch's sources and targets (flat launches)
        std::vector<uint32_t> bp(2 * (size_t)(nb + 1), 0);
        for (int j = 0; j < nb; ++j) {
          const int ia = regs[g0 + j];
          bp[j + 1] = bp[j] + (hsrc[ia + 1] - hsrc[ia]);
          bp[nb + 1 + j + 1] = bp[nb + 1 + j] + (htgt[ia + 1] - htgt[ia]);
        }
        PYFOF_TRY(upload(ctx, dbatch, regs.data() + g0, sizeof(int32_t) * nb, s));
        PYFOF_TRY(upload(ctx, dbpre, bp.data(), sizeof(uint32_t) * bp.size(), s));
        const int64_t ng = (int64_t)nb * sup * sup * sup;
        PYFOF_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * ng, s));
        pm_batch_scale_kernel<<<(unsigned)ceil_div(nb, 128), 128, 0, s>>>(dH, dbatch, nb, dA, dinv);
        PYFOF_CHECK_LAUNCH();
        const unsigned gd = (unsigned)std::min<int64_t>(ceil_div(std::max<uint32_t>(bp[nb], 1), BLK), 148 * 16);
        tl_deposit_kernel<<<gd, BLK, 0, s>>>(m, dH, dA, dbatch, dbpre, nb, src_start, src, keep, sup, acc);
        PYFOF_CHECK_LAUNCH();
        if (ctx.timing) ctx.conv_timer.begin(s);
        PYFOF_TRY(pm_convolve_batch<R>(rho, spec, gin, nin, sup, nb, s, acc, dinv, waves(nin)));
        if (ctx.timing) ctx.conv_timer.end(s);
        ctx.last_pm_solves += nb;
        ctx.last_pm_fft_bytes += 4.0 * sizeof(R) * nb * (nin + 2.0) * nin * nin;
        const unsigned gg = (unsigned)std::min<int64_t>(
            ceil_div(std::max<uint32_t>(bp[2 * nb + 1], 1), BLK), 148 * 16);
        tl_gather_kernel<R><<<gg, BLK, 0, s>>>(m, dH, dA, dbatch, dbpre + nb + 1, nb, tgt_start, tgt, keep,
                                               tl_self_in, sup, rho, a.a_val, phi_in);
        PYFOF_CHECK_LAUNCH();
      }
    }
    PYFOF_CUDA(cudaMemsetAsync(sr_next, 0, sizeof(unsigned), s));
    if (pass == 1) {
      sr_gather_kernel<R, false><<<gS, 256, 0, s>>>(dH, mhalo, keep, pr, chunks, nchunk, cstart, cmem, src4,
                                                    nullptr, nullptr, a.a_val, a.softening, c2, sr_next);
      PYFOF_CHECK_LAUNCH();
    } else {
      sr_removed_flag_kernel<<<gP, BLK, 0, s>>>(cmem, npm, jd, rflag);
      PYFOF_CHECK_LAUNCH();
      PYFOF_TRY(exclusive_scan_u32(rflag, rpos, (int64_t)npm + 1, nullptr, W, s));
      sr_removed_fill_kernel<<<gP, BLK, 0, s>>>(rflag, rpos, npm, rsrc);
      PYFOF_CHECK_LAUNCH();
      sr_gather_kernel<R, true><<<gS, 256, 0, s>>>(dH, mhalo, keep, pr, chunks, nchunk, cstart, cmem, src4,
                                                   rpos, rsrc, a.a_val, a.softening, c2, sr_next);
      PYFOF_CHECK_LAUNCH();
    }
    if (!pend_small.empty()) {
      PYFOF_CUDA(wait_velocities(ctx, s));
      pm_inner_kernel<R><<<(unsigned)pend_small.size(), IBLK, 0, s>>>(m, dH, dpend, (int)pend_small.size(), keep,
                                                                     jd, c1, phi_in, c2, phi, en,
                                                                     (float)a.b_val, a.np_halo_min, phi_only,
                                                                     ctx.d_flags);
      PYFOF_CHECK_LAUNCH();
    }
    if (nbig) PYFOF_TRY(big_removal<R>(ctx, m, dB, nbig, dCh, nchb, dH, keep, jd, c1, phi_in, c2, phi, en, bpart,
                                       bucount, bulist, beq, nactive, (float)a.b_val, a.np_halo_min,
                                       phi_only));
    if (ctx.timing) ctx.gap_timer.begin(s);
    PYFOF_CUDA(cudaMemcpyAsync(H.data(), dH, sizeof(PmHalo) * nh, cudaMemcpyDeviceToHost, s));
    PYFOF_CUDA(cudaMemcpyAsync(ctx.h_flags, ctx.d_flags, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    PYFOF_CUDA(cudaStreamSynchronize(s));
    if (ctx.timing) ctx.conv_timer.collect();
    if (ctx.h_flags[FLAG_ERR]) {
      set_error("particle-mesh unbinding failed (error %d)", ctx.h_flags[FLAG_ERR]);
      return ctx.h_flags[FLAG_ERR];
    }
  }
  std::vector<HaloResult> hr(nh);
  for (int h = 0; h < nh; ++h) {
    hr[h].status = H[h].pending ? 5 : H[h].status;
    hr[h].np_bound = H[h].np_bound;
  }
  for (int h = 0; h < nh; ++h)
    PYFOF_TRY(upload(ctx, res + list[h], &hr[h], sizeof(HaloResult), s));
  if (phi_out) PYFOF_CUDA(cudaMemcpyAsync(phi_out, phi, sizeof(float) * M, cudaMemcpyDeviceToDevice, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  return kOk;
}

}  // namespace

int32_t unbind_pm(Context &ctx, const FofArgs &a, const GridRules &rules, const Members &m,
                  const std::vector<HaloTask> &tasks, const std::vector<int32_t> &list,
                  HaloResult *res, uint8_t *keep, float *phi_out, int phi_only) {
  if (a.bound_fp64 || a.bound_per_halo) return run_pm<double>(ctx, a, rules, m, tasks, list, res, keep, phi_out, phi_only);
  return run_pm<float>(ctx, a, rules, m, tasks, list, res, keep, phi_out, phi_only);
}

}  // namespace pyfof
