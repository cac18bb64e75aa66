// Friends-of-friends linking on the device.
//
// Replaces process_single_region + the fof_fortran driver
// (fof_fortran.f90:109-362, :496-949) and atomic_dsu.c.  All input regions of
// a call are processed together:
//   1. fof_bbox_kernel    per-region unwrap about the first particle + bbox
//   2. host               reference cell geometry per region (same formulas,
//                         same libm pow) -> region table
//   3. fof_key_kernel     global cell key per particle + cell histogram
//   4. stable cell order  (cell key, particle index): the reference CRS order,
//                         by a scatter to per-cell slots and a sort of each
//                         cell (a stable radix sort when a cell is large)
//   5. fof_gather_kernel  FP32 sorted coordinates (real(x_rel,4))
//   6. link kernels       pair tests over the reference's neighbour cells
//                         (fof_link_dense_kernel for cells with more than
//                         DENSE_T particles and their pairs with sparse
//                         cells, fof_link_kernel for sparse-cell pairs),
//                         lock-free atomicCAS union (lower index wins)
//   7. fof_root_kernel    full compression + warp-aggregated group sizes
//   8. scan of root flags -> candidate ranks (region order, then root CRS
//                         position: the reference halo numbering)
//   9. outputs, FP64 centre-of-mass / angular momentum per candidate
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>

#include "context.cuh"
#include "fof.cuh"
#include "fof_internal.cuh"
#include "primitives.cuh"
#include "unbind.cuh"

namespace pyfof {

namespace {

constexpr int TILE = 4096;  // particles per block of the bbox and key kernels (16 per thread)
constexpr int BLK = 256;

__device__ __forceinline__ int region_of_key(const uint64_t *cell_off, int nreg, uint64_t key) {
  int lo = 0, hi = nreg;  // first r with cell_off[r] > key, minus one
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (cell_off[mid] <= key) lo = mid + 1; else hi = mid;
  }
  return lo - 1;
}

__device__ __forceinline__ void warp_minmax(double &mn, double &mx) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
}

__global__ void __launch_bounds__(BLK) fof_bbox_kernel(Coords xp, const RegionDev *__restrict__ R,
                                                       const Tile *__restrict__ T, double L,
                                                       double half,
                                                       unsigned long long *__restrict__ bbox,
                                                       int32_t *flags) {
  const Tile t = T[blockIdx.x];
  const RegionDev &r = R[t.region];
  if (!r.active) return;
  double anc[3], mn[3], mx[3];
  for (int d = 0; d < 3; ++d) {
    anc[d] = xp.get(r.start, d);
    mn[d] = INFINITY;
    mx[d] = -INFINITY;
  }
  bool bad = false;
  for (int64_t i = t.begin + threadIdx.x; i < t.end; i += BLK) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double x = xp.get(i, d);
      bad |= !isfinite(x);
      double v = unwrap(x, anc[d], half, L);
      mn[d] = fmin(mn[d], v);
      mx[d] = fmax(mx[d], v);
    }
  }
  if (bad) atomicExch(&flags[FLAG_ERR], kNonFinite);
  __shared__ double smn[3][BLK / 32], smx[3][BLK / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int d = 0; d < 3; ++d) {
    warp_minmax(mn[d], mx[d]);
    if (lane == 0) { smn[d][warp] = mn[d]; smx[d][warp] = mx[d]; }
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int d = threadIdx.x;
    double a = INFINITY, b = -INFINITY;
    for (int w = 0; w < BLK / 32; ++w) { a = fmin(a, smn[d][w]); b = fmax(b, smx[d][w]); }
    if (a <= b) {
      atomicMin(&bbox[6 * (int64_t)t.region + d], dbl_to_ord(a));
      atomicMax(&bbox[6 * (int64_t)t.region + 3 + d], dbl_to_ord(b));
    }
  }
}

__device__ __forceinline__ int64_t cell_coord(double x, double origin, double size, int32_t n) {
  double f = floor(__ddiv_rn(__dadd_rn(x, -origin), size)) + 1.0;
  if (!(f >= 1.0)) f = 1.0;
  if (f > (double)n) f = (double)n;
  return (int64_t)f - 1;
}

__global__ void __launch_bounds__(BLK) fof_key_kernel(Coords xp, const RegionDev *__restrict__ R,
                                                      const Tile *__restrict__ T, double L,
                                                      double half, uint32_t sentinel,
                                                      uint32_t *__restrict__ keys,
                                                      uint32_t *__restrict__ counts,
                                                      uint32_t *__restrict__ rank) {
  const Tile t = T[blockIdx.x];
  const RegionDev &r = R[t.region];
  if (!r.active) {
    for (int64_t i = t.begin + threadIdx.x; i < t.end; i += BLK) {
      keys[i] = sentinel;
      rank[i] = atomicAdd(&counts[sentinel], 1u);
    }
    return;
  }
  double anc[3];
  for (int d = 0; d < 3; ++d) anc[d] = xp.get(r.start, d);
  for (int64_t i = t.begin + threadIdx.x; i < t.end; i += BLK) {
    int64_t c[3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
      c[d] = cell_coord(unwrap(xp.get(i, d), anc[d], half, L), r.origin[d], r.size[d], r.N[d]);
    uint64_t key = r.cell_off + (uint64_t)(c[0] + (int64_t)r.N[0] * (c[1] + (int64_t)r.N[1] * c[2]));
    keys[i] = (uint32_t)key;
    rank[i] = atomicAdd(&counts[key], 1u);  // a slot in the cell, in no particular order
  }
}

// ---- cell order without a radix sort ---------------------------------------
// The key kernel's counters give every particle a distinct slot in its
// cell; scattering to cell start + slot groups the particles by cell, and
// sorting each cell's original indices restores the stable order of the
// reference's counting sort (ascending original index within a cell).

__global__ void fof_max_count_kernel(const uint32_t *__restrict__ counts, int64_t ncell,
                                     uint32_t *__restrict__ out) {
  uint32_t m = 0;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (int64_t)gridDim.x * blockDim.x)
    m = max(m, counts[c]);
  m = __reduce_max_sync(0xffffffffu, m);
  if ((threadIdx.x & 31) == 0 && m > 0) atomicMax(out, m);
}

__global__ void fof_cell_scatter_kernel(const uint32_t *__restrict__ keys, const uint32_t *__restrict__ rank,
                                        const uint32_t *__restrict__ cstart, int64_t n,
                                        uint32_t *__restrict__ skey, uint32_t *__restrict__ sidx) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t k = keys[i];
    const uint32_t p = cstart[k] + rank[i];
    skey[p] = k;
    sidx[p] = (uint32_t)i;
  }
}

constexpr int CELL_SORT_SMALL = 32;   // cells up to this size: one thread, insertion sort
constexpr int CELL_SORT_MAX = 8192;   // cells up to this size: one block, bitonic sort

__global__ void fof_cell_sort_small_kernel(const uint32_t *__restrict__ cstart, int64_t ncell,
                                           uint32_t *__restrict__ sidx, uint32_t *__restrict__ big,
                                           uint32_t *__restrict__ nbig) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t b = cstart[c], m = cstart[c + 1] - b;
    if (m < 2) continue;
    if (m > (uint32_t)CELL_SORT_SMALL) {
      big[atomicAdd(nbig, 1u)] = (uint32_t)c;
      continue;
    }
    uint32_t *a = sidx + b;
    for (uint32_t i = 1; i < m; ++i) {
      const uint32_t v = a[i];
      uint32_t j = i;
      while (j > 0 && a[j - 1] > v) {
        a[j] = a[j - 1];
        --j;
      }
      a[j] = v;
    }
  }
}

__global__ void __launch_bounds__(1024) fof_cell_sort_big_kernel(const uint32_t *__restrict__ cstart,
                                                               const uint32_t *__restrict__ big,
                                                               const uint32_t *__restrict__ nbig,
                                                               uint32_t *__restrict__ sidx) {
  __shared__ uint32_t v[CELL_SORT_MAX];
  const uint32_t nb = *nbig;
  for (uint32_t j = blockIdx.x; j < nb; j += gridDim.x) {
    const uint32_t c = big[j];
    const uint32_t b = cstart[c], m = cstart[c + 1] - b;
    uint32_t np2 = 1;
    while (np2 < m) np2 <<= 1;
    for (uint32_t i = threadIdx.x; i < np2; i += blockDim.x) v[i] = i < m ? sidx[b + i] : 0xffffffffu;
    __syncthreads();
    for (uint32_t k = 2; k <= np2; k <<= 1)
      for (uint32_t h = k >> 1; h > 0; h >>= 1) {
        for (uint32_t i = threadIdx.x; i < np2; i += blockDim.x) {
          const uint32_t l = i ^ h;
          if (l > i) {
            const bool up = (i & k) == 0;
            const uint32_t x = v[i], y = v[l];
            if ((x > y) == up) {
              v[i] = y;
              v[l] = x;
            }
          }
        }
        __syncthreads();
      }
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) sidx[b + i] = v[i];
    __syncthreads();
  }
}

__global__ void __launch_bounds__(BLK) fof_gather_kernel(
    Coords xp, const RegionDev *__restrict__ R, const uint64_t *__restrict__ cell_off, int nreg,
    const uint32_t *__restrict__ skey, const uint32_t *__restrict__ sidx, int64_t n_active,
    double L, double half, float4 *__restrict__ pos, uint32_t *__restrict__ prid) {
  for (int64_t p = (int64_t)blockIdx.x * BLK + threadIdx.x; p < n_active;
       p += (int64_t)gridDim.x * BLK) {
    const int rid = nreg == 1 ? 0 : region_of_key(cell_off, nreg, skey[p]);
    const RegionDev &r = R[rid];
    const int64_t i = sidx[p];
    float v[3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
      v[d] = __double2float_rn(unwrap(xp.get(i, d), xp.get(r.start, d), half, L));
    pos[p] = make_float4(v[0], v[1], v[2], __int_as_float((int)i));
    prid[p] = (uint32_t)rid;
  }
}

// ---- lock-free disjoint-set union over sorted positions -------------------
// parent[x] == x marks a root; parent pointers only ever point to smaller
// indices, so the root of every set is its minimum element, exactly as in
// atomic_dsu.c (a higher root is hung under a lower one by CAS).

__device__ __forceinline__ int dsu_find(int *parent, int x) {
  int y = __ldcg(parent + x);
  while (y != x) {
    int z = __ldcg(parent + y);
    if (z != y) parent[x] = z;  // path halving; z is an ancestor of x
    x = y;
    y = z;
  }
  return x;
}

__device__ __forceinline__ void dsu_union(int *parent, int a, int b, int32_t *flags) {
  for (int it = 0; it < (1 << 22); ++it) {
    a = dsu_find(parent, a);
    b = dsu_find(parent, b);
    if (a == b) return;
    if (a > b) { int t = a; a = b; b = t; }
    int old = atomicCAS(parent + b, b, a);
    if (old == b) return;
  }
  atomicExch(&flags[FLAG_ERR], kInvalid);  // unreachable: retry cap as a safety net
}

struct LinkParams {
  double L, half, rp2;
  float rp2_open;   // largest float f with (double)f <= link^2
  float rp2_lo, rp2_hi;  // FP32 fast-path brackets of link^2 for periodic tests
  int fast_periodic;
};

// Exact reference distance tests.  Open regions: FP32 differences, squares
// and sum (fof_fortran.f90:636).  Periodic regions: dist2_pbc
// (fof_fortran.f90:483-491) in FP64; an FP32 estimate settles all pairs
// whose distance is far from the linking length and only the rest take the
// FP64 path, which decides them exactly.
__device__ __forceinline__ bool linked_open(float4 a, float4 b, float thr) {
  float d0 = __fsub_rn(a.x, b.x), d1 = __fsub_rn(a.y, b.y), d2 = __fsub_rn(a.z, b.z);
  float s = __fmul_rn(d0, d0);
  s = __fadd_rn(s, __fmul_rn(d1, d1));
  s = __fadd_rn(s, __fmul_rn(d2, d2));
  return s <= thr;
}

__device__ __forceinline__ bool linked_pbc(float4 a, float4 b, const LinkParams &P) {
  float d0 = __fsub_rn(a.x, b.x), d1 = __fsub_rn(a.y, b.y), d2 = __fsub_rn(a.z, b.z);
  if (P.fast_periodic) {
    const float hf = (float)P.half, Lf = (float)P.L;
    float e0 = fabsf(d0), e1 = fabsf(d1), e2 = fabsf(d2);
    e0 = e0 > hf ? Lf - e0 : e0;
    e1 = e1 > hf ? Lf - e1 : e1;
    e2 = e2 > hf ? Lf - e2 : e2;
    float s = e0 * e0 + e1 * e1 + e2 * e2;
    if (s < P.rp2_lo) return true;
    if (s > P.rp2_hi) return false;
  }
  double x = fabs((double)d0), y = fabs((double)d1), z = fabs((double)d2);
  if (x > P.half) x = __dadd_rn(P.L, -x);
  if (y > P.half) y = __dadd_rn(P.L, -y);
  if (z > P.half) z = __dadd_rn(P.L, -z);
  double r2 = __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
  return r2 <= P.rp2;
}

// Cells with more than DENSE_T particles carry a sub-cell index (sub[d]
// slabs per axis, each at least one linking length wide; a single slab when
// the cell is narrower than two linking lengths): the particles of the cell
// are listed by sub-cell in dpos[], sub_tab holds the offsets.  A pair test
// against such a cell only visits the sub-cells that overlap the cube of
// half-width `reach` around the particle, which contains every partner the
// exact distance test can accept.  Their particles, and every pair between
// a dense and a sparse cell, are linked by the dense-cell kernel; pairs of
// sparse cells by the per-particle kernel.
constexpr int DENSE_T = 24;
constexpr int SUB_MAX = 216;

struct DenseIndex {
  const uint32_t *rank;  // exclusive scan of dense-cell flags, per cell
  const uint32_t *tab;   // per dense cell: S+1 offsets (relative to cell start)
  const float4 *dpos;    // dense cells' particles listed by sub-cell; .w = sorted position
  const uint32_t *order; // work order: dense-cell particles first, then the rest
  int stride;            // entries per dense cell in tab
  float reach;           // linking length plus FP32 rounding slack
};

// Sub-cell of a coordinate inside a cell whose lower corner is lo.  FP32,
// monotone in x; the same function places particles and bounds queries, and
// `reach` carries slack for the FP32 rounding of the query endpoints.
__device__ __forceinline__ int sub_of(float x, float lo, float inv_sub, int s) {
  float t = floorf(__fmul_rn(__fsub_rn(x, lo), inv_sub));
  if (!(t >= 0.0f)) t = 0.0f;
  if (t > (float)(s - 1)) t = (float)(s - 1);
  return (int)t;
}

// Sub-cell layout of a dense cell with n particles: about SUB_OCC particles
// per sub-cell (floor(cbrt(n / SUB_OCC)) slabs per axis), at most the
// region's sub[d] (slabs at least one linking length wide).  Few, well
// filled sub-cells keep the number of source ranges a query walks small.
// Build and queries use this one function, so they agree on every cell.
constexpr float SUB_OCC = 6.0f;

struct SubGrid {
  int s[3];
  float inv[3];  // sub-cells per unit length
};

// Very dense cell: a dense cell whose merge sub-cells hold VD_OCC particles
// or more on average.  All pairs inside one merge sub-cell are linked, so
// such cells are linked sub-cell by sub-cell (fof_vd_intra_kernel,
// fof_vd_inter_kernel) instead of pair by pair.
constexpr int VD_OCC = 4;
__device__ __forceinline__ bool is_vd(const RegionDev &r, int64_t n) {
  return r.vd_k[0] > 0 && n > DENSE_T && n >= (int64_t)VD_OCC * r.vd_k[0] * r.vd_k[1] * r.vd_k[2];
}

__device__ __forceinline__ SubGrid dense_sub(const RegionDev &r, int64_t n) {
  SubGrid g;
  if (is_vd(r, n)) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      g.s[d] = r.vd_k[d];
      g.inv[d] = r.vd_inv[d];
    }
    return g;
  }
  const int k = max(1, (int)cbrtf(__fdiv_rn((float)n, SUB_OCC)));
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    g.s[d] = min(k, r.sub[d]);
    g.inv[d] = g.s[d] == r.sub[d] ? r.inv_sub[d] : __double2float_rn((double)g.s[d] / r.size[d]);
  }
  return g;
}

__device__ __forceinline__ float cell_lower(const RegionDev &r, int d, int64_t i) {
  return __double2float_rn(__dadd_rn(r.origin[d], __dmul_rn((double)i, r.size[d])));
}

// Union of a linked pair (p, q); rp caches p's root between calls.
__device__ __forceinline__ void link_pair(int *parent, int p, int q, int &rp, int32_t *flags) {
  if (rp < 0) rp = dsu_find(parent, p);
  const int y = __ldcg(parent + q);
  if (y == rp) return;  // q already hangs directly under p's root
  const int rq = dsu_find(parent, q);
  if (rq != rp) {
    dsu_union(parent, rp, rq, flags);
    rp = dsu_find(parent, rp);
  }
}

// Root hints: a root of q's set found earlier in the call.  Sets only
// merge, so a hint equal to p's cached root rp means p and q already share a
// set and the pair needs neither its distance test nor a union; any other
// hint decides nothing (either may have been hung under a lower root since).
// The dense kernel finds the hints of a batch of 32 sources in parallel, one
// find per lane, instead of one dependent parent read per source and pair.

// Ordered-integer image of a float (monotone: a < b  <=>  key(a) < key(b)
// for non-NaN values), so warp min/max reductions of coordinates can use the
// integer reduction instructions.  The map is its own inverse.
// Sparse-cell particles, a warp per 32 consecutive entries of the sparse
// work order.  Each lane lists the source ranges of its particle: the
// sparse cells among the neighbour cells that the cube of half-width
// `reach` around it touches, from its own cell on (higher keys; in the own
// cell, the higher sorted positions).  That is at most 8 cells where cells
// are wider than two linking lengths; narrower cells, and the key order of
// wrapped periodic neighbours, allow up to all 27, and a lane tests the
// ranges beyond the first MAX_RANGES itself, right away.  The warp then
// runs all pairs of all lanes in rounds of 32, one pair per lane (a lane
// finds its pair's particle by a binary search over the lanes' pair
// offsets and its source by walking that particle's ranges), so the lanes
// stay busy however unevenly the pairs are spread over the particles.
// Pairs with dense-cell particles are the dense kernel's.
constexpr int MAX_RANGES = 8;

__global__ void __launch_bounds__(BLK, 4) fof_link_kernel(
    const float4 *__restrict__ pos, const uint32_t *__restrict__ skey,
    const uint32_t *__restrict__ prid, const RegionDev *__restrict__ R,
    const uint32_t *__restrict__ cell_start, int *parent, int64_t w0, int64_t w1, LinkParams P,
    DenseIndex D, int32_t *flags) {
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ uint2 ranges[BLK][MAX_RANGES];  // (first source, count)
  const int lane = threadIdx.x & 31;
  const int wbase_t = threadIdx.x & ~31;
  const int64_t nw = ((int64_t)gridDim.x * BLK) >> 5;
  for (int64_t wb = w0 + (((int64_t)blockIdx.x * BLK + threadIdx.x) >> 5) * 32; wb < w1; wb += nw * 32) {
    const int64_t w = wb + lane;
    const bool valid = w < w1;
    const int ip = valid ? (int)D.order[w] : 0;
    const float4 me = valid ? pos[ip] : make_float4(0.f, 0.f, 0.f, 0.f);
    const RegionDev &r = R[valid ? prid[ip] : 0];
    uint32_t total = 0;
    int nr = 0;
    if (valid) {
      const uint32_t local = skey[ip] - (uint32_t)r.cell_off;
      const int64_t N0 = r.N[0], N1 = r.N[1], N2 = r.N[2];
      int64_t ixyz[3];
      {
        const uint32_t n0 = (uint32_t)N0, n1 = (uint32_t)N1;
        const uint32_t q0 = local / n0;
        ixyz[0] = local - q0 * n0;
        ixyz[1] = q0 % n1;
        ixyz[2] = q0 / n1;
      }
      const int64_t Nd[3] = {N0, N1, N2};
      const float mexyz[3] = {me.x, me.y, me.z};
      int lo[3], hi[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const bool pd = (r.pdim >> d) & 1;
        if (Nd[d] == 1) { lo[d] = 0; hi[d] = 0; continue; }
        const float clo = cell_lower(r, d, ixyz[d]);
        const float chi = cell_lower(r, d, ixyz[d] + 1);
        const bool below = __fsub_rn(mexyz[d], D.reach) < clo;
        const bool above = __fadd_rn(mexyz[d], D.reach) >= chi;
        if (pd && Nd[d] == 2) { lo[d] = 0; hi[d] = (below || above) ? 1 : 0; }
        else { lo[d] = below ? -1 : 0; hi[d] = above ? 1 : 0; }
      }
      // (the distance test takes the minimum image itself: a wrapped cell
      // needs no coordinate shift)
      for (int dz = lo[2]; dz <= hi[2]; ++dz) {
        int64_t jz = ixyz[2] + dz;
        if ((r.pdim >> 2) & 1) {
          if (jz < 0) jz += N2; else if (jz >= N2) jz -= N2;
        } else if (jz < 0 || jz >= N2) continue;
        for (int dy = lo[1]; dy <= hi[1]; ++dy) {
          int64_t jy = ixyz[1] + dy;
          if ((r.pdim >> 1) & 1) {
            if (jy < 0) jy += N1; else if (jy >= N1) jy -= N1;
          } else if (jy < 0 || jy >= N1) continue;
          for (int dx = lo[0]; dx <= hi[0]; ++dx) {
            int64_t jx = ixyz[0] + dx;
            if (r.pdim & 1) {
              if (jx < 0) jx += N0; else if (jx >= N0) jx -= N0;
            } else if (jx < 0 || jx >= N0) continue;
            const int64_t jl = jx + N0 * (jy + N1 * jz);
            if (jl < (int64_t)local) continue;
            const uint64_t jc = r.cell_off + (uint64_t)jl;
            uint32_t b = cell_start[jc];
            const uint32_t e = cell_start[jc + 1];
            if (e - b > (uint32_t)DENSE_T) continue;  // pairs with a dense cell: the dense kernel
            if (jl == (int64_t)local) b = (uint32_t)ip + 1;
            if (e <= b) continue;
            if (nr < MAX_RANGES) {
              ranges[threadIdx.x][nr++] = make_uint2(b, e - b);
              total += e - b;
            } else {
              const bool per = r.periodic != 0;
              for (uint32_t q = b; q < e; ++q) {
                const float4 o = pos[q];
                const bool lk = per ? linked_pbc(me, o, P) : linked_open(me, o, P.rp2_open);
                if (lk) {
                  int rp = -1;
                  link_pair(parent, ip, (int)q, rp, flags);
                }
              }
            }
          }
        }
      }
    }
    // pair offsets of the lanes
    uint32_t incl = total;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += v;
    }
    const uint32_t excl = incl - total;
    const uint32_t T = __shfl_sync(FULL, incl, 31);
    __syncwarp();
    for (uint32_t g0 = 0; g0 < T; g0 += 32) {
      const uint32_t g = g0 + (uint32_t)lane;
      // owner lane of pair g: the number of lanes whose pairs end at or before g
      int owner = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const uint32_t v = __shfl_sync(FULL, incl, owner + step - 1);
        if (v <= g) owner += step;
      }
      owner &= 31;
      const uint32_t oexcl = __shfl_sync(FULL, excl, owner);
      const int po = __shfl_sync(FULL, ip, owner);
      float4 pm;
      pm.x = __shfl_sync(FULL, me.x, owner);
      pm.y = __shfl_sync(FULL, me.y, owner);
      pm.z = __shfl_sync(FULL, me.z, owner);
      pm.w = 0.f;
      const bool per = __shfl_sync(FULL, r.periodic, owner) != 0;
      if (g < T) {
        uint32_t j = g - oexcl;
        const uint2 *rg = ranges[wbase_t + owner];
        int k = 0;
        while (j >= rg[k].y) {
          j -= rg[k].y;
          ++k;
        }
        const int q = (int)(rg[k].x + j);
        const float4 o = pos[q];
        const bool lk = per ? linked_pbc(pm, o, P) : linked_open(pm, o, P.rp2_open);
        if (lk) {
          int rp = -1;
          link_pair(parent, po, q, rp, flags);
        }
      }
    }
    __syncwarp();
  }
}

// Dense cells, warp-cooperative: a warp takes a chunk of up to 32 particles
// of one dense cell (consecutive in sub-cell order, so the chunk is
// compact) and walks the neighbour cells and sub-cells that the chunk's
// bounding box widened by `reach` can touch.  Sources come in coalesced
// batches of 32; a source enters the pair loop only if it lies inside the
// widened box, and then every lane tests it against its own particle with
// the exact reference test.
//
// Which side tests a pair: two dense cells, this kernel from the lower cell
// (in one cell, from the lower sorted position); a dense and a sparse cell,
// this kernel from the dense cell, whichever key is lower; two sparse cells,
// the per-particle kernel.  Every pair within reach is tested once, and the
// reference test is symmetric (|a - b| = |b - a| in IEEE arithmetic), so
// the set of linked pairs, and with it the partition, equals the
// reference's.
struct DenseChunk {
  uint32_t cell, e0;  // dense cell (global cell index), first index in its dpos list
};

__global__ void __launch_bounds__(BLK, 3) fof_link_dense_kernel(
    const float4 *__restrict__ pos, const uint32_t *__restrict__ prid, const RegionDev *__restrict__ R,
    const uint32_t *__restrict__ cell_start, int *parent, const DenseChunk *__restrict__ chunks,
    int64_t nchunks, LinkParams P, DenseIndex D, int32_t *flags) {
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ float4 sbuf[BLK];
  __shared__ int shint[BLK];
  const int lane = threadIdx.x & 31;
  float4 *wbuf = sbuf + (threadIdx.x & ~31);
  int *whint = shint + (threadIdx.x & ~31);
  const int64_t nw = ((int64_t)gridDim.x * BLK) >> 5;
  for (int64_t ch = ((int64_t)blockIdx.x * BLK + threadIdx.x) >> 5; ch < nchunks; ch += nw) {
    const DenseChunk C = chunks[ch];
    const int64_t cb = cell_start[C.cell];
    const int64_t cn = (int64_t)cell_start[C.cell + 1] - cb;
    const int64_t k = (int64_t)C.e0 + lane;
    const bool valid = k < cn;
    float4 me = make_float4(0.f, 0.f, 0.f, 0.f);
    if (valid) me = D.dpos[cb + k];
    const int ip = valid ? __float_as_int(me.w) : -1;
    const RegionDev &r = R[prid[cb]];
    const bool my_vd = is_vd(r, cn);
    const int64_t local = (int64_t)C.cell - (int64_t)r.cell_off;
    const int64_t N0 = r.N[0], N1 = r.N[1], N2 = r.N[2];
    const int64_t ixyz[3] = {local % N0, (local / N0) % N1, local / (N0 * N1)};
    const int64_t Nd[3] = {N0, N1, N2};
    const bool per = r.periodic != 0;
    // chunk bounding box
    float bl[3] = {valid ? me.x : 3e38f, valid ? me.y : 3e38f, valid ? me.z : 3e38f};
    float bh[3] = {valid ? me.x : -3e38f, valid ? me.y : -3e38f, valid ? me.z : -3e38f};
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        bl[d] = fminf(bl[d], __shfl_xor_sync(FULL, bl[d], o));
        bh[d] = fmaxf(bh[d], __shfl_xor_sync(FULL, bh[d], o));
      }
    int lo[3], hi[3];
    bool open_ax[3];  // periodic axes of one or two cells: no box along them
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const bool pd = (r.pdim >> d) & 1;
      open_ax[d] = pd && Nd[d] <= 2;
      if (Nd[d] == 1) { lo[d] = 0; hi[d] = 0; continue; }
      const float clo = cell_lower(r, d, ixyz[d]);
      const float chi = cell_lower(r, d, ixyz[d] + 1);
      const bool below = __fsub_rn(bl[d], D.reach) < clo;
      const bool above = __fadd_rn(bh[d], D.reach) >= chi;
      if (pd && Nd[d] == 2) { lo[d] = 0; hi[d] = (below || above) ? 1 : 0; }
      else { lo[d] = below ? -1 : 0; hi[d] = above ? 1 : 0; }
    }
    // --- neighbour cells, one per lane (lane = 9 (dz+1) + 3 (dy+1) + dx+1)
    bool use = false, dense = false, own = false, single = false;
    int64_t nb_b = 0, nb_e = 0, jcoord[3] = {0, 0, 0};
    uint64_t jc = 0;
    float sh[3] = {0.f, 0.f, 0.f};
    if (lane < 27) {
      const int off[3] = {lane % 3 - 1, (lane / 3) % 3 - 1, lane / 9 - 1};
      use = true;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (off[d] < lo[d] || off[d] > hi[d]) use = false;
        int64_t j = ixyz[d] + off[d];
        if ((r.pdim >> d) & 1) {
          if (j < 0) { j += Nd[d]; sh[d] = (float)P.L; } else if (j >= Nd[d]) { j -= Nd[d]; sh[d] = -(float)P.L; }
        } else if (j < 0 || j >= Nd[d]) use = false;
        jcoord[d] = j;
      }
      if (use) {
        const int64_t jl = jcoord[0] + N0 * (jcoord[1] + N1 * jcoord[2]);
        jc = r.cell_off + (uint64_t)jl;
        nb_b = cell_start[jc];
        nb_e = cell_start[jc + 1];
        dense = nb_e - nb_b > DENSE_T;
        // pairs with a lower dense cell are that cell's; pairs with sparse
        // cells are all tested here; pairs of two very dense cells are the
        // merge kernels'
        if ((dense && jl < local) || nb_e == nb_b) use = false;
        if (use && dense && my_vd && is_vd(r, nb_e - nb_b)) use = false;
        own = jl == local;
        if (use) {
          const SubGrid g = dense ? dense_sub(r, nb_e - nb_b) : SubGrid{{1, 1, 1}, {0.f, 0.f, 0.f}};
          single = g.s[0] * g.s[1] * g.s[2] == 1;
        }
      }
    }
    int rp = valid ? dsu_find(parent, ip) : -1;  // cached root of this lane's particle
    // --- cells that are one source range (sparse cells, dense cells of one
    // sub-cell): their sources packed into shared batches of 32
    {
      const uint32_t cnt = (use && single) ? (uint32_t)(nb_e - nb_b) : 0u;
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
        const uint32_t ob = (uint32_t)__shfl_sync(FULL, (unsigned)nb_b, owner);
        const uint32_t oex = __shfl_sync(FULL, excl, owner);
        const bool od = __shfl_sync(FULL, (int)dense, owner) != 0;
        const bool oown = __shfl_sync(FULL, (int)own, owner) != 0;
        const float osh0 = __shfl_sync(FULL, sh[0], owner), osh1 = __shfl_sync(FULL, sh[1], owner),
                    osh2 = __shfl_sync(FULL, sh[2], owner);
        bool cand = false;
        if (g < T) {
          const uint32_t t = ob + (g - oex);
          float4 o;
          int q;
          if (od) {
            o = D.dpos[t];
            q = __float_as_int(o.w);
          } else {
            o = pos[t];
            q = (int)t;
          }
          const float osh[3] = {osh0, osh1, osh2};
          const float oc[3] = {o.x, o.y, o.z};
          cand = true;
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            if (open_ax[d]) continue;
            const float wl = __fsub_rn(__fadd_rn(bl[d], osh[d]), D.reach);
            const float wh = __fadd_rn(__fadd_rn(bh[d], osh[d]), D.reach);
            cand = cand && oc[d] >= wl && oc[d] <= wh;
          }
          o.w = __int_as_float(oown ? ~q : q);  // own-cell sources carry their flag
          wbuf[lane] = o;
          whint[lane] = cand ? dsu_find(parent, q) : -2;
        }
        __syncwarp();
        unsigned mask = __ballot_sync(FULL, cand);
        while (mask) {
          const int src = __ffs(mask) - 1;
          mask &= mask - 1;
          const float4 so = wbuf[src];
          const int qw = __float_as_int(so.w);
          const bool sown = qw < 0;
          const int qs = sown ? ~qw : qw;
          if (valid && whint[src] != rp && !(sown && qs <= ip)) {
            const bool lk = per ? linked_pbc(me, so, P) : linked_open(me, so, P.rp2_open);
            if (lk) link_pair(parent, ip, qs, rp, flags);
          }
        }
        __syncwarp();
      }
    }
    // --- dense cells of several sub-cells: one after the other, a source
    // range per sub-cell row the widened box overlaps
    unsigned multi = __ballot_sync(FULL, use && !single);
    while (multi) {
      const int nl = __ffs(multi) - 1;
      multi &= multi - 1;
      const int64_t b = (int64_t)__shfl_sync(FULL, (unsigned long long)nb_b, nl);
      const int64_t e = (int64_t)__shfl_sync(FULL, (unsigned long long)nb_e, nl);
      const uint64_t jcn = __shfl_sync(FULL, (unsigned long long)jc, nl);
      const bool own_n = __shfl_sync(FULL, (int)own, nl) != 0;
      int64_t jcn3[3];
      float wl[3], wh[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        jcn3[d] = (int64_t)__shfl_sync(FULL, (unsigned long long)jcoord[d], nl);
        const float s = __shfl_sync(FULL, sh[d], nl);
        if (open_ax[d]) {
          wl[d] = -3e38f;
          wh[d] = 3e38f;
        } else {
          wl[d] = __fsub_rn(__fadd_rn(bl[d], s), D.reach);
          wh[d] = __fadd_rn(__fadd_rn(bh[d], s), D.reach);
        }
      }
      const uint32_t *tab = D.tab + (int64_t)D.rank[jcn] * D.stride;
      const SubGrid g = dense_sub(r, e - b);
      int slo[3], shi[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float clo = cell_lower(r, d, jcn3[d]);
        slo[d] = sub_of(wl[d], clo, g.inv[d], g.s[d]);
        shi[d] = sub_of(wh[d], clo, g.inv[d], g.s[d]);
      }
      for (int sz = slo[2]; sz <= shi[2]; ++sz)
        for (int sy = slo[1]; sy <= shi[1]; ++sy) {
          const int s0 = slo[0] + g.s[0] * (sy + g.s[1] * sz);
          const int64_t k0 = tab[s0], k1 = tab[s0 + (shi[0] - slo[0]) + 1];
          for (int64_t base = k0; base < k1; base += 32) {
            const int64_t t = base + lane;
            float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
            int q = -1, hq = -2;
            bool cand = false;
            if (t < k1) {
              o = D.dpos[b + t];
              q = __float_as_int(o.w);
              cand = o.x >= wl[0] && o.x <= wh[0] && o.y >= wl[1] && o.y <= wh[1] && o.z >= wl[2] &&
                     o.z <= wh[2];
              if (cand) hq = dsu_find(parent, q);
            }
            unsigned mask = __ballot_sync(FULL, cand);
            while (mask) {
              const int src = __ffs(mask) - 1;
              mask &= mask - 1;
              float4 so;
              so.x = __shfl_sync(FULL, o.x, src);
              so.y = __shfl_sync(FULL, o.y, src);
              so.z = __shfl_sync(FULL, o.z, src);
              so.w = 0.f;
              const int qs = __shfl_sync(FULL, q, src);
              const int hs = __shfl_sync(FULL, hq, src);
              if (valid && hs != rp && !(own_n && qs <= ip)) {
                const bool lk = per ? linked_pbc(me, so, P) : linked_open(me, so, P.rp2_open);
                if (lk) link_pair(parent, ip, qs, rp, flags);
              }
            }
          }
        }
    }
  }
}

// Chunks of up to 32 particles per dense cell.
__global__ void fof_dense_chunk_count_kernel(const uint32_t *__restrict__ list, const uint32_t *__restrict__ cs,
                                             int64_t ndense, uint32_t *__restrict__ cnt) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ndense;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t c = list[i];
    cnt[i] = (cs[c + 1] - cs[c] + 31u) / 32u;
  }
}

__global__ void fof_dense_chunk_fill_kernel(const uint32_t *__restrict__ list, const uint32_t *__restrict__ cs,
                                            const uint32_t *__restrict__ off, int64_t ndense,
                                            DenseChunk *__restrict__ chunks) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ndense;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t c = list[i];
    const uint32_t n = (cs[c + 1] - cs[c] + 31u) / 32u;
    for (uint32_t j = 0; j < n; ++j) chunks[off[i] + j] = DenseChunk{c, 32u * j};
  }
}

__global__ void fof_dense_flag_kernel(const uint32_t *__restrict__ cs,
                                      const uint64_t *__restrict__ cell_off,
                                      const RegionDev *__restrict__ R, int nreg, int64_t ncell,
                                      uint32_t *__restrict__ flag) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell;
       c += (int64_t)gridDim.x * blockDim.x) {
    flag[c] = cs[c + 1] - cs[c] > (uint32_t)DENSE_T ? 1u : 0u;
  }
}

__global__ void fof_dense_pos_flag_kernel(const uint32_t *__restrict__ skey,
                                          const uint32_t *__restrict__ cflag, int64_t n,
                                          uint32_t *__restrict__ pflag) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x)
    pflag[p] = cflag[skey[p]];
}

// Dense-cell particles first (they carry most of the pair tests, so they
// start early), the rest after them; both parts keep the sorted order.
__global__ void fof_order_kernel(const uint32_t *__restrict__ pflag,
                                 const uint32_t *__restrict__ prank, int64_t n, int64_t ndense_p,
                                 uint32_t *__restrict__ order) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = pflag[p] ? (int64_t)prank[p] : ndense_p + (p - (int64_t)prank[p]);
    order[k] = (uint32_t)p;
  }
}

__global__ void fof_dense_list_kernel(const uint32_t *__restrict__ flag,
                                      const uint32_t *__restrict__ rank, int64_t ncell,
                                      uint32_t *__restrict__ list) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell;
       c += (int64_t)gridDim.x * blockDim.x)
    if (flag[c]) list[rank[c]] = (uint32_t)c;
}

// One block per dense cell: counting sort of its particles by sub-cell.
__global__ void __launch_bounds__(BLK) fof_dense_build_kernel(
    const uint32_t *__restrict__ list, const uint32_t *__restrict__ cs,
    const float4 *__restrict__ pos, const RegionDev *__restrict__ R,
    const uint64_t *__restrict__ cell_off, int nreg, int stride, uint32_t *__restrict__ tab,
    float4 *__restrict__ dpos) {
  __shared__ uint32_t hist[SUB_MAX + 1];
  __shared__ uint32_t cur[SUB_MAX + 1];
  const uint32_t c = list[blockIdx.x];
  const int rid = nreg == 1 ? 0 : region_of_key(cell_off, nreg, (uint64_t)c);
  const RegionDev &r = R[rid];
  const int64_t local = (int64_t)c - (int64_t)r.cell_off;
  const int64_t N0 = r.N[0], N1 = r.N[1];
  const int64_t ic[3] = {local % N0, (local / N0) % N1, local / (N0 * N1)};
  float clo[3];
  for (int d = 0; d < 3; ++d) clo[d] = cell_lower(r, d, ic[d]);
  for (int k = threadIdx.x; k <= SUB_MAX; k += BLK) hist[k] = 0;
  __syncthreads();
  const int64_t base = cs[c];
  const int64_t n = (int64_t)cs[c + 1] - base;
  const SubGrid g = dense_sub(r, n);
  const int S = g.s[0] * g.s[1] * g.s[2];
  for (int64_t k = threadIdx.x; k < n; k += BLK) {
    const float4 v = pos[base + k];
    const int sx = sub_of(v.x, clo[0], g.inv[0], g.s[0]);
    const int sy = sub_of(v.y, clo[1], g.inv[1], g.s[1]);
    const int sz = sub_of(v.z, clo[2], g.inv[2], g.s[2]);
    atomicAdd(&hist[sx + g.s[0] * (sy + g.s[1] * sz)], 1u);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (int k = 0; k < S; ++k) {
      const uint32_t h = hist[k];
      cur[k] = run;
      run += h;
    }
    cur[S] = run;
  }
  __syncthreads();
  uint32_t *t = tab + (int64_t)blockIdx.x * stride;
  for (int k = threadIdx.x; k <= S; k += BLK) t[k] = cur[k];
  __syncthreads();
  for (int64_t k = threadIdx.x; k < n; k += BLK) {
    const float4 v = pos[base + k];
    const int sx = sub_of(v.x, clo[0], g.inv[0], g.s[0]);
    const int sy = sub_of(v.y, clo[1], g.inv[1], g.s[1]);
    const int sz = sub_of(v.z, clo[2], g.inv[2], g.s[2]);
    const uint32_t slot = atomicAdd(&cur[sx + g.s[0] * (sy + g.s[1] * sz)], 1u);
    dpos[base + slot] = make_float4(v.x, v.y, v.z, __int_as_float((int)(base + k)));
  }
}

// Very dense cells, step 1: every particle of a merge sub-cell joins the
// sub-cell's first particle (every pair inside one passes the exact test,
// see region_geometry).  One block per dense cell; the others return.
__global__ void __launch_bounds__(BLK) fof_vd_intra_kernel(
    const uint32_t *__restrict__ list, const uint32_t *__restrict__ cs, const RegionDev *__restrict__ R,
    const uint64_t *__restrict__ cell_off, int nreg, int stride, const uint32_t *__restrict__ tab,
    const float4 *__restrict__ dpos, int *parent, int32_t *flags) {
  const uint32_t c = list[blockIdx.x];
  const int64_t base = cs[c];
  const int64_t n = (int64_t)cs[c + 1] - base;
  const RegionDev &r = R[nreg == 1 ? 0 : region_of_key(cell_off, nreg, (uint64_t)c)];
  if (!is_vd(r, n)) return;
  if (threadIdx.x == 0) atomicAdd(&flags[FLAG_VD], 1);
  const SubGrid g = dense_sub(r, n);
  const int S = g.s[0] * g.s[1] * g.s[2];
  const uint32_t *t = tab + (int64_t)blockIdx.x * stride;
  const int lane = threadIdx.x & 31;
  for (int sc = threadIdx.x >> 5; sc < S; sc += BLK / 32) {
    const int64_t m0 = base + t[sc], m1 = base + t[sc + 1];
    if (m1 - m0 < 2) continue;
    const int lead = __float_as_int(dpos[m0].w);
    int rp = -1;
    for (int64_t k = m0 + 1 + lane; k < m1; k += 32) link_pair(parent, lead, __float_as_int(dpos[k].w), rp, flags);
  }
}

// Very dense cells, step 2: merge sub-cells A (of cell c) and B (of c or of
// a neighbour very dense cell; pairs of cells from the lower cell, in one
// cell B > A) whose grid boxes come within `reach` are joined when any of
// their pairs passes the exact test.  The pairs are tested only while the
// two roots differ, 32 members of A at a time against each member of B
// inside A's widened box, up to the first link: sub-cells already joined
// cost two root look-ups, and linking one pair joins the whole of both.
// A warp per sub-cell A, a block per dense cell.
__global__ void __launch_bounds__(BLK) fof_vd_inter_kernel(
    const uint32_t *__restrict__ list, const uint32_t *__restrict__ cs, const RegionDev *__restrict__ R,
    const uint64_t *__restrict__ cell_off, int nreg, int stride, const uint32_t *__restrict__ tab,
    const uint32_t *__restrict__ rank, const float4 *__restrict__ dpos, int *parent, LinkParams P,
    float reach, int32_t *flags) {
  constexpr unsigned FULL = 0xffffffffu;
  const uint32_t c = list[blockIdx.x];
  const int64_t base = cs[c];
  const int64_t n = (int64_t)cs[c + 1] - base;
  const RegionDev &r = R[nreg == 1 ? 0 : region_of_key(cell_off, nreg, (uint64_t)c)];
  if (!is_vd(r, n)) return;
  const SubGrid g = dense_sub(r, n);
  const int S = g.s[0] * g.s[1] * g.s[2];
  const uint32_t *t = tab + (int64_t)blockIdx.x * stride;
  const int lane = threadIdx.x & 31;
  const int64_t local = (int64_t)c - (int64_t)r.cell_off;
  const int64_t Nd[3] = {r.N[0], r.N[1], r.N[2]};
  const int64_t ixyz[3] = {local % Nd[0], (local / Nd[0]) % Nd[1], local / (Nd[0] * Nd[1])};
  const bool per = r.periodic != 0;
  for (int A = threadIdx.x >> 5; A < S; A += BLK / 32) {
    const int64_t a0 = base + t[A], a1 = base + t[A + 1];
    if (a1 == a0) continue;
    // A's bounding box from its members
    float lo[3] = {3e38f, 3e38f, 3e38f}, hi[3] = {-3e38f, -3e38f, -3e38f};
    for (int64_t k = a0 + lane; k < a1; k += 32) {
      const float4 v = dpos[k];
      lo[0] = fminf(lo[0], v.x); lo[1] = fminf(lo[1], v.y); lo[2] = fminf(lo[2], v.z);
      hi[0] = fmaxf(hi[0], v.x); hi[1] = fmaxf(hi[1], v.y); hi[2] = fmaxf(hi[2], v.z);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        lo[d] = fminf(lo[d], __shfl_xor_sync(FULL, lo[d], o));
        hi[d] = fmaxf(hi[d], __shfl_xor_sync(FULL, hi[d], o));
      }
    const int leadA = __float_as_int(dpos[a0].w);
    for (int nb = 0; nb < 27; ++nb) {
      const int off[3] = {nb % 3 - 1, (nb / 3) % 3 - 1, nb / 9 - 1};
      int64_t jcoord[3];
      float sh[3] = {0.f, 0.f, 0.f};
      bool ok = true;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        int64_t j = ixyz[d] + off[d];
        if ((r.pdim >> d) & 1) {
          if (j < 0) { j += Nd[d]; sh[d] = (float)P.L; } else if (j >= Nd[d]) { j -= Nd[d]; sh[d] = -(float)P.L; }
        } else if (j < 0 || j >= Nd[d]) ok = false;
        jcoord[d] = j;
      }
      if (!ok) continue;
      const int64_t jl = jcoord[0] + Nd[0] * (jcoord[1] + Nd[1] * jcoord[2]);
      if (jl < local) continue;
      const uint64_t jc = r.cell_off + (uint64_t)jl;
      const int64_t jb = cs[jc], nj = (int64_t)cs[jc + 1] - jb;
      if (!is_vd(r, nj)) continue;
      const SubGrid gj = dense_sub(r, nj);
      const uint32_t *tj = tab + (int64_t)rank[jc] * stride;
      float wl[3], wh[3];
      int slo[3], shi[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        wl[d] = __fsub_rn(__fadd_rn(lo[d], sh[d]), reach);
        wh[d] = __fadd_rn(__fadd_rn(hi[d], sh[d]), reach);
        const float cl = cell_lower(r, d, jcoord[d]);
        slo[d] = sub_of(wl[d], cl, gj.inv[d], gj.s[d]);
        shi[d] = sub_of(wh[d], cl, gj.inv[d], gj.s[d]);
      }
      for (int bz = slo[2]; bz <= shi[2]; ++bz)
        for (int by = slo[1]; by <= shi[1]; ++by)
          for (int bx = slo[0]; bx <= shi[0]; ++bx) {
            const int B = bx + gj.s[0] * (by + gj.s[1] * bz);
            if (jl == local && B <= A) continue;
            const int64_t b0 = jb + tj[B], b1 = jb + tj[B + 1];
            if (b1 == b0) continue;
            int same = 0;
            if (lane == 0) same = dsu_find(parent, leadA) == dsu_find(parent, __float_as_int(dpos[b0].w));
            if (__shfl_sync(FULL, same, 0)) continue;
            bool done = false;
            for (int64_t ka = a0; ka < a1 && !done; ka += 32) {
              const int64_t k = ka + lane;
              const bool valid = k < a1;
              const float4 me = valid ? dpos[k] : make_float4(0.f, 0.f, 0.f, 0.f);
              for (int64_t kb = b0; kb < b1; ++kb) {
                const float4 o = dpos[kb];
                if (!(o.x >= wl[0] && o.x <= wh[0] && o.y >= wl[1] && o.y <= wh[1] && o.z >= wl[2] &&
                      o.z <= wh[2]))
                  continue;
                const bool lk = valid && (per ? linked_pbc(me, o, P) : linked_open(me, o, P.rp2_open));
                const unsigned m = __ballot_sync(FULL, lk);
                if (m) {
                  if (lane == __ffs(m) - 1) {
                    int rp = -1;
                    link_pair(parent, __float_as_int(me.w), __float_as_int(o.w), rp, flags);
                  }
                  done = true;
                  break;
                }
              }
            }
          }
    }
  }
}

__global__ void fof_init_parent(int *parent, int64_t n) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x)
    parent[p] = (int)p;
}

// Final labels.  The forest is static after linking; find() may still
// shorten paths with halving stores (each store points a node at one of its
// ancestors, so concurrent finds stay correct), but the label of every
// particle goes to a separate array: a store into parent[] could be
// overwritten by another thread's halving store with a non-root ancestor.
__global__ void __launch_bounds__(BLK) fof_root_kernel(int *parent, int *lab, uint32_t *gsize,
                                                       int64_t n) {
  for (int64_t base = (int64_t)blockIdx.x * BLK; base < n; base += (int64_t)gridDim.x * BLK) {
    const int64_t p = base + threadIdx.x;
    int root = -1;
    if (p < n) {
      root = dsu_find(parent, (int)p);
      lab[p] = root;
    }
    const unsigned peers = __match_any_sync(0xffffffffu, root);
    const int leader = __ffs(peers) - 1;
    if (root >= 0 && (int)(threadIdx.x & 31) == leader) atomicAdd(&gsize[root], (uint32_t)__popc(peers));
  }
}

__global__ void fof_cand_flag_kernel(const int *lab, const uint32_t *gsize, int64_t n,
                                     uint32_t np_min, uint32_t *flag) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x)
    flag[p] = (lab[p] == (int)p && gsize[p] >= np_min) ? 1u : 0u;
}

// Candidate of every sorted particle (-1 if its group is too small), plus
// the no-unbinding outputs (fof_fortran.f90:207-222).
__global__ void fof_member_kernel(const int *lab, const uint32_t *gsize,
                                  const uint32_t *crank, const float4 *pos, int64_t n,
                                  uint32_t np_min, int write_out, int32_t *pcand,
                                  int32_t *in_halo, int32_t *halo_id) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int r = lab[p];
    int32_t c = -1;
    if (gsize[r] >= np_min) c = (int32_t)crank[r];
    pcand[p] = c;
    if (write_out && c >= 0) {
      const int i = __float_as_int(pos[p].w);
      in_halo[i] = 1;
      halo_id[i] = c + 1;
    }
  }
}

// Per-candidate weighted sums for the centre of mass and mean velocity
// (fof_fortran.f90:225-238): acc[c] = {w, w*dx, w*dv}.
__global__ void __launch_bounds__(BLK) fof_com_kernel(Coords xp, Coords vp, const double *mp,
                                                      const float4 *pos, const int32_t *pcand,
                                                      const int64_t *cand_anchor, int64_t n,
                                                      double L, double half, double *acc) {
  for (int64_t base = (int64_t)blockIdx.x * BLK; base < n; base += (int64_t)gridDim.x * BLK) {
    const int64_t p = base + threadIdx.x;
    int32_t c = p < n ? pcand[p] : -1;
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    if (c >= 0) {
      const int64_t i = __float_as_int(pos[p].w);
      const int64_t a = cand_anchor[c];
      const double w = mp ? mp[i] : 1.0;
      v[0] = w;
      for (int d = 0; d < 3; ++d) {
        v[1 + d] = w * unwrap(xp.get(i, d), xp.get(a, d), half, L);
        v[4 + d] = w * vp.get(i, d);
      }
    }
    const unsigned peers = __match_any_sync(0xffffffffu, c);
    if (peers == 0xffffffffu) {
      for (int k = 0; k < 7; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
      if ((threadIdx.x & 31) == 0 && c >= 0)
        for (int k = 0; k < 7; ++k) atomicAdd(&acc[7 * (int64_t)c + k], v[k]);
    } else if (c >= 0) {
      for (int k = 0; k < 7; ++k) atomicAdd(&acc[7 * (int64_t)c + k], v[k]);
    }
  }
}

// Angular momentum about the candidate centre (fof_fortran.f90:239-247),
// accumulated per candidate.
__global__ void __launch_bounds__(BLK) fof_angmom_kernel(Coords xp, Coords vp, const double *mp,
                                                         const float4 *pos, const int32_t *pcand,
                                                         const int64_t *cand_anchor,
                                                         const double *acc, int64_t n, double L,
                                                         double half, double *am) {
  for (int64_t base = (int64_t)blockIdx.x * BLK; base < n; base += (int64_t)gridDim.x * BLK) {
    const int64_t p = base + threadIdx.x;
    int32_t c = p < n ? pcand[p] : -1;
    double v[3] = {0, 0, 0};
    if (c >= 0 && acc[7 * (int64_t)c] > 0.0) {
      const int64_t i = __float_as_int(pos[p].w);
      const int64_t a = cand_anchor[c];
      const double ws = acc[7 * (int64_t)c];
      const double w = mp ? mp[i] : 1.0;
      double dx[3], dv[3];
      for (int d = 0; d < 3; ++d) {
        dx[d] = unwrap(xp.get(i, d), xp.get(a, d), half, L) - acc[7 * (int64_t)c + 1 + d] / ws;
        dv[d] = vp.get(i, d) - acc[7 * (int64_t)c + 4 + d] / ws;
      }
      v[0] = w * (dx[1] * dv[2] - dx[2] * dv[1]);
      v[1] = w * (dx[2] * dv[0] - dx[0] * dv[2]);
      v[2] = w * (dx[0] * dv[1] - dx[1] * dv[0]);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, c);
    if (peers == 0xffffffffu) {
      for (int k = 0; k < 3; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
      if ((threadIdx.x & 31) == 0 && c >= 0)
        for (int k = 0; k < 3; ++k) atomicAdd(&am[3 * (int64_t)c + k], v[k]);
    } else if (c >= 0) {
      for (int k = 0; k < 3; ++k) atomicAdd(&am[3 * (int64_t)c + k], v[k]);
    }
  }
}

// anchor (first member in CRS order = the root) and region of each candidate
__global__ void fof_cand_info_kernel(const uint32_t *flag, const uint32_t *crank,
                                     const float4 *pos, const uint32_t *prid,
                                     const uint32_t *gsize, int64_t n, int64_t *cand_anchor,
                                     int32_t *cand_region, int32_t *cand_np, int32_t *cand_root) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x)
    if (flag[p]) {
      const uint32_t c = crank[p];
      cand_anchor[c] = __float_as_int(pos[p].w);
      cand_region[c] = (int32_t)prid[p];
      cand_np[c] = (int32_t)gsize[p];
      cand_root[c] = (int32_t)p;
    }
}

int bits_for(uint64_t v) {
  int b = 0;
  while (b < 64 && (v >> b) != 0) ++b;
  return b;
}

}  // namespace

// ------------------------------------------------------- host geometry

// Reference cell geometry of one region (fof_fortran.f90:528-570) from its
// unwrapped bounding box.  64-bit integers are used where the reference's
// default integers would overflow (N >= 2**29).
void region_geometry(double L, double link, int32_t np, const double *xmin, const double *xmax,
                     RegionDev &r) {
  const double half = 0.5 * L;
  double range[3];
  int pd = 0;
  for (int d = 0; d < 3; ++d) {
    range[d] = xmax[d] - xmin[d];
    if (range[d] + 2.0 * link >= L) pd |= 1 << d;
  }
  const double vol = std::max(range[0], link) * std::max(range[1], link) * std::max(range[2], link);
  auto geom = [&](double L_mesh, int64_t *N) {
    for (int d = 0; d < 3; ++d) {
      if ((pd >> d) & 1) {
        r.origin[d] = -half;
        int64_t a = (int64_t)(L / link), b = (int64_t)(L / L_mesh);
        N[d] = std::max<int64_t>(1, std::min(a, b));
        r.size[d] = L / (double)N[d];
      } else {
        r.origin[d] = xmin[d];
        N[d] = std::max<int64_t>(1, (int64_t)std::ceil(range[d] / L_mesh));
        r.size[d] = L_mesh;
      }
    }
  };
  int64_t N[3];
  double L_mesh = std::max(link, std::pow(vol / (double)std::max(1, np), 1.0 / 3.0));
  geom(L_mesh, N);
  const int64_t cap = std::max<int64_t>(262144, 4 * (int64_t)np);
  if ((double)N[0] * (double)N[1] * (double)N[2] > (double)cap) {
    L_mesh = std::pow(vol / (double)((int64_t)std::max(1, np) * 2), 1.0 / 3.0);
    L_mesh = std::max(link, L_mesh);
    geom(L_mesh, N);
  }
  for (int d = 0; d < 3; ++d) r.N[d] = (int32_t)std::min<int64_t>(N[d], INT32_MAX);
  r.pdim = pd;
  r.periodic = pd != 0;
  r.ncell = N[0] * N[1] * N[2];
  // sub-cells for dense cells: slabs at least one linking length wide; none
  // along periodic axes with fewer than 3 cells (both images are adjacent)
  int prod = 1;
  for (int d = 0; d < 3; ++d) {
    int sd = (int)std::floor(r.size[d] / link);
    if (sd < 1 || !std::isfinite(r.size[d] / link)) sd = 1;
    if (sd > 6) sd = 6;
    if (((pd >> d) & 1) && N[d] < 3) sd = 1;
    r.sub[d] = sd;
    prod *= sd;
  }
  r.sub_ok = prod > 1 ? 1 : 0;
  for (int d = 0; d < 3; ++d) r.inv_sub[d] = (float)((double)r.sub[d] / r.size[d]);
  // merge sub-cells: width at most link/sqrt(3) * 0.999 less 8 FP32 ulps of
  // the box size (the rounding of positions and sub-cell boundaries), so the
  // largest distance inside one, as the FP32/FP64 test computes it, stays
  // below the linking length; only where a cell holds at most SUB_MAX of
  // them and no periodic axis has fewer than 3 cells
  const double mw = link / std::sqrt(3.0) * 0.999 - 8.0 * 1.1920928955078125e-07 * (std::fabs(L) + 1.0);
  int64_t km = 1;
  int k[3] = {0, 0, 0};
  bool vd = mw > 0.0 && std::isfinite(mw);
  for (int d = 0; d < 3 && vd; ++d) {
    const double kk = std::ceil(r.size[d] / mw);
    if (!(kk >= 1.0) || kk > (double)SUB_MAX || (((pd >> d) & 1) && N[d] < 3)) vd = false;
    else { k[d] = (int)kk; km *= k[d]; }
  }
  if (vd && km > SUB_MAX) vd = false;
  for (int d = 0; d < 3; ++d) {
    r.vd_k[d] = vd ? k[d] : 0;
    r.vd_inv[d] = vd ? (float)((double)k[d] / r.size[d]) : 0.0f;
  }
}

int32_t fof_link_stage(Context &ctx, const FofArgs &a, FofState &st) {
  cudaStream_t s = ctx.stream;
  Arena &W = ctx.work;
  const int64_t n = a.total_np;
  const int nreg = a.nhalo;
  const double L = a.L_Box, half = 0.5 * a.L_Box;
  st.n = n;
  st.nreg = nreg;
  Coords xp{a.xp, n, a.soa};

  // --- region table and tiles (host)
  std::vector<RegionDev> reg(nreg);
  std::vector<Tile> tiles;
  int64_t start = 0;
  for (int r = 0; r < nreg; ++r) {
    RegionDev &R = reg[r];
    memset(&R, 0, sizeof(R));
    R.start = start;
    R.np = a.np_halo[r];
    R.active = (R.np >= a.np_halo_min && R.np > 0) ? 1 : 0;
    for (int64_t b = start; b < start + R.np; b += TILE)
      tiles.push_back(Tile{r, 0, b, std::min<int64_t>(start + R.np, b + TILE)});
    start += R.np;
  }
  if (start != n) {
    set_error("sum(np_halo)=%lld != total_np=%lld", (long long)start, (long long)n);
    return kInvalid;
  }
  const int64_t ntiles = (int64_t)tiles.size();
  RegionDev *dR = W.carve<RegionDev>(nreg);
  Tile *dT = W.carve<Tile>(std::max<int64_t>(ntiles, 1));
  unsigned long long *dbb = W.carve<unsigned long long>(6 * (size_t)nreg);
  if (!dR || !dT || !dbb) { set_error("workspace exhausted (regions)"); return kAlloc; }
  PYFOF_TRY(upload(ctx, dR, reg.data(), sizeof(RegionDev) * nreg, s));
  PYFOF_TRY(upload(ctx, dT, tiles.data(), sizeof(Tile) * ntiles, s));
  {
    std::vector<unsigned long long> init(6 * (size_t)nreg);
    for (int r = 0; r < nreg; ++r)
      for (int d = 0; d < 3; ++d) { init[6 * r + d] = ~0ull; init[6 * r + 3 + d] = 0ull; }
    PYFOF_TRY(upload(ctx, dbb, init.data(), sizeof(unsigned long long) * init.size(), s));
  }
  PYFOF_CUDA(cudaMemsetAsync(ctx.d_flags, 0, sizeof(int32_t) * FLAG_COUNT, s));
  if (ntiles) {
    fof_bbox_kernel<<<(unsigned)ntiles, BLK, 0, s>>>(xp, dR, dT, L, half, dbb, ctx.d_flags);
    PYFOF_CHECK_LAUNCH();
  }
  std::vector<unsigned long long> bb(6 * (size_t)nreg);
  PYFOF_CUDA(cudaMemcpyAsync(bb.data(), dbb, sizeof(unsigned long long) * bb.size(),
                             cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaMemcpyAsync(ctx.h_flags, ctx.d_flags, sizeof(int32_t) * FLAG_COUNT,
                             cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  if (ctx.h_flags[FLAG_ERR]) {
    set_error("non-finite particle coordinates");
    return ctx.h_flags[FLAG_ERR];
  }

  // --- reference geometry per region (host)
  uint64_t total_cells = 0;
  int64_t n_active = 0;
  std::vector<uint64_t> cell_off(nreg + 1);
  for (int r = 0; r < nreg; ++r) {
    RegionDev &R = reg[r];
    cell_off[r] = total_cells;
    R.cell_off = total_cells;
    if (!R.active) continue;
    double xmin[3], xmax[3];
    for (int d = 0; d < 3; ++d) {
      xmin[d] = ord_to_dbl(bb[6 * r + d]);
      xmax[d] = ord_to_dbl(bb[6 * r + 3 + d]);
    }
    region_geometry(L, a.link, R.np, xmin, xmax, R);
    total_cells += (uint64_t)R.ncell;
    n_active += R.np;
  }
  cell_off[nreg] = total_cells;
  if (total_cells >= 0xffffffffull) {
    set_error("total cell count %llu exceeds the 32-bit key range",
              (unsigned long long)total_cells);
    return kAlloc;
  }
  st.n_active = n_active;
  st.total_cells = total_cells;
  ctx.last_cells = (int64_t)total_cells;
  ctx.last_active = n_active;
  PYFOF_TRY(upload(ctx, dR, reg.data(), sizeof(RegionDev) * nreg, s));
  uint64_t *dcoff = W.carve<uint64_t>(nreg + 1);
  uint32_t *keys = W.carve<uint32_t>(std::max<int64_t>(n, 1));
  uint32_t *cstart = W.carve<uint32_t>(total_cells + 2);
  uint32_t *ka = W.carve<uint32_t>(std::max<int64_t>(n, 1));
  uint32_t *va = W.carve<uint32_t>(std::max<int64_t>(n, 1));
  uint32_t *kb = W.carve<uint32_t>(std::max<int64_t>(n, 1));
  uint32_t *vb = W.carve<uint32_t>(std::max<int64_t>(n, 1));
  if (!dcoff || !keys || !cstart || !ka || !va || !kb || !vb) {
    set_error("workspace exhausted (keys)");
    return kAlloc;
  }
  PYFOF_TRY(upload(ctx, dcoff, cell_off.data(), sizeof(uint64_t) * (nreg + 1), s));
  PYFOF_CUDA(cudaMemsetAsync(cstart, 0, sizeof(uint32_t) * (total_cells + 2), s));
  const uint32_t sentinel = (uint32_t)total_cells;
  // slots within the cells go to va (radix scratch when the sort is needed)
  if (ntiles) {
    fof_key_kernel<<<(unsigned)ntiles, BLK, 0, s>>>(xp, dR, dT, L, half, sentinel, keys, cstart, va);
    PYFOF_CHECK_LAUNCH();
  }
  // Per-cell sorts pay off where the radix sort needs a fourth pass (keys of
  // more than 24 bits) and every cell fits one block's sort; otherwise, and
  // always with cell_order 2, a stable radix sort of all keys.
  const uint64_t max_key = (n_active < n) ? total_cells : (total_cells ? total_cells - 1 : 0);
  const bool try_cells = a.cell_order == 1 || (a.cell_order == 0 && bits_for(max_key) > 24);
  uint32_t *dmax = reinterpret_cast<uint32_t *>(ctx.d_flags + FLAG_COUNT_A);
  PYFOF_CUDA(cudaMemsetAsync(dmax, 0, sizeof(uint32_t), s));
  const unsigned cgrid0 = (unsigned)std::max<int64_t>(
      1, std::min<int64_t>(ceil_div((int64_t)std::max<uint64_t>(total_cells, 1), (int64_t)BLK),
                           (int64_t)kNumSMs * 16));
  if (total_cells > 0) {
    fof_max_count_kernel<<<cgrid0, BLK, 0, s>>>(cstart, (int64_t)total_cells, dmax);
    PYFOF_CHECK_LAUNCH();
  }
  PYFOF_CUDA(cudaMemcpyAsync(ctx.h_flags + FLAG_COUNT_A, dmax, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  PYFOF_TRY(exclusive_scan_u32(cstart, cstart, (int64_t)total_cells + 1, nullptr, W, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  const uint32_t max_occ = (uint32_t)ctx.h_flags[FLAG_COUNT_A];
  ctx.last_max_cell = max_occ;
  ctx.last_cell_sorts = 0;
  uint32_t *skey, *sidx;
  if (try_cells && max_occ <= (uint32_t)CELL_SORT_MAX) {
    ctx.last_cell_sorts = 1;
    // cells of more than CELL_SORT_SMALL particles: at most n / (CELL_SORT_SMALL + 1)
    uint32_t *big = W.carve<uint32_t>(
        (size_t)std::min<int64_t>(n_active / (CELL_SORT_SMALL + 1) + 1, (int64_t)total_cells + 1));
    uint32_t *nbig = W.carve<uint32_t>(1);
    if (!big || !nbig) { set_error("workspace exhausted (cell sort)"); return kAlloc; }
    PYFOF_CUDA(cudaMemsetAsync(nbig, 0, sizeof(uint32_t), s));
    const unsigned sgrid = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>(ceil_div(std::max<int64_t>(n, 1), (int64_t)BLK), (int64_t)kNumSMs * 16));
    fof_cell_scatter_kernel<<<sgrid, BLK, 0, s>>>(keys, va, cstart, n, ka, vb);
    PYFOF_CHECK_LAUNCH();
    if (total_cells > 0) {
      fof_cell_sort_small_kernel<<<cgrid0, BLK, 0, s>>>(cstart, (int64_t)total_cells, vb, big, nbig);
      PYFOF_CHECK_LAUNCH();
      fof_cell_sort_big_kernel<<<kNumSMs * 2, 1024, 0, s>>>(cstart, big, nbig, vb);
      PYFOF_CHECK_LAUNCH();
    }
    skey = ka;
    sidx = vb;
  } else {
    PYFOF_TRY(radix_sort_pairs(keys, nullptr, n, bits_for(max_key), ka, va, kb, vb, &skey, &sidx,
                               W, s));
  }
  // --- sorted FP32 coordinates, DSU
  float4 *pos = W.carve<float4>(std::max<int64_t>(n_active, 1));
  uint32_t *prid = W.carve<uint32_t>(std::max<int64_t>(n_active, 1));
  int *parent = W.carve<int>(std::max<int64_t>(n_active, 1));
  if (!pos || !prid || !parent) { set_error("workspace exhausted (link)"); return kAlloc; }
  const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(std::max<int64_t>(n_active, 1), BLK),
                                                    (int64_t)kNumSMs * 16);
  if (n_active > 0) {
    fof_gather_kernel<<<grid, BLK, 0, s>>>(xp, dR, dcoff, nreg, skey, sidx, n_active, L, half, pos,
                                           prid);
    PYFOF_CHECK_LAUNCH();
    fof_init_parent<<<grid, BLK, 0, s>>>(parent, n_active);
    PYFOF_CHECK_LAUNCH();
    LinkParams P;
    P.L = L;
    P.half = half;
    P.rp2 = a.link * a.link;
    {
      float f = (float)P.rp2;
      if ((double)f > P.rp2) f = std::nextafter(f, -INFINITY);
      P.rp2_open = f;
    }
    P.fast_periodic = (P.rp2 > 1e-20 && P.rp2 < 1e20 && L < 1e30) ? 1 : 0;
    P.rp2_lo = (float)(P.rp2 * (1.0 - 4e-6));
    P.rp2_hi = (float)(P.rp2 * (1.0 + 4e-6));
    DenseIndex D{};
    const uint32_t *D_list = nullptr;  // dense cells in rank order
    bool any_vd = false;               // a region where very dense cells can occur
    for (int r = 0; r < nreg; ++r) any_vd = any_vd || (reg[r].active && reg[r].vd_k[0] > 0);
    int64_t ndense_p = 0;  // particles in dense cells (the head of D.order)
    int64_t ndense_chunks = 0;
    DenseChunk *dchunks = nullptr;
    // slack: relative 1e-4 for the FP32 distance arithmetic, 8 FP32 ulps of
    // the box size for the rounding of positions and query endpoints
    D.reach = (float)(a.link * (1.0 + 1e-4) + 8.0 * 1.1920928955078125e-07 * (std::fabs(L) + 1.0));
    {
      int smax = 1;
      for (int r = 0; r < nreg; ++r)
        if (reg[r].active) {
          smax = std::max(smax, reg[r].sub[0] * reg[r].sub[1] * reg[r].sub[2]);
          smax = std::max(smax, reg[r].vd_k[0] * reg[r].vd_k[1] * reg[r].vd_k[2]);
        }
      D.stride = smax + 1;
      const int64_t nc = (int64_t)total_cells;
      uint32_t *dflag = W.carve<uint32_t>(nc + 1);
      uint32_t *drank = W.carve<uint32_t>(nc + 1);
      float4 *dpos = W.carve<float4>(n_active);
      uint32_t *order = W.carve<uint32_t>(n_active);
      uint32_t *pflag = W.carve<uint32_t>(n_active + 1);
      uint32_t *prank = W.carve<uint32_t>(n_active + 1);
      if (!dflag || !drank || !dpos || !order || !pflag || !prank) {
        set_error("workspace exhausted (dense index)");
        return kAlloc;
      }
      const unsigned cgrid = (unsigned)std::min<int64_t>(ceil_div(nc, BLK), (int64_t)kNumSMs * 16);
      fof_dense_flag_kernel<<<cgrid, BLK, 0, s>>>(cstart, dcoff, dR, nreg, nc, dflag);
      PYFOF_CHECK_LAUNCH();
      PYFOF_TRY(exclusive_scan_u32(dflag, drank, nc, reinterpret_cast<uint32_t *>(ctx.d_flags + FLAG_COUNT_B), W, s));
      fof_dense_pos_flag_kernel<<<grid, BLK, 0, s>>>(skey, dflag, n_active, pflag);
      PYFOF_CHECK_LAUNCH();
      PYFOF_TRY(exclusive_scan_u32(pflag, prank, n_active, reinterpret_cast<uint32_t *>(ctx.d_flags + FLAG_COUNT_C), W, s));
      PYFOF_CUDA(cudaMemcpyAsync(ctx.h_flags, ctx.d_flags, sizeof(int32_t) * FLAG_COUNT,
                                 cudaMemcpyDeviceToHost, s));
      PYFOF_CUDA(cudaStreamSynchronize(s));
      const int64_t ndense = (uint32_t)ctx.h_flags[FLAG_COUNT_B];
      ndense_p = (uint32_t)ctx.h_flags[FLAG_COUNT_C];
      fof_order_kernel<<<grid, BLK, 0, s>>>(pflag, prank, n_active, ndense_p, order);
      PYFOF_CHECK_LAUNCH();
      uint32_t *tab = W.carve<uint32_t>(std::max<int64_t>(ndense, 1) * D.stride);
      uint32_t *list = W.carve<uint32_t>(std::max<int64_t>(ndense, 1));
      if (!tab || !list) { set_error("workspace exhausted (dense tables)"); return kAlloc; }
      if (ndense > 0) {
        fof_dense_list_kernel<<<cgrid, BLK, 0, s>>>(dflag, drank, nc, list);
        PYFOF_CHECK_LAUNCH();
        fof_dense_build_kernel<<<(unsigned)ndense, BLK, 0, s>>>(list, cstart, pos, dR, dcoff, nreg,
                                                                D.stride, tab, dpos);
        PYFOF_CHECK_LAUNCH();
        // warp chunks of the dense cells
        uint32_t *coff = W.carve<uint32_t>(ndense + 1);
        if (!coff) { set_error("workspace exhausted (dense chunks)"); return kAlloc; }
        PYFOF_CUDA(cudaMemsetAsync(coff, 0, sizeof(uint32_t) * (ndense + 1), s));
        const unsigned lgrid = (unsigned)std::min<int64_t>(ceil_div(ndense, BLK), (int64_t)kNumSMs * 16);
        fof_dense_chunk_count_kernel<<<lgrid, BLK, 0, s>>>(list, cstart, ndense, coff);
        PYFOF_CHECK_LAUNCH();
        PYFOF_TRY(exclusive_scan_u32(coff, coff, ndense + 1, nullptr, W, s));
        uint32_t nch = 0;
        PYFOF_CUDA(cudaMemcpyAsync(&nch, coff + ndense, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        PYFOF_CUDA(cudaStreamSynchronize(s));
        ndense_chunks = nch;
        dchunks = W.carve<DenseChunk>(std::max<uint32_t>(nch, 1));
        if (!dchunks) { set_error("workspace exhausted (dense chunks)"); return kAlloc; }
        fof_dense_chunk_fill_kernel<<<lgrid, BLK, 0, s>>>(list, cstart, coff, ndense, dchunks);
        PYFOF_CHECK_LAUNCH();
      }
      D.rank = drank;
      D_list = list;
      D.tab = tab;
      D.dpos = dpos;
      D.order = order;
      ctx.last_dense = ndense;
    }
    // dense-cell particles and the rest as two launches: the long pair loops
    // of the dense part do not hold back blocks of the short sparse work
    if (ctx.timing) cudaEventRecord(ctx.ev[0], s);
    PYFOF_CUDA(cudaMemsetAsync(ctx.d_flags + FLAG_VD, 0, sizeof(int32_t), s));
    if (ctx.last_dense > 0 && any_vd) {
      fof_vd_intra_kernel<<<(unsigned)ctx.last_dense, BLK, 0, s>>>(D_list, cstart, dR, dcoff, nreg, D.stride,
                                                                   D.tab, D.dpos, parent, ctx.d_flags);
      PYFOF_CHECK_LAUNCH();
      fof_vd_inter_kernel<<<(unsigned)ctx.last_dense, BLK, 0, s>>>(D_list, cstart, dR, dcoff, nreg, D.stride,
                                                                   D.tab, D.rank, D.dpos, parent, P, D.reach,
                                                                   ctx.d_flags);
      PYFOF_CHECK_LAUNCH();
    }
    PYFOF_CUDA(cudaMemcpyAsync(ctx.h_flags + FLAG_VD, ctx.d_flags + FLAG_VD, sizeof(int32_t),
                               cudaMemcpyDeviceToHost, s));
    if (ndense_chunks > 0) {
      const unsigned dgrid = (unsigned)std::min<int64_t>(ceil_div(ndense_chunks * 32, BLK), (int64_t)kNumSMs * 24);
      fof_link_dense_kernel<<<dgrid, BLK, 0, s>>>(pos, prid, dR, cstart, parent, dchunks, ndense_chunks, P, D,
                                                  ctx.d_flags);
      PYFOF_CHECK_LAUNCH();
    }
    if (n_active > ndense_p) {
      fof_link_kernel<<<grid, BLK, 0, s>>>(pos, skey, prid, dR, cstart, parent, ndense_p, n_active, P,
                                           D, ctx.d_flags);
      PYFOF_CHECK_LAUNCH();
    }
    if (ctx.timing) cudaEventRecord(ctx.ev[1], s);
  }
  st.dR = dR;
  st.pos = pos;
  st.prid = prid;
  st.parent = parent;
  st.skey = skey;
  st.sidx = sidx;
  st.cell_start = cstart;
  st.keys_free = keys;
  st.reg = reg;
  return kOk;
}

int32_t fof_candidates_stage(Context &ctx, const FofArgs &a, FofState &st, bool write_plain) {
  cudaStream_t s = ctx.stream;
  Arena &W = ctx.work;
  const int64_t na = st.n_active;
  uint32_t *gsize = W.carve<uint32_t>(std::max<int64_t>(na, 1));
  uint32_t *flag = W.carve<uint32_t>(std::max<int64_t>(na, 1) + 1);
  uint32_t *crank = W.carve<uint32_t>(std::max<int64_t>(na, 1) + 1);
  int32_t *pcand = W.carve<int32_t>(std::max<int64_t>(na, 1));
  if (!gsize || !flag || !crank || !pcand) { set_error("workspace exhausted (labels)"); return kAlloc; }
  st.ncand = 0;
  if (na > 0) {
    const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(na, BLK), (int64_t)kNumSMs * 16);
    PYFOF_CUDA(cudaMemsetAsync(gsize, 0, sizeof(uint32_t) * na, s));
    st.lab = reinterpret_cast<int *>(st.keys_free);  // keys are dead after the sort
    fof_root_kernel<<<grid, BLK, 0, s>>>(st.parent, st.lab, gsize, na);
    PYFOF_CHECK_LAUNCH();
    fof_cand_flag_kernel<<<grid, BLK, 0, s>>>(st.lab, gsize, na, (uint32_t)a.np_halo_min, flag);
    PYFOF_CHECK_LAUNCH();
    PYFOF_TRY(exclusive_scan_u32(flag, crank, na, reinterpret_cast<uint32_t *>(ctx.d_flags + FLAG_COUNT_A), W, s));
    fof_member_kernel<<<grid, BLK, 0, s>>>(st.lab, gsize, crank, st.pos, na,
                                           (uint32_t)a.np_halo_min, write_plain ? 1 : 0, pcand,
                                           a.in_halo, a.halo_id);
    PYFOF_CHECK_LAUNCH();
    PYFOF_CUDA(cudaMemcpyAsync(ctx.h_flags, ctx.d_flags, sizeof(int32_t) * FLAG_COUNT,
                               cudaMemcpyDeviceToHost, s));
    PYFOF_CUDA(cudaStreamSynchronize(s));
    if (ctx.h_flags[FLAG_ERR]) {
      set_error("linking failed (DSU retry cap)");
      return ctx.h_flags[FLAG_ERR];
    }
    st.ncand = (uint32_t)ctx.h_flags[FLAG_COUNT_A];
  }
  ctx.last_candidates = st.ncand;
  st.gsize = gsize;
  st.flag = flag;
  st.crank = crank;
  st.pcand = pcand;
  const int64_t nc = std::max<int64_t>(st.ncand, 1);
  st.cand_anchor = W.carve<int64_t>(nc);
  st.cand_region = W.carve<int32_t>(nc);
  st.cand_np = W.carve<int32_t>(nc);
  st.cand_root = W.carve<int32_t>(nc);
  if (!st.cand_anchor || !st.cand_region || !st.cand_np || !st.cand_root) {
    set_error("workspace exhausted (candidates)");
    return kAlloc;
  }
  if (st.ncand > 0) {
    const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(na, BLK), (int64_t)kNumSMs * 16);
    fof_cand_info_kernel<<<grid, BLK, 0, s>>>(flag, crank, st.pos, st.prid, gsize, na,
                                              st.cand_anchor, st.cand_region, st.cand_np,
                                              st.cand_root);
    PYFOF_CHECK_LAUNCH();
  }
  return kOk;
}

// ang_mom per input region over all candidates (no unbinding):
// fof_fortran.f90:224-248.
int32_t fof_plain_angmom(Context &ctx, const FofArgs &a, FofState &st) {
  cudaStream_t s = ctx.stream;
  Arena &W = ctx.work;
  const int nreg = a.nhalo;
  std::vector<double> am_host(3 * (size_t)nreg, 0.0);
  if (st.ncand > 0 && a.vp) {
    const int64_t na = st.n_active, nc = st.ncand;
    double *acc = W.carve<double>(7 * (size_t)nc);
    double *am = W.carve<double>(3 * (size_t)nc);
    if (!acc || !am) { set_error("workspace exhausted (ang_mom)"); return kAlloc; }
    PYFOF_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * 7 * nc, s));
    PYFOF_CUDA(cudaMemsetAsync(am, 0, sizeof(double) * 3 * nc, s));
    Coords xp{a.xp, a.total_np, a.soa}, vp{a.vp, a.total_np, a.soa};
    const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(na, BLK), (int64_t)kNumSMs * 16);
    fof_com_kernel<<<grid, BLK, 0, s>>>(xp, vp, a.mp, st.pos, st.pcand, st.cand_anchor, na,
                                        a.L_Box, 0.5 * a.L_Box, acc);
    PYFOF_CHECK_LAUNCH();
    fof_angmom_kernel<<<grid, BLK, 0, s>>>(xp, vp, a.mp, st.pos, st.pcand, st.cand_anchor, acc,
                                           na, a.L_Box, 0.5 * a.L_Box, am);
    PYFOF_CHECK_LAUNCH();
    std::vector<double> amc(3 * (size_t)nc);
    std::vector<int32_t> creg(nc);
    PYFOF_CUDA(cudaMemcpyAsync(amc.data(), am, sizeof(double) * 3 * nc, cudaMemcpyDeviceToHost, s));
    PYFOF_CUDA(cudaMemcpyAsync(creg.data(), st.cand_region, sizeof(int32_t) * nc,
                               cudaMemcpyDeviceToHost, s));
    PYFOF_CUDA(cudaStreamSynchronize(s));
    for (int64_t c = 0; c < nc; ++c)
      for (int d = 0; d < 3; ++d) am_host[3 * (size_t)creg[c] + d] += amc[3 * c + d];
  }
  memcpy(a.ang_mom, am_host.data(), sizeof(double) * am_host.size());
  return kOk;
}

// Every mass positive and finite (py_fof/__init__.py:259-260); with
// m_div != 1 each checked mass is then converted to code units, mp / m_grid
// (py_fof/__init__.py:318-319), in the same pass.
__global__ void check_mass_kernel(double *__restrict__ mp, int64_t n, int32_t *__restrict__ bad, double m_div) {
  int found = 0;
  const bool conv = m_div != 1.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double m = mp[i];
    found |= !(m > 0.0 && m <= 1.7976931348623157e308);
    if (conv) mp[i] = m / m_div;
  }
  if (__syncthreads_or(found) && threadIdx.x == 0) atomicExch(bad, 1);
}

__global__ void divide_kernel(double *__restrict__ x, int64_t n, double d) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = x[i] / d;
}

__global__ void multiply_kernel(double *__restrict__ x, int64_t n, double f) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = x[i] * f;
}

__global__ void fill_kernel(double *__restrict__ x, int64_t n, double v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = v;
}

// mask[i] = halo_id[i] > 0 as 0/1 bytes, four particles per thread
__global__ void member_mask_kernel(const int32_t *__restrict__ id, int64_t n, uint8_t *__restrict__ mask) {
  const int64_t n4 = n / 4;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
    const int4 v = reinterpret_cast<const int4 *>(id)[i];
    const uint32_t w = (uint32_t)(v.x > 0) | ((uint32_t)(v.y > 0) << 8) | ((uint32_t)(v.z > 0) << 16) |
                       ((uint32_t)(v.w > 0) << 24);
    reinterpret_cast<uint32_t *>(mask)[i] = w;
  }
  if (blockIdx.x == 0 && threadIdx.x < (unsigned)(n - 4 * n4)) {
    const int64_t i = 4 * n4 + threadIdx.x;
    mask[i] = id[i] > 0 ? 1 : 0;
  }
}

static unsigned stream_grid(int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, BLK), (int64_t)kNumSMs * 8));
}

int32_t divide_inplace(double *x, int64_t n, double d, cudaStream_t s) {
  if (n <= 0) return kOk;
  divide_kernel<<<stream_grid(n), BLK, 0, s>>>(x, n, d);
  PYFOF_CHECK_LAUNCH();
  return kOk;
}

int32_t multiply_inplace(double *x, int64_t n, double f, cudaStream_t s) {
  if (n <= 0) return kOk;
  multiply_kernel<<<stream_grid(n), BLK, 0, s>>>(x, n, f);
  PYFOF_CHECK_LAUNCH();
  return kOk;
}

int32_t fill_value(double *x, int64_t n, double v, cudaStream_t s) {
  if (n <= 0) return kOk;
  fill_kernel<<<stream_grid(n), BLK, 0, s>>>(x, n, v);
  PYFOF_CHECK_LAUNCH();
  return kOk;
}

int32_t member_mask(const int32_t *halo_id, int64_t n, uint8_t *mask, cudaStream_t s) {
  if (n <= 0) return kOk;
  member_mask_kernel<<<stream_grid(ceil_div(n, 4)), BLK, 0, s>>>(halo_id, n, mask);
  PYFOF_CHECK_LAUNCH();
  return kOk;
}

int32_t check_masses(Context &ctx, const double *mp, int64_t n, double m_div) {
  cudaStream_t s = ctx.stream;
  int32_t *bad = ctx.d_flags + FLAG_COUNT_C;
  PYFOF_CUDA(cudaMemsetAsync(bad, 0, sizeof(int32_t), s));
  // the mass array is only written when m_div != 1, and then it is the
  // library's own copy of the caller's masses
  check_mass_kernel<<<stream_grid(n), BLK, 0, s>>>(const_cast<double *>(mp), n, bad, m_div);
  PYFOF_CHECK_LAUNCH();
  PYFOF_CUDA(cudaMemcpyAsync(ctx.h_flags + FLAG_COUNT_C, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  if (ctx.h_flags[FLAG_COUNT_C]) {
    set_error("all particle masses must be positive and finite");
    return kMass;
  }
  return kOk;
}

int32_t fof_run(Context &ctx, const FofArgs &a) {
  FofState st;
  ctx.stage_reset();
  ctx.conv_timer.reset();
  ctx.gap_timer.reset();
  ctx.last_pm_passes = 0;
  ctx.side_timed = false;
  ctx.last_pm_solves = 0;
  ctx.last_pm_fft_bytes = 0.0;
  if (ctx.timing) cudaEventRecord(ctx.ev[2], ctx.stream);
  PYFOF_TRY(fof_link_stage(ctx, a, st));
  PYFOF_TRY(fof_candidates_stage(ctx, a, st, !a.bound_check));
  if (a.masses_ready) PYFOF_CUDA(cudaStreamWaitEvent(ctx.stream, a.masses_ready, 0));
  if (a.mp) PYFOF_TRY(check_masses(ctx, a.mp, a.total_np, a.m_div));
  if (ctx.timing) cudaEventRecord(ctx.ev[3], ctx.stream);
  if (!a.bound_check) {
    if (a.inputs_ready) PYFOF_CUDA(cudaStreamWaitEvent(ctx.stream, a.inputs_ready, 0));
    PYFOF_TRY(fof_plain_angmom(ctx, a, st));
  } else {
    // the velocities may still be copying: unbind_stage orders their use
    PYFOF_TRY(unbind_stage(ctx, a, st));
  }
  if (ctx.timing) cudaEventRecord(ctx.ev[4], ctx.stream);
  return kOk;
}

}  // namespace pyfof
