// Gravitational unbinding of FoF candidates (bound_fortran.f90) on the
// device: the bound_check=True branch of fof_fortran (fof_fortran.f90:252-360).
//
//   1. members of every candidate, ascending global index (the stable-id
//      order of bound_check_grid, bound_fortran.f90:2504-2528), packed as FP32
//      positions relative to the candidate anchor, FP32 velocities and masses
//      (fof_fortran.f90:281-308)
//   2. per-candidate span and lower corner -> host classification
//      (bound_classify, :2901-3073): 15 Mpc guard, method/grid/level choice
//   3. solvers: direct summation (N <= 1000) in one launch with one block
//      per halo running the whole removal loop; particle-mesh halos in
//      unbind_pm.cu
//   4. outputs: kept members of converged halos with >= np_halo_min members,
//      renumbered in candidate order, and angular momentum per input region
//      (fof_fortran.f90:313-355)
#include <algorithm>
#include <mutex>
#include <cmath>
#include <cstring>
#include <vector>

#include "context.cuh"
#include "primitives.cuh"
#include "unbind.cuh"
#include "unbind_direct.cuh"
#include "unbind_internal.cuh"

namespace pyfof {

namespace {

constexpr int BLK = 256;
constexpr double kPi = 3.141592653589793238462643383279502884197;

__global__ void ub_mark_kernel(const int32_t *__restrict__ pcand, const float4 *__restrict__ pos,
                               int64_t n, uint32_t *__restrict__ cand_of) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = pcand[p];
    if (c >= 0) cand_of[__float_as_int(pos[p].w)] = (uint32_t)c;
  }
}

__global__ void ub_fill_kernel(uint32_t *a, int64_t n, uint32_t v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    a[i] = v;
}

// xv packing (fof_fortran.f90:297-305): positions unwrapped about the
// candidate's first CRS member in FP64, then rounded to FP32.
__global__ void ub_pack_kernel(Coords xp, const double *__restrict__ mp,
                               const uint32_t *__restrict__ mcand,
                               const uint32_t *__restrict__ midx,
                               const int64_t *__restrict__ cand_anchor, int64_t M, double L,
                               double half, Members m) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < M;
       k += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t c = mcand[k];
    const int64_t i = midx[k];
    const int64_t a = cand_anchor[c];
#pragma unroll
    for (int d = 0; d < 3; ++d) m.q[d][k] = __double2float_rn(unwrap(xp.get(i, d), xp.get(a, d), half, L));
    m.w[k] = mp ? __double2float_rn(mp[i]) : 1.0f;
    m.pid[k] = (int32_t)i;
  }
}

// The members' velocities, packed apart from the rest: in a host-memory
// call they are the last input to arrive.
__global__ void ub_pack_v_kernel(Coords vp, const uint32_t *__restrict__ midx, int64_t M, Members m) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < M;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = midx[k];
#pragma unroll
    for (int d = 0; d < 3; ++d) m.v[d][k] = __double2float_rn(vp.get(i, d));
  }
}

// Span and lower corner of every candidate (bound_classify :2955-2965): the
// anchor member sits at q = 0; lo and hi start at 0.  The FP32 extremes of
// min/max are order-free, so many blocks per candidate (one per chunk of
// kSpanChunk members, the (candidate, chunk) pairs of `work`) fold theirs
// in with integer atomics on the ordered images of the floats; a
// non-finite coordinate marks the candidate.
constexpr int64_t kSpanChunk = 16384;

__device__ __forceinline__ uint32_t span_ord(float v) {
  const uint32_t b = __float_as_uint(v);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float span_flt(uint32_t o) {
  return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

// olo/ohi (3 per candidate) start at the ordered image of 0.0f, bad at 0
__global__ void span_init_kernel(uint32_t *__restrict__ olo, uint32_t *__restrict__ ohi, int32_t *__restrict__ bad,
                                 int ncand) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * ncand; i += gridDim.x * blockDim.x) {
    olo[i] = ohi[i] = 0x80000000u;
    if (i < ncand) bad[i] = 0;
  }
}

__global__ void __launch_bounds__(BLK) ub_span_kernel(Members m, const int64_t *__restrict__ off,
                                                      const int2 *__restrict__ work, uint32_t *__restrict__ olo,
                                                      uint32_t *__restrict__ ohi, int32_t *__restrict__ badc) {
  const int c = work[blockIdx.x].x;
  const int64_t b = off[c] + (int64_t)work[blockIdx.x].y * kSpanChunk;
  const int64_t e = min(off[c + 1], b + kSpanChunk);
  uint32_t lo[3] = {0x80000000u, 0x80000000u, 0x80000000u}, hi[3] = {0x80000000u, 0x80000000u, 0x80000000u};
  bool bad = false;
  for (int64_t k = b + threadIdx.x; k < e; k += BLK)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float v = m.q[d][k];
      if (!isfinite(v)) {
        bad = true;
        continue;
      }
      const uint32_t o = span_ord(v);
      lo[d] = min(lo[d], o);
      hi[d] = max(hi[d], o);
    }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    lo[d] = __reduce_min_sync(0xffffffffu, lo[d]);
    hi[d] = __reduce_max_sync(0xffffffffu, hi[d]);
  }
  bad = __any_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      atomicMin(&olo[3 * c + d], lo[d]);
      atomicMax(&ohi[3 * c + d], hi[d]);
    }
    if (bad) atomicOr(&badc[c], 1);
  }
}

__global__ void ub_span_final_kernel(const uint32_t *__restrict__ olo, const uint32_t *__restrict__ ohi,
                                     const int32_t *__restrict__ bad, int ncand, float *__restrict__ lo_out,
                                     float *__restrict__ span_out) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncand; c += gridDim.x * blockDim.x) {
    float span = 0.f;
    for (int d = 0; d < 3; ++d) {
      const float a = span_flt(olo[3 * c + d]), z = span_flt(ohi[3 * c + d]);
      lo_out[3 * c + d] = a;
      const float sd = z - a;
      span = d == 0 ? sd : fmaxf(span, sd);
    }
    span_out[c] = bad[c] ? NAN : span;
  }
}

// Launches the span kernels for candidates with member counts np (host).
static int32_t candidate_spans(Context &ctx, const Members &m, const int64_t *off, const int32_t *np, int ncand,
                               float *lo, float *span, cudaStream_t s) {
  Arena &W = ctx.work;
  std::vector<int2> work;
  for (int c = 0; c < ncand; ++c)
    for (int64_t k = 0; k * kSpanChunk < std::max<int64_t>(np[c], 1); ++k) work.push_back(make_int2(c, (int)k));
  uint32_t *olo = W.carve<uint32_t>(3 * (size_t)ncand), *ohi = W.carve<uint32_t>(3 * (size_t)ncand);
  int32_t *bad = W.carve<int32_t>(ncand);
  int2 *dwork = W.carve<int2>(std::max<size_t>(work.size(), 1));
  if (!olo || !ohi || !bad || !dwork) { set_error("workspace exhausted (spans)"); return kAlloc; }
  PYFOF_TRY(upload(ctx, dwork, work.data(), sizeof(int2) * work.size(), s));
  const unsigned g = (unsigned)std::min<int64_t>(ceil_div(3 * (int64_t)ncand, BLK), (int64_t)kNumSMs * 8);
  span_init_kernel<<<g, BLK, 0, s>>>(olo, ohi, bad, ncand);
  PYFOF_CHECK_LAUNCH();
  if (!work.empty()) {
    ub_span_kernel<<<(unsigned)work.size(), BLK, 0, s>>>(m, off, dwork, olo, ohi, bad);
    PYFOF_CHECK_LAUNCH();
  }
  ub_span_final_kernel<<<g, BLK, 0, s>>>(olo, ohi, bad, ncand, lo, span);
  PYFOF_CHECK_LAUNCH();
  return kOk;
}

// ---------------------------------------------------------------- direct

// Valid halos (status 0 and np_bound >= np_halo_min) in candidate order.
__global__ void ub_valid_kernel(const HaloResult *__restrict__ res, int ncand, int nmin,
                                uint32_t *__restrict__ valid) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncand; c += gridDim.x * blockDim.x)
    valid[c] = (res[c].status == 0 && res[c].np_bound >= nmin) ? 1u : 0u;
}

__global__ void ub_write_kernel(const uint32_t *__restrict__ mcand, const Members m,
                                const uint8_t *__restrict__ keep, const uint32_t *__restrict__ valid,
                                const uint32_t *__restrict__ vrank, int64_t M,
                                int32_t *__restrict__ in_halo, int32_t *__restrict__ halo_id) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < M;
       k += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t c = mcand[k];
    if (valid[c] && keep[k]) {
      const int32_t i = m.pid[k];
      in_halo[i] = 1;
      halo_id[i] = (int32_t)vrank[c] + 1;
    }
  }
}

// Sums of K values over each run of equal keys among the lanes of a warp
// (a segmented suffix scan over runs of consecutive lanes).  Returns true on
// the first lane of a run, which then holds the run's sums.  All 32 lanes
// must call it.
template <int K>
__device__ __forceinline__ bool warp_run_sums(uint32_t key, double (&v)[K]) {
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const uint32_t prev = __shfl_up_sync(FULL, key, 1);
  const bool head = lane == 0 || prev != key;
  const unsigned heads = __ballot_sync(FULL, head);
  const int run = 31 - __clz(heads & (FULL >> (31 - lane)));  // the run's first lane
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int orun = __shfl_down_sync(FULL, run, o);
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const double t = __shfl_down_sync(FULL, v[j], o);
      if (lane + o < 32 && orun == run) v[j] += t;
    }
  }
  return head;
}

// Angular momentum of the kept members of valid halos about their centre
// (fof_fortran.f90:321-350), accumulated per candidate in two passes.  A
// candidate's members are consecutive, so each warp first sums its lanes per
// candidate and adds those sums with one atomic per candidate and value
// (summation order differs from the reference's serial loop; the tests
// allow for that).
__global__ void ub_com_kernel(Coords xp, Coords vp, const double *mp,
                              const uint32_t *__restrict__ mcand, const Members m,
                              const uint8_t *__restrict__ keep, const uint32_t *__restrict__ valid,
                              const int64_t *__restrict__ cand_anchor, int64_t M, double L,
                              double half, double *acc) {
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < M; base += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = base + threadIdx.x;
    uint32_t c = 0xffffffffu;
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // weight, 3 weighted positions, 3 weighted velocities, count
    if (k < M) {
      c = mcand[k];
      if (valid[c] && keep[k]) {
        const int64_t i = m.pid[k], a = cand_anchor[c];
        const double wi = mp ? mp[i] : 1.0;
        v[0] = wi;
        for (int d = 0; d < 3; ++d) {
          v[1 + d] = wi * unwrap(xp.get(i, d), xp.get(a, d), half, L);
          v[4 + d] = wi * vp.get(i, d);
        }
        v[7] = 1.0;
      }
    }
    if (warp_run_sums<8>(c, v) && v[7] > 0.0)
      for (int j = 0; j < 7; ++j) atomicAdd(&acc[7 * (int64_t)c + j], v[j]);
  }
}

__global__ void ub_angmom_kernel(Coords xp, Coords vp, const double *mp,
                                 const uint32_t *__restrict__ mcand, const Members m,
                                 const uint8_t *__restrict__ keep,
                                 const uint32_t *__restrict__ valid,
                                 const int64_t *__restrict__ cand_anchor, const double *acc,
                                 int64_t M, double L, double half, double *am) {
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < M; base += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = base + threadIdx.x;
    uint32_t c = 0xffffffffu;
    double v[4] = {0, 0, 0, 0};  // angular momentum, count
    if (k < M) {
      c = mcand[k];
      const double ws = valid[c] && keep[k] ? acc[7 * (int64_t)c] : 0.0;
      if (ws > 0.0) {
        const int64_t i = m.pid[k], a = cand_anchor[c];
        const double wi = mp ? mp[i] : 1.0;
        double dx[3], dv[3];
        for (int d = 0; d < 3; ++d) {
          dx[d] = unwrap(xp.get(i, d), xp.get(a, d), half, L) - acc[7 * (int64_t)c + 1 + d] / ws;
          dv[d] = vp.get(i, d) - acc[7 * (int64_t)c + 4 + d] / ws;
        }
        v[0] = wi * (dx[1] * dv[2] - dx[2] * dv[1]);
        v[1] = wi * (dx[2] * dv[0] - dx[0] * dv[2]);
        v[2] = wi * (dx[0] * dv[1] - dx[1] * dv[0]);
        v[3] = 1.0;
      }
    }
    if (warp_run_sums<4>(c, v) && v[3] > 0.0)
      for (int j = 0; j < 3; ++j) atomicAdd(&am[3 * (int64_t)c + j], v[j]);
  }
}

int bits_for(uint64_t v) {
  int b = 0;
  while (b < 64 && (v >> b) != 0) ++b;
  return b;
}

}  // namespace

// ------------------------------------------------------------ grid rules

// bound_set_context / bound_grid_levels / bound_fgl_init / ladder
// (bound_fortran.f90:291-330, :1854-1955): the grid classes 48/64/128/256
// (capped at ng), their spacing levels 1/32, 1/16, ... while the coverage
// (n/2-3)*spacing stays below s_15, plus spacing_max = s_15/m_max on the
// largest enabled class.
void GridRules::init(int64_t ng_in, double s15_in) {
  static const int cand[4] = {48, 64, 128, 256};
  ng = ng_in > 0 ? ng_in : 256;
  const int ngi = (int)ng;
  ngrid = 1 + (ngi >= 64) + (ngi >= 128) + (ngi >= 256);
  for (int g = 0; g < 4; ++g) bn[g] = std::min(cand[g], ngi);
  const int n_max = std::min(256, ngi);
  const int m_max = n_max / 2 - 3;
  s15 = s15_in;
  spacing_max = s15 / (double)m_max;
  for (int g = 1; g <= 4; ++g) {
    std::vector<double> &sp = levels[g - 1];
    sp.clear();
    if (g > ngrid) continue;
    const int m = bn[g - 1] / 2 - 3;
    double s = 1.0 / 32.0;
    while ((double)m * s < s15 && (int)sp.size() < 32) { sp.push_back(s); s *= 2.0; }
    if (g == ngrid && (int)sp.size() < 32) sp.push_back(spacing_max);
  }
  // global ladder by coverage, selection sort as in bound_build_ladder
  struct E { int g, l; double sp, cov; };
  std::vector<E> t;
  for (int g = 1; g <= ngrid; ++g)
    for (int l = 0; l < (int)levels[g - 1].size(); ++l)
      t.push_back(E{g, l, levels[g - 1][l], (double)(bn[g - 1] / 2 - 3) * levels[g - 1][l]});
  for (size_t j = 0; j + 1 < t.size(); ++j) {
    size_t k = j;
    for (size_t i = j + 1; i < t.size(); ++i) if (t[i].cov < t[k].cov) k = i;
    if (k != j) std::swap(t[j], t[k]);
  }
  ladder_g.clear(); ladder_l.clear(); ladder_cov.clear();
  for (auto &e : t) { ladder_g.push_back(e.g); ladder_l.push_back(e.l); ladder_cov.push_back(e.cov); }
}

double GridRules::coverage(int g, int l) const {
  return (double)(bn[g - 1] / 2 - 3) * levels[g - 1][l];
}

// bound_select_grid_and_level (:1963-2019).  Returns false when no enabled
// grid class can cover the span.
bool GridRules::select(int64_t np, double span, int &gid, int &lev, double &sp) const {
  gid = 0; lev = -1; sp = 0.0;
  if (np <= 1000) return true;
  // candidate sequences per size band; spacing < 0 stands for spacing_max
  static const int nb[3] = {11, 10, 8};
  static const int cg[3][11] = {{1, 2, 2, 3, 3, 3, 4, 4, 4, 4, 4},
                                {3, 3, 4, 4, 4, 4, 4, 4, 4, 4, 0},
                                {4, 4, 4, 4, 4, 4, 4, 4, 0, 0, 0}};
  static const double cs[3][11] = {
      {0.125, 0.125, 0.25, 0.125, 0.25, 0.5, 0.0625, 0.125, 0.25, 0.5, -1.0},
      {0.0625, 0.125, 0.0625, 0.125, 0.25, 0.5, 1.0, 2.0, 4.0, -1.0, 0.0},
      {0.0625, 0.125, 0.25, 0.5, 1.0, 2.0, 4.0, -1.0, 0.0, 0.0, 0.0}};
  const int band = np <= 5000 ? 0 : (np <= 20000 ? 1 : 2);
  for (int s = 0; s < nb[band]; ++s) {
    const int g = cg[band][s];
    if (g < 1 || g > ngrid) continue;
    double want = cs[band][s];
    if (want == -1.0) want = spacing_max;
    int l = -1;
    for (int q = 0; q < (int)levels[g - 1].size(); ++q)
      if (std::fabs(levels[g - 1][q] - want) <= 1e-12 * std::max(1.0, std::fabs(want))) { l = q; break; }
    if (l < 0) continue;
    if (coverage(g, l) < span) continue;
    gid = g; lev = l; sp = levels[g - 1][l];
    return true;
  }
  if (span <= s15) {
    for (size_t i = 0; i < ladder_cov.size(); ++i)
      if (ladder_cov[i] >= span) {
        const int g = ladder_g[i], l = ladder_l[i];
        if (g >= 1 && g <= ngrid) { gid = g; lev = l; sp = levels[g - 1][l]; return true; }
        break;
      }
  }
  return false;
}

// ------------------------------------------------------------ stage

// Orders the context's side stream after the work issued so far on `s`
// (creating the stream and its events on first use).
static int32_t fork_side(Context &ctx, cudaStream_t s) {
  if (!ctx.side_stream) {
    PYFOF_CUDA(cudaStreamCreateWithFlags(&ctx.side_stream, cudaStreamNonBlocking));
    PYFOF_CUDA(cudaEventCreateWithFlags(&ctx.ev_fork, cudaEventDisableTiming));
    PYFOF_CUDA(cudaEventCreateWithFlags(&ctx.ev_join, cudaEventDisableTiming));
  }
  PYFOF_CUDA(cudaEventRecord(ctx.ev_fork, s));
  PYFOF_CUDA(cudaStreamWaitEvent(ctx.side_stream, ctx.ev_fork, 0));
  return kOk;
}

// The direct-summation removal loop over `nb` halos of at most `cap`
// members, with `threads` threads per block.
template <bool FP64, int NT>
static int32_t launch_direct_nt(unsigned nb, int cap, const Members &m, const int64_t *off, const int32_t *list,
                                const direct::DirectParams &P, HaloResult *res, uint8_t *keep, float *phi_out,
                                int32_t *flags, const double *phi1, cudaStream_t s) {
  // the shared-memory limit is a property of the kernel, shared by every
  // thread that launches it: set it once, to the largest size any launch
  // asks for, so concurrent calls (serving slots) never lower it
  static std::once_flag once;
  static cudaError_t attr = cudaSuccess;
  std::call_once(once, [] {
    attr = cudaFuncSetAttribute(direct::ub_direct_kernel<FP64, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)direct::direct_smem(kDirectMax));
  });
  PYFOF_CUDA(attr);
  const size_t smem = direct::direct_smem(cap);
  direct::ub_direct_kernel<FP64, NT><<<nb, NT, smem, s>>>(m, off, list, P, res, keep, phi_out, flags, phi1, cap);
  PYFOF_CHECK_LAUNCH();
  return kOk;
}

static int32_t launch_direct_loop(bool fp64, int threads, unsigned nb, int cap, const Members &m,
                                  const int64_t *off, const int32_t *list, const direct::DirectParams &P,
                                  HaloResult *res, uint8_t *keep, float *phi_out, int32_t *flags,
                                  const double *phi1, cudaStream_t s) {
#define PYFOF_DIRECT_NT(NT)                                                                           \
  return fp64 ? launch_direct_nt<true, NT>(nb, cap, m, off, list, P, res, keep, phi_out, flags, phi1, s) \
              : launch_direct_nt<false, NT>(nb, cap, m, off, list, P, res, keep, phi_out, flags, phi1, s)
  switch (threads) {
    case 32: PYFOF_DIRECT_NT(32);
    case 64: PYFOF_DIRECT_NT(64);
    case 128: PYFOF_DIRECT_NT(128);
    default: PYFOF_DIRECT_NT(256);
  }
#undef PYFOF_DIRECT_NT
}

int32_t unbind_stage(Context &ctx, const FofArgs &a, FofState &st) {
  cudaStream_t s = ctx.stream;
  Arena &W = ctx.work;
  const int nreg = a.nhalo;
  std::vector<double> am_host(3 * (size_t)nreg, 0.0);
  const int ncand = (int)st.ncand;
  if (ncand == 0) {
    std::memcpy(a.ang_mom, am_host.data(), sizeof(double) * am_host.size());
    return kOk;
  }
  GridRules rules;
  rules.init(a.ng, a.s15);
  if (rules.ngrid != 4) {
    set_error("bound_check_batch: fixed groups require ng >= 256");
    return kInvalid;
  }
  if (!std::isfinite(a.a_val) || a.a_val <= 0.0 || !std::isfinite(a.b_val)) {
    set_error("bound_check_batch: invalid physical context");
    return kInvalid;
  }
  const int64_t n = a.total_np;
  const double L = a.L_Box, half = 0.5 * a.L_Box;
  Coords xp{a.xp, n, a.soa}, vp{a.vp, n, a.soa};

  // 1. members grouped by candidate, ascending global index
  uint32_t *cand_of = W.carve<uint32_t>(n);
  uint32_t *ka = W.carve<uint32_t>(n), *va = W.carve<uint32_t>(n);
  uint32_t *kb = W.carve<uint32_t>(n), *vb = W.carve<uint32_t>(n);
  int64_t *off = W.carve<int64_t>(ncand + 1);
  if (!cand_of || !ka || !va || !kb || !vb || !off) { set_error("workspace exhausted (members)"); return kAlloc; }
  const unsigned grid_n = (unsigned)std::min<int64_t>(ceil_div(n, BLK), (int64_t)kNumSMs * 16);
  ub_fill_kernel<<<grid_n, BLK, 0, s>>>(cand_of, n, (uint32_t)ncand);
  PYFOF_CHECK_LAUNCH();
  ub_mark_kernel<<<grid_n, BLK, 0, s>>>(st.pcand, st.pos, st.n_active, cand_of);
  PYFOF_CHECK_LAUNCH();
  uint32_t *mcand, *midx;
  PYFOF_TRY(radix_sort_pairs(cand_of, nullptr, n, bits_for((uint64_t)ncand), ka, va, kb, vb, &mcand,
                             &midx, W, s));
  std::vector<int32_t> cnp(ncand);
  PYFOF_CUDA(cudaMemcpyAsync(cnp.data(), st.cand_np, sizeof(int32_t) * ncand, cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  std::vector<int64_t> hoff(ncand + 1, 0);
  for (int c = 0; c < ncand; ++c) hoff[c + 1] = hoff[c] + cnp[c];
  const int64_t M = hoff[ncand];
  PYFOF_TRY(upload(ctx, off, hoff.data(), sizeof(int64_t) * (ncand + 1), s));
  Members m;
  for (int d = 0; d < 3; ++d) {
    m.q[d] = W.carve<float>(M);
    m.v[d] = W.carve<float>(M);
    if (!m.q[d] || !m.v[d]) { set_error("workspace exhausted (xv)"); return kAlloc; }
  }
  m.w = W.carve<float>(M);
  m.pid = W.carve<int32_t>(M);
  float *lo = W.carve<float>(3 * (size_t)ncand), *span = W.carve<float>(ncand);
  HaloResult *res = W.carve<HaloResult>(ncand);
  uint8_t *keep = W.carve<uint8_t>(M);
  if (!m.w || !m.pid || !lo || !span || !res || !keep) { set_error("workspace exhausted (xv)"); return kAlloc; }
  const unsigned grid_m = (unsigned)std::min<int64_t>(ceil_div(M, BLK), (int64_t)kNumSMs * 16);
  ub_pack_kernel<<<grid_m, BLK, 0, s>>>(xp, a.mp, mcand, midx, st.cand_anchor, M, L, half, m);
  PYFOF_CHECK_LAUNCH();
  // The velocities of a host-memory call may still be copying: their pack
  // runs on the input stream after the copy, and the kernels that read
  // them wait for it (wait_velocities); every return orders `s` after it
  // (the caller frees this call's memory on `s`).
  struct VelocityJoin {
    Context &c;
    cudaStream_t s;
    ~VelocityJoin() {
      if (c.vel_wait) cudaStreamWaitEvent(s, c.vel_wait, 0);
      c.vel_wait = nullptr;
    }
  } velocity_join{ctx, s};
  if (a.inputs_ready && a.input_stream) {
    PYFOF_CUDA(cudaEventRecord(ctx.ev_pack, s));
    PYFOF_CUDA(cudaStreamWaitEvent(a.input_stream, ctx.ev_pack, 0));
    PYFOF_CUDA(cudaStreamWaitEvent(a.input_stream, a.inputs_ready, 0));
    ub_pack_v_kernel<<<grid_m, BLK, 0, a.input_stream>>>(vp, midx, M, m);
    PYFOF_CHECK_LAUNCH();
    PYFOF_CUDA(cudaEventRecord(ctx.ev_vel, a.input_stream));
    ctx.vel_wait = ctx.ev_vel;
  } else {
    ub_pack_v_kernel<<<grid_m, BLK, 0, s>>>(vp, midx, M, m);
    PYFOF_CHECK_LAUNCH();
  }
  PYFOF_TRY(candidate_spans(ctx, m, off, cnp.data(), ncand, lo, span, s));

  // 2. classification, in candidate order (first error wins)
  std::vector<float> hlo(3 * (size_t)ncand), hspan(ncand);
  PYFOF_CUDA(cudaMemcpyAsync(hlo.data(), lo, sizeof(float) * 3 * ncand, cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaMemcpyAsync(hspan.data(), span, sizeof(float) * ncand, cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  std::vector<HaloTask> tasks(ncand);
  std::vector<int32_t> direct, pm;
  for (int c = 0; c < ncand; ++c) {
    HaloTask &t = tasks[c];
    t.off = hoff[c];
    t.np = cnp[c];
    const float sp_c = hspan[c];
    if (!std::isfinite(sp_c)) { set_error("bound_classify: non-finite span"); return kInvalid; }
    if (t.np > 1000 && sp_c > (float)a.s15) {
      set_error("candidate %d: span %g exceeds D_max = 15 Mpc (s_15 = %g)", c, (double)sp_c, a.s15);
      return kSpan;
    }
    int g, l;
    double sp;
    if (!rules.select(t.np, (double)sp_c, g, l, sp)) {
      set_error("candidate %d: no enabled grid class can cover span %g", c, (double)sp_c);
      return kInvalid;
    }
    t.gid = g;
    t.n = g > 0 ? rules.bn[g - 1] : 0;
    if (g > 0) {
      const float spf = (float)sp;
      t.spacing = spf;
      for (int d = 0; d < 3; ++d) t.origin[d] = hlo[3 * c + d] - spf;
      if ((double)(rules.bn[g - 1] / 2 - 3) * (double)spf < (double)sp_c) {
        set_error("candidate %d: single precision spacing does not cover span", c);
        return kInvalid;
      }
      pm.push_back(c);
    } else {
      direct.push_back(c);
    }
  }
  ctx.last_direct = (int64_t)direct.size();
  ctx.last_pm = (int64_t)pm.size();

  // 3. solvers
  PYFOF_CUDA(cudaMemsetAsync(ctx.d_flags, 0, sizeof(int32_t), s));
  // Once the direct path is forked onto the side stream, every return
  // orders `s` after it (the caller frees this call's memory on `s`).
  bool side_forked = false;
  struct SideJoin {
    Context &c;
    cudaStream_t s;
    bool &on;
    ~SideJoin() {
      if (on) cudaStreamWaitEvent(s, c.ev_join, 0);
    }
  } side_join{ctx, s, side_forked};
  if (!direct.empty()) {
    int32_t *dl = W.carve<int32_t>(direct.size());
    if (!dl) { set_error("workspace exhausted (direct list)"); return kAlloc; }
    PYFOF_TRY(upload(ctx, dl, direct.data(), sizeof(int32_t) * direct.size(), s));
    direct::DirectParams P;
    P.fac = a.a_val / (6.0 * kPi);
    P.app = a.softening;
    P.b = (float)a.b_val;
    P.nmin = a.np_halo_min;
    P.phi_only = 0;
    const size_t smem = kDirectSmem;
    if (a.bound_per_halo) {
      // plain baseline: one halo per launch, waited for before the next
      PYFOF_CUDA(cudaFuncSetAttribute(direct::ub_direct_kernel<true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      PYFOF_CUDA(wait_velocities(ctx, s));
      for (size_t i = 0; i < direct.size(); ++i) {
        direct::ub_direct_kernel<true><<<1, BLK, smem, s>>>(m, off, dl + i, P, res, keep, st.phi_out,
                                                            ctx.d_flags);
        PYFOF_CHECK_LAUNCH();
        PYFOF_CUDA(cudaStreamSynchronize(s));
      }
    } else {
      // first-pass potentials flat over (halo, 64-target tile), then the
      // removal loops, one block per halo, launched per halo-size bucket
      // with the tile table's block size and shared memory for the bucket's
      // largest halo
      std::vector<int2> tl;
      for (size_t e = 0; e < direct.size(); ++e)
        for (int t0 = 0; t0 < tasks[direct[e]].np; t0 += direct::PT) tl.push_back(make_int2((int)e, t0));
      int2 *dtl = W.carve<int2>(tl.size());
      double *phi1 = W.carve<double>((size_t)std::max<int64_t>(M, 1));
      int32_t *dbl = W.carve<int32_t>(direct.size());
      if (!dtl || !phi1 || !dbl) { set_error("workspace exhausted (direct potentials)"); return kAlloc; }
      PYFOF_TRY(upload(ctx, dtl, tl.data(), sizeof(int2) * tl.size(), s));
      if (a.bound_fp64)
        direct::ub_direct_phi1_kernel<true><<<(unsigned)tl.size(), direct::PT, 0, s>>>(m, off, dl, dtl, P, phi1);
      else
        direct::ub_direct_phi1_kernel<false><<<(unsigned)tl.size(), direct::PT, 0, s>>>(m, off, dl, dtl, P, phi1);
      PYFOF_CHECK_LAUNCH();
      // per bucket, largest halos first (they run longest)
      std::vector<int32_t> bl;
      std::vector<size_t> bstart(7, 0);
      for (int b = 0; b < 6; ++b) {
        const size_t b0 = bl.size();
        for (int32_t c : direct) {
          const int np = tasks[c].np;
          if (np <= kDirectBucketEdge[b] && (b == 0 || np > kDirectBucketEdge[b - 1])) bl.push_back(c);
        }
        std::stable_sort(bl.begin() + b0, bl.end(),
                         [&](int32_t x, int32_t y) { return tasks[x].np > tasks[y].np; });
        bstart[b + 1] = bl.size();
      }
      PYFOF_TRY(upload(ctx, dbl, bl.data(), sizeof(int32_t) * bl.size(), s));
      // the removal loops run on the side stream, overlapping the
      // particle-mesh halos on `s` (disjoint halos, disjoint outputs)
      PYFOF_TRY(fork_side(ctx, s));
      side_forked = true;
      if (ctx.timing) {
        cudaEventRecord(ctx.ev[9], ctx.side_stream);
        ctx.side_timed = true;
      }
      PYFOF_CUDA(wait_velocities(ctx, ctx.side_stream));
      for (int b = 5; b >= 0; --b) {
        const unsigned nb = (unsigned)(bstart[b + 1] - bstart[b]);
        if (!nb) continue;
        const int cap = (kDirectBucketEdge[b] + 31) / 32 * 32;
        PYFOF_TRY(launch_direct_loop(a.bound_fp64 != 0, a.tiles.direct_threads[b], nb, cap, m, off,
                                     dbl + bstart[b], P, res, keep, st.phi_out, ctx.d_flags, phi1,
                                     ctx.side_stream));
      }
      if (ctx.timing) cudaEventRecord(ctx.ev[10], ctx.side_stream);
      PYFOF_CUDA(cudaEventRecord(ctx.ev_join, ctx.side_stream));
    }
    PYFOF_CHECK_LAUNCH();
  }
  if (!pm.empty()) {
    if (a.bound_per_halo) {
      // each halo on its own: its members as the whole member set, its
      // scratch sized by and freed with it
      for (int32_t c : pm) {
        const HaloTask &t = tasks[c];
        Members mh = m;
        for (int d = 0; d < 3; ++d) {
          mh.q[d] += t.off;
          mh.v[d] += t.off;
        }
        mh.w += t.off;
        mh.pid += t.off;
        std::vector<HaloTask> th(1, t);
        th[0].off = 0;
        const std::vector<int32_t> one(1, 0);
        const size_t mk = W.mark();
        PYFOF_TRY(unbind_pm(ctx, a, rules, mh, th, one, res + c, keep + t.off,
                            st.phi_out ? st.phi_out + t.off : nullptr, 0));
        W.release_to(mk);
      }
    } else {
      PYFOF_TRY(unbind_pm(ctx, a, rules, m, tasks, pm, res, keep, st.phi_out, 0));
    }
  }
  if (side_forked) {
    if (ctx.timing) cudaEventRecord(ctx.ev[11], s);
    PYFOF_CUDA(cudaStreamWaitEvent(s, ctx.ev_join, 0));
    side_forked = false;
  }
  // the outputs read the velocities too
  PYFOF_CUDA(wait_velocities(ctx, s));
  ctx.vel_wait = nullptr;
  PYFOF_CUDA(cudaMemcpyAsync(ctx.h_flags, ctx.d_flags, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  if (ctx.h_flags[FLAG_ERR]) {
    set_error("unbinding failed (error %d)", ctx.h_flags[FLAG_ERR]);
    return ctx.h_flags[FLAG_ERR];
  }

  // 4. outputs
  uint32_t *valid = W.carve<uint32_t>(ncand + 1), *vrank = W.carve<uint32_t>(ncand + 1);
  double *acc = W.carve<double>(7 * (size_t)ncand), *am = W.carve<double>(3 * (size_t)ncand);
  if (!valid || !vrank || !acc || !am) { set_error("workspace exhausted (outputs)"); return kAlloc; }
  const unsigned grid_c = (unsigned)std::min<int64_t>(ceil_div(ncand, BLK), (int64_t)kNumSMs * 8);
  ub_valid_kernel<<<grid_c, BLK, 0, s>>>(res, ncand, a.np_halo_min, valid);
  PYFOF_CHECK_LAUNCH();
  PYFOF_TRY(exclusive_scan_u32(valid, vrank, ncand, nullptr, W, s));
  ub_write_kernel<<<grid_m, BLK, 0, s>>>(mcand, m, keep, valid, vrank, M, a.in_halo, a.halo_id);
  PYFOF_CHECK_LAUNCH();
  PYFOF_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * 7 * ncand, s));
  PYFOF_CUDA(cudaMemsetAsync(am, 0, sizeof(double) * 3 * ncand, s));
  ub_com_kernel<<<grid_m, BLK, 0, s>>>(xp, vp, a.mp, mcand, m, keep, valid, st.cand_anchor, M, L,
                                       half, acc);
  PYFOF_CHECK_LAUNCH();
  ub_angmom_kernel<<<grid_m, BLK, 0, s>>>(xp, vp, a.mp, mcand, m, keep, valid, st.cand_anchor,
                                          acc, M, L, half, am);
  PYFOF_CHECK_LAUNCH();
  std::vector<double> amc(3 * (size_t)ncand);
  std::vector<int32_t> creg(ncand);
  std::vector<HaloResult> hres(ncand);
  PYFOF_CUDA(cudaMemcpyAsync(amc.data(), am, sizeof(double) * 3 * ncand, cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaMemcpyAsync(creg.data(), st.cand_region, sizeof(int32_t) * ncand,
                             cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaMemcpyAsync(hres.data(), res, sizeof(HaloResult) * ncand, cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  int64_t nvalid = 0, nmax = 0;
  for (int c = 0; c < ncand; ++c) {
    for (int d = 0; d < 3; ++d) am_host[3 * (size_t)creg[c] + d] += amc[3 * c + d];
    nvalid += hres[c].status == 0 && hres[c].np_bound >= a.np_halo_min;
    nmax += hres[c].status == 5;
  }
  ctx.last_valid = nvalid;
  if (a.verbose >= 1)
    fprintf(stderr, "[BOUND_STATUS] candidates=%d direct=%zu pm=%zu valid=%lld max_iter=%lld\n",
            ncand, direct.size(), pm.size(), (long long)nvalid, (long long)nmax);
  std::memcpy(a.ang_mom, am_host.data(), sizeof(double) * am_host.size());
  return kOk;
}

int32_t unbind_potential(Context &ctx, const float *q_soa, const float *w, int32_t np,
                         double softening, double a_val, double s15, int64_t ng, int fp64,
                         float *phi, int32_t *method) {
  cudaStream_t s = ctx.stream;
  Arena &W = ctx.work;
  ctx.stage_reset();
  GridRules rules;
  rules.init(ng, s15);
  if (rules.ngrid != 4 || np <= 0) {
    set_error("unbind_potential: invalid grid or member count");
    return kInvalid;
  }
  Members m;
  for (int d = 0; d < 3; ++d) {
    m.q[d] = W.carve<float>(np);
    m.v[d] = W.carve<float>(np);
    if (!m.q[d] || !m.v[d]) { set_error("workspace exhausted"); return kAlloc; }
    PYFOF_CUDA(cudaMemcpyAsync(m.q[d], q_soa + (size_t)d * np, sizeof(float) * np, cudaMemcpyHostToDevice, s));
    PYFOF_CUDA(cudaMemsetAsync(m.v[d], 0, sizeof(float) * np, s));
  }
  m.w = W.carve<float>(np);
  m.pid = W.carve<int32_t>(np);
  int64_t *off = W.carve<int64_t>(2);
  float *lo = W.carve<float>(3), *span = W.carve<float>(1), *phid = W.carve<float>(np);
  HaloResult *res = W.carve<HaloResult>(1);
  uint8_t *keep = W.carve<uint8_t>(np);
  int32_t *dl = W.carve<int32_t>(1);
  if (!m.w || !m.pid || !off || !lo || !span || !phid || !res || !keep || !dl) {
    set_error("workspace exhausted");
    return kAlloc;
  }
  PYFOF_CUDA(cudaMemcpyAsync(m.w, w, sizeof(float) * np, cudaMemcpyHostToDevice, s));
  const int64_t hoff[2] = {0, np};
  PYFOF_CUDA(cudaMemcpyAsync(off, hoff, sizeof(hoff), cudaMemcpyHostToDevice, s));
  PYFOF_TRY(candidate_spans(ctx, m, off, &np, 1, lo, span, s));
  float hlo[3], hspan;
  PYFOF_CUDA(cudaMemcpyAsync(hlo, lo, sizeof(hlo), cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaMemcpyAsync(&hspan, span, sizeof(float), cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  if (!std::isfinite(hspan)) { set_error("non-finite span"); return kInvalid; }
  if (np > 1000 && hspan > (float)s15) { set_error("span exceeds s_15"); return kSpan; }
  int g, l;
  double sp;
  if (!rules.select(np, (double)hspan, g, l, sp)) { set_error("no grid covers the span"); return kInvalid; }
  *method = g;
  std::vector<HaloTask> tasks(1);
  tasks[0].off = 0;
  tasks[0].np = np;
  tasks[0].gid = g;
  tasks[0].n = g > 0 ? rules.bn[g - 1] : 0;
  FofArgs a;
  a.softening = softening;
  a.a_val = a_val;
  a.b_val = 0.0;
  a.s15 = s15;
  a.ng = ng;
  a.np_halo_min = 1;
  a.bound_fp64 = fp64;
  PYFOF_CUDA(cudaMemsetAsync(ctx.d_flags, 0, sizeof(int32_t), s));
  if (g == 0) {
    const int32_t zero = 0;
    PYFOF_CUDA(cudaMemcpyAsync(dl, &zero, sizeof(int32_t), cudaMemcpyHostToDevice, s));
    direct::DirectParams P;
    P.fac = a_val / (6.0 * kPi);
    P.app = softening;
    P.b = 0.0f;
    P.nmin = 1;
    P.phi_only = 1;
    if (fp64) {
      PYFOF_CUDA(cudaFuncSetAttribute(direct::ub_direct_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kDirectSmem));
      direct::ub_direct_kernel<true><<<1, BLK, kDirectSmem, s>>>(m, off, dl, P, res, keep, phid, ctx.d_flags);
    } else {
      PYFOF_CUDA(cudaFuncSetAttribute(direct::ub_direct_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kDirectSmem));
      direct::ub_direct_kernel<false><<<1, BLK, kDirectSmem, s>>>(m, off, dl, P, res, keep, phid, ctx.d_flags);
    }
    PYFOF_CHECK_LAUNCH();
  } else {
    const float spf = (float)sp;
    tasks[0].spacing = spf;
    for (int d = 0; d < 3; ++d) tasks[0].origin[d] = hlo[d] - spf;
    std::vector<int32_t> list(1, 0);
    PYFOF_TRY(unbind_pm(ctx, a, rules, m, tasks, list, res, keep, phid, 1));
  }
  PYFOF_CUDA(cudaMemcpyAsync(phi, phid, sizeof(float) * np, cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaMemcpyAsync(ctx.h_flags, ctx.d_flags, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  if (ctx.h_flags[FLAG_ERR]) {
    set_error("potential failed (error %d)", ctx.h_flags[FLAG_ERR]);
    return ctx.h_flags[FLAG_ERR];
  }
  return kOk;
}

}  // namespace pyfof
