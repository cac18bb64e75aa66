// Direct-summation solver of the unbinding removal loop (bound_check_grid
// for gid 0, bound_fortran.f90:2611-2864), shared by the batched stage
// (unbind.cu) and the static-scratch entry point (direct_static.cu).
#pragma once

#include "unbind_internal.cuh"

namespace pyfof {
namespace direct {

constexpr int BLK = 256;

// bound_depth_continuous (bound_fortran.f90:3080-3102): spline-softened 1/r.
template <typename T>
__device__ __forceinline__ T depth_continuous(T r, T h);

template <>
__device__ __forceinline__ double depth_continuous<double>(double r, double h) {
  if (r <= 0.0) return __ddiv_rn(208.0, __dmul_rn(70.0, h));
  if (r >= h) return __ddiv_rn(1.0, r);
  const double e = __ddiv_rn(__dmul_rn(2.0, r), h);
  if (e <= 1.0) {
    double t = __dadd_rn(8.0, __dmul_rn(-3.0, e));
    t = __dadd_rn(14.0, __dmul_rn(e, t));
    t = __dadd_rn(-56.0, __dmul_rn(e, t));
    t = __dadd_rn(112.0, __dmul_rn(__dmul_rn(e, e), t));
    const double prim = __dmul_rn(__dmul_rn(e, e), t);
    return __ddiv_rn(__dadd_rn(208.0, -prim), __dmul_rn(70.0, h));
  }
  double t = __dadd_rn(-8.0, e);
  t = __dadd_rn(14.0, __dmul_rn(e, t));
  t = __dadd_rn(56.0, __dmul_rn(e, t));
  t = __dadd_rn(-280.0, __dmul_rn(e, t));
  t = __dadd_rn(448.0, __dmul_rn(e, t));
  double prim = __dmul_rn(__dmul_rn(e, e), t);
  prim = __dadd_rn(prim, -__dmul_rn(224.0, e));
  prim = __dadd_rn(prim, -__ddiv_rn(12.0, e));
  return __ddiv_rn(__dadd_rn(128.0, -prim), __dmul_rn(70.0, h));
}

// FP32 product-path kernel: same piecewise polynomial, with the
// reciprocals precomputed by the caller (inv70h = 1/(70h), inv_h = 1/h).
__device__ __forceinline__ float depth_f32(float r2, float h, float inv_h, float inv70h) {
  if (r2 >= h * h) return rsqrtf(r2);
  const float r = sqrtf(r2);
  const float e = 2.0f * r * inv_h;
  if (e <= 1.0f) {
    const float e2 = e * e;
    const float prim = e2 * (112.0f + e2 * (-56.0f + e * (14.0f + e * (8.0f - 3.0f * e))));
    return (208.0f - prim) * inv70h;
  }
  const float prim = e * e * (448.0f + e * (-280.0f + e * (56.0f + e * (14.0f + e * (-8.0f + e))))) -
                     224.0f * e - 12.0f / e;
  return (128.0f - prim) * inv70h;
}

// Compensated (Fast2Sum/Kahan) FP32 accumulator.
struct Kahan {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

__device__ __forceinline__ int block_sum_i(int v, int *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  int t = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  return t;
}

struct DirectParams {
  double fac;     // a / (6 pi)
  double app;     // softening (standard grid units)
  float b;        // real(b_bound, 4)
  int nmin;       // np_halo_min
  int phi_only;   // stop after the first potential
};

// Sources j0 .. j0+cnt-1 (staged at sx[0..cnt)) of a target's first-pass
// potential, in ascending index, skipping the target itself: the
// reference's accumulation order (bound_fortran.f90:2619-2640; its i<j loop
// adds each pair term to both ends, so every target sums its sources in
// ascending order) and the same operations as the in-kernel first pass of
// ub_direct_kernel.
template <bool FP64>
__device__ __forceinline__ void phi1_sources(const float *sx, const float *sy, const float *sz,
                                             const float *sw, int j0, int cnt, int i, float xi, float yi,
                                             float zi, const DirectParams &P, double &acc64, Kahan &acc32,
                                             float h32, float inv_h, float inv70h) {
  for (int k = 0; k < cnt; ++k) {
    if (j0 + k == i) continue;
    if (FP64) {
      const double dx = (double)__fsub_rn(sx[k], xi);
      const double dy = (double)__fsub_rn(sy[k], yi);
      const double dz = (double)__fsub_rn(sz[k], zi);
      const double r = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                                            __dmul_rn(dz, dz)));
      const double dd = __dmul_rn(P.fac, depth_continuous<double>(r, P.app));
      acc64 = __dadd_rn(acc64, -__dmul_rn((double)sw[k], dd));
    } else {
      const float dx = sx[k] - xi, dy = sy[k] - yi, dz = sz[k] - zi;
      const float r2 = dx * dx + dy * dy + dz * dz;
      acc32.add(-sw[k] * depth_f32(r2, h32, inv_h, inv70h));
    }
  }
}

// The first-pass potentials of many direct-summation halos, spread over
// the whole GPU: block b takes the PT targets tiles[b] = (entry of list,
// first target) of one halo and streams the halo's members through shared
// memory in ascending order.  Each target's sum has exactly the order and
// operations of the in-kernel first pass of ub_direct_kernel, so the
// results are the same bits; the removal loop then starts from phi1.
constexpr int PT = 64;
template <bool FP64>
__global__ void __launch_bounds__(PT) ub_direct_phi1_kernel(Members m, const int64_t *__restrict__ off,
                                                            const int32_t *__restrict__ list,
                                                            const int2 *__restrict__ tiles, DirectParams P,
                                                            double *__restrict__ phi1) {
  __shared__ float sx[PT], sy[PT], sz[PT], sw[PT];
  const int2 t = tiles[blockIdx.x];
  const int c = list[t.x];
  const int64_t b0 = off[c];
  const int np = (int)(off[c + 1] - b0);
  const int i = t.y + threadIdx.x;
  const bool act = i < np;
  const float xi = act ? m.q[0][b0 + i] : 0.f, yi = act ? m.q[1][b0 + i] : 0.f,
              zi = act ? m.q[2][b0 + i] : 0.f;
  const float h32 = (float)P.app, inv_h = (float)(1.0 / P.app), inv70h = (float)(1.0 / (70.0 * P.app));
  double acc64 = 0.0;
  Kahan acc32;
  for (int j0 = 0; j0 < np; j0 += PT) {
    const int j = j0 + threadIdx.x;
    if (j < np) {
      sx[threadIdx.x] = m.q[0][b0 + j];
      sy[threadIdx.x] = m.q[1][b0 + j];
      sz[threadIdx.x] = m.q[2][b0 + j];
      sw[threadIdx.x] = m.w[b0 + j];
    }
    __syncthreads();
    if (act)
      phi1_sources<FP64>(sx, sy, sz, sw, j0, min(PT, np - j0), i, xi, yi, zi, P, acc64, acc32, h32, inv_h,
                         inv70h);
    __syncthreads();
  }
  if (act) phi1[b0 + i] = FP64 ? acc64 : (double)((float)P.fac * acc32.s);
}

// Dynamic shared memory of ub_direct_kernel for halos of up to cap members
// (cap a multiple of 32): nine float and two int arrays, one double array
// and the keep flags.
__host__ __device__ constexpr size_t direct_smem(int cap) { return (size_t)cap * (11 * 4 + 8 + 1); }

// One block of NT threads per halo: bound_check_grid for gid 0
// (:2611-2864).  FP64=true is the plain FP64 path, bit-exact with the
// reference arithmetic; FP64=false the FP32 product path with compensated
// sums.  phi1 (optional): the first-pass potentials from
// ub_direct_phi1_kernel; null computes them here.  Every halo of the launch
// has at most cap members.  No result depends on NT: every sum runs in an
// order fixed by the member indices alone (per-target serial sums, the
// FP64 centre sums in thread 0, the FP32 ones in warp 0 by index mod 32).
template <bool FP64, int NT = BLK>
__global__ void __launch_bounds__(NT) ub_direct_kernel(Members m, const int64_t *__restrict__ off,
                                                       const int32_t *__restrict__ list,
                                                       DirectParams P, HaloResult *__restrict__ res,
                                                       uint8_t *__restrict__ keep_out,
                                                       float *__restrict__ phi_out,
                                                       int32_t *flags,
                                                       const double *__restrict__ phi1 = nullptr,
                                                       int cap = kDirectMax) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int c = list[blockIdx.x];
  const int64_t b0 = off[c];
  const int np = (int)(off[c + 1] - b0);
  float *qx = reinterpret_cast<float *>(smem);
  float *qy = qx + cap, *qz = qy + cap;
  float *vx = qz + cap, *vy = vx + cap, *vz = vy + cap;
  float *w = vz + cap, *phi = w + cap, *en = phi + cap;
  int *jdel = reinterpret_cast<int *>(en + cap);
  int *unb = jdel + cap;
  double *phid = reinterpret_cast<double *>(unb + cap);
  unsigned char *keep = reinterpret_cast<unsigned char *>(phid + cap);
  __shared__ int red_i[NT / 32];
  __shared__ double s_qc[3], s_vc[3], s_sum[7];
  __shared__ int s_nu, s_err;

  for (int i = threadIdx.x; i < np; i += NT) {
    const int64_t k = b0 + i;
    qx[i] = m.q[0][k]; qy[i] = m.q[1][k]; qz[i] = m.q[2][k];
    vx[i] = m.v[0][k]; vy[i] = m.v[1][k]; vz[i] = m.v[2][k];
    w[i] = m.w[k];
    keep[i] = 1;
    phid[i] = 0.0;
  }
  if (threadIdx.x == 0) s_err = 0;
  __syncthreads();
  const float h32 = (float)P.app, inv_h = (float)(1.0 / P.app), inv70h = (float)(1.0 / (70.0 * P.app));
  const float fac32 = (float)P.fac;
  int np_bound = np, njd = 0, status = 5;

  for (int pass = 1; pass <= kMaxPasses; ++pass) {
    int ks = 0;
    for (int i = threadIdx.x; i < np; i += NT) ks += keep[i];
    const int n_source = block_sum_i(ks, red_i);
    // potential: full sum on the first pass, later passes add back the
    // sources removed since the previous refresh
    for (int i = threadIdx.x; i < np; i += NT) {
      if (pass == 1 && phi1) {
        phid[i] = phi1[b0 + i];
      } else if (pass == 1) {
        if (FP64) {
          double acc = 0.0;
          for (int j = 0; j < np; ++j) {
            if (j == i) continue;
            const double dx = (double)__fsub_rn(qx[j], qx[i]);
            const double dy = (double)__fsub_rn(qy[j], qy[i]);
            const double dz = (double)__fsub_rn(qz[j], qz[i]);
            const double r = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                                                  __dmul_rn(dz, dz)));
            const double dd = __dmul_rn(P.fac, depth_continuous<double>(r, P.app));
            acc = __dadd_rn(acc, -__dmul_rn((double)w[j], dd));
          }
          phid[i] = acc;
        } else {
          Kahan acc;
          const float xi = qx[i], yi = qy[i], zi = qz[i];
          for (int j = 0; j < np; ++j) {
            if (j == i) continue;
            const float dx = qx[j] - xi, dy = qy[j] - yi, dz = qz[j] - zi;
            const float r2 = dx * dx + dy * dy + dz * dz;
            acc.add(-w[j] * depth_f32(r2, h32, inv_h, inv70h));
          }
          phid[i] = (double)(fac32 * acc.s);
        }
      } else if (keep[i]) {
        if (FP64) {
          double acc = phid[i];
          for (int k = 0; k < njd; ++k) {
            const int j = jdel[k];
            const double dx = (double)__fsub_rn(qx[j], qx[i]);
            const double dy = (double)__fsub_rn(qy[j], qy[i]);
            const double dz = (double)__fsub_rn(qz[j], qz[i]);
            const double r = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                                                  __dmul_rn(dz, dz)));
            acc = __dadd_rn(acc, __dmul_rn(__dmul_rn((double)w[j], P.fac),
                                           depth_continuous<double>(r, P.app)));
          }
          phid[i] = acc;
        } else {
          Kahan acc;
          const float xi = qx[i], yi = qy[i], zi = qz[i];
          for (int k = 0; k < njd; ++k) {
            const int j = jdel[k];
            const float dx = qx[j] - xi, dy = qy[j] - yi, dz = qz[j] - zi;
            acc.add(w[j] * depth_f32(dx * dx + dy * dy + dz * dz, h32, inv_h, inv70h));
          }
          phid[i] += (double)(fac32 * acc.s);
        }
      }
    }
    njd = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < np; i += NT) {
      if (!keep[i]) continue;
      float v = FP64 ? __double2float_rn(phid[i]) : (float)phid[i];
      if (np_bound == 1 || n_source == 1) v = 0.0f;
      if (!isfinite(v)) s_err = kNonFinite;
      phi[i] = v;
    }
    __syncthreads();
    if (s_err) break;
    if (P.phi_only) { status = 0; break; }
    int deleted = 0;
    for (;;) {
      // centre of mass and mean velocity of the kept set, FP64
      if (FP64) {
        // seven sequential sums in ascending index (the reference's order),
        // one per lane of warp 0: the kept mass and the mass-weighted
        // positions and velocities
        if (threadIdx.x < 7) {
          const int qi = threadIdx.x;
          const float *src = qi == 1 ? qx : qi == 2 ? qy : qi == 3 ? qz : qi == 4 ? vx : qi == 5 ? vy : vz;
          double acc = 0.0;
#pragma unroll 4
          for (int i = 0; i < np; ++i) {
            if (!keep[i]) continue;
            const double wi = (double)w[i];
            acc = __dadd_rn(acc, qi == 0 ? wi : __dmul_rn(wi, (double)src[i]));
          }
          s_sum[qi] = acc;
        }
        __syncwarp();
        if (threadIdx.x == 0) {
          const double ws = s_sum[0];
          for (int d = 0; d < 3; ++d) {
            s_qc[d] = __ddiv_rn(s_sum[1 + d], ws);
            s_vc[d] = __ddiv_rn(s_sum[4 + d], ws);
          }
        }
      } else if (threadIdx.x < 32) {
        // warp 0: lane l sums the members l, l+32, ...; then a butterfly
        double a[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int i = threadIdx.x; i < np; i += 32) {
          if (!keep[i]) continue;
          const double wi = (double)w[i];
          a[0] += wi;
          a[1] += wi * qx[i]; a[2] += wi * qy[i]; a[3] += wi * qz[i];
          a[4] += wi * vx[i]; a[5] += wi * vy[i]; a[6] += wi * vz[i];
        }
        for (int k = 0; k < 7; ++k)
          for (int o = 16; o > 0; o >>= 1) a[k] += __shfl_xor_sync(0xffffffffu, a[k], o);
        if (threadIdx.x == 0) {
          for (int d = 0; d < 3; ++d) { s_qc[d] = a[1 + d] / a[0]; s_vc[d] = a[4 + d] / a[0]; }
        }
      }
      if (threadIdx.x == 0) s_nu = 0;
      __syncthreads();
      const float qc0 = __double2float_rn(s_qc[0]), qc1 = __double2float_rn(s_qc[1]),
                  qc2 = __double2float_rn(s_qc[2]);
      const float vc0 = __double2float_rn(s_vc[0]), vc1 = __double2float_rn(s_vc[1]),
                  vc2 = __double2float_rn(s_vc[2]);
      // specific energies (bound_fortran.f90:2773-2786), FP32
      for (int i = threadIdx.x; i < np; i += NT) {
        if (!keep[i]) continue;
        const float d0 = __fadd_rn(__fsub_rn(vx[i], vc0), __fmul_rn(P.b, __fsub_rn(qx[i], qc0)));
        const float d1 = __fadd_rn(__fsub_rn(vy[i], vc1), __fmul_rn(P.b, __fsub_rn(qy[i], qc1)));
        const float d2 = __fadd_rn(__fsub_rn(vz[i], vc2), __fmul_rn(P.b, __fsub_rn(qz[i], qc2)));
        float s = __fmul_rn(d0, d0);
        s = __fadd_rn(s, __fmul_rn(d1, d1));
        s = __fadd_rn(s, __fmul_rn(d2, d2));
        const float e = __fadd_rn(__fdiv_rn(s, 2.0f), phi[i]);
        if (!isfinite(e)) s_err = kInvalid;
        en[i] = e;
        if (e >= 0.0f) unb[atomicAdd(&s_nu, 1)] = i;
      }
      __syncthreads();
      if (s_err) break;
      const int nu = s_nu;
      if (nu == 0) {
        if (deleted == 0) { status = 0; break; }
        break;
      }
      // delete the nb highest energies; ties go to the lower local index
      // first (bound_fortran.f90:2808-2844)
      int nb = (int)ceil(0.02 * (double)np_bound);
      nb = max(1, nb);
      nb = min(nu, nb);
      for (int t = threadIdx.x; t < nu; t += NT) {
        const int i = unb[t];
        const float ei = en[i];
        int rank = 0;
        for (int u = 0; u < nu; ++u) {
          const int j = unb[u];
          const float ej = en[j];
          rank += (ej > ei) || (ej == ei && j < i);
        }
        if (rank < nb) {
          keep[i] = 0;
          jdel[njd + rank] = i;
        }
      }
      __syncthreads();
      njd += nb;
      np_bound -= nb;
      deleted += nb;
      if (np_bound < P.nmin) { status = 1; break; }
      if ((double)deleted >= 0.2 * (double)np_bound) break;
    }
    __syncthreads();
    if (s_err || status != 5) break;
    if (pass == kMaxPasses) break;
  }
  if (s_err) {
    if (threadIdx.x == 0) atomicCAS(&flags[FLAG_ERR], 0, s_err);
    return;
  }
  for (int i = threadIdx.x; i < np; i += NT) {
    keep_out[b0 + i] = keep[i];
    if (phi_out) phi_out[b0 + i] = phi[i];
  }
  if (threadIdx.x == 0) {
    res[c].status = status;
    res[c].np_bound = np_bound;
  }
}

}  // namespace direct
}  // namespace pyfof
