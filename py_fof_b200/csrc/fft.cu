// Batched zero-padded 3-D FFT convolution for the particle-mesh solver.
// See fft.cuh for layouts.
//
// Every line transform of length N = N1 * N2 runs as two register-resident
// DFTs with one shared-memory exchange between them (Cooley-Tukey with the
// input index e = s + N2 q and the output index k = k1 + N1 k2):
//   stage A  thread (line, s):  Y[s][k1] = sum_q x[s + N2 q] W_N1^(q k1),
//            times the twiddle W_N^(s k1), written to shared memory;
//   stage B  thread (line, k1): X[k1 + N1 k2] = sum_s Y[s][k1] W_N2^(s k2).
// The register DFTs are mixed-radix (4, 2, 3) decompositions unrolled at
// compile time with constant twiddles.  A block works on a tile of W lines
// that are adjacent in memory (consecutive kx), so every global access of a
// warp covers whole 128-byte segments.  The z pass does forward transform,
// Green multiplication and inverse transform in one kernel (stage B holds a
// full frequency line per thread; the inverse walks the same stages back),
// and loops over the halos of a batch with the Green values held in
// registers, so the table is read once per block.
#include <utility>

#include "fft.cuh"

namespace pyfof {

namespace {

// ------------------------------------------------------------ compile time

template <class F, int... I>
__device__ __forceinline__ void sfor_impl(F &&f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void sfor(F &&f) {
  sfor_impl(static_cast<F &&>(f), std::make_integer_sequence<int, N>{});
}

constexpr double kQuarterPi = 0.785398163397448309615660845819875721;

__host__ __device__ constexpr double taylor_sin(double x) {
  double x2 = x * x, term = x, sum = x;
  for (int k = 1; k < 12; ++k) {
    term *= -x2 / (double)((2 * k) * (2 * k + 1));
    sum += term;
  }
  return sum;
}
__host__ __device__ constexpr double taylor_cos(double x) {
  double x2 = x * x, term = 1.0, sum = 1.0;
  for (int k = 1; k < 12; ++k) {
    term *= -x2 / (double)((2 * k - 1) * (2 * k));
    sum += term;
  }
  return sum;
}

struct CosSin {
  double c, s;
};

// cos and sin of the angle 2 pi num / den: exact octant reduction of the
// rational angle, then Taylor series on [0, pi/4].
__host__ __device__ constexpr CosSin turn(int num, int den) {
  num %= den;
  if (num < 0) num += den;
  const long long e = 8LL * num;
  const int o = (int)(e / den);
  const long long r = e - (long long)o * den;
  const double th = kQuarterPi * (double)r / (double)den;          // [0, pi/4)
  const double ph = kQuarterPi * (double)(den - r) / (double)den;  // pi/4 - th
  switch (o) {
    case 0: return {taylor_cos(th), taylor_sin(th)};
    case 1: return {taylor_sin(ph), taylor_cos(ph)};
    case 2: return {-taylor_sin(th), taylor_cos(th)};
    case 3: return {-taylor_cos(ph), taylor_sin(ph)};
    case 4: return {-taylor_cos(th), -taylor_sin(th)};
    case 5: return {-taylor_sin(ph), -taylor_cos(ph)};
    case 6: return {taylor_sin(th), -taylor_cos(th)};
    default: return {taylor_cos(ph), -taylor_sin(ph)};
  }
}

// ---------------------------------------------------------------- complex

template <typename C>
__device__ __forceinline__ C mk(decltype(C{}.x) x, decltype(C{}.x) y) {
  C r;
  r.x = x;
  r.y = y;
  return r;
}
template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C>
__device__ __forceinline__ C cmulc(C a, C b) {
  return mk<C>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// v * exp(SIGN 2 pi i J / M), J and M known at compile time
template <int SIGN, int J, int M, typename C>
__device__ __forceinline__ C twc(C v) {
  constexpr int j = J % M;
  if constexpr (j == 0) {
    return v;
  } else if constexpr (2 * j == M) {
    return mk<C>(-v.x, -v.y);
  } else if constexpr (4 * j == M) {  // times SIGN i
    return SIGN < 0 ? mk<C>(v.y, -v.x) : mk<C>(-v.y, v.x);
  } else if constexpr (4 * j == 3 * M) {  // times -SIGN i
    return SIGN < 0 ? mk<C>(-v.y, v.x) : mk<C>(v.y, -v.x);
  } else {
    using R = decltype(v.x);
    constexpr CosSin w = turn(j, M);
    constexpr R c = (R)w.c;
    constexpr R s = (R)(SIGN * w.s);
    return mk<C>(v.x * c - v.y * s, v.x * s + v.y * c);
  }
}

// In-register DFT of length M: v[k] <- sum_e v[e] exp(SIGN 2 pi i e k / M).
template <int M, int SIGN, typename C>
__device__ __forceinline__ void dft(C (&v)[M]) {
  using R = decltype(v[0].x);
  if constexpr (M == 1) {
  } else if constexpr (M == 2) {
    const C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (M == 3) {
    const R h = (R)0.866025403784438646763723170752936183;  // sqrt(3)/2
    const C t1 = cadd(v[1], v[2]);
    const C t2 = mk<C>(v[0].x - (R)0.5 * t1.x, v[0].y - (R)0.5 * t1.y);
    const C d = csub(v[1], v[2]);
    const C t3 = SIGN < 0 ? mk<C>(h * d.y, -h * d.x) : mk<C>(-h * d.y, h * d.x);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
  } else if constexpr (M == 4) {
    const C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    const C t2 = cadd(v[1], v[3]), d = csub(v[1], v[3]);
    const C t3 = SIGN < 0 ? mk<C>(d.y, -d.x) : mk<C>(-d.y, d.x);
    v[0] = cadd(t0, t2);
    v[1] = cadd(t1, t3);
    v[2] = csub(t0, t2);
    v[3] = csub(t1, t3);
  } else {
    // decimation in time: e = p + P q, k = k' + Q j
    constexpr int P = (M % 4 == 0) ? 4 : ((M % 2 == 0) ? 2 : 3);
    constexpr int Q = M / P;
    static_assert(P * Q == M, "DFT length must be 2^a 3^b");
    C sub[P][Q];
#pragma unroll
    for (int p = 0; p < P; ++p) {
#pragma unroll
      for (int q = 0; q < Q; ++q) sub[p][q] = v[p + P * q];
      dft<Q, SIGN>(sub[p]);
    }
    sfor<Q>([&](auto kc) {
      constexpr int k = decltype(kc)::value;
      C t[P];
      sfor<P>([&](auto pc) {
        constexpr int p = decltype(pc)::value;
        t[p] = twc<SIGN, p * k, M>(sub[p][k]);
      });
      dft<P, SIGN>(t);
#pragma unroll
      for (int j = 0; j < P; ++j) v[k + Q * j] = t[j];
    });
  }
}

// ------------------------------------------------------------------ plans

// Lines per tile: 128 bytes of complex values per row of the tile.
template <typename R>
constexpr int kW = sizeof(R) == 4 ? 16 : 8;

// N = N1 * N2 and threads per block.
template <typename R, int N>
struct Cfg;
template <> struct Cfg<float, 48> { static constexpr int N1 = 8, N2 = 6, T = 128; };
template <> struct Cfg<float, 64> { static constexpr int N1 = 8, N2 = 8, T = 128; };
template <> struct Cfg<float, 128> { static constexpr int N1 = 16, N2 = 8, T = 128; };
template <> struct Cfg<float, 216> { static constexpr int N1 = 12, N2 = 18, T = 96; };
template <> struct Cfg<float, 256> { static constexpr int N1 = 16, N2 = 16, T = 256; };
template <> struct Cfg<double, 48> { static constexpr int N1 = 8, N2 = 6, T = 64; };
template <> struct Cfg<double, 64> { static constexpr int N1 = 8, N2 = 8, T = 64; };
template <> struct Cfg<double, 128> { static constexpr int N1 = 16, N2 = 8, T = 64; };
template <> struct Cfg<double, 216> { static constexpr int N1 = 12, N2 = 18, T = 96; };
template <> struct Cfg<double, 256> { static constexpr int N1 = 16, N2 = 16, T = 128; };

// Shared memory of the line kernels: twiddles and one tile of N rows of W+1
// complex (one pad column).  Every stage runs in place: stage B rewrites
// exactly the column each thread read, stage A reads all its inputs into
// registers before a barrier (x passes); the plain y passes write stage B
// straight to the spectrum.
template <typename R, int N>
constexpr size_t smem_lines_bytes() {
  return sizeof(cplx_t<R>) * (size_t)(N + (kW<R> + 1) * N);
}

// Shared memory of the fused z pass: the tile plus two staging buffers of
// N/2+1 rows for the next halo's input.
template <typename R, int N>
constexpr size_t smem_conv_bytes() {
  return smem_lines_bytes<R, N>() + sizeof(cplx_t<R>) * (size_t)(2 * (N / 2 + 1) * kW<R>);
}

// 16-byte asynchronous copy global -> shared (completion by wait_group)
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int K>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(K) : "memory"); }

// tw[j] = exp(-2 pi i j / N), from double-precision sincospi
template <typename R, int N, int T>
__device__ __forceinline__ void load_twiddles(cplx_t<R> *tw) {
  for (int j = threadIdx.x; j < N; j += T) {
    double s, c;
    sincospi(2.0 * (double)j / (double)N, &s, &c);
    tw[j] = mk<cplx_t<R>>((R)c, (R)-s);
  }
}

// Stage A in place on `buf`: every thread first reads all the elements of
// its units into registers, then (after a barrier) writes the results over
// the tile.
template <typename R, int N, int SIGN>
__device__ __forceinline__ void stage_a_inplace(cplx_t<R> *buf, const cplx_t<R> *tw, int in_lim) {
  using C = cplx_t<R>;
  constexpr int N1 = Cfg<R, N>::N1, N2 = Cfg<R, N>::N2, T = Cfg<R, N>::T;
  constexpr int W = kW<R>, WP = W + 1, UA = W * N2, IA = (UA + T - 1) / T;
  C v[IA][N1];
#pragma unroll
  for (int it = 0; it < IA; ++it) {
    const int u = threadIdx.x + it * T;
    const int li = u % W, s = u / W;
#pragma unroll
    for (int q = 0; q < N1; ++q) {
      const int e = s + N2 * q;
      v[it][q] = (u < UA && e < in_lim) ? buf[li + WP * e] : mk<C>(0, 0);
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < IA; ++it) {
    const int u = threadIdx.x + it * T;
    if (u < UA) {
      const int li = u % W, s = u / W;
      dft<N1, SIGN>(v[it]);
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1)
        buf[li + WP * (k1 + N1 * s)] = SIGN < 0 ? cmul(v[it][k1], tw[s * k1]) : cmulc(v[it][k1], tw[s * k1]);
    }
  }
}

// Stage B from `src` (stage A layout) into tile layout `dst` (li + (W+1) k).
// Unit (li, k1) reads and writes only the elements li + (W+1) (k1 + N1 j),
// so src may equal dst.
template <typename R, int N, int SIGN>
__device__ __forceinline__ void stage_b_smem(const cplx_t<R> *src, cplx_t<R> *dst) {
  using C = cplx_t<R>;
  constexpr int N1 = Cfg<R, N>::N1, N2 = Cfg<R, N>::N2, T = Cfg<R, N>::T;
  constexpr int W = kW<R>, WP = W + 1, UB = W * N1;
#pragma unroll
  for (int it = 0; it < (UB + T - 1) / T; ++it) {
    const int u = threadIdx.x + it * T;
    if (u < UB) {
      const int li = u % W, k1 = u / W;
      C v[N2];
#pragma unroll
      for (int s = 0; s < N2; ++s) v[s] = src[li + WP * (k1 + N1 * s)];
      dft<N2, SIGN>(v);
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) dst[li + WP * (k1 + N1 * k2)] = v[k2];
    }
  }
}

// ------------------------------------------------------------------ kernels

// x pass, forward r2c.  Real lines L = (b*SUP + z)*SUP + y, x < SUP
// (SUP = N/2 + 1), are taken in pairs as one complex line (a + i b); the two
// half spectra are separated with the Hermitian symmetry of real
// transforms.  All loops have compile-time trip counts, so every thread
// issues its loads before the first one returns.
// FIX: the input is the fixed-point deposit grid (64-bit integers, grid b
// scaled by inv_scale[b]) instead of R values.
template <typename R, int N, bool FIX>
__global__ void __launch_bounds__(Cfg<R, N>::T) k_x_r2c(const R *__restrict__ rho, cplx_t<R> *__restrict__ spec,
                                                        int nhp, int nlines,
                                                        const unsigned long long *__restrict__ acc,
                                                        const double *__restrict__ inv_scale) {
  using C = cplx_t<R>;
  constexpr int T = Cfg<R, N>::T, W = kW<R>, WP = W + 1, NH = N / 2 + 1, SUP = N / 2 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *tw = reinterpret_cast<C *>(smem_raw);
  C *t0 = tw + N;
  load_twiddles<R, N, T>(tw);
  const int L0 = blockIdx.x * (2 * W);
  const int nl = min(2 * W, nlines - L0);
  const R *src = rho + (int64_t)L0 * SUP;
#pragma unroll
  for (int it = 0; it < (W * SUP + T - 1) / T; ++it) {
    const int idx = threadIdx.x + it * T;
    if (idx < W * SUP) {
      const int p = idx / SUP, x = idx - p * SUP;
      R va, vb;
      if constexpr (FIX) {
        const int la = L0 + 2 * p;
        va = 2 * p < nl ? (R)((double)acc[(int64_t)la * SUP + x] * inv_scale[la / (SUP * SUP)]) : (R)0;
        vb = 2 * p + 1 < nl ? (R)((double)acc[(int64_t)(la + 1) * SUP + x] * inv_scale[(la + 1) / (SUP * SUP)])
                            : (R)0;
      } else {
        va = 2 * p < nl ? src[(2 * p) * SUP + x] : (R)0;
        vb = 2 * p + 1 < nl ? src[(2 * p + 1) * SUP + x] : (R)0;
      }
      t0[p + WP * x] = mk<C>(va, vb);
    }
  }
  __syncthreads();
  stage_a_inplace<R, N, -1>(t0, tw, SUP);
  __syncthreads();
  stage_b_smem<R, N, -1>(t0, t0);
  __syncthreads();
#pragma unroll
  for (int it = 0; it < (2 * W * NH + T - 1) / T; ++it) {
    const int idx = threadIdx.x + it * T;
    const int lr = idx / NH, kx = idx - lr * NH;
    if (lr < nl) {
      const int L = L0 + lr, p = lr >> 1;
      const int b = L / (SUP * SUP), rem = L - b * (SUP * SUP);
      const int z = rem / SUP, y = rem - z * SUP;
      const C zk = t0[p + WP * kx];
      const C zm = t0[p + WP * ((N - kx) % N)];
      C out;
      if ((lr & 1) == 0) out = mk<C>((R)0.5 * (zk.x + zm.x), (R)0.5 * (zk.y - zm.y));
      else out = mk<C>((R)0.5 * (zk.y + zm.y), (R)0.5 * (zm.x - zk.x));
      spec[(((int64_t)b * N + z) * N + y) * nhp + kx] = out;
    }
  }
}

// x pass, c2r into compact cubes of side OLIM: lines L = (b*OLIM + z)*OLIM
// + y, out[L*OLIM + x] = x-th real value / scale.  Two Hermitian half
// spectra become one complex line (a + i b); only the real parts of the DC
// and Nyquist bins are used.
template <typename R, int N, int OLIM>
__global__ void __launch_bounds__(Cfg<R, N>::T) k_x_c2r(const cplx_t<R> *__restrict__ spec, R *__restrict__ out,
                                                        int nhp, int nlines, R scale) {
  using C = cplx_t<R>;
  constexpr int T = Cfg<R, N>::T, W = kW<R>, WP = W + 1, NH = N / 2 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *tw = reinterpret_cast<C *>(smem_raw);
  C *t0 = tw + N;
  load_twiddles<R, N, T>(tw);
  const int L0 = blockIdx.x * (2 * W);
  const int nl = min(2 * W, nlines - L0);
#pragma unroll
  for (int it = 0; it < (W * NH + T - 1) / T; ++it) {
    const int idx = threadIdx.x + it * T;
    if (idx < W * NH) {
      const int p = idx / NH, kx = idx - p * NH;
      C a = mk<C>(0, 0), b = mk<C>(0, 0);
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const int lr = 2 * p + hh;
        if (lr < nl) {
          const int L = L0 + lr;
          const int bb = L / (OLIM * OLIM), rem = L - bb * (OLIM * OLIM);
          const int z = rem / OLIM, y = rem - z * OLIM;
          const C v = spec[(((int64_t)bb * N + z) * N + y) * nhp + kx];
          if (hh == 0) a = v;
          else b = v;
        }
      }
      if (kx == 0 || kx == N / 2) {
        a.y = 0;
        b.y = 0;
      }
      t0[p + WP * kx] = mk<C>(a.x - b.y, a.y + b.x);
      if (kx > 0 && kx < N / 2) t0[p + WP * (N - kx)] = mk<C>(a.x + b.y, b.x - a.y);
    }
  }
  __syncthreads();
  stage_a_inplace<R, N, +1>(t0, tw, N);
  __syncthreads();
  stage_b_smem<R, N, +1>(t0, t0);
  __syncthreads();
  R *dst = out + (int64_t)L0 * OLIM;
#pragma unroll
  for (int it = 0; it < (W * OLIM + T - 1) / T; ++it) {
    const int idx = threadIdx.x + it * T;
    if (idx < W * OLIM) {
      const int p = idx / OLIM, x = idx - p * OLIM;
      const C v = t0[p + WP * x];
      if (2 * p < nl) dst[(2 * p) * OLIM + x] = v.x / scale;
      if (2 * p + 1 < nl) dst[(2 * p + 1) * OLIM + x] = v.y / scale;
    }
  }
}

// Strided pass over tiles of W consecutive kx.  Line (b, other, kx) starts at
// spec + b*bstride + other*ostride + kx, element e at + e*estride.  Elements
// e >= in_lim are zero; elements e < out_lim are written.  CONV: forward
// transform, multiplication by the real Green table (index ((e*N + other)*NH
// + kx)) and inverse transform; otherwise one transform of sign SIGN.  A
// block handles halos [b0, b0 + nbb) of the batch.
template <typename R, int N, int SIGN, bool CONV>
__global__ void __launch_bounds__(Cfg<R, N>::T) k_lines(cplx_t<R> *__restrict__ spec, const R *__restrict__ green,
                                                        int64_t bstride, int64_t ostride, int64_t estride,
                                                        int nother, int ntiles, int nbb, int batch, int in_lim,
                                                        int out_lim) {
  using C = cplx_t<R>;
  constexpr int N1 = Cfg<R, N>::N1, N2 = Cfg<R, N>::N2, T = Cfg<R, N>::T;
  constexpr int W = kW<R>, WP = W + 1, NH = N / 2 + 1;
  constexpr int UA = W * N2, UB = W * N1;
  constexpr int IA = (UA + T - 1) / T, IB = (UB + T - 1) / T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *tw = reinterpret_cast<C *>(smem_raw);
  C *const buf0 = tw + N;
  load_twiddles<R, N, T>(tw);
  int64_t bid = blockIdx.x;
  const int tile = (int)(bid % ntiles);
  bid /= ntiles;
  const int other = (int)(bid % nother);
  const int b0 = (int)(bid / nother) * nbb;
  const int b1 = min(batch, b0 + nbb);
  const int kx0 = tile * W;
  R g[CONV ? IB : 1][CONV ? N2 : 1];
  if constexpr (CONV) {
#pragma unroll
    for (int it = 0; it < IB; ++it) {
      const int u = threadIdx.x + it * T;
      const int li = u % W, k1 = u / W, kx = kx0 + li;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) {
        const int e = k1 + N1 * k2;
        g[it][k2] = (u < UB && kx < NH) ? green[((int64_t)e * N + other) * NH + kx] : (R)0;
      }
    }
  }
  __syncthreads();
  // CONV: the input rows of the next halo are copied into a staging buffer
  // while the current one is transformed (two buffers of N/2+1 rows of W
  // complex; in_lim <= N/2+1 there)
  constexpr int SROWS = N / 2 + 1, CPR = (int)(W * sizeof(C) / 16);
  C *const stage0 = buf0 + WP * N;
  auto prefetch = [&](int bb, int slot) {
    const C *src = spec + (int64_t)bb * bstride + (int64_t)other * ostride + kx0;
    C *dst = stage0 + slot * (SROWS * W);
    for (int c = threadIdx.x; c < in_lim * CPR; c += T) {
      const int e = c / CPR, part = c - e * CPR;
      cp_async16(reinterpret_cast<char *>(dst + e * W) + 16 * part,
                 reinterpret_cast<const char *>(src + (int64_t)e * estride) + 16 * part);
    }
    cp_async_commit();
  };
  if constexpr (CONV) {
    if (b0 < b1) prefetch(b0, 0);
  }
  for (int b = b0, i = 0; b < b1; ++b, ++i) {
    C *base = spec + (int64_t)b * bstride + (int64_t)other * ostride + kx0;
    C *bA = buf0;
    const C *stg = stage0 + (i & 1) * (SROWS * W);
    if constexpr (CONV) {
      if (b + 1 < b1) {
        prefetch(b + 1, (i + 1) & 1);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();
    }
    // stage A: input -> registers -> DFT over q -> twiddle -> shared
#pragma unroll
    for (int it = 0; it < IA; ++it) {
      const int u = threadIdx.x + it * T;
      if (u < UA) {
        const int li = u % W, s = u / W;
        const bool col = kx0 + li < NH;
        C v[N1];
#pragma unroll
        for (int q = 0; q < N1; ++q) {
          const int e = s + N2 * q;
          if constexpr (CONV) v[q] = (col && e < in_lim) ? stg[e * W + li] : mk<C>(0, 0);
          else v[q] = (col && e < in_lim) ? base[(int64_t)e * estride + li] : mk<C>(0, 0);
        }
        dft<N1, CONV ? -1 : SIGN>(v);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) {
          const C w = tw[s * k1];
          bA[li + WP * (k1 + N1 * s)] = (CONV || SIGN < 0) ? cmul(v[k1], w) : cmulc(v[k1], w);
        }
      }
    }
    __syncthreads();
    // stage B: DFT over s (and for CONV: Green, inverse DFT over k2, twiddle,
    // written back in place: unit (li, k1) reads and rewrites only its own
    // elements li + WP (k1 + N1 s))
    C *bB = buf0;
#pragma unroll
    for (int it = 0; it < IB; ++it) {
      const int u = threadIdx.x + it * T;
      if (u < UB) {
        const int li = u % W, k1 = u / W;
        C v[N2];
#pragma unroll
        for (int s = 0; s < N2; ++s) v[s] = bA[li + WP * (k1 + N1 * s)];
        dft<N2, CONV ? -1 : SIGN>(v);
        if constexpr (CONV) {
#pragma unroll
          for (int k2 = 0; k2 < N2; ++k2) {
            v[k2].x *= g[it][k2];
            v[k2].y *= g[it][k2];
          }
          dft<N2, +1>(v);
#pragma unroll
          for (int s = 0; s < N2; ++s) bB[li + WP * (k1 + N1 * s)] = cmulc(v[s], tw[s * k1]);
        } else {
          if (kx0 + li < NH) {
#pragma unroll
            for (int k2 = 0; k2 < N2; ++k2) {
              const int e = k1 + N1 * k2;
              if (e < out_lim) base[(int64_t)e * estride + li] = v[k2];
            }
          }
        }
      }
    }
    if constexpr (CONV) {
      __syncthreads();
      // stage A': inverse DFT over k1 -> element s + N2 q
#pragma unroll
      for (int it = 0; it < IA; ++it) {
        const int u = threadIdx.x + it * T;
        if (u < UA) {
          const int li = u % W, s = u / W;
          C v[N1];
#pragma unroll
          for (int k1 = 0; k1 < N1; ++k1) v[k1] = bB[li + WP * (k1 + N1 * s)];
          dft<N1, +1>(v);
          if (kx0 + li < NH) {
#pragma unroll
            for (int q = 0; q < N1; ++q) {
              const int e = s + N2 * q;
              if (e < out_lim) base[(int64_t)e * estride + li] = v[q];
            }
          }
        }
      }
    }
    // the next halo's stage A rewrites the tile: every thread must have
    // finished reading it (CONV: the barrier at the top of the loop)
    if constexpr (!CONV) __syncthreads();
  }
}

template <typename R>
__global__ void k_real_to_cplx(const R *__restrict__ g, cplx_t<R> *__restrict__ spec, int n, int nhp) {
  const int nh = n / 2 + 1;
  const int64_t cnt = (int64_t)nh * n * n;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = i / nh;
    const int kx = (int)(i - row * nh);
    spec[row * nhp + kx] = mk<cplx_t<R>>(g[i], (R)0);
  }
}

template <typename K>
int32_t allow_smem(K kernel, size_t bytes) {
  PYFOF_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return kOk;
}

// Shared-memory limits of every kernel of grid N, set once per process.
template <typename R, int N>
int32_t prepare() {
  static std::once_flag once;
  static int32_t status = kOk;
  std::call_once(once, [] {
    const size_t sm = smem_lines_bytes<R, N>();
    int32_t r = kOk;
    if (r == kOk) r = allow_smem(k_x_r2c<R, N, false>, sm);
    if (r == kOk) r = allow_smem(k_x_r2c<R, N, true>, sm);
    if (r == kOk) r = allow_smem(k_x_c2r<R, N, N / 2 + 1>, sm);
    if (r == kOk) r = allow_smem(k_x_c2r<R, N, N>, sm);
    if (r == kOk) r = allow_smem(k_lines<R, N, -1, false>, smem_lines_bytes<R, N>());
    if (r == kOk) r = allow_smem(k_lines<R, N, +1, false>, smem_lines_bytes<R, N>());
    if (r == kOk) r = allow_smem(k_lines<R, N, -1, true>, smem_conv_bytes<R, N>());
    status = r;
  });
  return status;
}

template <typename R, int N>
int32_t convolve_n(R *rho, cplx_t<R> *spec, const R *green, int sup, int batch, cudaStream_t s,
                   const unsigned long long *acc, const double *inv_scale, int waves) {
  PYFOF_TRY((prepare<R, N>()));
  constexpr int W = kW<R>, T = Cfg<R, N>::T;
  const int nhp = (int)spec_row<R>(N);
  const int ntiles = nhp / W;
  const size_t sm = smem_lines_bytes<R, N>();
  const int64_t bstride = (int64_t)N * N * nhp;
  const int64_t nlines = (int64_t)batch * sup * sup;
  if (acc)
    k_x_r2c<R, N, true><<<(unsigned)ceil_div(nlines, 2 * W), T, sm, s>>>(rho, spec, nhp, (int)nlines, acc,
                                                                         inv_scale);
  else
    k_x_r2c<R, N, false><<<(unsigned)ceil_div(nlines, 2 * W), T, sm, s>>>(rho, spec, nhp, (int)nlines, nullptr,
                                                                          nullptr);
  PYFOF_CHECK_LAUNCH();
  // y forward: lines (kx, z < sup), input y < sup, output all y
  k_lines<R, N, -1, false><<<(unsigned)((int64_t)ntiles * sup * batch), T, smem_lines_bytes<R, N>(), s>>>(
      spec, nullptr, bstride, (int64_t)N * nhp, nhp, sup, ntiles, 1, batch, sup, N);
  PYFOF_CHECK_LAUNCH();
  // z: forward, Green, inverse; lines (kx, ky), input and output z < sup;
  // halos split into chunks so that the grid is at least `waves` full waves
  const int64_t per = (int64_t)ntiles * N;
  static int conv_blocks_per_sm = 0;
  if (!conv_blocks_per_sm) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_lines<R, N, -1, true>, T,
                                                      smem_conv_bytes<R, N>()) != cudaSuccess || b < 1)
      b = 1;
    conv_blocks_per_sm = b;
  }
  const int64_t slots = (int64_t)conv_blocks_per_sm * kNumSMs;
  const int nchunk = (int)std::max<int64_t>(1, std::min<int64_t>(batch, ceil_div((int64_t)waves * slots, per)));
  const int nbb = (int)ceil_div(batch, nchunk);
  const int nchunk_used = (int)ceil_div(batch, nbb);
  k_lines<R, N, -1, true><<<(unsigned)(per * nchunk_used), T, smem_conv_bytes<R, N>(), s>>>(
      spec, green, bstride, nhp, (int64_t)N * nhp, N, ntiles, nbb, batch, sup, sup);
  PYFOF_CHECK_LAUNCH();
  // y inverse: lines (kx, z < sup), input all y, output y < sup
  k_lines<R, N, +1, false><<<(unsigned)((int64_t)ntiles * sup * batch), T, smem_lines_bytes<R, N>(), s>>>(
      spec, nullptr, bstride, (int64_t)N * nhp, nhp, sup, ntiles, 1, batch, N, sup);
  PYFOF_CHECK_LAUNCH();
  const R n3 = (R)((double)N * N * N);
  k_x_c2r<R, N, N / 2 + 1><<<(unsigned)ceil_div(nlines, 2 * W), T, sm, s>>>(spec, rho, nhp, (int)nlines, n3);
  PYFOF_CHECK_LAUNCH();
  return kOk;
}

template <typename R, int N>
int32_t c2r_full_n(const R *green, cplx_t<R> *spec, R *out, cudaStream_t s) {
  PYFOF_TRY((prepare<R, N>()));
  constexpr int W = kW<R>, T = Cfg<R, N>::T;
  const int nhp = (int)spec_row<R>(N);
  const int ntiles = nhp / W;
  const size_t sm = smem_lines_bytes<R, N>();
  const int64_t cnt = (int64_t)(N / 2 + 1) * N * N;
  k_real_to_cplx<R><<<(unsigned)std::min<int64_t>(ceil_div(cnt, 256), 4096), 256, 0, s>>>(green, spec, N, nhp);
  PYFOF_CHECK_LAUNCH();
  const int64_t bstride = (int64_t)N * N * nhp;
  // z inverse over all ky, then y inverse over all z
  k_lines<R, N, +1, false><<<(unsigned)((int64_t)ntiles * N), T, smem_lines_bytes<R, N>(), s>>>(
      spec, nullptr, bstride, nhp, (int64_t)N * nhp, N, ntiles, 1, 1, N, N);
  PYFOF_CHECK_LAUNCH();
  k_lines<R, N, +1, false><<<(unsigned)((int64_t)ntiles * N), T, smem_lines_bytes<R, N>(), s>>>(
      spec, nullptr, bstride, (int64_t)N * nhp, nhp, N, ntiles, 1, 1, N, N);
  PYFOF_CHECK_LAUNCH();
  const int64_t nlines = (int64_t)N * N;
  k_x_c2r<R, N, N><<<(unsigned)ceil_div(nlines, 2 * W), T, sm, s>>>(spec, out, nhp, (int)nlines, (R)1);
  PYFOF_CHECK_LAUNCH();
  return kOk;
}

}  // namespace

template <typename R>
int32_t pm_convolve_batch(R *rho, cplx_t<R> *spec, const R *green, int n, int sup, int batch,
                          cudaStream_t s, const unsigned long long *acc, const double *inv_scale, int waves) {
  if (sup != n / 2 + 1 || batch < 1 || (int64_t)batch * sup * sup >= (int64_t)1 << 30) {
    set_error("invalid convolution batch (n %d, support %d, batch %d)", n, sup, batch);
    return kInvalid;
  }
  switch (n) {
    case 48: return convolve_n<R, 48>(rho, spec, green, sup, batch, s, acc, inv_scale, waves);
    case 64: return convolve_n<R, 64>(rho, spec, green, sup, batch, s, acc, inv_scale, waves);
    case 128: return convolve_n<R, 128>(rho, spec, green, sup, batch, s, acc, inv_scale, waves);
    case 216: return convolve_n<R, 216>(rho, spec, green, sup, batch, s, acc, inv_scale, waves);
    case 256: return convolve_n<R, 256>(rho, spec, green, sup, batch, s, acc, inv_scale, waves);
    default: set_error("unsupported FFT size %d", n); return kInvalid;
  }
}

template <typename R>
int32_t c2r_full(const R *green, cplx_t<R> *spec, R *out, int n, cudaStream_t s) {
  switch (n) {
    case 48: return c2r_full_n<R, 48>(green, spec, out, s);
    case 64: return c2r_full_n<R, 64>(green, spec, out, s);
    case 128: return c2r_full_n<R, 128>(green, spec, out, s);
    case 216: return c2r_full_n<R, 216>(green, spec, out, s);
    case 256: return c2r_full_n<R, 256>(green, spec, out, s);
    default: set_error("unsupported FFT size %d", n); return kInvalid;
  }
}

template int32_t pm_convolve_batch<float>(float *, float2 *, const float *, int, int, int, cudaStream_t,
                                          const unsigned long long *, const double *, int);
template int32_t pm_convolve_batch<double>(double *, double2 *, const double *, int, int, int, cudaStream_t,
                                           const unsigned long long *, const double *, int);
template int32_t c2r_full<float>(const float *, float2 *, float *, int, cudaStream_t);
template int32_t c2r_full<double>(const double *, double2 *, double *, int, cudaStream_t);

}  // namespace pyfof
