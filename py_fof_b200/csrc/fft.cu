// Batched zero-padded 3-D FFT convolution for the particle-mesh solver.
// See fft.cuh for layouts.  Each kernel transforms whole lines held in
// shared memory with a Stockham autosort FFT (radices 4, 2, 3).
#include "fft.cuh"

namespace pyfof {

namespace {

constexpr int FT = 256;  // threads per block

template <typename R>
__device__ __forceinline__ void sincospi_t(R x, R *s, R *c);
template <>
__device__ __forceinline__ void sincospi_t<float>(float x, float *s, float *c) { sincospif(x, s, c); }
template <>
__device__ __forceinline__ void sincospi_t<double>(double x, double *s, double *c) { sincospi(x, s, c); }

template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }

struct Radices {
  int nf;
  int f[12];
};

Radices factor(int n) {
  Radices r{};
  while (n % 4 == 0) { r.f[r.nf++] = 4; n /= 4; }
  while (n % 2 == 0) { r.f[r.nf++] = 2; n /= 2; }
  while (n % 3 == 0) { r.f[r.nf++] = 3; n /= 3; }
  if (n != 1) r.nf = -1;
  return r;
}

// tw[k] = exp(-2 pi i k / n)
template <typename R>
__device__ __forceinline__ void make_twiddles(cplx_t<R> *tw, int n) {
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    R s, c;
    sincospi_t<R>((R)(2 * k) / (R)n, &s, &c);
    tw[k].x = c;
    tw[k].y = -s;
  }
}

// Stockham FFT of `lines` lines of length n held in A (A[l*n+e]); B is
// scratch.  sign = -1 forward, +1 inverse (unnormalised).  Returns the
// buffer that holds the result.
template <typename R>
__device__ cplx_t<R> *fft_lines(cplx_t<R> *A, cplx_t<R> *B, const cplx_t<R> *tw, int n, int lines,
                                const Radices &rad, int sign) {
  typedef cplx_t<R> C;
  int m = 1;
  const R s3 = (R)0.86602540378443864676;  // sqrt(3)/2
  for (int st = 0; st < rad.nf; ++st) {
    const int r = rad.f[st];
    const int l = n / (m * r);
    const int step = n / (l * r);
    const int nb = n / r;
    for (int t = threadIdx.x; t < lines * nb; t += blockDim.x) {
      const int line = t / nb, bf = t - line * nb;
      const int j = bf / m, k = bf - j * m;
      const C *a = A + line * n;
      C *b = B + line * n;
      C v[4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (q < r) v[q] = a[(q * l + j) * m + k];
      C o[4];
      if (r == 2) {
        o[0] = cadd(v[0], v[1]);
        o[1] = csub(v[0], v[1]);
      } else if (r == 4) {
        const C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]), t2 = cadd(v[1], v[3]);
        const C d = csub(v[1], v[3]);
        C t3;  // d * (-i) forward, d * (+i) inverse
        if (sign < 0) { t3.x = d.y; t3.y = -d.x; } else { t3.x = -d.y; t3.y = d.x; }
        o[0] = cadd(t0, t2);
        o[1] = cadd(t1, t3);
        o[2] = csub(t0, t2);
        o[3] = csub(t1, t3);
      } else {
        const C t1 = cadd(v[1], v[2]);
        C t2;
        t2.x = v[0].x - (R)0.5 * t1.x;
        t2.y = v[0].y - (R)0.5 * t1.y;
        const C d = csub(v[1], v[2]);
        C t3;  // s3 * d * (-i) forward, s3 * d * (+i) inverse
        if (sign < 0) { t3.x = s3 * d.y; t3.y = -s3 * d.x; } else { t3.x = -s3 * d.y; t3.y = s3 * d.x; }
        o[0] = cadd(v[0], t1);
        o[1] = cadd(t2, t3);
        o[2] = csub(t2, t3);
      }
      // decimation in frequency: output u of butterfly j takes w^(j*u)
      C *ob = b + (j * r) * m + k;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (u < r) {
          C val = o[u];
          if (u > 0 && j > 0) {
            C w = tw[j * u * step];
            if (sign > 0) w.y = -w.y;
            val = cmul(val, w);
          }
          ob[u * m] = val;
        }
      }
    }
    __syncthreads();
    C *tmp = A; A = B; B = tmp;
    m *= r;
  }
  return A;
}

template <typename R>
__device__ __forceinline__ cplx_t<R> *smem_base() {
  extern __shared__ __align__(16) unsigned char fft_smem[];
  return reinterpret_cast<cplx_t<R> *>(fft_smem);
}

// x pass, forward r2c: lines (y,z) in [0,sup)^2 of every grid.
template <typename R>
__global__ void __launch_bounds__(FT) k_fft_x_r2c(const R *__restrict__ rho, cplx_t<R> *__restrict__ spec,
                                                  int n, int sup, int lpb, int64_t nlines, Radices rad) {
  typedef cplx_t<R> C;
  C *tw = smem_base<R>();
  C *A = tw + n, *B = A + lpb * n;
  make_twiddles<R>(tw, n);
  const int nh = n / 2 + 1;
  const int64_t l0 = (int64_t)blockIdx.x * lpb;
  const int nl = (int)(nlines - l0 < (int64_t)lpb ? nlines - l0 : (int64_t)lpb);
  for (int t = threadIdx.x; t < nl * n; t += blockDim.x) {
    const int li = t / n, x = t - li * n;
    const int64_t L = l0 + li;  // (b*sup + z)*sup + y
    C v;
    v.x = x < sup ? rho[L * sup + x] : (R)0;
    v.y = 0;
    A[li * n + x] = v;
  }
  __syncthreads();
  C *res = fft_lines<R>(A, B, tw, n, nl, rad, -1);
  for (int t = threadIdx.x; t < nl * nh; t += blockDim.x) {
    const int li = t / nh, kx = t - li * nh;
    const int64_t L = l0 + li;
    const int64_t b = L / ((int64_t)sup * sup);
    const int rem = (int)(L - b * sup * sup);
    const int z = rem / sup, y = rem - z * sup;
    spec[((b * n + z) * n + y) * nh + kx] = res[li * n + kx];
  }
}

// y or z pass over tiles of `lpb` consecutive kx.  AXIS 1: lines (kx, z),
// z < other_lim, elements y; AXIS 2: lines (kx, ky), ky < other_lim,
// elements z.  Elements >= in_lim are zero; elements < out_lim are written.
// With green != null (AXIS 2 only) the forward transform is followed by the
// Green multiplication and the inverse transform.
template <typename R, int AXIS>
__global__ void __launch_bounds__(FT) k_fft_yz(cplx_t<R> *__restrict__ spec, const R *__restrict__ green,
                                               int n, int other_lim, int in_lim, int out_lim,
                                               int sign, int lpb, Radices rad) {
  typedef cplx_t<R> C;
  C *tw = smem_base<R>();
  C *A = tw + n, *B = A + lpb * n;
  make_twiddles<R>(tw, n);
  const int nh = n / 2 + 1;
  const int ntx = (nh + lpb - 1) / lpb;
  int64_t bid = blockIdx.x;
  const int tx = (int)(bid % ntx);
  bid /= ntx;
  const int other = (int)(bid % other_lim);
  const int64_t b = bid / other_lim;
  const int kx0 = tx * lpb;
  const int nl = min(lpb, nh - kx0);
  auto addr = [&](int e, int kx) -> int64_t {
    return AXIS == 1 ? ((b * n + other) * n + e) * nh + kx : ((b * n + e) * n + other) * nh + kx;
  };
  for (int t = threadIdx.x; t < nl * n; t += blockDim.x) {
    const int e = t / nl, li = t - e * nl;
    C v;
    if (e < in_lim) v = spec[addr(e, kx0 + li)];
    else { v.x = 0; v.y = 0; }
    A[li * n + e] = v;
  }
  __syncthreads();
  C *res = fft_lines<R>(A, B, tw, n, nl, rad, sign);
  if (AXIS == 2 && green) {
    C *other_buf = (res == A) ? B : A;
    for (int t = threadIdx.x; t < nl * n; t += blockDim.x) {
      const int li = t / n, e = t - li * n;
      const R g = green[((int64_t)e * n + other) * nh + kx0 + li];
      res[t].x *= g;
      res[t].y *= g;
    }
    __syncthreads();
    res = fft_lines<R>(res, other_buf, tw, n, nl, rad, +1);
  }
  for (int t = threadIdx.x; t < nl * out_lim; t += blockDim.x) {
    const int e = t / nl, li = t - e * nl;
    spec[addr(e, kx0 + li)] = res[li * n + e];
  }
}

// x pass, c2r: lines (y,z) in [0,out)^2; out[x] = Re(line[x]) / scale for
// x < out, written to a compact cube of side `ostride`.
template <typename R>
__global__ void __launch_bounds__(FT) k_fft_x_c2r(const cplx_t<R> *__restrict__ spec, R *__restrict__ out,
                                                  int n, int olim, int lpb, int64_t nlines, R scale,
                                                  Radices rad) {
  typedef cplx_t<R> C;
  C *tw = smem_base<R>();
  C *A = tw + n, *B = A + lpb * n;
  make_twiddles<R>(tw, n);
  const int nh = n / 2 + 1;
  const int64_t l0 = (int64_t)blockIdx.x * lpb;
  const int nl = (int)(nlines - l0 < (int64_t)lpb ? nlines - l0 : (int64_t)lpb);
  for (int t = threadIdx.x; t < nl * nh; t += blockDim.x) {
    const int li = t / nh, kx = t - li * nh;
    const int64_t L = l0 + li;  // (b*olim + z)*olim + y
    const int64_t b = L / ((int64_t)olim * olim);
    const int rem = (int)(L - b * olim * olim);
    const int z = rem / olim, y = rem - z * olim;
    C c = spec[((b * n + z) * n + y) * nh + kx];
    if (kx == 0 || kx == n / 2) {
      c.y = 0;
      A[li * n + kx] = c;
    } else {
      A[li * n + kx] = c;
      C cc;
      cc.x = c.x;
      cc.y = -c.y;
      A[li * n + n - kx] = cc;
    }
  }
  __syncthreads();
  C *res = fft_lines<R>(A, B, tw, n, nl, rad, +1);
  for (int t = threadIdx.x; t < nl * olim; t += blockDim.x) {
    const int li = t / olim, x = t - li * olim;
    out[(l0 + li) * olim + x] = res[li * n + x].x / scale;
  }
}

template <typename R>
__global__ void k_real_to_cplx(const R *__restrict__ g, cplx_t<R> *__restrict__ spec, int64_t cnt) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += (int64_t)gridDim.x * blockDim.x) {
    cplx_t<R> c;
    c.x = g[i];
    c.y = 0;
    spec[i] = c;
  }
}

template <typename R>
int lines_per_block(int n) {
  // two line buffers of lpb*n complex plus the twiddles within 48 KB
  const int bytes = (int)sizeof(cplx_t<R>);
  int lpb = (48 * 1024 / bytes - n) / (2 * n);
  if (lpb > 16) lpb = 16;
  return lpb < 1 ? 1 : lpb;
}

template <typename R>
size_t smem_for(int n, int lpb) {
  return sizeof(cplx_t<R>) * (size_t)(n + 2 * lpb * n);
}

}  // namespace

template <typename R>
int32_t pm_convolve_batch(R *rho, cplx_t<R> *spec, const R *green, int n, int sup, int batch,
                          cudaStream_t s) {
  const Radices rad = factor(n);
  if (rad.nf < 0 || n > 256 || sup > n / 2 + 1) {
    set_error("unsupported FFT size %d", n);
    return kInvalid;
  }
  const int nh = n / 2 + 1;
  const int lpb = lines_per_block<R>(n);
  const size_t sm = smem_for<R>(n, lpb);
  // x r2c
  {
    const int64_t nlines = (int64_t)batch * sup * sup;
    k_fft_x_r2c<R><<<(unsigned)ceil_div(nlines, lpb), FT, sm, s>>>(rho, spec, n, sup, lpb, nlines, rad);
    PYFOF_CHECK_LAUNCH();
  }
  const int ntx = (nh + lpb - 1) / lpb;
  // y forward: lines (kx, z<sup), input y<sup, output all y
  k_fft_yz<R, 1><<<(unsigned)((int64_t)batch * sup * ntx), FT, sm, s>>>(spec, nullptr, n, sup, sup, n, -1,
                                                                        lpb, rad);
  PYFOF_CHECK_LAUNCH();
  // z forward, Green multiply, z inverse: lines (kx, ky), input z<sup, output z<sup
  k_fft_yz<R, 2><<<(unsigned)((int64_t)batch * n * ntx), FT, sm, s>>>(spec, green, n, n, sup, sup, -1, lpb,
                                                                      rad);
  PYFOF_CHECK_LAUNCH();
  // y inverse: lines (kx, z<sup), input all y, output y<sup
  k_fft_yz<R, 1><<<(unsigned)((int64_t)batch * sup * ntx), FT, sm, s>>>(spec, nullptr, n, sup, n, sup, +1,
                                                                        lpb, rad);
  PYFOF_CHECK_LAUNCH();
  // x c2r into the support cube, divided by n^3
  {
    const int64_t nlines = (int64_t)batch * sup * sup;
    const R n3 = (R)((double)n * n * n);
    k_fft_x_c2r<R><<<(unsigned)ceil_div(nlines, lpb), FT, sm, s>>>(spec, rho, n, sup, lpb, nlines, n3, rad);
    PYFOF_CHECK_LAUNCH();
  }
  return kOk;
}

template <typename R>
int32_t c2r_full(const R *green, cplx_t<R> *spec, R *out, int n, cudaStream_t s) {
  const Radices rad = factor(n);
  if (rad.nf < 0 || n > 256) {
    set_error("unsupported FFT size %d", n);
    return kInvalid;
  }
  const int nh = n / 2 + 1;
  const int lpb = lines_per_block<R>(n);
  const size_t sm = smem_for<R>(n, lpb);
  const int64_t cnt = (int64_t)nh * n * n;
  k_real_to_cplx<R><<<(unsigned)std::min<int64_t>(ceil_div(cnt, 256), 4096), 256, 0, s>>>(green, spec, cnt);
  PYFOF_CHECK_LAUNCH();
  const int ntx = (nh + lpb - 1) / lpb;
  k_fft_yz<R, 2><<<(unsigned)((int64_t)n * ntx), FT, sm, s>>>(spec, nullptr, n, n, n, n, +1, lpb, rad);
  PYFOF_CHECK_LAUNCH();
  k_fft_yz<R, 1><<<(unsigned)((int64_t)n * ntx), FT, sm, s>>>(spec, nullptr, n, n, n, n, +1, lpb, rad);
  PYFOF_CHECK_LAUNCH();
  const int64_t nlines = (int64_t)n * n;
  k_fft_x_c2r<R><<<(unsigned)ceil_div(nlines, lpb), FT, sm, s>>>(spec, out, n, n, lpb, nlines, (R)1, rad);
  PYFOF_CHECK_LAUNCH();
  return kOk;
}

template int32_t pm_convolve_batch<float>(float *, float2 *, const float *, int, int, int, cudaStream_t);
template int32_t pm_convolve_batch<double>(double *, double2 *, const double *, int, int, int, cudaStream_t);
template int32_t c2r_full<float>(const float *, float2 *, float *, int, cudaStream_t);
template int32_t c2r_full<double>(const double *, double2 *, double *, int, cudaStream_t);

}  // namespace pyfof
