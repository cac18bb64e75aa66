// Batched 3-D real<->complex FFTs of zero-padded cubic grids, for the
// isolated particle-mesh convolution (replaces FFTW3f at
// bound_fortran.f90:2166-2169, :2675-2677, :894-906).
//
// Grids: n points per axis, n = 2^a 3^b <= 256 (48, 64, 128, 216, 256).
// The real grid keeps only its support cube [0,sup)^3 (sup <= n/2+1, the
// zero-padded half of the isolated convolution), compact:
//     rho[((b*sup + z)*sup + y)*sup + x]
// The spectrum is the r2c half spectrum, x halved, rows padded to a whole
// number of 128-byte line tiles (spec_row):
//     spec[((b*n + kz)*n + ky)*spec_row(n) + kx],  kx < n/2+1
// Line transforms are register-resident mixed-radix DFTs (fft.cu); zero
// blocks of the padded grid are neither read nor transformed.  The inverse follows FFTW's c2r definition (complex inverse
// transforms along z and y, then a Hermitian c2r along x that uses only the
// real parts of the DC and Nyquist bins) and is unnormalised.
#pragma once

#include <type_traits>

#include "common.cuh"

namespace pyfof {

template <typename R>
using cplx_t = typename std::conditional<std::is_same<R, float>::value, float2, double2>::type;

// Row length (complex elements) of the half spectrum of an n-point axis.
template <typename R>
constexpr int64_t spec_row(int n) {
  return (int64_t)((n / 2 + 1 + (sizeof(R) == 4 ? 15 : 7)) / (sizeof(R) == 4 ? 16 : 8)) *
         (sizeof(R) == 4 ? 16 : 8);
}

// Complex elements of one half spectrum of an n^3 grid.
template <typename R>
constexpr int64_t spec_elems(int n) {
  return spec_row<R>(n) * n * n;
}

// Runs out = G * FFT(rho) and rho <- iFFT(out) / n^3 over a batch:
//   rho   batch of compact support cubes (input: density, output: potential
//         divided by n^3 in R precision, as the reference's rho/real(n**3))
//   spec  batch of half spectra (scratch)
//   green half-spectrum table of real values, unpadded rows:
//         green[((kz*n + ky)*(n/2+1) + kx]
//   acc, inv_scale (optional): the density as 64-bit fixed-point cubes
//         (value of grid b = acc * inv_scale[b]) read in place of rho; the
//         output still goes to rho, which may alias acc
//   waves the fused z pass splits the batch so that its grid covers at
//         least this many full waves of the GPU (a launch shape only)
template <typename R>
int32_t pm_convolve_batch(R *rho, cplx_t<R> *spec, const R *green, int n, int sup, int batch,
                          cudaStream_t s, const unsigned long long *acc = nullptr,
                          const double *inv_scale = nullptr, int waves = 4);

// FFTW-style c2r of a real half-spectrum table (the Green's function) into a
// full n^3 real grid (unnormalised); used once per table to extract the
// self-potential kernel.
template <typename R>
int32_t c2r_full(const R *green, cplx_t<R> *spec, R *out, int n, cudaStream_t s);

}  // namespace pyfof
