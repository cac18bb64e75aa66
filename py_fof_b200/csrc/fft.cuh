// Batched 3-D real<->complex FFTs of zero-padded cubic grids, for the
// isolated particle-mesh convolution (replaces FFTW3f at
// bound_fortran.f90:2166-2169, :2675-2677, :894-906).
//
// Grids: n points per axis, n = 2^a 3^b <= 256 (48, 64, 128, 216, 256).
// The real grid keeps only its support cube [0,sup)^3 (sup <= n/2+1, the
// zero-padded half of the isolated convolution), compact:
//     rho[((b*sup + z)*sup + y)*sup + x]
// The spectrum is the r2c half spectrum, x halved:
//     spec[((b*n + kz)*n + ky)*(n/2+1) + kx]
// All passes are Stockham autosort radix-4/2/3 transforms of whole lines in
// shared memory; zero blocks of the padded grid are neither read nor
// transformed.  The inverse follows FFTW's c2r definition (complex inverse
// transforms along z and y, then a Hermitian c2r along x that uses only the
// real parts of the DC and Nyquist bins) and is unnormalised.
#pragma once

#include <type_traits>

#include "common.cuh"

namespace pyfof {

template <typename R>
using cplx_t = typename std::conditional<std::is_same<R, float>::value, float2, double2>::type;

template <typename R>
struct FftPlanDev {
  int n, nh, nf;
  int f[12];  // radices
};

// Runs out = G * FFT(rho) and rho <- iFFT(out) / n^3 over a batch:
//   rho   batch of compact support cubes (input: density, output: potential
//         divided by n^3 in R precision, as the reference's rho/real(n**3))
//   spec  batch of half spectra (scratch)
//   green half-spectrum table of real values (same layout, one copy)
template <typename R>
int32_t pm_convolve_batch(R *rho, cplx_t<R> *spec, const R *green, int n, int sup, int batch,
                          cudaStream_t s);

// FFTW-style c2r of a real half-spectrum table (the Green's function) into a
// full n^3 real grid (unnormalised); used once per table to extract the
// self-potential kernel.
template <typename R>
int32_t c2r_full(const R *green, cplx_t<R> *spec, R *out, int n, cudaStream_t s);

}  // namespace pyfof
