/* CPU oracle FFT helper -- TEST INFRASTRUCTURE ONLY (see oracle.h). */
#ifndef PYFOF_ORACLE_FFT_H
#define PYFOF_ORACLE_FFT_H
#include <complex.h>

void offt_1d(double complex *x, double complex *work, int n, int sign);
void offt_r2c_3d(const double *rho, double complex *spec, int n, int sup);
void offt_c2r_3d(double complex *spec, double *rho, int n, int out);

#endif
