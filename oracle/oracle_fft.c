/*
 * CPU oracle FFT helper -- TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * The reference calls FFTW3f (single precision r2c/c2r, FFTW_ESTIMATE) at
 * bound_fortran.f90:2166-2169,2373,2675-2677,894-906.  FFTW is not part of
 * the reference tree, so this oracle uses its own FP64 mixed-radix (2,3,4)
 * Stockham FFT.  The c2r direction reproduces FFTW's definition of the
 * multi-dimensional complex-to-real transform: complex inverse DFTs along the
 * two full axes, then a 1-D Hermitian c2r along the halved (first Fortran)
 * axis that reads only the real parts of the DC and Nyquist bins.
 */
#include <complex.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_fft.h"

typedef double complex cplx;

typedef struct {
    int n, nf, f[32];
    cplx *tw[32];  /* stage s: w_{l r}^{j q}, index j*r+q, forward sign */
} fft_plan;

#define MAX_PLANS 16
static fft_plan g_plans[MAX_PLANS];
static int g_nplans = 0;
static pthread_mutex_t g_plan_lock = PTHREAD_MUTEX_INITIALIZER;

static const fft_plan *get_plan(int n)
{
    pthread_mutex_lock(&g_plan_lock);
    for (int i = 0; i < g_nplans; ++i)
        if (g_plans[i].n == n) { pthread_mutex_unlock(&g_plan_lock); return &g_plans[i]; }
    fft_plan *p = &g_plans[g_nplans];
    memset(p, 0, sizeof(*p));
    p->n = n;
    int m = n;
    while (m % 4 == 0) { p->f[p->nf++] = 4; m /= 4; }
    while (m % 2 == 0) { p->f[p->nf++] = 2; m /= 2; }
    while (m % 3 == 0) { p->f[p->nf++] = 3; m /= 3; }
    if (m != 1) { pthread_mutex_unlock(&g_plan_lock); return NULL; }
    int mm = 1;
    for (int s = 0; s < p->nf; ++s) {
        int r = p->f[s], l = n / (mm * r);
        p->tw[s] = (cplx *)malloc(sizeof(cplx) * (size_t)l * r);
        for (int j = 0; j < l; ++j)
            for (int q = 0; q < r; ++q) {
                double ang = -2.0 * M_PI * (double)(j * q) / (double)(l * r);
                p->tw[s][j * r + q] = cos(ang) + I * sin(ang);
            }
        mm *= r;
    }
    ++g_nplans;
    pthread_mutex_unlock(&g_plan_lock);
    return p;
}

/* In-place complex DFT of length n, sign -1 (forward) or +1 (inverse),
 * unnormalised.  work must hold n values. */
void offt_1d(double complex *x, double complex *work, int n, int sign)
{
    const fft_plan *p = get_plan(n);
    if (!p) return;
    cplx *a = x, *b = work;
    int m = 1;
    const double s3 = sqrt(3.0) * 0.5;
    for (int s = 0; s < p->nf; ++s) {
        int r = p->f[s], l = n / (m * r);
        const cplx *tw = p->tw[s];
        for (int j = 0; j < l; ++j) {
            cplx w[4];
            for (int u = 0; u < r; ++u) w[u] = sign < 0 ? tw[j * r + u] : conj(tw[j * r + u]);
            for (int k = 0; k < m; ++k) {
                cplx v[4], o[4];
                for (int q = 0; q < r; ++q) v[q] = a[(q * l + j) * m + k];
                if (r == 2) {
                    o[0] = v[0] + v[1];
                    o[1] = v[0] - v[1];
                } else if (r == 4) {
                    cplx t0 = v[0] + v[2], t1 = v[0] - v[2], t2 = v[1] + v[3];
                    cplx t3 = (v[1] - v[3]) * (sign < 0 ? -I : I);
                    o[0] = t0 + t2;
                    o[1] = t1 + t3;
                    o[2] = t0 - t2;
                    o[3] = t1 - t3;
                } else { /* r == 3 */
                    cplx t1 = v[1] + v[2];
                    cplx t2 = v[0] - 0.5 * t1;
                    cplx t3 = (sign < 0 ? -I : I) * s3 * (v[1] - v[2]);
                    o[0] = v[0] + t1;
                    o[1] = t2 + t3;
                    o[2] = t2 - t3;
                }
                /* Stockham decimation in frequency: twiddle after the butterfly */
                for (int u = 0; u < r; ++u) b[(j * r + u) * m + k] = o[u] * w[u];
            }
        }
        m *= r;
        cplx *t = a; a = b; b = t;
    }
    if (a != x) memcpy(x, a, sizeof(cplx) * (size_t)n);
}

/* Forward r2c of a real (n,n,n) grid (x fastest) whose support lies in
 * [0,sup)^3, producing the half spectrum spec[(kz*n+ky)*(n/2+1)+kx]. */
void offt_r2c_3d(const double *rho, double complex *spec, int n, int sup)
{
    const int nh = n / 2 + 1;
    memset(spec, 0, sizeof(cplx) * (size_t)nh * n * n);
#pragma omp parallel
    {
        cplx *line = (cplx *)malloc(sizeof(cplx) * (size_t)n);
        cplx *work = (cplx *)malloc(sizeof(cplx) * (size_t)n);
#pragma omp for collapse(2)
        for (int z = 0; z < sup; ++z)
            for (int y = 0; y < sup; ++y) {
                for (int x = 0; x < n; ++x) line[x] = rho[((size_t)z * n + y) * n + x];
                offt_1d(line, work, n, -1);
                for (int kx = 0; kx < nh; ++kx) spec[((size_t)z * n + y) * nh + kx] = line[kx];
            }
#pragma omp for collapse(2)
        for (int z = 0; z < sup; ++z)
            for (int kx = 0; kx < nh; ++kx) {
                for (int y = 0; y < n; ++y) line[y] = spec[((size_t)z * n + y) * nh + kx];
                offt_1d(line, work, n, -1);
                for (int y = 0; y < n; ++y) spec[((size_t)z * n + y) * nh + kx] = line[y];
            }
#pragma omp for collapse(2)
        for (int y = 0; y < n; ++y)
            for (int kx = 0; kx < nh; ++kx) {
                for (int z = 0; z < n; ++z) line[z] = spec[((size_t)z * n + y) * nh + kx];
                offt_1d(line, work, n, -1);
                for (int z = 0; z < n; ++z) spec[((size_t)z * n + y) * nh + kx] = line[z];
            }
        free(line);
        free(work);
    }
}

/* Unnormalised c2r with FFTW semantics; only outputs in [0,out)^3 are
 * produced (rho[(z*n+y)*n+x]).  spec is overwritten. */
void offt_c2r_3d(double complex *spec, double *rho, int n, int out)
{
    const int nh = n / 2 + 1;
#pragma omp parallel
    {
        cplx *line = (cplx *)malloc(sizeof(cplx) * (size_t)n);
        cplx *work = (cplx *)malloc(sizeof(cplx) * (size_t)n);
#pragma omp for collapse(2)
        for (int y = 0; y < n; ++y)
            for (int kx = 0; kx < nh; ++kx) {
                for (int z = 0; z < n; ++z) line[z] = spec[((size_t)z * n + y) * nh + kx];
                offt_1d(line, work, n, +1);
                for (int z = 0; z < out; ++z) spec[((size_t)z * n + y) * nh + kx] = line[z];
            }
#pragma omp for collapse(2)
        for (int z = 0; z < out; ++z)
            for (int kx = 0; kx < nh; ++kx) {
                for (int y = 0; y < n; ++y) line[y] = spec[((size_t)z * n + y) * nh + kx];
                offt_1d(line, work, n, +1);
                for (int y = 0; y < out; ++y) spec[((size_t)z * n + y) * nh + kx] = line[y];
            }
#pragma omp for collapse(2)
        for (int z = 0; z < out; ++z)
            for (int y = 0; y < out; ++y) {
                const cplx *c = spec + ((size_t)z * n + y) * nh;
                line[0] = creal(c[0]);
                for (int kx = 1; kx < n / 2; ++kx) { line[kx] = c[kx]; line[n - kx] = conj(c[kx]); }
                line[n / 2] = creal(c[n / 2]);
                offt_1d(line, work, n, +1);
                for (int x = 0; x < out; ++x) rho[((size_t)z * n + y) * n + x] = creal(line[x]);
            }
        free(line);
        free(work);
    }
}
