/*
 * CPU oracle, gravitational-unbinding part -- TEST INFRASTRUCTURE ONLY
 * (see oracle.h).
 *
 * Restates bound_fortran.f90: context and grid tables (:291-330, :1854-2040),
 * candidate classification (:2901-3073), Green's function and self kernel
 * (:2300-2382, :3563-3583), the per-halo solver bound_check_grid
 * (:2436-2888) with the FP64 direct sum, TSC particle-mesh C1 term, C2
 * short-range residual (:3125-3223, :3403-3552), two-level inner PM/PP
 * (:531-942, :944-1498) and the removal loop.  The FFT is this oracle's own
 * FP64 transform (oracle_fft.c) instead of FFTW3f, so PM results agree with
 * the reference to FFT rounding only ("parity unpinned" for PM).  The
 * multi-threaded team variants of C2/PP (used by the reference only for
 * 256-grid halos with >= 20000 members and 2-thread teams) are replaced by
 * their serial counterparts, which give the same sums in a fixed order.
 */
#include <complex.h>
#include <math.h>
#include <omp.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "oracle_fft.h"

#define PI 3.141592653589793238462643383279502884197
#define MAX_PASSES 20
#define H_SPLIT 3.5
#define TL_N12 3926
#define TL_N24 14688
#define TL_NR2 128
#define TL_NR4 216

/* ---------------------------------------------------------------- context */

typedef struct {
    int64_t ng;
    int ngrid, bn[4], n_max, m_max;
    double s15, spacing_max, app, a, b;
    int np_min, verbose;
    int fgl_nlev[4];
    double fgl_sp[4][32], fgl_cov[4][32];
    int ntotal, tab_gid[64], tab_lev[64];
    double tab_sp[64], tab_cov[64];
} bctx;

static const int k_cand_n[4] = {48, 64, 128, 256};

/* bound_grid_levels (bound_fortran.f90:1854-1876); gid is 1-based */
static int grid_levels(const bctx *c, int gid, double *sp_out, int cap)
{
    int nlev = 0;
    if (gid < 1 || gid > c->ngrid) return 0;
    int m = c->bn[gid - 1] / 2 - 3;
    double sp = 1.0 / 32.0;
    while ((double)m * sp < c->s15 && nlev < cap) { sp_out[nlev++] = sp; sp = 2.0 * sp; }
    if (gid == c->ngrid && nlev < cap) sp_out[nlev++] = c->spacing_max;
    return nlev;
}

static void ctx_init(bctx *c, double app, double a, double b, double s15, int np_min,
                     int verbose, int64_t ng_in, double ng_global_in)
{
    memset(c, 0, sizeof(*c));
    c->ng = ng_in > 0 ? ng_in : 256;
    (void)ng_global_in;
    int ngi = (int)c->ng;
    c->ngrid = 1 + (ngi >= 64) + (ngi >= 128) + (ngi >= 256);
    for (int g = 0; g < 4; ++g) c->bn[g] = k_cand_n[g] < ngi ? k_cand_n[g] : ngi;
    c->n_max = ngi < 256 ? ngi : 256;
    c->m_max = c->n_max / 2 - 3;
    c->app = app; c->a = a; c->b = b; c->s15 = s15;
    c->spacing_max = s15 / (double)c->m_max;
    c->np_min = np_min; c->verbose = verbose;
    for (int g = 1; g <= c->ngrid; ++g) {
        double sp[32];
        int nl = grid_levels(c, g, sp, 32);
        c->fgl_nlev[g - 1] = nl;
        for (int l = 0; l < nl; ++l) {
            c->fgl_sp[g - 1][l] = sp[l];
            c->fgl_cov[g - 1][l] = (double)(c->bn[g - 1] / 2 - 3) * sp[l];
        }
    }
    /* bound_build_ladder (:1882-1916): selection sort by coverage */
    int nt = 0, tg[64], tl[64];
    double ts[64], tc[64];
    for (int g = 1; g <= c->ngrid; ++g)
        for (int l = 0; l < c->fgl_nlev[g - 1]; ++l) {
            tg[nt] = g; tl[nt] = l; ts[nt] = c->fgl_sp[g - 1][l]; tc[nt] = c->fgl_cov[g - 1][l];
            ++nt;
        }
    for (int j = 0; j < nt - 1; ++j) {
        int k = j;
        for (int i = j + 1; i < nt; ++i) if (tc[i] < tc[k]) k = i;
        if (k != j) {
            int it; double t;
            it = tg[j]; tg[j] = tg[k]; tg[k] = it;
            it = tl[j]; tl[j] = tl[k]; tl[k] = it;
            t = tc[j]; tc[j] = tc[k]; tc[k] = t;
            t = ts[j]; ts[j] = ts[k]; ts[k] = t;
        }
    }
    c->ntotal = nt;
    for (int i = 0; i < nt; ++i) {
        c->tab_gid[i] = tg[i]; c->tab_lev[i] = tl[i]; c->tab_sp[i] = ts[i]; c->tab_cov[i] = tc[i];
    }
}

/* bound_fgl_init candidate sequences (bound_fortran.f90:1936-1952);
 * spacing -1 stands for spacing_max */
static const int k_band_n[3] = {11, 10, 8};
static const int k_band_gid[3][11] = {{1, 2, 2, 3, 3, 3, 4, 4, 4, 4, 4},
                                      {3, 3, 4, 4, 4, 4, 4, 4, 4, 4, 0},
                                      {4, 4, 4, 4, 4, 4, 4, 4, 0, 0, 0}};
static const double k_band_sp[3][11] = {
    {0.125, 0.125, 0.25, 0.125, 0.25, 0.5, 0.0625, 0.125, 0.25, 0.5, -1.0},
    {0.0625, 0.125, 0.0625, 0.125, 0.25, 0.5, 1.0, 2.0, 4.0, -1.0, 0},
    {0.0625, 0.125, 0.25, 0.5, 1.0, 2.0, 4.0, -1.0, 0, 0, 0}};

/* bound_select_grid_and_level (:1963-2019).  Returns 0 ok, 2 no combination. */
static int select_grid(const bctx *c, int64_t np, double span, int *gid, int *lev, double *sp_out)
{
    *gid = 0; *lev = -1; *sp_out = 0.0;
    if (np <= 1000) return 0;
    int band = np <= 5000 ? 0 : (np <= 20000 ? 1 : 2);
    for (int s = 0; s < k_band_n[band]; ++s) {
        int g = k_band_gid[band][s];
        if (g < 1 || g > c->ngrid) continue;
        double sp = k_band_sp[band][s];
        if (sp == -1.0) sp = c->spacing_max;
        int l = -1;
        for (int q = 0; q < c->fgl_nlev[g - 1]; ++q)
            if (fabs(c->fgl_sp[g - 1][q] - sp) <= 1e-12 * (fabs(sp) > 1.0 ? fabs(sp) : 1.0)) { l = q; break; }
        if (l < 0) continue;
        if (c->fgl_cov[g - 1][l] < span) continue;
        *gid = g; *lev = l; *sp_out = c->fgl_sp[g - 1][l];
        return 0;
    }
    if (span <= c->s15) {
        for (int i = 0; i < c->ntotal; ++i)
            if (c->tab_cov[i] >= span) {
                int g = c->tab_gid[i], l = c->tab_lev[i];
                if (g >= 1 && g <= c->ngrid) {
                    *gid = g; *lev = l; *sp_out = c->fgl_sp[g - 1][l];
                    return 0;
                }
                break;
            }
    }
    return 2;
}

/* ------------------------------------------------------- kernels (:3080) */

static double depth_continuous(double r, double h)
{
    if (r <= 0.0) return 208.0 / (70.0 * h);
    if (r >= h) return 1.0 / r;
    double e = 2.0 * r / h;
    if (e <= 1.0) {
        double prim = e * e * (112.0 + e * e * (-56.0 + e * (14.0 + e * (8.0 - 3.0 * e))));
        return (208.0 - prim) / (70.0 * h);
    }
    double prim = e * e * (448.0 + e * (-280.0 + e * (56.0 + e * (14.0 + e * (-8.0 + e))))) -
                  224.0 * e - 12.0 / e;
    return (128.0 - prim) / (70.0 * h);
}

static double c2_delta_depth(double r, double ht, double hs)
{
    if (r <= 0.0) return (208.0 / 70.0) * (1.0 / ht - 1.0 / hs);
    if (r >= ht && r >= hs) return 0.0;
    return depth_continuous(r, ht) - depth_continuous(r, hs);
}

/* --------------------------------------------------- Green + self kernel */

static double wave_number(int idx0, int n) /* idx0 = 0-based array index */
{
    int mode = ((idx0 + n / 2) % n) - n / 2;
    return 2.0 * PI * (double)mode / (double)n;
}

static double window_sq(const double *k)
{
    double s = 1.0;
    for (int d = 0; d < 3; ++d) {
        double x = 0.5 * k[d];
        if (x != 0.0) s = s * sin(x) / x;
    }
    double s2 = s * s, s3 = s2 * s;
    return s3 * s3; /* real**6 as gfortran expands it: (x^2*x)^2 */
}

int32_t oracle_green_and_self(int32_t n, double apm_soft, double apm_range, int32_t truncated,
                              float *green, float *self_out)
{
    const int nh = n / 2 + 1;
    const double radius = 0.5 * (double)n;
    int bad = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(| : bad)
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < nh; ++i) {
                double kv[3] = {wave_number(i, n), wave_number(j, n), wave_number(k, n)};
                double asum = 0.0, bsum = 0.0;
                for (int ka = -2; ka <= 2; ++ka)
                    for (int ja = -2; ja <= 2; ++ja)
                        for (int ia = -2; ia <= 2; ++ia) {
                            double kal[3] = {kv[0] + 2.0 * PI * (double)ia, kv[1] + 2.0 * PI * (double)ja,
                                             kv[2] + 2.0 * PI * (double)ka};
                            double kmag = sqrt(kal[0] * kal[0] + kal[1] * kal[1] + kal[2] * kal[2]);
                            double uk2 = window_sq(kal);
                            asum += uk2;
                            double target;
                            if (kmag == 0.0) {
                                if (apm_range == 0.0) target = -4.0 * PI * radius * radius / 6.0;
                                else if (truncated) target = 0.0;
                                else target = -2.0 * PI * (apm_range * apm_range - apm_soft * apm_soft) / 15.0;
                            } else {
                                double y = apm_soft * kmag / 2.0;
                                double y2 = y * y, y4 = y2 * y2;
                                double ssoft = 12.0 * (1.0 / y4) * (2.0 - 2.0 * cos(y) - y * sin(y));
                                double srange = 0.0;
                                if (apm_range != 0.0) {
                                    y = apm_range * kmag / 2.0;
                                    y2 = y * y; y4 = y2 * y2;
                                    srange = 12.0 * (1.0 / y4) * (2.0 - 2.0 * cos(y) - y * sin(y));
                                }
                                double cut = 1.0;
                                if (truncated) { double kr = kmag * radius; cut = 1.0 - sin(kr) / kr; }
                                target = -4.0 * PI * (ssoft * ssoft - srange * srange) * cut / (kmag * kmag);
                            }
                            bsum += uk2 * target;
                        }
                if (asum <= 2.2250738585072014e-308) { bad = 1; continue; }
                green[((size_t)k * n + j) * nh + i] = (float)(bsum / (asum * asum));
            }
    if (bad) return 1;
    /* self kernel: FFTW-style c2r of the real table evaluated at offsets
     * -2..2 (mod n), divided by n^3 in FP32 */
    double complex *ph = (double complex *)malloc(sizeof(double complex) * (size_t)n * 5);
    for (int t = 0; t < n; ++t)
        for (int o = 0; o < 5; ++o) {
            int x = ((o - 2) % n + n) % n;
            double ang = 2.0 * PI * (double)(((int64_t)t * x) % n) / (double)n;
            ph[t * 5 + o] = cos(ang) + I * sin(ang);
        }
    /* A[i][j][oz] = sum_k G(i,j,k) e^{+2 pi i k z / n} */
    double complex *A = (double complex *)calloc((size_t)nh * n * 5, sizeof(double complex));
#pragma omp parallel for
    for (int j = 0; j < n; ++j)
        for (int k = 0; k < n; ++k)
            for (int i = 0; i < nh; ++i) {
                double g = green[((size_t)k * n + j) * nh + i];
                for (int oz = 0; oz < 5; ++oz) A[((size_t)i * n + j) * 5 + oz] += g * ph[k * 5 + oz];
            }
    for (int oz = 0; oz < 5; ++oz)
        for (int oy = 0; oy < 5; ++oy) {
            double complex C[nh];
            for (int i = 0; i < nh; ++i) {
                double complex s = 0;
                for (int j = 0; j < n; ++j) s += A[((size_t)i * n + j) * 5 + oz] * ph[j * 5 + oy];
                C[i] = s;
            }
            for (int ox = 0; ox < 5; ++ox) {
                int x = ((ox - 2) % n + n) % n;
                double f = creal(C[0]) + creal(C[n / 2]) * ((x & 1) ? -1.0 : 1.0);
                for (int i = 1; i < n / 2; ++i) f += 2.0 * creal(C[i] * ph[i * 5 + ox]);
                self_out[(oz * 5 + oy) * 5 + ox] = (float)f / (float)((double)n * n * n);
            }
        }
    free(A);
    free(ph);
    return 0;
}

typedef struct {
    int n;
    double soft, range;
    int trunc;
    float *green;
    float self[125];
} green_entry;

static green_entry g_green[8];
static int g_ngreen = 0;
static pthread_mutex_t g_green_lock = PTHREAD_MUTEX_INITIALIZER;

static const green_entry *get_green(int n, double soft, double range, int trunc)
{
    pthread_mutex_lock(&g_green_lock);
    for (int i = 0; i < g_ngreen; ++i)
        if (g_green[i].n == n && g_green[i].soft == soft && g_green[i].range == range &&
            g_green[i].trunc == trunc) {
            pthread_mutex_unlock(&g_green_lock);
            return &g_green[i];
        }
    green_entry *e = &g_green[g_ngreen];
    e->n = n; e->soft = soft; e->range = range; e->trunc = trunc;
    e->green = (float *)malloc(sizeof(float) * (size_t)(n / 2 + 1) * n * n);
    if (!e->green || oracle_green_and_self(n, soft, range, trunc, e->green, e->self)) {
        free(e->green);
        pthread_mutex_unlock(&g_green_lock);
        return NULL;
    }
    ++g_ngreen;
    pthread_mutex_unlock(&g_green_lock);
    return e;
}

/* Convolve a real (n,n,n) FP32 grid with a Green table the way the reference
 * does: r2c, multiply, c2r, divide by n^3 in FP32.  Source/target support is
 * [0, sup). */
static void pm_convolve(float *rho, const float *green, int n, int sup)
{
    const int nh = n / 2 + 1;
    double *r = (double *)malloc(sizeof(double) * (size_t)n * n * n);
    double complex *spec = (double complex *)malloc(sizeof(double complex) * (size_t)nh * n * n);
    for (size_t i = 0; i < (size_t)n * n * n; ++i) r[i] = rho[i];
    offt_r2c_3d(r, spec, n, sup);
    for (size_t i = 0; i < (size_t)nh * n * n; ++i) {
        /* FFTW-float spectrum times complex(G,0) */
        float re = (float)creal(spec[i]), im = (float)cimag(spec[i]);
        spec[i] = (double)(re * green[i]) + I * (double)(im * green[i]);
    }
    offt_c2r_3d(spec, r, n, sup);
    const float n3 = (float)((double)n * n * n);
    for (int z = 0; z < sup; ++z)
        for (int y = 0; y < sup; ++y)
            for (int x = 0; x < sup; ++x) {
                size_t idx = ((size_t)z * n + y) * n + x;
                rho[idx] = (float)r[idx] / n3;
            }
    free(r);
    free(spec);
}

/* ---------------------------------------------------------- TSC helpers */

static inline int fnint(float x) { return (int)lroundf(x); } /* Fortran NINT */

static void tsc_weights(float t, int *first, float *w)
{
    int nearest = fnint(t);
    float d = t - (float)nearest;
    *first = nearest;
    float a = 0.5f - d, b = 0.5f + d;
    w[0] = 0.5f * (a * a);
    w[1] = 0.75f - d * d;
    w[2] = 0.5f * (b * b);
}

static float tsc_self(const float *wt /*[3][3] axis-major*/, const float *self_phi)
{
    double acc = 0.0;
    for (int sz = 0; sz < 3; ++sz)
        for (int sy = 0; sy < 3; ++sy)
            for (int sx = 0; sx < 3; ++sx) {
                float sw = wt[0 * 3 + sx] * wt[1 * 3 + sy] * wt[2 * 3 + sz];
                for (int tz = 0; tz < 3; ++tz)
                    for (int ty = 0; ty < 3; ++ty)
                        for (int tx = 0; tx < 3; ++tx) {
                            float tw = wt[0 * 3 + tx] * wt[1 * 3 + ty] * wt[2 * 3 + tz];
                            int o = ((tz - sz + 2) * 5 + (ty - sy + 2)) * 5 + (tx - sx + 2);
                            acc = acc + (double)(sw * tw) * (double)self_phi[o];
                        }
            }
    return (float)acc;
}

/* ------------------------------------------------------ C2 cell lists */

typedef struct {
    int nc[3];
    double u_min[3];
    int32_t *cell_id, *cell_start, *cell_part;
} c2cells;

/* bound_build_cells (:3125-3223); 0-based cells */
static void build_cells(c2cells *cc, const float *q, int np, float spacing, double cw)
{
    double umin[3] = {1e30, 1e30, 1e30}, umax[3] = {-1e30, -1e30, -1e30};
    for (int i = 0; i < np; ++i)
        for (int d = 0; d < 3; ++d) {
            double u = (double)q[3 * i + d] / (double)spacing;
            if (u < umin[d]) umin[d] = u;
            if (u > umax[d]) umax[d] = u;
        }
    for (int d = 0; d < 3; ++d) {
        int v = (int)floor((umax[d] - umin[d]) / cw) + 1;
        cc->nc[d] = v > 1 ? v : 1;
        cc->u_min[d] = umin[d];
    }
    int nt = cc->nc[0] * cc->nc[1] * cc->nc[2];
    cc->cell_id = (int32_t *)malloc(sizeof(int32_t) * (size_t)(np > 0 ? np : 1));
    cc->cell_part = (int32_t *)malloc(sizeof(int32_t) * (size_t)(np > 0 ? np : 1));
    cc->cell_start = (int32_t *)calloc((size_t)nt + 1, sizeof(int32_t));
    for (int i = 0; i < np; ++i) {
        int ic[3];
        for (int d = 0; d < 3; ++d) {
            double u = (double)q[3 * i + d] / (double)spacing;
            int v = (int)floor((u - umin[d]) / cw) + 1;
            if (v < 1) v = 1;
            if (v > cc->nc[d]) v = cc->nc[d];
            ic[d] = v - 1;
        }
        int c = ic[0] + ic[1] * cc->nc[0] + ic[2] * cc->nc[0] * cc->nc[1];
        cc->cell_id[i] = c;
        cc->cell_start[c + 1]++;
    }
    for (int c = 0; c < nt; ++c) cc->cell_start[c + 1] += cc->cell_start[c];
    int *cur = (int *)malloc(sizeof(int) * (size_t)(nt > 0 ? nt : 1));
    memcpy(cur, cc->cell_start, sizeof(int) * (size_t)nt);
    for (int i = 0; i < np; ++i) cc->cell_part[cur[cc->cell_id[i]]++] = i;
    free(cur);
}

static void free_cells(c2cells *cc)
{
    free(cc->cell_id); free(cc->cell_start); free(cc->cell_part);
    memset(cc, 0, sizeof(*cc));
}

/* bound_c2_stencil (:154-159): the 13 offsets that follow (0,0,0) */
static const int k_c2_sten[13][3] = {{-1, -1, 1}, {0, -1, 1}, {1, -1, 1}, {-1, 0, 1}, {0, 0, 1},
                                     {1, 0, 1},   {-1, 1, 1}, {0, 1, 1},  {1, 1, 1},  {-1, 1, 0},
                                     {0, 1, 0},   {1, 1, 0},  {1, 0, 0}};

static inline void c2_pair(const float *q, const float *w, int i1, int i2, double r2cut,
                           double spacing, double ht, float pref, float *phi)
{
    double dx = (double)(q[3 * i2 + 0] - q[3 * i1 + 0]);
    double dy = (double)(q[3 * i2 + 1] - q[3 * i1 + 1]);
    double dz = (double)(q[3 * i2 + 2] - q[3 * i1 + 2]);
    double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 < r2cut) {
        double r = sqrt(r2) / spacing;
        float dphi = -pref * (float)c2_delta_depth(r, ht, H_SPLIT);
        phi[i1] = phi[i1] + w[i2] * dphi;
        phi[i2] = phi[i2] + w[i1] * dphi;
    }
}

/* bound_c2_calc_cells (:3403-3483) */
static void c2_full(const c2cells *cc, const float *q, const float *w, const char *keep, int np,
                    float spacing, float app_f, double a, float *phi)
{
    for (int i = 0; i < np; ++i) phi[i] = 0.0f;
    int nk = 0;
    for (int i = 0; i < np; ++i) nk += keep[i];
    if (nk <= 1 || spacing <= 0.0f) return;
    double ht = (double)app_f / (double)spacing;
    double r2cut = 12.25 * (double)spacing * (double)spacing;
    float pref = (float)(a / (6.0 * PI * (double)spacing));
    const int *nc = cc->nc;
    for (int cz = 0; cz < nc[2]; ++cz)
        for (int cy = 0; cy < nc[1]; ++cy)
            for (int cx = 0; cx < nc[0]; ++cx) {
                int c1 = cx + cy * nc[0] + cz * nc[0] * nc[1];
                for (int p1 = cc->cell_start[c1]; p1 < cc->cell_start[c1 + 1]; ++p1) {
                    int i1 = cc->cell_part[p1];
                    if (!keep[i1]) continue;
                    for (int p2 = p1 + 1; p2 < cc->cell_start[c1 + 1]; ++p2) {
                        int i2 = cc->cell_part[p2];
                        if (!keep[i2]) continue;
                        c2_pair(q, w, i1, i2, r2cut, spacing, ht, pref, phi);
                    }
                    for (int s = 0; s < 13; ++s) {
                        int nx = cx + k_c2_sten[s][0], ny = cy + k_c2_sten[s][1], nz = cz + k_c2_sten[s][2];
                        if (nx < 0 || nx >= nc[0] || ny < 0 || ny >= nc[1] || nz < 0 || nz >= nc[2]) continue;
                        int c2 = nx + ny * nc[0] + nz * nc[0] * nc[1];
                        for (int p2 = cc->cell_start[c2]; p2 < cc->cell_start[c2 + 1]; ++p2) {
                            int i2 = cc->cell_part[p2];
                            if (!keep[i2]) continue;
                            c2_pair(q, w, i1, i2, r2cut, spacing, ht, pref, phi);
                        }
                    }
                }
            }
}

/* bound_c2_update_incremental_cells (:3490-3552) */
static void c2_update(const c2cells *cc, const float *q, const float *w, const char *keep,
                      int np, const int *del, int ndel, float spacing, float app_f, double a,
                      float *phi)
{
    int nk = 0;
    for (int i = 0; i < np; ++i) nk += keep[i];
    if (ndel <= 0 || nk <= 0 || spacing <= 0.0f) return;
    double ht = (double)app_f / (double)spacing;
    double r2cut = 12.25 * (double)spacing * (double)spacing;
    float pref = (float)(a / (6.0 * PI * (double)spacing));
    const int *nc = cc->nc;
    for (int k = 0; k < ndel; ++k) {
        int j = del[k];
        int cj = cc->cell_id[j];
        int cz = cj / (nc[0] * nc[1]), cy = (cj % (nc[0] * nc[1])) / nc[0], cx = cj % nc[0];
        for (int nz = cz - 1; nz <= cz + 1; ++nz) {
            if (nz < 0 || nz >= nc[2]) continue;
            for (int ny = cy - 1; ny <= cy + 1; ++ny) {
                if (ny < 0 || ny >= nc[1]) continue;
                for (int nx = cx - 1; nx <= cx + 1; ++nx) {
                    if (nx < 0 || nx >= nc[0]) continue;
                    int c2 = nx + ny * nc[0] + nz * nc[0] * nc[1];
                    for (int p = cc->cell_start[c2]; p < cc->cell_start[c2 + 1]; ++p) {
                        int i2 = cc->cell_part[p];
                        if (!keep[i2]) continue;
                        double dx = (double)(q[3 * i2 + 0] - q[3 * j + 0]);
                        double dy = (double)(q[3 * i2 + 1] - q[3 * j + 1]);
                        double dz = (double)(q[3 * i2 + 2] - q[3 * j + 2]);
                        double r2 = dx * dx + dy * dy + dz * dz;
                        if (r2 < r2cut) {
                            double r = sqrt(r2) / (double)spacing;
                            float dphi = -pref * (float)c2_delta_depth(r, ht, H_SPLIT);
                            phi[i2] = phi[i2] - w[j] * dphi;
                        }
                    }
                }
            }
        }
    }
}

/* ------------------------------------------------- two-level inner PM/PP */

typedef struct {
    int n_active;
    int active[512], region_r[512];
    int *particle_r, *target_reg, *target_start, *target_part;
    int *source_start, *source_part, *first_src, *first_tgt;
    float *wt_src, *wt_tgt, *self_in;
    /* PP cells */
    int pnc[3], k_search;
    double pu_min[3], pcw;
    int *pcell_id, *pcell_start, *pcell_part;
    double *cell_max_a;
    int ntask, *task_c1, *task_p1, *task_p2;
    double *task_max_a;
} tl_ctx;

static void tl_free(tl_ctx *t)
{
    free(t->particle_r); free(t->target_reg); free(t->target_start); free(t->target_part);
    free(t->source_start); free(t->source_part); free(t->first_src); free(t->first_tgt);
    free(t->wt_src); free(t->wt_tgt); free(t->self_in);
    free(t->pcell_id); free(t->pcell_start); free(t->pcell_part); free(t->cell_max_a);
    free(t->task_c1); free(t->task_p1); free(t->task_p2); free(t->task_max_a);
    memset(t, 0, sizeof(*t));
}

static void region_bounds(int b, float *lo, float *hi)
{
    int bx = b % 8, by = (b / 8) % 8, bz = b / 64;
    int bb[3] = {bx, by, bz};
    for (int d = 0; d < 3; ++d) {
        lo[d] = (float)(bb[d] * 16);
        hi[d] = lo[d] + 16.0f < 127.0f ? lo[d] + 16.0f : 127.0f;
    }
}

static int region_id(const float *t)
{
    int c[3];
    for (int d = 0; d < 3; ++d) {
        int v = (int)floor((double)t[d]) / 16; /* Fortran integer division truncates */
        c[d] = v < 0 ? 0 : (v > 7 ? 7 : v);
    }
    return c[0] + c[1] * 8 + c[2] * 64;
}

/* bound_two_level_build_halo (:614-823).  Returns error code (0 ok). */
static int tl_build(tl_ctx *t, const float *q, int np, float spacing, const float *origin,
                    float app_f, const green_entry *g2, const green_entry *g4)
{
    memset(t, 0, sizeof(*t));
    t->particle_r = (int *)malloc(sizeof(int) * np);
    t->target_reg = (int *)malloc(sizeof(int) * np);
    int cnt[512] = {0};
    float *tt = (float *)malloc(sizeof(float) * 3 * (size_t)np);
    for (int i = 0; i < np; ++i) {
        for (int d = 0; d < 3; ++d)
            tt[3 * i + d] = (float)(((double)q[3 * i + d] - (double)origin[d]) / (double)spacing);
        int b = region_id(tt + 3 * i);
        t->target_reg[i] = b;
        cnt[b]++;
    }
    for (int b = 0; b < 512; ++b) {
        int r = cnt[b] < TL_N12 ? 1 : (cnt[b] < TL_N24 ? 2 : 4);
        if (r == 4 && H_SPLIT * ((double)spacing / 4.0) < (double)app_f) r = 2;
        if (r == 2 && H_SPLIT * ((double)spacing / 2.0) < (double)app_f) r = 1;
        t->region_r[b] = r;
    }
    int any = 0;
    for (int i = 0; i < np; ++i) { t->particle_r[i] = t->region_r[t->target_reg[i]]; any |= t->particle_r[i] != 1; }
    if (!any) { free(tt); return 0; }
    int n_act = 0;
    for (int b = 0; b < 512; ++b)
        if (cnt[b] > 0 && t->region_r[b] > 1) t->active[n_act++] = b;
    t->n_active = n_act;
    if (!n_act) { free(tt); return 0; }
    int need2 = 0, need4 = 0;
    for (int i = 0; i < np; ++i) { need2 |= t->particle_r[i] == 2; need4 |= t->particle_r[i] == 4; }
    if ((need2 && !g2) || (need4 && !g4)) { free(tt); return 1; }
    t->target_start = (int *)calloc(513, sizeof(int));
    t->target_part = (int *)malloc(sizeof(int) * np);
    for (int b = 0; b < 512; ++b) t->target_start[b + 1] = t->target_start[b] + cnt[b];
    int fill[512] = {0};
    for (int i = 0; i < np; ++i) {
        int b = t->target_reg[i];
        t->target_part[t->target_start[b] + fill[b]++] = i;
    }
    int scnt[512] = {0};
    for (int a = 0; a < n_act; ++a) {
        int b = t->active[a], r = t->region_r[b];
        float lo[3], hi[3];
        region_bounds(b, lo, hi);
        float bo = 3.5f + 3.0f / (float)r;
        for (int j = 0; j < np; ++j) {
            const float *p = tt + 3 * j;
            if (p[0] >= lo[0] - bo && p[0] <= hi[0] + bo && p[1] >= lo[1] - bo && p[1] <= hi[1] + bo &&
                p[2] >= lo[2] - bo && p[2] <= hi[2] + bo)
                scnt[b]++;
        }
    }
    t->source_start = (int *)calloc(513, sizeof(int));
    for (int b = 0; b < 512; ++b) t->source_start[b + 1] = t->source_start[b] + scnt[b];
    int tot = t->source_start[512];
    t->source_part = (int *)malloc(sizeof(int) * (size_t)(tot > 0 ? tot : 1));
    t->first_src = (int *)malloc(sizeof(int) * 3 * (size_t)(tot > 0 ? tot : 1));
    t->wt_src = (float *)malloc(sizeof(float) * 9 * (size_t)(tot > 0 ? tot : 1));
    memset(scnt, 0, sizeof(scnt));
    for (int a = 0; a < n_act; ++a) {
        int b = t->active[a], r = t->region_r[b];
        int nin = r == 2 ? TL_NR2 : TL_NR4;
        float lo[3], hi[3];
        region_bounds(b, lo, hi);
        float bo = 3.5f + 3.0f / (float)r;
        float u0[3];
        for (int d = 0; d < 3; ++d) u0[d] = lo[d] - bo - (1.0f / (float)r) + (0.0f / (float)r);
        for (int j = 0; j < np; ++j) {
            const float *p = tt + 3 * j;
            if (!(p[0] >= lo[0] - bo && p[0] <= hi[0] + bo && p[1] >= lo[1] - bo && p[1] <= hi[1] + bo &&
                  p[2] >= lo[2] - bo && p[2] <= hi[2] + bo))
                continue;
            int s = t->source_start[b] + scnt[b];
            t->source_part[s] = j;
            for (int d = 0; d < 3; ++d) {
                float tf = (p[d] - u0[d]) * (float)r;
                int f;
                tsc_weights(tf, &f, t->wt_src + 9 * s + 3 * d);
                t->first_src[3 * s + d] = f;
                if (f < 1 || f + 2 > nin / 2) { free(tt); return 1; }
            }
            scnt[b]++;
        }
    }
    t->self_in = (float *)calloc((size_t)np, sizeof(float));
    t->wt_tgt = (float *)malloc(sizeof(float) * 9 * (size_t)np);
    t->first_tgt = (int *)malloc(sizeof(int) * 3 * (size_t)np);
    for (int a = 0; a < n_act; ++a) {
        int b = t->active[a], r = t->region_r[b];
        int nin = r == 2 ? TL_NR2 : TL_NR4;
        float lo[3], hi[3];
        region_bounds(b, lo, hi);
        float bo = 3.5f + 3.0f / (float)r;
        float u0[3];
        for (int d = 0; d < 3; ++d) u0[d] = lo[d] - bo - (1.0f / (float)r) + (0.0f / (float)r);
        for (int p = t->target_start[b]; p < t->target_start[b + 1]; ++p) {
            int i = t->target_part[p];
            for (int d = 0; d < 3; ++d) {
                float tf = (tt[3 * i + d] - u0[d]) * (float)r;
                int f;
                tsc_weights(tf, &f, t->wt_tgt + 9 * i + 3 * d);
                t->first_tgt[3 * i + d] = f;
                if (f < 1 || f + 2 > nin / 2) { free(tt); return 1; }
            }
            t->self_in[i] = tsc_self(t->wt_tgt + 9 * i, r == 2 ? g2->self : g4->self);
        }
    }
    for (int a = 0; a < n_act; ++a) {
        int b = t->active[a], r = t->region_r[b];
        int nin = r == 2 ? TL_NR2 : TL_NR4;
        int slo[3] = {1 << 30, 1 << 30, 1 << 30}, shi[3] = {-(1 << 30), -(1 << 30), -(1 << 30)};
        int tlo[3] = {1 << 30, 1 << 30, 1 << 30}, thi[3] = {-(1 << 30), -(1 << 30), -(1 << 30)};
        for (int s = t->source_start[b]; s < t->source_start[b + 1]; ++s)
            for (int d = 0; d < 3; ++d) {
                int f = t->first_src[3 * s + d];
                if (f < slo[d]) slo[d] = f;
                if (f + 2 > shi[d]) shi[d] = f + 2;
            }
        for (int p = t->target_start[b]; p < t->target_start[b + 1]; ++p)
            for (int d = 0; d < 3; ++d) {
                int f = t->first_tgt[3 * t->target_part[p] + d];
                if (f < tlo[d]) tlo[d] = f;
                if (f + 2 > thi[d]) thi[d] = f + 2;
            }
        for (int d = 0; d < 3; ++d) {
            int gap = abs(thi[d] - slo[d]) > abs(shi[d] - tlo[d]) ? abs(thi[d] - slo[d]) : abs(shi[d] - tlo[d]);
            if (slo[d] < 1 || shi[d] > nin / 2 || tlo[d] < 1 || thi[d] > nin / 2 || gap >= nin / 2) {
                free(tt);
                return 1;
            }
        }
    }
    free(tt);
    return 0;
}

/* bound_two_level_run_pm (:825-942) */
static void tl_run_pm(const tl_ctx *t, const char *keep, const float *w, float spacing, double a,
                      const green_entry *g2, const green_entry *g4, float *phi_in, int np)
{
    for (int i = 0; i < np; ++i) phi_in[i] = 0.0f;
    for (int ra = 0; ra < t->n_active; ++ra) {
        int b = t->active[ra], r = t->region_r[b];
        int nin = r == 2 ? TL_NR2 : TL_NR4;
        const green_entry *g = r == 2 ? g2 : g4;
        float *rho = (float *)calloc((size_t)nin * nin * nin, sizeof(float));
        for (int s = t->source_start[b]; s < t->source_start[b + 1]; ++s) {
            int j = t->source_part[s];
            if (!keep[j]) continue;
            const float *wt = t->wt_src + 9 * s;
            const int *f = t->first_src + 3 * s;
            for (int sz = 0; sz < 3; ++sz)
                for (int sy = 0; sy < 3; ++sy)
                    for (int sx = 0; sx < 3; ++sx) {
                        size_t idx = ((size_t)(f[2] + sz - 1) * nin + (f[1] + sy - 1)) * nin + (f[0] + sx - 1);
                        rho[idx] = rho[idx] + w[j] * wt[sx] * wt[3 + sy] * wt[6 + sz];
                    }
        }
        pm_convolve(rho, g->green, nin, nin / 2 + 1);
        float pref = (float)(a * (double)r / (6.0 * PI * (double)spacing));
        for (int p = t->target_start[b]; p < t->target_start[b + 1]; ++p) {
            int i = t->target_part[p];
            if (!keep[i]) continue;
            const float *wt = t->wt_tgt + 9 * i;
            const int *f = t->first_tgt + 3 * i;
            float raw = 0.0f;
            for (int sz = 0; sz < 3; ++sz)
                for (int sy = 0; sy < 3; ++sy)
                    for (int sx = 0; sx < 3; ++sx) {
                        size_t idx = ((size_t)(f[2] + sz - 1) * nin + (f[1] + sy - 1)) * nin + (f[0] + sx - 1);
                        raw = raw + rho[idx] * wt[sx] * wt[3 + sy] * wt[6 + sz];
                    }
            phi_in[i] = pref * (raw - w[i] * t->self_in[i]);
        }
        free(rho);
    }
}

/* bound_two_level_pp_build (:944-1086) */
static void tl_pp_build(tl_ctx *t, const float *q, int np, float spacing)
{
    int rmax = 1, rmin = 4, any1 = 0;
    for (int i = 0; i < np; ++i) {
        int r = t->particle_r[i];
        if (r > rmax) rmax = r;
        if (r < rmin) rmin = r;
        any1 |= r == 1;
    }
    double at[5] = {0, 3.5 * (double)spacing, H_SPLIT * (double)spacing / 2.0, 0.0, H_SPLIT * (double)spacing / 4.0};
    double cw = rmax == 1 ? 3.5 * (double)spacing : H_SPLIT * (double)spacing / (double)rmax;
    if (cw <= 0.0) cw = 3.5 * (double)spacing;
    double amax = rmin == 1 ? 3.5 * (double)spacing : H_SPLIT * (double)spacing / (double)rmin;
    if (any1 && 3.5 * (double)spacing > amax) amax = 3.5 * (double)spacing;
    int ks = (int)ceil(amax / cw);
    t->k_search = ks < 1 ? 1 : (ks > 4 ? 4 : ks);
    double umin[3] = {1e30, 1e30, 1e30}, umax[3] = {-1e30, -1e30, -1e30};
    for (int i = 0; i < np; ++i)
        for (int d = 0; d < 3; ++d) {
            double u = (double)q[3 * i + d];
            if (u < umin[d]) umin[d] = u;
            if (u > umax[d]) umax[d] = u;
        }
    for (int d = 0; d < 3; ++d) {
        int v = (int)floor((umax[d] - umin[d]) / cw) + 1;
        t->pnc[d] = v > 1 ? v : 1;
        t->pu_min[d] = umin[d];
    }
    t->pcw = cw;
    int nt = t->pnc[0] * t->pnc[1] * t->pnc[2];
    t->pcell_id = (int *)malloc(sizeof(int) * np);
    t->pcell_part = (int *)malloc(sizeof(int) * np);
    t->pcell_start = (int *)calloc((size_t)nt + 1, sizeof(int));
    t->cell_max_a = (double *)calloc((size_t)nt, sizeof(double));
    for (int i = 0; i < np; ++i) {
        int ic[3];
        for (int d = 0; d < 3; ++d) {
            int v = (int)floor(((double)q[3 * i + d] - umin[d]) / cw) + 1;
            if (v < 1) v = 1;
            if (v > t->pnc[d]) v = t->pnc[d];
            ic[d] = v - 1;
        }
        int c = ic[0] + ic[1] * t->pnc[0] + ic[2] * t->pnc[0] * t->pnc[1];
        t->pcell_id[i] = c;
        t->pcell_start[c + 1]++;
        double ai = at[t->particle_r[i]];
        if (ai > t->cell_max_a[c]) t->cell_max_a[c] = ai;
    }
    for (int c = 0; c < nt; ++c) t->pcell_start[c + 1] += t->pcell_start[c];
    int *cur = (int *)malloc(sizeof(int) * (size_t)nt);
    memcpy(cur, t->pcell_start, sizeof(int) * (size_t)nt);
    for (int i = 0; i < np; ++i) t->pcell_part[cur[t->pcell_id[i]]++] = i;
    free(cur);
    int ntask = 0;
    for (int c = 0; c < nt; ++c) {
        int pc = t->pcell_start[c + 1] - t->pcell_start[c];
        if (pc > 0) ntask += (pc + 1023) / 1024;
    }
    t->ntask = ntask;
    t->task_c1 = (int *)malloc(sizeof(int) * (size_t)(ntask > 0 ? ntask : 1));
    t->task_p1 = (int *)malloc(sizeof(int) * (size_t)(ntask > 0 ? ntask : 1));
    t->task_p2 = (int *)malloc(sizeof(int) * (size_t)(ntask > 0 ? ntask : 1));
    t->task_max_a = (double *)malloc(sizeof(double) * (size_t)(ntask > 0 ? ntask : 1));
    ntask = 0;
    for (int c = 0; c < nt; ++c) {
        int beg = t->pcell_start[c], end = t->pcell_start[c + 1];
        for (int p = beg; p < end; p += 1024) {
            int pe = p + 1024 < end ? p + 1024 : end;
            double am = 0.0;
            for (int k = p; k < pe; ++k) {
                double ai = at[t->particle_r[t->pcell_part[k]]];
                if (ai > am) am = ai;
            }
            t->task_c1[ntask] = c; t->task_p1[ntask] = p; t->task_p2[ntask] = pe; t->task_max_a[ntask] = am;
            ++ntask;
        }
    }
}

static inline void tl_pp_pair(const float *q, const float *w, const int *pr, const double *at,
                              int i1, int i2, double eps, double factor, float *phi)
{
    double a1 = at[pr[i1]], a2 = at[pr[i2]];
    double dx = (double)q[3 * i2 + 0] - (double)q[3 * i1 + 0];
    double dy = (double)q[3 * i2 + 1] - (double)q[3 * i1 + 1];
    double dz = (double)q[3 * i2 + 2] - (double)q[3 * i1 + 2];
    double r2 = dx * dx + dy * dy + dz * dz;
    double am = a1 > a2 ? a1 : a2;
    if (r2 < am * am) {
        double d = sqrt(r2);
        double pe = depth_continuous(d, eps);
        if (r2 < a1 * a1) {
            float dp = -(float)(factor * (pe - depth_continuous(d, a1)));
            phi[i1] = phi[i1] + w[i2] * dp;
        }
        if (r2 < a2 * a2) {
            float dp = -(float)(factor * (pe - depth_continuous(d, a2)));
            phi[i2] = phi[i2] + w[i1] * dp;
        }
    }
}

/* bound_two_level_pp_full serial branch (:1252-1341) */
static void tl_pp_full(const tl_ctx *t, const float *q, const float *w, const char *keep, int np,
                       float spacing, float app_f, double a, float *phi)
{
    for (int i = 0; i < np; ++i) phi[i] = 0.0f;
    int nk = 0;
    for (int i = 0; i < np; ++i) nk += keep[i];
    if (nk <= 1) return;
    double at[5] = {0, 3.5 * (double)spacing / 1.0, H_SPLIT * (double)spacing / 2.0, 0.0, H_SPLIT * (double)spacing / 4.0};
    double eps = (double)app_f, factor = a / (6.0 * PI);
    const int *nc = t->pnc;
    double cw2 = t->pcw * t->pcw;
    int ks = t->k_search;
    for (int it = 0; it < t->ntask; ++it) {
        int c1 = t->task_c1[it], pb = t->task_p1[it], pe = t->task_p2[it];
        double tmax = t->task_max_a[it];
        int cz = c1 / (nc[0] * nc[1]), cy = (c1 % (nc[0] * nc[1])) / nc[0], cx = c1 % nc[0];
        for (int p1 = pb; p1 < pe; ++p1) {
            int i1 = t->pcell_part[p1];
            if (!keep[i1]) continue;
            for (int p2 = p1 + 1; p2 < t->pcell_start[c1 + 1]; ++p2) {
                int i2 = t->pcell_part[p2];
                if (!keep[i2]) continue;
                tl_pp_pair(q, w, t->particle_r, at, i1, i2, eps, factor, phi);
            }
        }
        for (int dz = 0; dz <= ks; ++dz) {
            int nz = cz + dz;
            if (nz < 0 || nz >= nc[2]) continue;
            int gz = abs(dz) - 1 > 0 ? abs(dz) - 1 : 0;
            for (int dy = -ks; dy <= ks; ++dy) {
                int ny = cy + dy;
                if (ny < 0 || ny >= nc[1]) continue;
                int gy = abs(dy) - 1 > 0 ? abs(dy) - 1 : 0;
                for (int dx = -ks; dx <= ks; ++dx) {
                    if (dz == 0 && (dy < 0 || (dy == 0 && dx <= 0))) continue;
                    int nx = cx + dx;
                    if (nx < 0 || nx >= nc[0]) continue;
                    int gx = abs(dx) - 1 > 0 ? abs(dx) - 1 : 0;
                    int c2 = nx + ny * nc[0] + nz * nc[0] * nc[1];
                    if (t->pcell_start[c2] >= t->pcell_start[c2 + 1]) continue;
                    double dmin2 = cw2 * (double)(gx * gx + gy * gy + gz * gz);
                    double rc = tmax > t->cell_max_a[c2] ? tmax : t->cell_max_a[c2];
                    if (dmin2 >= rc * rc) continue;
                    for (int p1 = pb; p1 < pe; ++p1) {
                        int i1 = t->pcell_part[p1];
                        if (!keep[i1]) continue;
                        for (int p2 = t->pcell_start[c2]; p2 < t->pcell_start[c2 + 1]; ++p2) {
                            int i2 = t->pcell_part[p2];
                            if (!keep[i2]) continue;
                            tl_pp_pair(q, w, t->particle_r, at, i1, i2, eps, factor, phi);
                        }
                    }
                }
            }
        }
    }
}

/* bound_two_level_pp_update serial branch (:1455-1496) */
static void tl_pp_update(const tl_ctx *t, const float *q, const float *w, const char *keep,
                         int np, const int *del, int ndel, float spacing, float app_f, double a,
                         float *phi)
{
    int nk = 0;
    for (int i = 0; i < np; ++i) nk += keep[i];
    if (ndel <= 0 || nk <= 0) return;
    double at[5] = {0, 3.5 * (double)spacing / 1.0, H_SPLIT * (double)spacing / 2.0, 0.0, H_SPLIT * (double)spacing / 4.0};
    double eps = (double)app_f, factor = a / (6.0 * PI);
    const int *nc = t->pnc;
    double cw2 = t->pcw * t->pcw;
    int ks = t->k_search;
    for (int k = 0; k < ndel; ++k) {
        int j = del[k];
        int cj = t->pcell_id[j];
        int cz = cj / (nc[0] * nc[1]), cy = (cj % (nc[0] * nc[1])) / nc[0], cx = cj % nc[0];
        for (int dz = -ks; dz <= ks; ++dz) {
            int nz = cz + dz;
            if (nz < 0 || nz >= nc[2]) continue;
            int gz = abs(dz) - 1 > 0 ? abs(dz) - 1 : 0;
            for (int dy = -ks; dy <= ks; ++dy) {
                int ny = cy + dy;
                if (ny < 0 || ny >= nc[1]) continue;
                int gy = abs(dy) - 1 > 0 ? abs(dy) - 1 : 0;
                for (int dx = -ks; dx <= ks; ++dx) {
                    int nx = cx + dx;
                    if (nx < 0 || nx >= nc[0]) continue;
                    int gx = abs(dx) - 1 > 0 ? abs(dx) - 1 : 0;
                    int c2 = nx + ny * nc[0] + nz * nc[0] * nc[1];
                    if (t->pcell_start[c2] >= t->pcell_start[c2 + 1]) continue;
                    double dmin2 = cw2 * (double)(gx * gx + gy * gy + gz * gz);
                    double rc = t->cell_max_a[c2];
                    if (dmin2 >= rc * rc) continue;
                    for (int p = t->pcell_start[c2]; p < t->pcell_start[c2 + 1]; ++p) {
                        int i = t->pcell_part[p];
                        if (!keep[i]) continue;
                        double ai = at[t->particle_r[i]];
                        double dx_ = (double)q[3 * i + 0] - (double)q[3 * j + 0];
                        double dy_ = (double)q[3 * i + 1] - (double)q[3 * j + 1];
                        double dz_ = (double)q[3 * i + 2] - (double)q[3 * j + 2];
                        double r2 = dx_ * dx_ + dy_ * dy_ + dz_ * dz_;
                        if (r2 < ai * ai) {
                            double d = sqrt(r2);
                            float dp = -(float)(factor * (depth_continuous(d, eps) - depth_continuous(d, ai)));
                            phi[i] = phi[i] - w[j] * dp;
                        }
                    }
                }
            }
        }
    }
}

/* ------------------------------------------------------- per-halo solver */

typedef struct {
    int gid;       /* 0 direct, 1..4 PM grid class */
    int lev;
    double spacing; /* double mirror of the FP32 spacing */
    float span, anchor[3], origin[3];
} htask;

/* heap sort of members by pid ascending (:2504-2528) -- any correct sort of
 * unique keys gives the same order */
static int cmp_i64(const void *a, const void *b, void *ctx)
{
    const int64_t *pid = (const int64_t *)ctx;
    int64_t x = pid[*(const int32_t *)a], y = pid[*(const int32_t *)b];
    return (x > y) - (x < y);
}

/* removal order: ascending energy; equal energies put the larger local index
 * first, so deletion from the top removes the smaller index first (:2808-2835) */
static int cmp_energy(const void *a, const void *b, void *ctx)
{
    const float *e = (const float *)ctx;
    int32_t i = *(const int32_t *)a, j = *(const int32_t *)b;
    if (e[i] < e[j]) return -1;
    if (e[i] > e[j]) return 1;
    return (i < j) - (i > j);
}

/* bound_check_grid (:2436-2888).  members: positions in xv of this
 * candidate (table order); returns ierr, fills status/np_bound/keep/member. */
static int check_grid(const bctx *c, const htask *tk, const float *xv, const float *mp,
                      const int64_t *pid, int32_t *member, int np, int *status_out,
                      int *np_bound_out, char *keep, float *phi_out, int phi_only,
                      float *energy_tab, float *phimax_out)
{
    const double a = c->a;
    const int nmin = c->np_min;
    *status_out = 0;
    qsort_r(member, (size_t)np, sizeof(int32_t), cmp_i64, (void *)pid);
    for (int i = 1; i < np; ++i) if (pid[member[i]] == pid[member[i - 1]]) return 1;
    float *q = (float *)malloc(sizeof(float) * 3 * (size_t)np);
    float *w = (float *)malloc(sizeof(float) * (size_t)np);
    float *phi = (float *)calloc((size_t)np, sizeof(float));
    float *energy = (float *)calloc((size_t)np, sizeof(float));
    double *phid = (double *)calloc((size_t)np, sizeof(double));
    int32_t *order = (int32_t *)malloc(sizeof(int32_t) * (size_t)np);
    int32_t *jdel = (int32_t *)malloc(sizeof(int32_t) * (size_t)np);
    float *selfp = NULL, *wt = NULL, *phi_c1 = NULL, *phi_c2 = NULL, *phi_in = NULL;
    int *first = NULL;
    c2cells cells = {0};
    tl_ctx tl;
    memset(&tl, 0, sizeof(tl));
    int use_tl = 0, ierr = 0, njd = 0;
    int np_bound = np;
    for (int i = 0; i < np; ++i) {
        keep[i] = 1;
        w[i] = mp ? mp[member[i]] : 1.0f;
        for (int d = 0; d < 3; ++d) q[3 * i + d] = (xv[6 * (size_t)member[i] + d] - tk->anchor[d]) * 1.0f;
    }
    const int gid = tk->gid;
    const float spacing = (float)tk->spacing;
    const green_entry *ge = NULL, *g2 = NULL, *g4 = NULL;
    int n = 0;
    if (gid >= 1) {
        n = c->bn[gid - 1];
        ge = get_green(n, H_SPLIT, 0.0, 1);
        if (!ge) { ierr = 1; goto out; }
        selfp = (float *)malloc(sizeof(float) * (size_t)np);
        wt = (float *)malloc(sizeof(float) * 9 * (size_t)np);
        first = (int *)malloc(sizeof(int) * 3 * (size_t)np);
        phi_c1 = (float *)calloc((size_t)np, sizeof(float));
        phi_c2 = (float *)calloc((size_t)np, sizeof(float));
        phi_in = (float *)calloc((size_t)np, sizeof(float));
        for (int i = 0; i < np; ++i) {
            float t[3];
            for (int d = 0; d < 3; ++d) t[d] = (q[3 * i + d] - tk->origin[d]) / spacing;
            for (int d = 0; d < 3; ++d) {
                if (!isfinite(t[d])) { ierr = 1; goto out; }
                if (t[d] < 0.0f || t[d] >= (float)(n / 2 - 1)) { ierr = 1; goto out; }
            }
            for (int d = 0; d < 3; ++d) tsc_weights(t[d], &first[3 * i + d], wt + 9 * i + 3 * d);
            selfp[i] = tsc_self(wt + 9 * i, ge->self);
        }
        if (gid == 4) {
            int need2 = H_SPLIT * tk->spacing / 2.0 >= c->app;
            int need4 = H_SPLIT * tk->spacing / 4.0 >= c->app;
            if (need2) g2 = get_green(TL_NR2, H_SPLIT, 7.0, 0);
            if (need4) g4 = get_green(TL_NR4, H_SPLIT, 14.0, 0);
            int e = tl_build(&tl, q, np, spacing, tk->origin, (float)c->app, g2, g4);
            if (e) { ierr = e; goto out; }
            use_tl = tl.n_active > 0;
        }
        if (!use_tl) build_cells(&cells, q, np, spacing, 3.5);
    }

    for (int pass = 1; pass <= MAX_PASSES; ++pass) {
        int n_source = 0;
        for (int i = 0; i < np; ++i) n_source += keep[i];
        if (gid == 0) {
            const double fac = a / (6.0 * PI);
            if (pass == 1) {
                for (int i = 0; i < np; ++i) phid[i] = 0.0;
                for (int i = 0; i < np - 1; ++i)
                    for (int j = i + 1; j < np; ++j) {
                        double dx = (double)(q[3 * j + 0] - q[3 * i + 0]);
                        double dy = (double)(q[3 * j + 1] - q[3 * i + 1]);
                        double dz = (double)(q[3 * j + 2] - q[3 * i + 2]);
                        double r = sqrt(dx * dx + dy * dy + dz * dz);
                        double dd = fac * depth_continuous(r, c->app);
                        phid[i] = phid[i] - (double)w[j] * dd;
                        phid[j] = phid[j] - (double)w[i] * dd;
                    }
            } else {
                for (int k = 0; k < njd; ++k) {
                    int j = jdel[k];
                    for (int i = 0; i < np; ++i) {
                        if (!keep[i]) continue;
                        double dx = (double)(q[3 * j + 0] - q[3 * i + 0]);
                        double dy = (double)(q[3 * j + 1] - q[3 * i + 1]);
                        double dz = (double)(q[3 * j + 2] - q[3 * i + 2]);
                        double r = sqrt(dx * dx + dy * dy + dz * dz);
                        phid[i] = phid[i] + (double)w[j] * fac * depth_continuous(r, c->app);
                    }
                }
            }
            njd = 0;
            for (int i = 0; i < np; ++i) if (keep[i]) phi[i] = (float)phid[i];
        } else {
            int full = pass == 1;
            const int sup = n / 2 + 1;
            float *rho = (float *)calloc((size_t)n * n * n, sizeof(float));
            for (int i = 0; i < np; ++i) {
                if (!keep[i]) continue;
                const float *wi = wt + 9 * i;
                const int *f = first + 3 * i;
                for (int sz = 0; sz < 3; ++sz)
                    for (int sy = 0; sy < 3; ++sy)
                        for (int sx = 0; sx < 3; ++sx) {
                            size_t idx = ((size_t)(f[2] + sz - 1) * n + (f[1] + sy - 1)) * n + (f[0] + sx - 1);
                            rho[idx] = rho[idx] + w[i] * wi[sx] * wi[3 + sy] * wi[6 + sz];
                        }
            }
            pm_convolve(rho, ge->green, n, sup);
            const float radius_r = (float)n / 2.0f;
            double mkeep = 0.0;
            for (int i = 0; i < np; ++i) if (keep[i]) mkeep += (double)w[i];
            const float pref = (float)(a / (6.0 * PI * (double)spacing));
            for (int i = 0; i < np; ++i) {
                if (!keep[i]) continue;
                double mrest = mkeep - (double)w[i];
                float dz0 = (float)(mrest > 0.0 ? mrest : 0.0) / radius_r;
                const float *wi = wt + 9 * i;
                const int *f = first + 3 * i;
                float raw = 0.0f;
                for (int sz = 0; sz < 3; ++sz)
                    for (int sy = 0; sy < 3; ++sy)
                        for (int sx = 0; sx < 3; ++sx) {
                            size_t idx = ((size_t)(f[2] + sz - 1) * n + (f[1] + sy - 1)) * n + (f[0] + sx - 1);
                            raw = raw + rho[idx] * wi[sx] * wi[3 + sy] * wi[6 + sz];
                        }
                phi_c1[i] = pref * ((raw - w[i] * selfp[i]) - dz0);
                if (full) phi_c2[i] = 0.0f;
            }
            free(rho);
            if (use_tl) {
                tl_run_pm(&tl, keep, w, spacing, a, g2, g4, phi_in, np);
                if (full) {
                    tl_pp_build(&tl, q, np, spacing);
                    tl_pp_full(&tl, q, w, keep, np, spacing, (float)c->app, a, phi_c2);
                } else {
                    tl_pp_update(&tl, q, w, keep, np, jdel, njd, spacing, (float)c->app, a, phi_c2);
                }
            } else {
                for (int i = 0; i < np; ++i) phi_in[i] = 0.0f;
                if (full) c2_full(&cells, q, w, keep, np, spacing, (float)c->app, a, phi_c2);
                else c2_update(&cells, q, w, keep, np, jdel, njd, spacing, (float)c->app, a, phi_c2);
            }
            njd = 0;
        }
        for (int i = 0; i < np; ++i) {
            if (!keep[i]) continue;
            if (gid >= 1) phi[i] = use_tl ? (phi_c1[i] + phi_in[i]) + phi_c2[i] : phi_c1[i] + phi_c2[i];
            if (np_bound == 1 || n_source == 1) phi[i] = 0.0f;
            if (!isfinite(phi[i])) { ierr = 4; goto out; }
        }
        if (pass == 1 && phimax_out) {
            float m = 0.0f;
            for (int i = 0; i < np; ++i) if (keep[i] && fabsf(phi[i]) > m) m = fabsf(phi[i]);
            *phimax_out = m;
        }
        if (phi_only) { *status_out = 0; goto done; }
        int deleted = 0;
        for (;;) {
            double wsum = 0, qc[3] = {0, 0, 0}, vc[3] = {0, 0, 0};
            for (int i = 0; i < np; ++i) {
                if (!keep[i]) continue;
                double wi = (double)w[i];
                wsum = wsum + wi;
                for (int d = 0; d < 3; ++d) {
                    qc[d] = qc[d] + wi * (double)q[3 * i + d];
                    vc[d] = vc[d] + wi * (double)xv[6 * (size_t)member[i] + 3 + d];
                }
            }
            for (int d = 0; d < 3; ++d) { qc[d] = qc[d] / wsum; vc[d] = vc[d] / wsum; }
            float vcf[3], qcf[3], bf = (float)c->b;
            for (int d = 0; d < 3; ++d) { vcf[d] = (float)vc[d]; qcf[d] = (float)qc[d]; }
            int nu = 0;
            for (int i = 0; i < np; ++i) {
                if (!keep[i]) continue;
                float dv[3];
                for (int d = 0; d < 3; ++d)
                    dv[d] = (xv[6 * (size_t)member[i] + 3 + d] - vcf[d]) + bf * (q[3 * i + d] - qcf[d]);
                float s = dv[0] * dv[0];
                s = s + dv[1] * dv[1];
                s = s + dv[2] * dv[2];
                energy[i] = s / 2.0f + phi[i];
                if (!isfinite(energy[i])) { ierr = 1; goto out; }
                if (energy[i] >= 0.0f) order[nu++] = i;
            }
            if (nu == 0) {
                if (deleted == 0) { *status_out = 0; goto done; }
                break;
            }
            if (nu > 1) qsort_r(order, (size_t)nu, sizeof(int32_t), cmp_energy, energy);
            int nb = (int)ceil(0.02 * (double)np_bound);
            if (nb < 1) nb = 1;
            if (nb > nu) nb = nu;
            for (int i = nu - 1; i >= nu - nb; --i) {
                keep[order[i]] = 0;
                jdel[njd++] = order[i];
            }
            np_bound -= nb;
            deleted += nb;
            if (np_bound < nmin) { *status_out = 1; goto done; }
            if ((double)deleted >= 0.20 * (double)np_bound) break;
        }
    }
    *status_out = 5;
    if (c->verbose >= 0)
        fprintf(stderr, " bound_check: MAX_ITER, retained members = %d\n", np_bound);
done:
    *np_bound_out = np_bound;
    if (phi_out)
        for (int i = 0; i < np; ++i) phi_out[i] = phi[i];
    /* diagnostics for the tests' energy band: each member's specific energy
     * at its last evaluation (the final one if kept, at removal otherwise) */
    if (energy_tab)
        for (int i = 0; i < np; ++i) energy_tab[member[i]] = energy[i];
out:
    free(q); free(w); free(phi); free(energy); free(phid); free(order); free(jdel);
    free(selfp); free(wt); free(first); free(phi_c1); free(phi_c2); free(phi_in);
    free_cells(&cells);
    tl_free(&tl);
    return ierr;
}

/* bound_classify (:2901-3073), without the cost-ordered queues (they only
 * decide the processing order).  Returns ierr. */
static int classify(const bctx *c, const float *xv, const int32_t *cand_np, const int64_t *off,
                    int32_t ncand, htask *tasks)
{
    for (int32_t h = 0; h < ncand; ++h) {
        htask *t = &tasks[h];
        memset(t, 0, sizeof(*t));
        const float *x0 = xv + 6 * (size_t)off[h];
        float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        for (int d = 0; d < 3; ++d) t->anchor[d] = x0[d];
        for (int32_t i = 0; i < cand_np[h]; ++i)
            for (int d = 0; d < 3; ++d) {
                float qv = (xv[6 * (size_t)(off[h] + i) + d] - t->anchor[d]) * 1.0f;
                lo[d] = fminf(lo[d], qv);
                hi[d] = fmaxf(hi[d], qv);
            }
        float span = hi[0] - lo[0];
        for (int d = 1; d < 3; ++d) if (hi[d] - lo[d] > span) span = hi[d] - lo[d];
        t->span = span;
        if (!isfinite(span)) return 1;
        if (cand_np[h] > 1000 && span > (float)c->s15) return 2;
        int g, l;
        double sp;
        if (select_grid(c, cand_np[h], (double)span, &g, &l, &sp)) return 1;
        t->gid = g;
        t->lev = l;
        if (g > 0) {
            t->spacing = (double)(float)sp;
            for (int d = 0; d < 3; ++d) t->origin[d] = lo[d] - (float)sp;
            if ((double)(c->bn[g - 1] / 2 - 3) * t->spacing < (double)span) return 1;
        }
    }
    return 0;
}

/* ------------------------------------------------ the reference's schedule
 *
 * bound_classify's groups and queues (bound_fortran.f90:2986-3067) and
 * compute_bound_parallel_config / the phase build of bound_check_batch
 * (:332-401, :1627-1665): group g = grid class (direct-summation halos join
 * group 1); cost = n(n-1)/2 for direct halos, 6 V log2 V + 12 V + 64 n +
 * 9 n log2 max(2,n) with V = bn(g)^3 for PM halos; each group's queue in
 * descending cost (ties: ascending candidate index); phase 1 runs group 4
 * with g4_team workers, phase 2 groups 1-3 with a greedy split of the
 * remaining threads (or one phase per group, 3 down to 1, when there are
 * fewer threads than groups); a worker takes halos only from its own
 * group's queue.  The reference's group-4 workers each own g4_nest threads
 * for their short-range sums (a nested team whose per-thread partial sums
 * make results thread-count dependent); here every halo's sums run on its
 * worker's thread alone, so results do not depend on the thread count. */
typedef struct {
    int nphases;
    int workers[5][4];
    int next[4], last[4];
    int32_t *queue;
} sched_t;

static void bound_parallel_config(int T, const int M[4], const double W[4], const double L[4],
                                  int nmax4, int *g4_team, int *g4_nest, int gteam[3])
{
    if (M[3] == 0) { *g4_team = 0; *g4_nest = 1; }
    else {
        *g4_nest = (T >= 2 && M[3] <= 10 * T && nmax4 > 10000) ? 2 : 1;
        int t = T / *g4_nest;
        if (t < 1) t = 1;
        *g4_team = M[3] < t ? M[3] : t;
    }
    int B = M[0] + M[1] + M[2];
    if (B > T) B = T;
    int K = (M[0] > 0) + (M[1] > 0) + (M[2] > 0);
    gteam[0] = gteam[1] = gteam[2] = 0;
    if (B >= K && K > 0) {
        for (int g = 0; g < 3; ++g) if (M[g] > 0) gteam[g] = 1;
        int used = gteam[0] + gteam[1] + gteam[2];
        while (used < B) {
            int best = -1;
            double best_gain = -1.0;
            for (int g = 0; g < 3; ++g)
                if (gteam[g] >= 1 && gteam[g] < M[g]) {
                    double before = fmax(L[g], W[g] / (double)gteam[g]);
                    double after = fmax(L[g], W[g] / (double)(gteam[g] + 1));
                    if (before - after > best_gain) { best_gain = before - after; best = g; }
                }
            if (best_gain <= 0.0) {
                double best_load = -1.0;
                for (int g = 0; g < 3; ++g)
                    if (gteam[g] >= 1 && gteam[g] < M[g] && W[g] / (double)gteam[g] > best_load) {
                        best_load = W[g] / (double)gteam[g];
                        best = g;
                    }
            }
            if (best < 0) break;
            ++gteam[best];
            ++used;
        }
    }
}

static const double *g_cost_sort;
static int cmp_cost_desc(const void *a, const void *b)
{
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    if (g_cost_sort[x] > g_cost_sort[y]) return -1;
    if (g_cost_sort[x] < g_cost_sort[y]) return 1;
    return (x > y) - (x < y);
}

static int schedule(const bctx *c, const htask *tasks, const int32_t *cand_np, int32_t ncand, int T,
                    sched_t *sc)
{
    static pthread_mutex_t mu = PTHREAD_MUTEX_INITIALIZER;
    memset(sc, 0, sizeof(*sc));
    int M[4] = {0, 0, 0, 0}, nmax4 = 0;
    double W[4] = {0, 0, 0, 0}, L[4] = {0, 0, 0, 0};
    double *cost = (double *)malloc(sizeof(double) * (size_t)(ncand > 0 ? ncand : 1));
    int *grp = (int *)malloc(sizeof(int) * (size_t)(ncand > 0 ? ncand : 1));
    sc->queue = (int32_t *)malloc(sizeof(int32_t) * (size_t)(ncand > 0 ? ncand : 1));
    if (!cost || !grp || !sc->queue) { free(cost); free(grp); free(sc->queue); sc->queue = NULL; return 1; }
    for (int32_t h = 0; h < ncand; ++h) {
        const double nn = (double)cand_np[h];
        int g;
        if (tasks[h].gid == 0) {
            g = 0;
            cost[h] = nn * (nn - 1.0) / 2.0;
        } else {
            g = tasks[h].gid - 1;
            const double vol = (double)c->bn[g] * (double)c->bn[g] * (double)c->bn[g];
            cost[h] = 6.0 * vol * log(vol) / log(2.0) + 12.0 * vol + 64.0 * nn +
                      9.0 * nn * log(fmax(2.0, nn)) / log(2.0);
        }
        grp[h] = g;
        ++M[g];
        W[g] += cost[h];
        if (cost[h] > L[g]) L[g] = cost[h];
        if (g == 3 && cand_np[h] > nmax4) nmax4 = cand_np[h];
    }
    int cur[4];
    cur[0] = 0;
    for (int g = 1; g < 4; ++g) cur[g] = cur[g - 1] + M[g - 1];
    for (int g = 0; g < 4; ++g) { sc->next[g] = cur[g]; sc->last[g] = cur[g] + M[g] - 1; }
    for (int32_t h = 0; h < ncand; ++h) sc->queue[cur[grp[h]]++] = h;
    pthread_mutex_lock(&mu);
    g_cost_sort = cost;
    for (int g = 0; g < 4; ++g)
        if (M[g] > 1) qsort(sc->queue + sc->next[g], (size_t)M[g], sizeof(int32_t), cmp_cost_desc);
    pthread_mutex_unlock(&mu);
    int g4_team, g4_nest, gt[3];
    bound_parallel_config(T, M, W, L, nmax4, &g4_team, &g4_nest, gt);
    if (g4_team > 0) {
        sc->workers[sc->nphases][3] = g4_team;
        ++sc->nphases;
    }
    if (M[0] + M[1] + M[2] > 0) {
        int B = M[0] + M[1] + M[2];
        if (B > T) B = T;
        int K = (M[0] > 0) + (M[1] > 0) + (M[2] > 0);
        if (B >= K) {
            for (int g = 0; g < 3; ++g) sc->workers[sc->nphases][g] = gt[g];
            ++sc->nphases;
        } else {
            for (int g = 2; g >= 0; --g)
                if (M[g] > 0) {
                    sc->workers[sc->nphases][g] = M[g] < B ? M[g] : B;
                    ++sc->nphases;
                }
        }
    }
    free(cost);
    free(grp);
    return 0;
}

int32_t oracle_bound_batch(const float *xv, const float *mp, const int64_t *pid,
                           const int32_t *cand_np, int32_t ncand, double softening,
                           double a_val, double b_val, double s15, int32_t np_halo_min,
                           int32_t verbose, int32_t n_threads, int64_t ng_val,
                           double ng_global_val, int32_t *np_bound, int32_t *status,
                           int32_t *final_members, float *phi_out, int32_t *method_out)
{
    return oracle_bound_batch_diag(xv, mp, pid, cand_np, ncand, softening, a_val, b_val, s15,
                                   np_halo_min, verbose, n_threads, ng_val, ng_global_val,
                                   np_bound, status, final_members, phi_out, method_out, NULL,
                                   NULL);
}

int32_t oracle_bound_batch_diag(const float *xv, const float *mp, const int64_t *pid,
                                const int32_t *cand_np, int32_t ncand, double softening,
                                double a_val, double b_val, double s15, int32_t np_halo_min,
                                int32_t verbose, int32_t n_threads, int64_t ng_val,
                                double ng_global_val, int32_t *np_bound, int32_t *status,
                                int32_t *final_members, float *phi_out, int32_t *method_out,
                                float *energy_tab, float *phimax)
{
    bctx c;
    ctx_init(&c, softening, a_val, b_val, s15, np_halo_min, verbose, ng_val, ng_global_val);
    int64_t *off = (int64_t *)malloc(sizeof(int64_t) * ((size_t)ncand + 1));
    htask *tasks = (htask *)calloc((size_t)ncand, sizeof(htask));
    if (!off || !tasks) { free(off); free(tasks); return 3; }
    off[0] = 0;
    for (int32_t h = 0; h < ncand; ++h) off[h + 1] = off[h] + cand_np[h];
    for (int64_t i = 0; i < off[ncand]; ++i) final_members[i] = -1;
    for (int32_t h = 0; h < ncand; ++h) { np_bound[h] = 0; status[h] = -1; }
    int ierr = 0;
    if (c.ngrid != 4) ierr = 1;
    if (!ierr && (!isfinite(a_val) || a_val <= 0.0 || !isfinite(b_val))) ierr = 1;
    if (!ierr) ierr = classify(&c, xv, cand_np, off, ncand, tasks);
    if (method_out)
        for (int32_t h = 0; h < ncand; ++h) method_out[h] = tasks[h].gid;
    if (!ierr) {
        /* Green tables are built once, before the parallel loop */
        for (int32_t h = 0; h < ncand && !ierr; ++h) {
            if (tasks[h].gid > 0 && !get_green(c.bn[tasks[h].gid - 1], H_SPLIT, 0.0, 1)) ierr = 1;
            if (tasks[h].gid == 4 && H_SPLIT * tasks[h].spacing / 2.0 >= c.app && cand_np[h] >= TL_N12 &&
                !get_green(TL_NR2, H_SPLIT, 7.0, 0)) ierr = 1;
            if (tasks[h].gid == 4 && H_SPLIT * tasks[h].spacing / 4.0 >= c.app && cand_np[h] >= TL_N24 &&
                !get_green(TL_NR4, H_SPLIT, 14.0, 0)) ierr = 1;
        }
        int T = n_threads > 0 ? n_threads : omp_get_max_threads();
        sched_t sc;
        if (schedule(&c, tasks, cand_np, ncand, T, &sc)) {
            ierr = 3;
        } else {
            omp_set_max_active_levels(2);
            for (int ph = 0; ph < sc.nphases && !ierr; ++ph) {
                int wg[1024], nslots = 0;
                for (int g = 3; g >= 0; --g)
                    for (int l = 0; l < sc.workers[ph][g] && nslots < 1024; ++l) wg[nslots++] = g;
                if (nslots <= 0) continue;
#pragma omp parallel num_threads(nslots)
                {
                    const int g = wg[omp_get_thread_num()];
                    for (;;) {
                        int e, pos;
#pragma omp atomic read
                        e = ierr;
                        if (e) break;
#pragma omp atomic capture
                        pos = sc.next[g]++;
                        if (pos > sc.last[g]) break;
                        const int32_t h = sc.queue[pos];
                        int np = cand_np[h];
                        int32_t *member = (int32_t *)malloc(sizeof(int32_t) * (size_t)np);
                        char *keep = (char *)malloc((size_t)np);
                        for (int i = 0; i < np; ++i) member[i] = (int32_t)(off[h] + i);
                        int st = -1, nb = 0;
                        e = check_grid(&c, &tasks[h], xv, mp, pid, member, np, &st, &nb, keep,
                                       phi_out ? phi_out + off[h] : NULL, 0, energy_tab,
                                       phimax ? phimax + h : NULL);
                        if (e) {
#pragma omp critical(oracle_bound_err)
                            if (!ierr) ierr = e;
                        } else {
                            status[h] = st;
                            np_bound[h] = nb;
                            if (st == 0) {
                                int cnt = 0;
                                for (int i = 0; i < np; ++i)
                                    if (keep[i]) final_members[off[h] + cnt++] = member[i];
                            }
                        }
                        free(member);
                        free(keep);
                    }
                }
            }
            free(sc.queue);
        }
    }
    free(off);
    free(tasks);
    return ierr;
}

int32_t oracle_bound_first_potential(const float *xv, const float *mp, const int64_t *pid,
                                     int32_t np, double softening, double a_val, double s15,
                                     int64_t ng_val, float *phi)
{
    bctx c;
    ctx_init(&c, softening, a_val, 0.0, s15, 1, -1, ng_val, 512.0);
    int64_t off[2] = {0, np};
    htask t;
    int e = classify(&c, xv, &np, off, 1, &t);
    if (e) return -e;
    int32_t *member = (int32_t *)malloc(sizeof(int32_t) * (size_t)np);
    char *keep = (char *)malloc((size_t)np);
    for (int i = 0; i < np; ++i) member[i] = i;
    int st, nb;
    e = check_grid(&c, &t, xv, mp, pid, member, np, &st, &nb, keep, phi, 1, NULL, NULL);
    free(member); free(keep);
    return e ? -e : t.gid;
}

void oracle_direct_potential_f64(const float *q, const float *w, int32_t np, double softening,
                                 double a_val, double *phi)
{
    const double fac = a_val / (6.0 * PI);
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < np; ++i) {
        double s = 0.0;
        for (int32_t j = 0; j < np; ++j) {
            if (j == i) continue;
            double dx = (double)q[3 * j] - (double)q[3 * i];
            double dy = (double)q[3 * j + 1] - (double)q[3 * i + 1];
            double dz = (double)q[3 * j + 2] - (double)q[3 * i + 2];
            s -= (double)w[j] * fac * depth_continuous(sqrt(dx * dx + dy * dy + dz * dz), softening);
        }
        phi[i] = s;
    }
}
