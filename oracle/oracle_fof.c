/*
 * CPU oracle, friends-of-friends part -- TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Restates fof_fortran.f90 (driver :109-362, region engine :496-949) and
 * atomic_dsu.c.  Floating-point rules that make the partition bit-exact:
 *   - gfortran MODULO for reals: r = fmod(a,p); r += p when r != 0 and the
 *     signs of a and p differ; r = +0 when r == 0 (oracle_modulo);
 *   - stored CRS coordinates are real(x,4) = round-to-nearest FP32;
 *   - non-periodic distance: FP32 differences, FP32 squares, FP32 sum in
 *     x,y,z order, widened to FP64 and compared with link**2 (FP64);
 *   - periodic distance (dist2_pbc): FP32 difference widened to FP64,
 *     minimum image in FP64, FP64 squares summed in x,y,z order;
 *   - compiled with -ffp-contract=off so no FMA contraction happens.
 * Integer expressions that overflow default (32-bit) integers in the
 * reference for N >= 2**29 (4*np, 2*np, Nx*Ny*Nz) are evaluated in 64 bits.
 */
#include "oracle.h"

#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static int32_t g_last_threads = 1;
int32_t oracle_last_threads(void) { return g_last_threads; }

/* gfortran lowering of MODULO(a,p) for real arguments. */
double oracle_modulo(double a, double p)
{
    double r = fmod(a, p);
    if (r != 0.0) {
        if ((a < 0.0) != (p < 0.0)) r += p;
    } else {
        r = copysign(0.0, p);
    }
    return r;
}

static inline double dmax(double a, double b) { return a > b ? a : b; }
static inline double dmin(double a, double b) { return a < b ? a : b; }

typedef struct {
    int32_t ncand;
    int32_t *cand_np;      /* [ncand] */
    int64_t *member_ptr;   /* [ncand+1], offsets into cand_members */
    int64_t *cand_members; /* global 0-based particle indices, CRS order per candidate */
    float *xm, *vm;        /* [3*ncand] preliminary centre / mean velocity */
} region_cands;

/* ---- disjoint-set union, reference semantics ---------------------------- */

/* dsu_union_serial (fof_fortran.f90:424-458): full path compression of both
 * operands, then the higher root is hung under the lower one. */
static void dsu_union_serial(int32_t *parent, int32_t i, int32_t j)
{
    int32_t ra = i, rb = j, cur, nxt;
    while (parent[ra] >= 0) ra = parent[ra];
    cur = i;
    while (cur != ra) { nxt = parent[cur]; parent[cur] = ra; cur = nxt; }
    while (parent[rb] >= 0) rb = parent[rb];
    cur = j;
    while (cur != rb) { nxt = parent[cur]; parent[cur] = rb; cur = nxt; }
    if (ra == rb) return;
    if (ra > rb) parent[ra] = rb; else parent[rb] = ra;
}

static int32_t dsu_find_root(int32_t *parent, int32_t i)
{
    int32_t r = i, cur = i, nxt;
    while (parent[r] >= 0) r = parent[r];
    while (cur != r) { nxt = parent[cur]; parent[cur] = r; cur = nxt; }
    return r;
}

/* atomic_dsu.c root(): path halving by CAS. */
static int32_t dsu_root_atomic(int32_t *parent, int32_t p)
{
    for (;;) {
        int32_t next = __atomic_load_n(&parent[p], __ATOMIC_RELAXED);
        if (next < 0) return p;
        int32_t after = __atomic_load_n(&parent[next], __ATOMIC_RELAXED);
        if (after >= 0) {
            int32_t expected = next;
            (void)__atomic_compare_exchange_n(&parent[p], &expected, after, 0,
                                              __ATOMIC_RELAXED, __ATOMIC_RELAXED);
        }
        p = next;
    }
}

/* atomic_dsu.c fof_atomic_union(): CAS parent[high] from -1 to low. */
static void dsu_union_atomic(int32_t *parent, int32_t i, int32_t j)
{
    for (;;) {
        int32_t a = dsu_root_atomic(parent, i);
        int32_t b = dsu_root_atomic(parent, j);
        if (a == b) return;
        int32_t lo = a < b ? a : b, hi = a < b ? b : a;
        int32_t expected = -1;
        if (__atomic_compare_exchange_n(&parent[hi], &expected, lo, 0,
                                        __ATOMIC_RELAXED, __ATOMIC_RELAXED))
            return;
    }
}

/* ---- distance tests ----------------------------------------------------- */

/* fof_fortran.f90:636 -- sum((x_crs(:,p1)-x_crs(:,p2))**2) in FP32. */
static inline double dist2_open(const float *a, const float *b)
{
    float d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
    float s = d0 * d0;
    s = s + d1 * d1;
    s = s + d2 * d2;
    return (double)s;
}

/* dist2_pbc (fof_fortran.f90:483-491). */
static inline double dist2_pbc(const float *a, const float *b, double L, double half)
{
    double dx = fabs((double)(a[0] - b[0])); if (dx > half) dx = L - dx;
    double dy = fabs((double)(a[1] - b[1])); if (dy > half) dy = L - dy;
    double dz = fabs((double)(a[2] - b[2])); if (dz > half) dz = L - dz;
    return dx * dx + dy * dy + dz * dz;
}

/* ---- cell geometry (fof_fortran.f90:538-570) ----------------------------- */

static void cell_geometry(const double *range, const double *xmin, const int *pdim,
                          double L, double half, double link, double L_mesh,
                          double *origin, double *size, int64_t *N)
{
    for (int d = 0; d < 3; ++d) {
        if (pdim[d]) {
            origin[d] = -half;
            int64_t a = (int64_t)(L / link), b = (int64_t)(L / L_mesh);
            int64_t n = a < b ? a : b;
            N[d] = n > 1 ? n : 1;
            size[d] = L / (double)N[d];
        } else {
            origin[d] = xmin[d];
            int64_t n = (int64_t)ceil(range[d] / L_mesh);
            N[d] = n > 1 ? n : 1;
            size[d] = L_mesh;
        }
    }
}

static inline int64_t cell_coord(double x, double origin, double size, int64_t n)
{
    double f = floor((x - origin) / size) + 1.0;
    if (!(f >= 1.0)) f = 1.0; /* also maps NaN to the first cell */
    if (f > (double)n) f = (double)n;
    return (int64_t)f;
}

/* ---- one region (process_single_region, fof_fortran.f90:496-949) ------- */

static int process_region(const double *xp, const double *vp, const double *mp,
                          int64_t istart, int32_t np, double L, double half,
                          double link, int32_t np_min, int nest, region_cands *out)
{
    const double rp2 = link * link;
    memset(out, 0, sizeof(*out));
    double *xr = (double *)malloc(sizeof(double) * 3 * (size_t)np);
    if (!xr) return 3;
    const double *anc = xp + 3 * istart;
    double xmin[3] = {INFINITY, INFINITY, INFINITY}, xmax[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int32_t i = 0; i < np; ++i)
        for (int d = 0; d < 3; ++d) {
            double v = oracle_modulo(xp[3 * (istart + i) + d] - anc[d] + half, L) - half;
            xr[3 * i + d] = v;
            if (v < xmin[d]) xmin[d] = v;
            if (v > xmax[d]) xmax[d] = v;
        }
    double range[3];
    int pdim[3], periodic = 0;
    for (int d = 0; d < 3; ++d) {
        range[d] = xmax[d] - xmin[d];
        pdim[d] = (range[d] + 2.0 * link >= L);
        periodic |= pdim[d];
    }
    double vol = dmax(range[0], link) * dmax(range[1], link) * dmax(range[2], link);
    double L_mesh = dmax(link, pow(vol / (double)(np > 1 ? np : 1), 1.0 / 3.0));
    double origin[3], size[3];
    int64_t N[3];
    cell_geometry(range, xmin, pdim, L, half, link, L_mesh, origin, size, N);
    int64_t cap = 4 * (int64_t)np;
    if (cap < 262144) cap = 262144;
    if ((double)N[0] * (double)N[1] * (double)N[2] > (double)cap) {
        L_mesh = pow(vol / (double)((int64_t)(np > 1 ? np : 1) * 2), 1.0 / 3.0);
        L_mesh = dmax(link, L_mesh);
        cell_geometry(range, xmin, pdim, L, half, link, L_mesh, origin, size, N);
    }
    const int64_t Nx = N[0], Ny = N[1], Nz = N[2];
    const int64_t ncell = Nx * Ny * Nz;

    int64_t *cell_ptr = (int64_t *)calloc((size_t)ncell + 1, sizeof(int64_t));
    int64_t *cellid = (int64_t *)malloc(sizeof(int64_t) * (size_t)np);
    float *xc = (float *)malloc(sizeof(float) * 3 * (size_t)np);
    int64_t *pid = (int64_t *)malloc(sizeof(int64_t) * (size_t)np);
    int32_t *parent = (int32_t *)malloc(sizeof(int32_t) * (size_t)np);
    if (!cell_ptr || !cellid || !xc || !pid || !parent) {
        free(xr); free(cell_ptr); free(cellid); free(xc); free(pid); free(parent);
        return 3;
    }
    /* two-pass CRS: count, prefix, stable scatter in particle order */
    for (int32_t i = 0; i < np; ++i) {
        int64_t ix = cell_coord(xr[3 * i + 0], origin[0], size[0], Nx);
        int64_t iy = cell_coord(xr[3 * i + 1], origin[1], size[1], Ny);
        int64_t iz = cell_coord(xr[3 * i + 2], origin[2], size[2], Nz);
        int64_t c = (ix - 1) + Nx * ((iy - 1) + Ny * (iz - 1));
        cellid[i] = c;
        cell_ptr[c + 1]++;
    }
    for (int64_t c = 0; c < ncell; ++c) cell_ptr[c + 1] += cell_ptr[c];
    {
        int64_t *cursor = (int64_t *)malloc(sizeof(int64_t) * (size_t)ncell);
        if (!cursor) { free(xr); free(cell_ptr); free(cellid); free(xc); free(pid); free(parent); return 3; }
        memcpy(cursor, cell_ptr, sizeof(int64_t) * (size_t)ncell);
        for (int32_t i = 0; i < np; ++i) {
            int64_t p = cursor[cellid[i]]++;
            for (int d = 0; d < 3; ++d) xc[3 * p + d] = (float)xr[3 * i + d];
            pid[p] = istart + i;
        }
        free(cursor);
    }
    free(xr);
    free(cellid);
    for (int32_t p = 0; p < np; ++p) parent[p] = -1;

    /* link: same-cell upper triangle plus every adjacent cell visited once */
#define LINK_PAIR(P1, P2)                                                          \
    do {                                                                           \
        double r2_ = periodic ? dist2_pbc(xc + 3 * (P1), xc + 3 * (P2), L, half)   \
                              : dist2_open(xc + 3 * (P1), xc + 3 * (P2));          \
        if (r2_ <= rp2) {                                                          \
            if (nest > 1) dsu_union_atomic(parent, (int32_t)(P1), (int32_t)(P2));  \
            else dsu_union_serial(parent, (int32_t)(P1), (int32_t)(P2));           \
        }                                                                          \
    } while (0)

    char *layer_done = NULL;
    if (nest > 1) {
        layer_done = (char *)calloc((size_t)Nz, 1);
        if (!layer_done) { free(cell_ptr); free(xc); free(pid); free(parent); return 3; }
    }
#pragma omp parallel num_threads(nest) if (nest > 1)
    {
        int nth = omp_get_num_threads(), tid = omp_get_thread_num();
        int64_t my_start = (Nz * tid) / nth;
        for (int64_t step = 0; step < Nz; ++step) {
            int64_t iz = (nest > 1) ? (my_start + step) % Nz : step;
            if (nest > 1) {
                char claimed;
                __atomic_exchange(&layer_done[iz], &(char){1}, &claimed, __ATOMIC_RELAXED);
                if (claimed) continue;
            }
            for (int64_t iy = 0; iy < Ny; ++iy)
                for (int64_t ix = 0; ix < Nx; ++ix) {
                    int64_t ic = ix + Nx * (iy + Ny * iz);
                    int64_t b0 = cell_ptr[ic], e0 = cell_ptr[ic + 1];
                    if (b0 >= e0) continue;
                    for (int64_t p1 = b0; p1 < e0; ++p1)
                        for (int64_t p2 = p1 + 1; p2 < e0; ++p2) LINK_PAIR(p1, p2);
                    int64_t nbr[27];
                    int nn = 0;
                    if (!periodic) {
                        /* half stencil: offsets that precede (0,0,0) in x-fastest order */
                        for (int dz = -1; dz <= 0; ++dz)
                            for (int dy = -1; dy <= 1; ++dy)
                                for (int dx = -1; dx <= 1; ++dx) {
                                    if (dz == 0 && (dy > 0 || (dy == 0 && dx >= 0))) continue;
                                    int64_t jx = ix + dx, jy = iy + dy, jz = iz + dz;
                                    if (jx < 0 || jx >= Nx || jy < 0 || jy >= Ny || jz < 0 || jz >= Nz) continue;
                                    nbr[nn++] = jx + Nx * (jy + Ny * jz);
                                }
                    } else {
                        for (int dz = -1; dz <= 1; ++dz) {
                            if (!pdim[2] && (iz + dz < 0 || iz + dz >= Nz)) continue;
                            int64_t jz = ((iz + dz) % Nz + Nz) % Nz;
                            for (int dy = -1; dy <= 1; ++dy) {
                                if (!pdim[1] && (iy + dy < 0 || iy + dy >= Ny)) continue;
                                int64_t jy = ((iy + dy) % Ny + Ny) % Ny;
                                for (int dx = -1; dx <= 1; ++dx) {
                                    if (!pdim[0] && (ix + dx < 0 || ix + dx >= Nx)) continue;
                                    int64_t jx = ((ix + dx) % Nx + Nx) % Nx;
                                    int64_t jc = jx + Nx * (jy + Ny * jz);
                                    if (jc <= ic) continue;
                                    int dup = 0;
                                    for (int k = 0; k < nn; ++k) if (nbr[k] == jc) { dup = 1; break; }
                                    if (!dup) nbr[nn++] = jc;
                                }
                            }
                        }
                    }
                    for (int k = 0; k < nn; ++k) {
                        int64_t b1 = cell_ptr[nbr[k]], e1 = cell_ptr[nbr[k] + 1];
                        if (b1 >= e1) continue;
                        for (int64_t p1 = b0; p1 < e0; ++p1)
                            for (int64_t p2 = b1; p2 < e1; ++p2) LINK_PAIR(p1, p2);
                    }
                }
        }
    }
#undef LINK_PAIR
    free(layer_done);
    free(cell_ptr);

    /* root sizes, candidates in root (CRS) order, members in CRS order */
    int32_t *root_size = (int32_t *)calloc((size_t)np, sizeof(int32_t));
    int32_t *root_map = (int32_t *)calloc((size_t)np, sizeof(int32_t));
    if (!root_size || !root_map) { free(root_size); free(root_map); free(xc); free(pid); free(parent); return 3; }
    for (int32_t p = 0; p < np; ++p) root_size[dsu_find_root(parent, p)]++;
    int32_t ncand = 0;
    int64_t nmem = 0;
    for (int32_t r = 0; r < np; ++r)
        if (root_size[r] >= np_min) { root_map[r] = ++ncand; nmem += root_size[r]; }
    out->ncand = ncand;
    if (ncand > 0) {
        out->cand_np = (int32_t *)malloc(sizeof(int32_t) * (size_t)ncand);
        out->member_ptr = (int64_t *)malloc(sizeof(int64_t) * ((size_t)ncand + 1));
        out->cand_members = (int64_t *)malloc(sizeof(int64_t) * (size_t)nmem);
        out->xm = (float *)malloc(sizeof(float) * 3 * (size_t)ncand);
        out->vm = (float *)malloc(sizeof(float) * 3 * (size_t)ncand);
        int64_t *cursor = (int64_t *)malloc(sizeof(int64_t) * (size_t)ncand);
        if (!out->cand_np || !out->member_ptr || !out->cand_members || !out->xm || !out->vm || !cursor) {
            free(cursor); free(root_size); free(root_map); free(xc); free(pid); free(parent);
            return 3;
        }
        out->member_ptr[0] = 0;
        int32_t g = 0;
        for (int32_t r = 0; r < np; ++r)
            if (root_size[r] >= np_min) {
                out->cand_np[g] = root_size[r];
                out->member_ptr[g + 1] = out->member_ptr[g] + root_size[r];
                ++g;
            }
        memcpy(cursor, out->member_ptr, sizeof(int64_t) * (size_t)ncand);
        for (int32_t p = 0; p < np; ++p) {
            int32_t gg = root_map[dsu_find_root(parent, p)];
            if (gg > 0) out->cand_members[cursor[gg - 1]++] = pid[p];
        }
        free(cursor);
        for (g = 0; g < ncand; ++g) {
            const double *xa = xp + 3 * out->cand_members[out->member_ptr[g]];
            double w_sum = 0, qc[3] = {0, 0, 0}, vc[3] = {0, 0, 0};
            for (int64_t p = out->member_ptr[g]; p < out->member_ptr[g + 1]; ++p) {
                int64_t o = out->cand_members[p];
                double wi = mp[o];
                w_sum += wi;
                for (int d = 0; d < 3; ++d) {
                    double dx = oracle_modulo(xp[3 * o + d] - xa[d] + half, L) - half;
                    qc[d] += wi * dx;
                    vc[d] += wi * vp[3 * o + d];
                }
            }
            for (int d = 0; d < 3; ++d) {
                out->xm[3 * g + d] = w_sum > 0 ? (float)(qc[d] / w_sum) : 0.0f;
                out->vm[3 * g + d] = w_sum > 0 ? (float)(vc[d] / w_sum) : 0.0f;
            }
        }
    }
    free(root_size); free(root_map); free(xc); free(pid); free(parent);
    return 0;
}

static void free_cands(region_cands *c)
{
    free(c->cand_np); free(c->member_ptr); free(c->cand_members); free(c->xm); free(c->vm);
    memset(c, 0, sizeof(*c));
}

static int cmp_desc(const void *a, const void *b, void *ctx)
{
    const int32_t *np = (const int32_t *)ctx;
    int32_t x = np[*(const int32_t *)a], y = np[*(const int32_t *)b];
    return (x < y) - (x > y);
}

/* angular momentum of a member list about its weighted centre
 * (fof_fortran.f90:224-248 and :323-350) */
static void add_ang_mom(const double *xp, const double *vp, const double *mp, double L,
                        double half, int64_t anchor, const int64_t *mem, int64_t n,
                        double *am)
{
    const double *xa = xp + 3 * anchor;
    double w_sum = 0, qc[3] = {0, 0, 0}, vc[3] = {0, 0, 0};
    for (int64_t k = 0; k < n; ++k) {
        int64_t o = mem[k];
        double wi = mp[o];
        w_sum += wi;
        for (int d = 0; d < 3; ++d) {
            double dx = oracle_modulo(xp[3 * o + d] - xa[d] + half, L) - half;
            qc[d] += wi * dx;
            vc[d] += wi * vp[3 * o + d];
        }
    }
    if (!(w_sum > 0.0)) return;
    for (int d = 0; d < 3; ++d) { qc[d] /= w_sum; vc[d] /= w_sum; }
    for (int64_t k = 0; k < n; ++k) {
        int64_t o = mem[k];
        double wi = mp[o], dx[3], dv[3];
        for (int d = 0; d < 3; ++d) {
            dx[d] = (oracle_modulo(xp[3 * o + d] - xa[d] + half, L) - half) - qc[d];
            dv[d] = vp[3 * o + d] - vc[d];
        }
        am[0] = am[0] + wi * (dx[1] * dv[2] - dx[2] * dv[1]);
        am[1] = am[1] + wi * (dx[2] * dv[0] - dx[0] * dv[2]);
        am[2] = am[2] + wi * (dx[0] * dv[1] - dx[1] * dv[0]);
    }
}

int32_t oracle_fof_fortran(const double *xp, const double *vp, const double *mp,
                           const int32_t *np_halo, int32_t nhalo, int64_t total_np,
                           double L_Box, double link, int32_t np_halo_min,
                           int32_t bound_check, int32_t verbose, double softening,
                           double a_val, double b_val, double s15_val,
                           int32_t n_threads, int64_t ng_val, double ng_global_val,
                           int32_t *in_halo, int32_t *halo_id, double *ang_mom)
{
    return oracle_fof_fortran_diag(xp, vp, mp, np_halo, nhalo, total_np, L_Box, link,
                                   np_halo_min, bound_check, verbose, softening, a_val, b_val,
                                   s15_val, n_threads, ng_val, ng_global_val, in_halo, halo_id,
                                   ang_mom, NULL, NULL);
}

int32_t oracle_fof_fortran_diag(const double *xp, const double *vp, const double *mp,
                                const int32_t *np_halo, int32_t nhalo, int64_t total_np,
                                double L_Box, double link, int32_t np_halo_min,
                                int32_t bound_check, int32_t verbose, double softening,
                                double a_val, double b_val, double s15_val,
                                int32_t n_threads, int64_t ng_val, double ng_global_val,
                                int32_t *in_halo, int32_t *halo_id, double *ang_mom,
                                float *energy, float *phi_scale)
{
    if (energy)
        for (int64_t i = 0; i < total_np; ++i) { energy[i] = NAN; phi_scale[i] = NAN; }
    for (int64_t i = 0; i < total_np; ++i) { in_halo[i] = 0; halo_id[i] = 0; }
    for (int64_t i = 0; i < 3 * (int64_t)(nhalo > 0 ? nhalo : 0); ++i) ang_mom[i] = 0.0;
    if (n_threads > 256) return 10;
    if (nhalo <= 0 || total_np <= 0) return 0;
    int T = n_threads <= 0 ? omp_get_max_threads() : n_threads;
    if (T > 256) T = 256;
    g_last_threads = T;

    int32_t N_max = 0;
    for (int32_t h = 0; h < nhalo; ++h) if (np_halo[h] > N_max) N_max = np_halo[h];
    /* compute_fof_parallel_config (fof_fortran.f90:369-379) */
    int nest = (T >= 2 && (int64_t)nhalo <= 10 * (int64_t)T && N_max > 10000) ? 2 : 1;
    int team = T / nest;
    if (team < 1) team = 1;
    if (team > nhalo) team = nhalo;
    const double half = 0.5 * L_Box;

    int64_t *reg_start = (int64_t *)malloc(sizeof(int64_t) * (size_t)nhalo);
    int32_t *order = (int32_t *)malloc(sizeof(int32_t) * (size_t)nhalo);
    region_cands *rc = (region_cands *)calloc((size_t)nhalo, sizeof(region_cands));
    double *vzero = NULL;
    if (!reg_start || !order || !rc) { free(reg_start); free(order); free(rc); return 3; }
    reg_start[0] = 0;
    for (int32_t h = 0; h + 1 < nhalo; ++h) reg_start[h + 1] = reg_start[h] + np_halo[h];
    for (int32_t h = 0; h < nhalo; ++h) order[h] = h;
    qsort_r(order, (size_t)nhalo, sizeof(int32_t), cmp_desc, (void *)np_halo);
    if (!vp) {
        vzero = (double *)calloc(3 * (size_t)total_np, sizeof(double));
        if (!vzero) { free(reg_start); free(order); free(rc); return 3; }
        vp = vzero;
    }

    omp_set_max_active_levels(2);
    omp_set_dynamic(0);
    int ierr = 0;
#pragma omp parallel for num_threads(team) schedule(dynamic, 1) if (team > 1)
    for (int32_t k = 0; k < nhalo; ++k) {
        int32_t h = order[k];
        int32_t np = np_halo[h];
        if (np >= np_halo_min && np > 0) {
            int e = process_region(xp, vp, mp, reg_start[h], np, L_Box, half, link, np_halo_min,
                                   nest, &rc[h]);
            if (e) {
#pragma omp atomic write
                ierr = e;
            }
        }
    }
    if (ierr) goto done;

    if (!bound_check) {
        int32_t hid = 0;
        for (int32_t h = 0; h < nhalo; ++h)
            for (int32_t g = 0; g < rc[h].ncand; ++g) {
                ++hid;
                const int64_t *mem = rc[h].cand_members + rc[h].member_ptr[g];
                int64_t n = rc[h].member_ptr[g + 1] - rc[h].member_ptr[g];
                for (int64_t k = 0; k < n; ++k) { in_halo[mem[k]] = 1; halo_id[mem[k]] = hid; }
                add_ang_mom(xp, vp, mp, L_Box, half, mem[0], mem, n, ang_mom + 3 * h);
            }
    } else {
        int64_t ncand = 0, ntot = 0;
        for (int32_t h = 0; h < nhalo; ++h) {
            ncand += rc[h].ncand;
            if (rc[h].ncand) ntot += rc[h].member_ptr[rc[h].ncand];
        }
        if (ncand == 0) goto done;
        float *xv = (float *)malloc(sizeof(float) * 6 * (size_t)ntot);
        float *mpf = (float *)malloc(sizeof(float) * (size_t)ntot);
        int64_t *pid = (int64_t *)malloc(sizeof(int64_t) * (size_t)ntot);
        int32_t *cnp = (int32_t *)malloc(sizeof(int32_t) * (size_t)ncand);
        int32_t *creg = (int32_t *)malloc(sizeof(int32_t) * (size_t)ncand);
        int32_t *nb = (int32_t *)malloc(sizeof(int32_t) * (size_t)ncand);
        int32_t *st = (int32_t *)malloc(sizeof(int32_t) * (size_t)ncand);
        int32_t *fm = (int32_t *)malloc(sizeof(int32_t) * (size_t)ntot);
        int64_t *mem = (int64_t *)malloc(sizeof(int64_t) * (size_t)ntot);
        if (!xv || !mpf || !pid || !cnp || !creg || !nb || !st || !fm || !mem) {
            ierr = 3;
        } else {
            int64_t off = 0, c = 0;
            for (int32_t h = 0; h < nhalo; ++h)
                for (int32_t g = 0; g < rc[h].ncand; ++g, ++c) {
                    cnp[c] = rc[h].cand_np[g];
                    creg[c] = h;
                    const int64_t *m = rc[h].cand_members + rc[h].member_ptr[g];
                    const double *xa = xp + 3 * m[0];
                    for (int32_t p = 0; p < cnp[c]; ++p) {
                        int64_t o = m[p];
                        for (int d = 0; d < 3; ++d) {
                            xv[6 * (off + p) + d] =
                                (float)(oracle_modulo(xp[3 * o + d] - xa[d] + half, L_Box) - half);
                            xv[6 * (off + p) + 3 + d] = (float)vp[3 * o + d];
                        }
                        mpf[off + p] = (float)mp[o];
                        pid[off + p] = o + 1;
                    }
                    off += cnp[c];
                }
            float *etab = energy ? (float *)malloc(sizeof(float) * (size_t)ntot) : NULL;
            float *pmax = energy ? (float *)calloc((size_t)ncand, sizeof(float)) : NULL;
            ierr = oracle_bound_batch_diag(xv, mpf, pid, cnp, (int32_t)ncand, softening, a_val,
                                           b_val, s15_val, np_halo_min, verbose, T, ng_val,
                                           ng_global_val, nb, st, fm, NULL, NULL, etab, pmax);
            if (ierr == 0 && etab && pmax) {
                int64_t o2 = 0;
                for (int64_t cc = 0; cc < ncand; ++cc) {
                    for (int32_t k = 0; k < cnp[cc]; ++k) {
                        energy[pid[o2 + k] - 1] = etab[o2 + k];
                        phi_scale[pid[o2 + k] - 1] = pmax[cc];
                    }
                    o2 += cnp[cc];
                }
            }
            free(etab);
            free(pmax);
            if (ierr == 0) {
                int32_t valid = 0;
                off = 0;
                for (c = 0; c < ncand; ++c) {
                    if (st[c] == 0 && nb[c] >= np_halo_min) {
                        ++valid;
                        for (int32_t k = 0; k < nb[c]; ++k) {
                            int64_t o = pid[fm[off + k]] - 1;
                            mem[k] = o;
                            in_halo[o] = 1;
                            halo_id[o] = valid;
                        }
                        add_ang_mom(xp, vp, mp, L_Box, half, pid[off] - 1, mem, nb[c],
                                    ang_mom + 3 * creg[c]);
                    }
                    off += cnp[c];
                }
            }
        }
        free(xv); free(mpf); free(pid); free(cnp); free(creg); free(nb); free(st); free(fm); free(mem);
    }
done:
    if (ierr) {
        for (int64_t i = 0; i < total_np; ++i) { in_halo[i] = 0; halo_id[i] = 0; }
        for (int64_t i = 0; i < 3 * (int64_t)nhalo; ++i) ang_mom[i] = 0.0;
    }
    for (int32_t h = 0; h < nhalo; ++h) free_cands(&rc[h]);
    free(rc); free(order); free(reg_start); free(vzero);
    (void)verbose;
    return ierr;
}
