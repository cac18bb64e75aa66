/*
 * CPU oracle for the py_fof hot paths -- TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference algorithm (friends-of-friends
 * linking in fof_fortran.f90 + atomic_dsu.c, gravitational unbinding in
 * bound_fortran.f90).  It exists to check the CUDA product path and to serve
 * as the timed CPU baseline.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it; the product library never does.
 *
 * Arrays follow the reference layout: xp/vp are (3,N) Fortran-order, i.e.
 * particle i, axis d lives at xp[3*i+d]; ang_mom is (3,nhalo) Fortran-order.
 * Particle and candidate indices in the public entry points are 0-based.
 */
#ifndef PYFOF_ORACLE_H
#define PYFOF_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Full restatement of fof_fortran (fof_fortran.f90:10-362).  Returns ierr. */
int32_t oracle_fof_fortran(const double *xp, const double *vp, const double *mp,
                           const int32_t *np_halo, int32_t nhalo, int64_t total_np,
                           double L_Box, double link, int32_t np_halo_min,
                           int32_t bound_check, int32_t verbose, double softening,
                           double a_val, double b_val, double s15_val,
                           int32_t n_threads, int64_t ng_val, double ng_global_val,
                           int32_t *in_halo, int32_t *halo_id, double *ang_mom);

/* oracle_fof_fortran plus diagnostics of the unbinding (both may be NULL):
 * energy[i] = the specific energy of candidate member i at its last
 * evaluation in the removal loop (kept: the final one; removed: the one that
 * removed it), phi_scale[i] = max |phi| of its candidate's first-pass
 * potential; NaN for particles of no candidate.  The tests bound the
 * energies of members the GPU classifies differently with them. */
int32_t oracle_fof_fortran_diag(const double *xp, const double *vp, const double *mp,
                                const int32_t *np_halo, int32_t nhalo, int64_t total_np,
                                double L_Box, double link, int32_t np_halo_min,
                                int32_t bound_check, int32_t verbose, double softening,
                                double a_val, double b_val, double s15_val,
                                int32_t n_threads, int64_t ng_val, double ng_global_val,
                                int32_t *in_halo, int32_t *halo_id, double *ang_mom,
                                float *energy, float *phi_scale);

/* Thread count actually used by the last oracle_fof_fortran call. */
int32_t oracle_last_threads(void);

/* Unbinding batch on pre-packed candidates (bound_fortran.f90:1527-1813).
 * xv: (6,ncand_np) F-order FP32 (pos relative to candidate anchor, vel),
 * mp: FP32 masses, pid: 1-based stable ids, cand_np[h]: member count of
 * candidate h, members stored contiguously in candidate order.
 * Outputs: np_bound[h], status[h]; final_members: for status==0 candidates,
 * the kept members' 0-based positions in xv, written at the candidate's
 * offset in ascending pid order.  phi_out (optional, may be NULL): final
 * FP32 potential per member at the candidate's offset, in pid order.
 * method_out (optional): chosen method gid per candidate (0 direct, 1..4 PM).
 * Returns ierr. */
int32_t oracle_bound_batch(const float *xv, const float *mp, const int64_t *pid,
                           const int32_t *cand_np, int32_t ncand,
                           double softening, double a_val, double b_val, double s15,
                           int32_t np_halo_min, int32_t verbose, int32_t n_threads,
                           int64_t ng_val, double ng_global_val,
                           int32_t *np_bound, int32_t *status, int32_t *final_members,
                           float *phi_out, int32_t *method_out);

/* oracle_bound_batch plus diagnostics (both may be NULL): energy_tab[k] =
 * the last specific energy of the member at table position k, phimax[h] =
 * max |phi| of candidate h's first-pass potential. */
int32_t oracle_bound_batch_diag(const float *xv, const float *mp, const int64_t *pid,
                                const int32_t *cand_np, int32_t ncand,
                                double softening, double a_val, double b_val, double s15,
                                int32_t np_halo_min, int32_t verbose, int32_t n_threads,
                                int64_t ng_val, double ng_global_val,
                                int32_t *np_bound, int32_t *status, int32_t *final_members,
                                float *phi_out, int32_t *method_out, float *energy_tab,
                                float *phimax);

/* First-pass potential of one candidate with the reference solver selected by
 * the reference rules (direct FP64 sum or PM+C2), members in pid order;
 * phi[i] is FP32 as used for the energy test.  Returns method gid, <0 on error. */
int32_t oracle_bound_first_potential(const float *xv, const float *mp, const int64_t *pid,
                                     int32_t np, double softening, double a_val,
                                     double s15, int64_t ng_val, float *phi);

/* Exact FP64 softened direct-sum potential (all pairs, same kernel as the
 * reference direct path) for physics error reports. */
void oracle_direct_potential_f64(const float *q, const float *w, int32_t np,
                                 double softening, double a_val, double *phi);

/* Green's function (bound_fortran.f90:2300-2382): half-spectrum table
 * green[(k*n + j)*(n/2+1) + i] (FP32, real part only) and 5x5x5 self
 * kernel self[(iz+2)*25 + (iy+2)*5 + (ix+2)].  Returns 0 on success. */
int32_t oracle_green_and_self(int32_t n, double apm_soft, double apm_range,
                              int32_t truncated, float *green, float *self_out);

/* gfortran MODULO for reals, exposed for unit tests. */
double oracle_modulo(double a, double p);

#ifdef __cplusplus
}
#endif
#endif
