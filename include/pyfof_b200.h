/*
 * libpyfof_b200 -- C-ABI of the B200 friends-of-friends + unbinding library.
 *
 * The library replaces the compiled extension module `fof_fortran` of
 * py_fof.  Its main entry point pyfof_run() has the argument list and the
 * error codes of the f2py binding of
 *     subroutine fof_fortran(xp_halo, vp_halo, mp_halo, np_halo, nhalo, L_Box,
 *        linking_length, np_halo_min, bound_check, verbose, softening, a_val,
 *        b_val, s_15_val, n_threads, total_np, in_halo, halo_id, ang_mom,
 *        ierr, ng_val, ng_global_val)          (fof_fortran.f90:10-58)
 * as called by _fof_core (py_fof/__init__.py:331-336), with the intent(out)
 * arrays passed in by the caller and ierr returned.
 *
 * Error codes (py_fof/__init__.py:338-348): 0 ok, 1 invalid input or
 * configuration, 2 candidate span exceeds s_15, 3 allocation failure,
 * 4 non-finite values, 10 n_threads > 256, 20 CUDA runtime failure.
 * pyfof_last_error() returns a message for the calling thread's last error.
 *
 * All pointers are plain host pointers unless the function name says
 * "device".  The caller owns every buffer; nothing is retained after return.
 * Calls on one device are serialised internally; the library keeps device
 * memory cached between calls.
 */
#ifndef PYFOF_B200_H
#define PYFOF_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PYFOF_B200_ABI_VERSION 2

/* Memory layout of the (3,N) float64 coordinate/velocity arrays. */
#define PYFOF_LAYOUT_AOS 0 /* Fortran order, x[3*i+d]: the f2py xp_halo layout */
#define PYFOF_LAYOUT_SOA 1 /* C order,       x[d*N+i]: numpy hstack output */

/* ABI version of the loaded library (PYFOF_B200_ABI_VERSION). */
int32_t pyfof_version(void);

/* Select the CUDA device used by later calls and create its context.
 * No reference counterpart (the reference is a CPU module). */
int32_t pyfof_init(int32_t device);

/* Release all device contexts and cached device memory. */
int32_t pyfof_shutdown(void);

/* Copies the calling thread's last error message into buf (NUL-terminated,
 * truncated to len) and returns its full length. */
int32_t pyfof_last_error(char *buf, int64_t len);

/* Library options: "unbind_fp64" (1 = FP64 unbinding, batched, the
 * default: the direct sums of candidates up to 1000 members reproduce the
 * reference's FP64 arithmetic bit for bit; 0 = the FP32 product path, whose
 * potentials differ by FP32 rounding, so particles with a specific energy
 * within about 1e-5 of the halo's |phi| scale of zero may be classified
 * differently), "unbind_per_halo" (1 = the plain FP64 baseline: one halo per
 * launch sequence), "timing" (1 = record stage times), "unbind_big_np"
 * (particle-mesh halos above this many members run their removal loop
 * spread over the whole GPU; 0 = the default of 32768), "cell_order" (how
 * the particles are put in cell order: 0 = per-cell sorts when cell keys
 * need more than 24 bits and no cell holds more than 8192 particles, else a
 * radix sort; 1 = per-cell sorts whenever no cell holds more than 8192; 2 =
 * always the radix sort; all give the same order). */
int32_t pyfof_set_option(const char *key, int64_t value);

/* Current value of a pyfof_set_option key.  No reference counterpart. */
int32_t pyfof_get_option(const char *key, int64_t *value);

/* Tile table: launch shapes that never change a result, tuned per device
 * by py_fof_b200.autotune (the reference's counterpart is its per-group
 * thread split, bound_fortran.f90:332-401).  Keys: "direct_threads" (index
 * = halo-size bucket 0..5 for halos of at most 32, 64, 128, 256, 512, 1000
 * members; value 32, 64, 128 or 256 threads per block of the
 * direct-summation removal loop), "pm_batch" (index = PM grid size 48, 64,
 * 128, 216 or 256; value = halos per convolution batch, 0 = as many as the
 * batch memory budget allows), "conv_waves" (index = grid size; value 1..64
 * = full GPU waves the fused z pass of a convolution is split into at
 * least).  Invalid keys or values give ierr 1 with a message. */
int32_t pyfof_set_tile(const char *key, int64_t index, int64_t value);
int32_t pyfof_get_tile(const char *key, int64_t index, int64_t *value);

/* Issue all later work of the selected device on `stream` (a cudaStream_t;
 * NULL restores the library's own stream).  Lets a caller order calls with
 * its own work and time them with events on that stream. */
int32_t pyfof_set_stream(void *stream);

/* Page-locked host memory for a caller's input staging: a list of regions
 * is concatenated into one array before the call (the reference does so in
 * NumPy, py_fof/__init__.py:213-231); concatenated into this memory, which
 * a caller keeps and reuses, it is not page-faulted again on every call and
 * copies to the device at the host link's full rate.  Free with
 * pyfof_host_free. */
int32_t pyfof_host_alloc(int64_t bytes, void **ptr);
int32_t pyfof_host_free(void *ptr);


/* Counters: "launches" (kernels launched by this process so far), and for
 * the last call on the selected device "cells" (reference cell grid size),
 * "active" (particles in linked regions), "candidates" (FoF groups with at
 * least np_halo_min members), "dense_cells" (cells given a sub-cell index),
 * "max_cell" (particles in the fullest cell), "vd_cells" (very dense cells,
 * linked by merge sub-cells narrower than link/sqrt(3)), "cell_sorts" (1 when the
 * cell order came from per-cell sorts, 0 from the radix sort),
 * "direct_halos" / "pm_halos" (candidates unbound by direct summation / the
 * particle mesh), "valid_halos" (halos written to the output),
 * "refined_regions" (two-level inner regions), "pm_passes" (passes of the
 * particle-mesh removal loop), "pm_solves" (halo-grid
 * convolutions over all passes), "pm_fft_bytes" (their algorithmic bytes:
 * 4 s (n+2) n^2 per solve on an n^3 grid of s-byte reals: a read and a
 * write of the padded grid per transform, two transforms). */
int32_t pyfof_get_stat(const char *key, int64_t *value);

/* Device time of the linking kernel of the last call, when timing is on. */
int32_t pyfof_last_link_ms(float *ms);

/* Device time (ms) of one stage of the last call, when timing is on:
 * "link" (the linking kernel), "fof" (binning, linking and labelling up to
 * the candidate list), "unbind" (unbinding and outputs with bound_check, the
 * ang_mom pass without), "call" (all of it), "pm_fft" (the particle-mesh
 * convolutions, summed over all solves), "pm_gaps" (device idle time
 * between the passes of the particle-mesh removal loop, while the host reads
 * a pass's results and launches the next), "before_link" / "after_link"
 * (the parts of "fof" before and after the linking kernel), "direct_loops"
 * / "pm_path" (from the fork of the direct-summation removal loops onto
 * their side stream: the loops, and the particle-mesh halos on the call
 * stream; 0 when nothing forked); after a
 * host-memory call also
 * "h2d_positions" (the copy of xp), "h2d_inputs" (from the first copy to the
 * end of the last input copy), "d2h" (the output copy after the device work)
 * and "host_call" (from the first input copy to the end of the output copy). */
int32_t pyfof_last_stage_ms(const char *stage, float *ms);

/* First-pass gravitational potential of one candidate, computed by the
 * solver the reference rules select for it (bound_select_grid_and_level,
 * bound_fortran.f90:1963): FP64 direct summation for np <= 1000
 * (:2613-2647), particle-mesh C1 + C2 otherwise (:2657-2735).  Diagnostic
 * counterpart of the first pass of bound_check_grid; no removal happens.
 *   q    (3,np) float32 C order: member positions relative to member 0, in
 *        stable-id order
 *   w    (np) float32 masses
 *   fp64 1 = plain FP64 path, 0 = FP32 product path
 *   phi  (np) output potential; *method = 0 direct, 1..4 PM grid class. */
int32_t pyfof_halo_potential(const float *q, const float *w, int32_t np, double softening,
                             double a_val, double s_15_val, int64_t ng_val, int32_t fp64,
                             float *phi, int32_t *method);

/* Allocation-free variant of pyfof_halo_potential for direct-summation
 * candidates (np <= 1000).  No counterpart in the reference: it exists for
 * callers that must not allocate device memory while running, e.g. a host
 * framework whose caching allocator already owns the device memory, or a
 * latency-bound loop that cannot afford an allocation failing mid-step.
 * All device scratch lives in a static array of the library (about 42 KiB
 * per GPU, held until exit); inputs q (3,np), w (np) and the output phi (np)
 * are host arrays as in pyfof_halo_potential; `stream` is a cudaStream_t
 * (NULL = legacy default stream).  Returns 1 for np > 1000.  The first call
 * on a device looks up the array's address; calls share the array, so calls
 * that overlap on the GPU race. */
int32_t pyfof_halo_potential_direct_static(const float *q, const float *w, int32_t np,
                                           double softening, double a_val, int32_t fp64,
                                           float *phi, void *stream);

/* Replaces fof_fortran.fof_fortran (fof_fortran.f90:10-58).
 *   xp, vp    (3,total_np) float64 in `layout`; vp may be NULL (all zero,
 *             the value _fof_core passes when vp_list is None,
 *             py_fof/__init__.py:233), but not when bound_check != 0
 *   mp        (total_np) float64, NULL means unit masses
 *   np_halo   (nhalo) particle count of every input region
 *   in_halo, halo_id  (total_np) int32 outputs; ang_mom (3,nhalo) float64
 *             Fortran order (ang_mom[3*h+d]) output; all three are written
 *             in full on success and zeroed on failure.  in_halo may be
 *             NULL: it equals halo_id > 0, so a caller can save its copy
 * Returns ierr: the reference codes (0 ok, 1 invalid input, 2 span above
 * s_15, 3 allocation, 4 non-finite, 10 n_threads > 256), plus 5 when a mass
 * is not positive and finite (the reference raises that in Python before
 * its call, py_fof/__init__.py:259-260; here the device checks it) and 20
 * for a CUDA failure (pyfof_last_error has the detail).  Positions are
 * copied first; velocity and mass copies overlap with the linking. */
int32_t pyfof_run(const double *xp, const double *vp, const double *mp, int32_t layout,
                  const int32_t *np_halo, int32_t nhalo, int64_t total_np, double L_Box,
                  double linking_length, int32_t np_halo_min, int32_t bound_check,
                  int32_t verbose, double softening, double a_val, double b_val,
                  double s_15_val, int32_t n_threads, int64_t ng_val, double ng_global_val,
                  int32_t *in_halo, int32_t *halo_id, double *ang_mom);

/* Same as pyfof_run with xp/vp/mp/in_halo/halo_id in device memory of the
 * selected device (np_halo and ang_mom stay on the host).  The inputs must
 * be complete before the call (synchronise the producing stream). */
int32_t pyfof_run_device(const double *d_xp, const double *d_vp, const double *d_mp,
                         int32_t layout, const int32_t *np_halo, int32_t nhalo, int64_t total_np,
                         double L_Box, double linking_length, int32_t np_halo_min,
                         int32_t bound_check, int32_t verbose, double softening, double a_val,
                         double b_val, double s_15_val, int32_t n_threads, int64_t ng_val,
                         double ng_global_val, int32_t *d_in_halo, int32_t *d_halo_id,
                         double *ang_mom);

/* Conversion of the inputs to code units, applied on the device after the
 * host-to-device copy.  The reference converts on the host before its call
 * (py_fof/__init__.py:266-326, units='physical'): positions / dx,
 * velocities * v_scale, masses / m_grid, or the constant mass
 * ng_eff^3 / n_sim when only n_sim is given.  The same IEEE operations on
 * the device give the same bits.  Masses are checked (positive, finite)
 * before the division, as the reference checks mp_list before converting.
 * {1, 1, 1, 1} converts nothing. */
typedef struct pyfof_units {
  double x_div;   /* positions are divided by x_div */
  double v_mul;   /* velocities are multiplied by v_mul */
  double m_div;   /* masses (mp != NULL) are divided by m_div */
  double m_const; /* the mass of every particle when mp is NULL */
} pyfof_units_t;

/* pyfof_run with the inputs in the caller's units, converted on the device
 * (`units` may be NULL: none).  slot: a slot handle or NULL (default
 * context); in_halo may be NULL (it is halo_id > 0). */
int32_t pyfof_run_units(void *slot, const pyfof_units_t *units, const double *xp, const double *vp,
                        const double *mp, int32_t layout, const int32_t *np_halo, int32_t nhalo,
                        int64_t total_np, double L_Box, double linking_length, int32_t np_halo_min,
                        int32_t bound_check, int32_t verbose, double softening, double a_val,
                        double b_val, double s_15_val, int32_t n_threads, int64_t ng_val,
                        double ng_global_val, int32_t *in_halo, int32_t *halo_id, double *ang_mom);

/* py_fof.fof (py_fof/__init__.py:354-447) returns in_halo alone: this is
 * pyfof_run_units with in_halo as one byte per particle (0 or 1, a numpy
 * bool array's layout) and no halo_id, so a quarter of the output bytes
 * cross back to the host.  ang_mom, units, slot and ierr as in
 * pyfof_run_units; in_halo is written in full on success and zeroed on
 * failure. */
int32_t pyfof_run_mask(void *slot, const pyfof_units_t *units, const double *xp, const double *vp,
                       const double *mp, int32_t layout, const int32_t *np_halo, int32_t nhalo,
                       int64_t total_np, double L_Box, double linking_length, int32_t np_halo_min,
                       int32_t bound_check, int32_t verbose, double softening, double a_val,
                       double b_val, double s_15_val, int32_t n_threads, int64_t ng_val,
                       double ng_global_val, uint8_t *in_halo, double *ang_mom);

/* fof_with_info on the device (py_fof/__init__.py:481-518): pyfof_run
 * (without in_halo, which is halo_id > 0) that also returns the halo
 * catalogue: members[0 .. offsets[n]) holds the particle indices of every
 * valid halo, ascending within a halo, halos in id order, and
 * offsets[h] .. offsets[h+1] delimits halo h+1 (n = *nhalo_found halos;
 * members needs total_np entries, offsets n+1, at most total_np /
 * max(1, np_halo_min) + 1).  slot: a slot handle or NULL (default context);
 * units: as in pyfof_run_units, or NULL.  Returns ierr like pyfof_run. */
int32_t pyfof_run_catalogue(void *slot, const pyfof_units_t *units, const double *xp, const double *vp,
                            const double *mp,
                            int32_t layout, const int32_t *np_halo, int32_t nhalo, int64_t total_np,
                            double L_Box, double linking_length, int32_t np_halo_min, int32_t bound_check,
                            int32_t verbose, double softening, double a_val, double b_val, double s_15_val,
                            int32_t n_threads, int64_t ng_val, double ng_global_val, int32_t *halo_id,
                            double *ang_mom, int32_t *members, int64_t *offsets, int64_t offsets_cap,
                            int32_t *nhalo_found);

/* Slots: contexts of their own (CUDA streams, device scratch, status
 * words) on one device, for callers that run several calls at once — the
 * serving loop of py_fof_b200.serve runs one host thread per slot, so the
 * calls of different slots overlap on the GPU.  No counterpart in the
 * reference (its f2py module is not re-entrant).  pm_budget_bytes bounds
 * the particle-mesh grid batches of the slot (0: the default of 8 GB).
 * Calls on one slot are serialised; slots share the device's Green tables. */
int32_t pyfof_slot_create(int32_t device, int64_t pm_budget_bytes, void **slot);
int32_t pyfof_slot_destroy(void *slot);

/* pyfof_run on a slot (same arguments, outputs and error codes). */
int32_t pyfof_slot_run(void *slot, const double *xp, const double *vp, const double *mp,
                       int32_t layout, const int32_t *np_halo, int32_t nhalo, int64_t total_np,
                       double L_Box, double linking_length, int32_t np_halo_min, int32_t bound_check,
                       int32_t verbose, double softening, double a_val, double b_val, double s_15_val,
                       int32_t n_threads, int64_t ng_val, double ng_global_val, int32_t *in_halo,
                       int32_t *halo_id, double *ang_mom);

/* Statistics of the slot's last call (the pyfof_get_stat keys), plus
 * "peak_bytes": the most device memory that call held at once. */
int32_t pyfof_slot_stat(void *slot, const char *key, int64_t *value);

#ifdef __cplusplus
}
#endif
#endif
