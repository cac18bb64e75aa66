// Shared declarations of the unbinding stage.
#pragma once

#include <vector>

#include "fof_internal.cuh"

namespace pyfof {

constexpr int kMaxPasses = 20;     // bound_max_passes (bound_fortran.f90:231)
constexpr int kDirectMax = 1024;   // direct summation handles N <= 1000
constexpr size_t kDirectSmem = 11 * kDirectMax * 4 + kDirectMax * 8 + kDirectMax;

// Packed members of all candidates, candidate-major, ascending global index
// inside a candidate (the xv/mp/pid arrays of fof_fortran.f90:265-305).
struct Members {
  float *q[3];    // position relative to the candidate anchor (FP32)
  float *v[3];    // velocity (FP32)
  float *w;       // mass (FP32)
  int32_t *pid;   // global particle index
};

struct HaloTask {
  int64_t off;      // first member
  int32_t np;
  int32_t gid;      // 0 direct summation, 1..4 particle-mesh grid class
  int32_t n;        // grid points per axis of the PM grid
  float spacing;    // PM grid spacing (standard grid units, FP32)
  float origin[3];  // PM source-domain origin relative to the anchor
};

struct HaloResult {
  int32_t status;   // 0 converged, 1 too few members, 5 max passes
  int32_t np_bound; // members kept
};

// Grid classes, spacing levels and the selection rules of
// bound_select_grid_and_level (bound_fortran.f90:1854-2040).
struct GridRules {
  int64_t ng = 256;
  int ngrid = 4;
  int bn[4] = {48, 64, 128, 256};
  double s15 = 0.0, spacing_max = 0.0;
  std::vector<double> levels[4];
  std::vector<int> ladder_g, ladder_l;
  std::vector<double> ladder_cov;
  void init(int64_t ng, double s15);
  double coverage(int g, int l) const;
  bool select(int64_t np, double span, int &gid, int &lev, double &sp) const;
};

// Particle-mesh halos (gid >= 1): unbind_pm.cu.
int32_t unbind_pm(Context &ctx, const FofArgs &a, const GridRules &rules, const Members &m,
                  const std::vector<HaloTask> &tasks, const std::vector<int32_t> &list,
                  HaloResult *res, uint8_t *keep, float *phi_out, int phi_only);

// First-pass potential of one halo (members in stable-id order, positions
// relative to the first member), by the solver the reference rules select.
int32_t unbind_potential(Context &ctx, const float *q_soa, const float *w, int32_t np,
                         double softening, double a_val, double s15, int64_t ng, int fp64,
                         float *phi, int32_t *method);

}  // namespace pyfof
