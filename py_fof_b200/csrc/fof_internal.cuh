// State shared between the FoF stages and the unbinding stage.
#pragma once

#include <vector>

#include "common.cuh"
#include "fof.cuh"

namespace pyfof {

// Slots of Context::d_flags.
// FLAG_VD: very dense cells linked by merge sub-cells in the last call
enum { FLAG_ERR = 0, FLAG_COUNT_A = 1, FLAG_COUNT_B = 2, FLAG_COUNT_C = 3, FLAG_VD = 4, FLAG_COUNT = 8 };

// One input region (one element of xp_list) with its reference cell grid.
struct RegionDev {
  double origin[3];
  double size[3];
  int64_t start;     // first particle (global index)
  int64_t ncell;     // Nx*Ny*Nz
  uint64_t cell_off; // first global cell key
  int32_t np;
  int32_t N[3];
  int32_t pdim;      // bit d set: axis d is periodic
  int32_t periodic;  // any axis periodic: dist2_pbc is used for every pair
  int32_t active;    // np >= np_halo_min
  int32_t sub_ok;    // dense cells of this region have more than one sub-cell
  int32_t sub[3];    // sub-cells per axis (each at least one linking length)
  float inv_sub[3];  // sub-cells per unit length
  // merge sub-cells of very dense cells (0: none in this region): per axis,
  // at most link/sqrt(3) less a rounding margin wide, so that every two
  // particles of one are linked by the exact distance test
  int32_t vd_k[3];
  float vd_inv[3];
};

struct Tile {
  int32_t region;
  int32_t pad;
  int64_t begin, end;
};

struct FofState {
  int64_t n = 0, n_active = 0;
  int nreg = 0;
  uint64_t total_cells = 0;
  std::vector<RegionDev> reg;
  RegionDev *dR = nullptr;
  float4 *pos = nullptr;      // sorted FP32 coordinates, .w = original index bits
  uint32_t *prid = nullptr;   // region of each sorted particle
  int *parent = nullptr;      // DSU forest over sorted positions
  int *lab = nullptr;         // root (minimum sorted position) of every particle
  uint32_t *skey = nullptr, *sidx = nullptr, *cell_start = nullptr, *keys_free = nullptr;
  uint32_t *gsize = nullptr, *flag = nullptr, *crank = nullptr;
  int32_t *pcand = nullptr;   // candidate of each sorted particle or -1
  uint32_t ncand = 0;
  int64_t *cand_anchor = nullptr;  // original index of each candidate's first CRS member
  int32_t *cand_region = nullptr, *cand_np = nullptr, *cand_root = nullptr;
  float *phi_out = nullptr;   // optional: final potential of every packed member
};

void region_geometry(double L, double link, int32_t np, const double *xmin, const double *xmax,
                     RegionDev &r);
int32_t fof_link_stage(Context &ctx, const FofArgs &a, FofState &st);
int32_t fof_candidates_stage(Context &ctx, const FofArgs &a, FofState &st, bool write_plain);
int32_t fof_plain_angmom(Context &ctx, const FofArgs &a, FofState &st);

}  // namespace pyfof
