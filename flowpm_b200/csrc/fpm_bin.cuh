// Eulerian binning of the particles (fpm_bin.cu): counting sort by
// force-mesh cell and the binned leapfrog step, used by the plan
// orchestration in fpm_plan.cu.
#pragma once

#include "fpm_kernels.cuh"

namespace fpm {

// One run of a plan (consecutive simulations of equal shape) as the sort
// kernels see it: slot p0 + r * np + t is particle t of simulation r, whose
// force-mesh cells start at m0 + r * ncell.
struct BinRun {
  int nx, ny, nz, bf, mx, my, mz;
  int ntx, nty, ntz;       // tiles per axis
  int count;               // simulations
  int qkb, qjb;            // bit widths of the packed lattice site
  int64_t np, ncell, p0, m0;
};

// Whether a run of `count` simulations of this shape can be binned: the
// packed lattice site fits 32 bits and every run-relative cell key stays
// below the sentinels the sort kernels keep for lanes past the end.
bool bin_run_supported(int nx, int ny, int nz, int64_t ncell, int count,
                       int* qkb, int* qjb);

// Particle arrays a sort moves: n float3 arrays (2: displacement and
// momentum; 4: displacement, momentum and the two cotangents of the
// reverse sweep), src[0] the displacement the cell keys come from.
struct BinPayload {
  int n;
  const float* src[4];
  float* dst[4];
};

// Tile sizes the binned step is built for (8 or 16 cells per side) and
// whether a force mesh divides into them.
bool bin_tile_supported(int tile, int mx, int my, int mz);

// Chunk sums the scan of ncells cell counts needs.
size_t bin_scan_blocks(int64_t ncells);

// Counting sort of the run's particles by tile-major cell key: cell counts
// into count[m0 ..) (all zero on entry, and left zero), their exclusive
// scan (plus p0: absolute slots) into cell[m0 ..), then the scatter of
// (d, p, packed lattice site) into the output arrays; afterwards cell[c]
// holds the end slot of cell c.  lag NULL: the input is in Lagrangian
// order (slot p0 + r np + t is lattice site t); the index written is the
// packed lattice site (pack_site).  counted: the counts are already in
// count (a step kernel made them), only the scan and the scatter run.
// sums: at least bin_scan_blocks(count * ncell) ints.
int launch_bin_sort(int tile, const BinRun& R, const float* d,
                    const float* p, const uint32_t* lag, int32_t* count,
                    int32_t* cell, int32_t* sums, float* d_out, float* p_out,
                    uint32_t* lag_out, bool counted, cudaStream_t st);

// The first half of a sort: counts of the cells of (d, lag) -- lag NULL:
// Lagrangian order -- into count (zero on entry), scanned into cell (the
// first slot of each cell, plus p0) with count left zero.
int launch_bin_count_scan(int tile, const BinRun& R, const float* d,
                          const uint32_t* lag, int32_t* count, int32_t* cell,
                          int32_t* sums, cudaStream_t st);

// The scan alone (counts already in count, left zero).
int launch_bin_scan(const BinRun& R, int32_t* count, int32_t* cell,
                    int32_t* sums, cudaStream_t st);

// The same sort of the payload's arrays.
int launch_bin_sort(int tile, const BinRun& R, const BinPayload& pay,
                    const uint32_t* lag, int32_t* count, int32_t* cell,
                    int32_t* sums, uint32_t* lag_out, cudaStream_t st);

// Sorted slots back to Lagrangian order (payload of 4 arrays): the slot of
// simulation r holding packed site (i, j, k) goes to p0 + r np +
// (i ny + j) nz + k.
int launch_bin_unsort(const BinRun& R, const BinPayload& pay,
                      const uint32_t* lag, cudaStream_t st);

// State of the binned step: the sorted particles (updated in place), their
// packed lattice sites and the cells' end slots of the last sort.  The
// StepArgs' disp, mom and force_out are the caller's Lagrangian arrays,
// written at the last step (and ckpt / inter through the index).
struct BinStepArgs {
  StepArgs a;
  float* bd;
  float* bp;
  const uint32_t* blag;
  const int32_t* cell_end;
  // k_step_sorted only: when set, the cells of the drifted particles are
  // counted into count (keys tile-major in tiles of 2^tile_log2 cells, per
  // simulation at its m_off) for the sort that follows the step
  int32_t* count;
  int tile_log2;
  // k_step_sorted only, the particles re-sorted as they move (FPM_BIN_FLOW):
  // with claim set, each particle claims claim[key of its cell at the start
  // of the step]++ (the scan of the previous step's counts) and writes its
  // updated (d, p, site) there in (od, op, olag) instead of in place; with
  // blag NULL the input (bd, bp) is in Lagrangian order
  int32_t* claim;
  float* od;
  float* op;
  uint32_t* olag;
};

// The step over the tile chunks [ch0, ch1) (whole simulations), painting
// through shared-memory tiles.
void launch_step_binned(int tile, const SimDev* sims, int nsims, int64_t ch0,
                        int64_t ch1, const BinStepArgs& b, cudaStream_t st);

// The step over the sorted particles in equal chunks (the particle chunks
// [ch0, ch1), whole simulations), painting straight into the density with
// warp-segmented sums of equal deposits.
void launch_step_sorted(const SimDev* sims, int nsims, int64_t ch0,
                        int64_t ch1, const BinStepArgs& b, cudaStream_t st);

}  // namespace fpm
