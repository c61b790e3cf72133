// sweep2d.cuh -- single-sweep (one fused pass per time step) 2D kernels and
// the kernel-family choice of the autotuner.
#pragma once
#include <cuda.h>

#include "solver2d_kernels.cuh"

namespace fomo {

// Work decomposition of one single-sweep launch.
struct SweepGeom {
  int nx, nz, ld;   // padded grid and row pitch
  long long plane;  // ld * nz
  int nbc;          // HABC zone
  int TX, W;        // strip width, TMA box width (TX + 2*halo, 8-aligned)
  int nstrip, ns;   // strips per shot, shots
};

// Upper bound on the persistent grid (size of the row-range table).
constexpr int kMaxGrid = 4096;

struct SweepPlan {
  int N = 0, variant = 0;
  int family = 0;            // 0: column-per-thread, 1: pair-blocked, 2: register-window
  int P = 0;                 // pair-blocked: prefetch depth (row pairs)
  int per_sm = 1, grid = 1;  // persistent CTAs per SM, grid size
  float frame_weight = 1.0f; // extra cost of a frame cell in the row-range split
  const long long* d_bounds = nullptr;  // [grid + 1] row ranges (device)
  size_t smem = 0;
  SweepGeom gm{};
  CUtensorMap tm[2][5];  // [ping-pong set][txx, tzz, txz, vx, vz]
};

// Kernel family for a problem (FOMO_KERNEL_TWO_PHASE / _SINGLE_SWEEP).
int pick_kernel_2d(int phys, int N, int nxp, int nzp, int ns);
bool sweep2d_supported(int phys, int N);
int sweep_num_variants();
// Candidate strip widths for a variant (multiples of 4 that fit its threads)
// on a padded grid nx columns wide.
int sweep_tx_candidates(int variant, int N, int nx, int* out, int max_out);
// per_sm: persistent CTAs per SM (capped by occupancy); each CTA owns a
// contiguous share of the flattened (strip, shot, row) space of equal
// estimated cost (frame cells weigh 1 + frame_weight); the row-range table is
// written to d_bounds (kMaxGrid + 1 entries) on stream st.
// sets: per ping-pong set the fields txx, tzz, txz, vx, vz.
cudaError_t make_sweep_plan(SweepPlan& sp, int N, int variant, int TX, int per_sm, const Geo2& g,
                            int ns, float* const sets[2][5], float frame_weight,
                            long long* d_bounds, cudaStream_t st);
cudaError_t launch_sweep_elastic(cudaStream_t st, const SweepPlan& sp, int set, const Coef& c,
                                 float dtx, float dtz, const HabcDev& h, const ElFields& a,
                                 const ElMat& m, const ElOut& o, int* err);
// Resident CTAs per SM for a plan (occupancy API).
int sweep_blocks_per_sm(const SweepPlan& sp);

}  // namespace fomo
