// sweep3d.cuh -- 3D grid geometry and the fused, TMA-staged 3D half steps
// (sweep3d.cu): each launch updates one field group (velocities, or stresses /
// pressure) and applies the Higdon boundary to it in the same pass.
#pragma once
#include <cuda.h>

#include <algorithm>
#include <vector>

#include "fomo_internal.cuh"

namespace fomo {

// Higdon weight ramps of the 3D boundary for the offsets 0, .25, .5, .75
// (habc_3d.jl:40-43): w = clamp((d - offset) / (pad - 1), 0, 1) for distances
// d = 0 .. wstride - 1, one ramp after the other.
inline std::vector<float> habc3_ramps(int pad, int wstride) {
  std::vector<float> wt(4 * (size_t)wstride);
  const double offs[4] = {0.0, 0.25, 0.5, 0.75};
  for (int k = 0; k < 4; ++k)
    for (int d = 0; d < wstride; ++d) {
      const double w = ((double)d - offs[k]) / (double)(pad - 1);
      wt[(size_t)k * wstride + d] = (float)std::min(std::max(w, 0.0), 1.0);
    }
  return wt;
}

// Padded 3D grid: x fastest, then y, then z; every field is one pitched volume.
struct Geo3 {
  int nx, ny, nz;       // padded
  int ld;               // x pitch
  long long sy, sz;     // strides of y and z (ld, ld*ny)
  long long vol;        // sz * nz
  int M, nbc;           // half stencil; HABC zone (pad - 1)
  // z-slabs of one model (fomo_slab3d): the volume holds global padded planes
  // [z0, z0 + nz) of a grid of gnz planes and updates its local planes
  // [zlo, zhi).  The whole grid is z0 = 0, gnz = nz, [0, nz).
  int z0 = 0, gnz = 0;
  int zlo = 0, zhi = 0;
};

// Work split of the fused half steps.  A CTA of 32 x 16 threads owns a tile of
// 30 x 14 output columns plus a one-column ring on every side (the ring's
// updated values feed the Higdon terms of the tile's edge cells) and marches
// down z.  Persistent CTAs (one or two per SM) take segments {tile x, tile y,
// z0, z1} from a list through a counter in device memory.
struct Fused3Plan {
  int N = 0;
  bool elastic = true;           // elastic3d (9 fields a set) or acoustic3d (4)
  int ntx = 0, nty = 0;          // tiles in x and y
  int grid_v = 0, grid_s = 0;    // persistent CTAs of the two half steps
  size_t smem_v = 0, smem_s = 0; // dynamic shared memory of the two kernels
  int4* d_segs = nullptr;        // segments in the order they are handed out
  int nseg = 0;
  int* d_sched = nullptr;        // [next segment, CTAs done]; zero between launches
  // tensor maps over the two field sets (4D: x, y, z, set * 9 + field) and the
  // materials (x, y, z, material)
  CUtensorMap c1, c3, c6, xh, yh, xyh, xyh3, m1, m3, m5;
};

// Whether the fused form runs for half-stencil N (TMA tensor-map encoder present).
bool fused3_supported(int N);
// Device bytes of the segment table for grid g.
size_t fused3_table_bytes(const Geo3& g);
// Builds the plan for the state `state` (2 sets x 9 fields of g.vol floats:
// vx vy vz txx tyy tzz txy txz tyz; acoustic: 2 sets x vx vy vz p) and the
// materials `mat` (bx by bz lam l2m mxy mxz myz; acoustic: bx by bz kappa);
// d_table: fused3_table_bytes(g) bytes of device memory, 256-byte aligned.
// Synchronizes `st`.
cudaError_t fused3_make_plan(Fused3Plan& p, const Geo3& g, int N, bool elastic, float* state,
                             const float* mat, void* d_table, cudaStream_t st);
// Velocity half step: set A -> B.v (update + Higdon).  Stress / pressure half
// step: A's stresses (pressure) and B.v -> B (update + Higdon).  err collects
// bounded-wait timeouts.
cudaError_t fused3_velocity(cudaStream_t st, const Fused3Plan& p, const Geo3& g, float* state,
                            int A, int B, const Coef& c, float dtdh, const HabcDev& h, int* err);
cudaError_t fused3_stress(cudaStream_t st, const Fused3Plan& p, const Geo3& g, float* state,
                          int A, int B, const Coef& c, float dtdh, const HabcDev& h, int* err);

// Materials (bx by bz lam l2m mxy mxz myz; acoustic bx by bz kappa) of the
// volume g (global padded planes g.z0 .. g.z0 + g.nz of g.gnz) from raw
// interior models of nx x ny x nz cells padded by `pad`, whose device arrays
// hold the raw planes from kz0 on (solver3d.cu).
cudaError_t medium3d(cudaStream_t st, bool elastic, const Geo3& g, const float* vp,
                     const float* vs, const float* rho, int nx, int ny, int nz, int pad, int kz0,
                     float* mat);
// Injection into set B (p | txx tyy tzz) and recording of B's vx vy vz at
// step it (1-based); negative linear indices are skipped (solver3d.cu).
cudaError_t inject_record3(cudaStream_t st, bool elastic, const Geo3& g, float* state, int B,
                           int it, int nt, int n_src, const int* src_lin, const float* wav,
                           int n_rec, const int* rec_lin, float* s0, float* s1, float* s2);

}  // namespace fomo
