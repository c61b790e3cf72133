// replica2d.cuh -- the CUDA C++ replica of Fomo.jl's elastic2d_batch launch
// sequence (replica2d.cu), a same-hardware measurement baseline.
#pragma once
#include "solver2d_kernels.cuh"

namespace fomo {

// In-place fields and their strip backups (one (ld, nz, ns) array each).
struct RepFields {
  float *vx, *vz, *txx, *tzz, *txz;
  float *vx_o, *vz_o, *txx_o, *tzz_o, *txz_o;
};
// Up to three fields of one det-HABC application: fields, backups, weights.
struct RepHabc {
  float* f[3];
  const float* fo[3];
  const float* w[3];
};

// Frame cells of the padded grid (_habc_frame_total, kernels_fused.jl:48-52).
long long replica_frame_total(int nx, int nz, int nbc);
// Fills the three HABC weight planes (vx, vz, tau) from the distance table.
cudaError_t replica_setup(cudaStream_t st, const Geo2& g, const HabcDev& h, float* wv, float* wz,
                          float* wt);
// One time step it (1-based) as the reference's eight launches.  scr holds
// 3 * replica_frame_total * ns floats.
cudaError_t replica_step(cudaStream_t st, int N, const Geo2& g, const Coef& c, float dtx,
                         float dtz, const HabcDev& h, const RepFields& w, const ElMat& m,
                         const float* w_vx, const float* w_vz, const float* w_tau, float* scr,
                         int ns, int it, int nt, int n_src, const int* src_lin, const float* wav,
                         int n_rec, const int* rec_lin, float* s0, float* s1);

}  // namespace fomo
