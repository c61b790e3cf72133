// sweep2d.cuh -- single-sweep (one fused pass per time step) 2D kernels and
// the kernel-family choice of the autotuner.
#pragma once
#include <cuda.h>
#include <cuda_fp16.h>

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
// Default extra cost of a frame row in the row-range split (the autotuner
// searches around it).
constexpr float kFrameWeight = 0.15f;

// Material pack of the lean single sweep: the five elastic planes copied into
// column-pair-interleaved rows with kPackRowPad zero rows above and below the
// grid and kPackColPad zero columns to its left (room for every row and column
// a CTA reads, so the kernel loads without bounds tests).  Element (z, pair p)
// of each region sits at (z + kPackRowPad) * pitch + p + kPackColPad / 2:
//   v : float4 {bx(2p), bx(2p+1), bz(2p), bz(2p+1)}
//   l : float4 {lam(2p), lam(2p+1), l2m(2p), l2m(2p+1)}
//   mu: float2 {mut(2p), mut(2p+1)}
constexpr int kPackRowPad = 32;
constexpr int kPackColPad = 8;
struct MatPack {
  const float4* v;
  const float4* l;
  const float2* mu;
  int pitch;  // column pairs per row
};
// Pairs per pack row and floats of the whole pack for a padded nx x nz grid.
int sweep_pack_pitch(int nx);
size_t sweep_pack_floats(int nx, int nz);
// Fills the pack at dst (16-byte aligned, sweep_pack_floats floats) from m's
// planes and records it in m (pack, pack_pitch).
cudaError_t build_sweep_pack(cudaStream_t st, const Geo2& g, ElMat& m, float* dst);

// Binary16 arrays of the output set (binary16 storage form; same index space
// as the FP32 arrays, which keep the band cells).
struct ElOut16 {
  __half* vx;
  __half* vz;
  __half* txx;
  __half* tzz;
  __half* txz;
};

struct SweepPlan {
  int N = 0, variant = 0;
  int family = 0;            // 0: column-per-thread, 1: pair-blocked, 2: register-window,
                             // 3: lean register-window, 4: warp-specialized,
                             // 5: shot pairs (packed FP32, pair-interleaved fields)
  int P = 0;                 // pair-blocked: prefetch depth (row pairs)
  int per_sm = 1, grid = 1;  // persistent CTAs per SM, grid size
  float frame_weight = 1.0f; // extra cost of a frame cell in the row-range split
  const long long* d_bounds = nullptr;  // [grid + 1] row ranges (device)
  size_t smem = 0;
  SweepGeom gm{};
  CUtensorMap tm[2][5];  // [ping-pong set][txx, tzz, txz, vx, vz]
  bool h16 = false;      // binary16 storage form (tm16 maps the binary16 arrays)
  CUtensorMap tm16[2][5];
};

// ---- shot-pair sweep (sweep2d_pair.cu) -------------------------------------
// Fields of a shot-pair run are pair-interleaved: element (x, z) of pair p is
// the float2 {shot 2p, shot 2p+1} at (p * plane + z * ld + x) float2 units;
// an odd batch carries one all-zero shot.  The materials come from a pack of
// duplicated values (both lanes of a float2 equal), kPairRowPad zero rows
// above and below the grid and kPairColPad zero columns left of it:
//   v : float4 {bx, bx, bz, bz}   l : float4 {lam, lam, l2m, l2m}   mu: float2 {mut, mut}
// element (z, x) of each region at (z + kPairRowPad) * pitch + x + kPairColPad.
constexpr int kPairRowPad = 32;
constexpr int kPairColPad = 16;
struct PairPack {
  const float4* v;
  const float4* l;
  const float2* mu;
  int pitch;  // cells per pack row
};
struct PairOut {
  float2* vx;
  float2* vz;
  float2* txx;
  float2* tzz;
  float2* txz;
};
// Stencil and Higdon constants, duplicated into both lanes.
struct PairCoef {
  float2 a[5];
  float2 dtx, dtz;
  float2 nq, nqt, nqxt;  // -q, -qt, -qxt
};
int pair_num_variants();
int pair_threads(int v);
int pair_txmax(int N, int v);       // widest strip of a variant (even)
int pair_box_width(int N, int v);   // TMA box width in float2 elements
size_t pair_smem(int N, int v, int wstride);
int pair_blocks_per_sm(int N, int v, size_t smem);
int pair_pack_pitch(int nx);
size_t pair_pack_floats(int nx, int nz);
cudaError_t build_pair_pack(cudaStream_t st, const Geo2& g, const ElMat& m, float* dst,
                            PairPack& out);
PairCoef make_pair_coef(const Coef& c, float dtx, float dtz, const HabcDev& h);
cudaError_t launch_pair_elastic(cudaStream_t st, const SweepPlan& sp, int v, int set,
                                const PairCoef& k, const HabcDev& h, const PairPack& mp,
                                const PairOut& o, int* err);
// Injection then recording of one step on pair-layout txx/tzz and vx/vz
// (k_inject_record's order and semantics), one block per shot.
cudaError_t launch_inject_record_pair(cudaStream_t st, int it, int nt, int ns, long long plane,
                                      int n_src, const int* src_lin, const float* wav, float* txx,
                                      float* tzz, int n_rec, const int* rec_lin, const float* vx,
                                      const float* vz, float* s0, float* s1);
// Columns [x0, x0 + nx) of rows [z0, z0 + nz) of shot `shot` of a pair-layout
// field into out (unpitched).
cudaError_t launch_pair_unpack(cudaStream_t st, const float* f, long long plane, int ld, int x0,
                               int z0, int nx, int nz, int shot, float* out);
// Is a sweep variant (the plan numbering) a shot-pair / warp-specialized variant?
bool sweep_variant_pair(int variant);
bool sweep_variant_ws(int variant);

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
// sets16: for the binary16 variants, the binary16 arrays [set * 5 + field] in
// the order of sets (null for the FP32 variants).
cudaError_t make_sweep_plan(SweepPlan& sp, int N, int variant, int TX, int per_sm, const Geo2& g,
                            int ns, float* const sets[2][5], float frame_weight,
                            long long* d_bounds, cudaStream_t st, __half* const* sets16 = nullptr);
// o16: the binary16 output arrays, for (and only for) a binary16 plan.
cudaError_t launch_sweep_elastic(cudaStream_t st, const SweepPlan& sp, int set, const Coef& c,
                                 float dtx, float dtz, const HabcDev& h, const ElFields& a,
                                 const ElMat& m, const ElOut& o, int* err,
                                 const ElOut16* o16 = nullptr);
// Is a variant the binary16 storage form?
bool sweep_variant_h16(int variant);
// Resident CTAs per SM for a plan (occupancy API).
int sweep_blocks_per_sm(const SweepPlan& sp);

}  // namespace fomo
