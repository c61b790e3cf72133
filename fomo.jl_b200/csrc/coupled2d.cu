// coupled2d.cu -- coupled P-S potential solver (equations/coupled2d/*, constant
// density, after Li et al. 2018).
//
// Medium (coupled2d/medium.jl:46-193), on the device: alpha = vp^2 and
// beta = vs^2 on the edge-replicated padded grid; a separable Gaussian of the
// two (x pass, then z pass, clamped indices); centered first derivatives and
// Laplacians of the smoothed fields.  These repeat the reference's CPU
// arithmetic: one multiply and one add per tap or stencil term, IEEE division.
//
// Step (coupled2d.jl:192-260, update_fields.jl:27-141), on ping-pong sets
// A -> B of {P, S, dP/dt, dS/dt}:
//   k_cp_vel: dP/dt, dS/dt += dt * RHS(P, S, medium), then the Higdon boundary
//             with weights w_vx and the coefficients of v_ref_p (dP/dt) and
//             v_ref_s (dS/dt);
//   k_cp_pos: P, S += dt * dP/dt, dS/dt, then the boundary with weights w_tau,
//             then, on source and receiver cells, injection into P and
//             recording of P and S.
// The reference applies its racy full-grid HABC kernel (boundary/habc/
// kernels.jl:122-190) here; these kernels fuse the same formula in the
// deterministic two-pass form (a frame cell reads its neighbour's
// pre-correction value, recomputed from A), as the other 2D solvers do.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "fomo_internal.cuh"
#include "solver2d_kernels.cuh"

namespace fomo {

// utils/FD_centered.jl:15-21: centered first-derivative coefficients.
const float kD1[6][5] = {
    {0, 0, 0, 0, 0},
    {(float)0.5, 0, 0, 0, 0},
    {(float)(2.0 / 3.0), (float)(-1.0 / 12.0), 0, 0, 0},
    {(float)(3.0 / 4.0), (float)(-3.0 / 20.0), (float)(1.0 / 60.0), 0, 0},
    {(float)(4.0 / 5.0), (float)(-1.0 / 5.0), (float)(4.0 / 105.0), (float)(-1.0 / 280.0), 0},
    {(float)(5.0 / 6.0), (float)(-5.0 / 21.0), (float)(5.0 / 84.0), (float)(-5.0 / 504.0),
     (float)(1.0 / 1260.0)},
};

namespace {

struct CCoef {
  float d1[5];
  float d2[5];
  float c0;
};

// The eight medium planes: alpha, beta, d alpha/dx, d alpha/dz, d beta/dx,
// d beta/dz, lap alpha, lap beta (CoupledMedium, medium.jl:16-34).
struct CpMat {
  const float* a;
  const float* b;
  const float* ax;
  const float* az;
  const float* bx;
  const float* bz;
  const float* la;
  const float* lb;
};

// medium.jl:121-126: taps exp(-0.5 (k/sigma)^2), k = -r..r, r = ceil(3 sigma),
// rounded to float and divided by their float sum (summed from k = -r).
std::vector<float> gaussian_taps(double sigma) {
  const int r = (int)std::ceil(3.0 * sigma);
  std::vector<float> k((size_t)(2 * r + 1));
  for (int q = -r; q <= r; ++q) {
    const double x = (double)q / sigma;
    k[(size_t)(q + r)] = (float)std::exp(-0.5 * (x * x));
  }
  float s = 0.0f;
  for (float v : k) s = s + v;
  for (float& v : k) v = v / s;
  return k;
}

// alpha = vp^2, beta = vs^2 on the padded grid (pad_array.jl:8-22 clamping).
__global__ void k_cp_square(int nx, int nz, int pad, int nxp, int nzp, int ld,
                            const float* __restrict__ vp, const float* __restrict__ vs,
                            float* __restrict__ a, float* __restrict__ b) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= nxp || z >= nzp) return;
  const int i = min(max(x - pad, 0), nx - 1), j = min(max(z - pad, 0), nz - 1);
  const long long q = (long long)j * nx + i, p = (long long)z * ld + x;
  const float u = __ldg(vp + q), v = __ldg(vs + q);
  a[p] = __fmul_rn(u, u);
  b[p] = __fmul_rn(v, v);
}

// medium.jl:127-151: one pass of the separable Gaussian along x (dir 0) or z (dir 1).
__global__ void k_cp_smooth(int nxp, int nzp, int ld, int dir, const float* __restrict__ taps,
                            int r, const float* __restrict__ f, float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= nxp || z >= nzp) return;
  float v = 0.0f;
  for (int q = -r; q <= r; ++q) {
    const int xx = dir == 0 ? min(max(x + q, 0), nxp - 1) : x;
    const int zz = dir == 1 ? min(max(z + q, 0), nzp - 1) : z;
    v = __fadd_rn(v, __fmul_rn(__ldg(taps + q + r), __ldg(f + (long long)zz * ld + xx)));
  }
  out[(long long)z * ld + x] = v;
}

// medium.jl:157-193: gradients (x: M <= x < nxp-M, every z; z: the transpose)
// and the Laplacian (both ranges) of a smoothed field; 0 elsewhere.
template <int N>
__global__ void __launch_bounds__(256) k_cp_derivs(Geo2 g, CCoef c, float h, float ih2,
                                                   const float* __restrict__ f,
                                                   float* __restrict__ dx,
                                                   float* __restrict__ dz,
                                                   float* __restrict__ lap) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= g.nx || z >= g.nz) return;
  const long long p = (long long)z * g.ld + x, s = g.ld;
  const bool ix = x >= N && x < g.nx - N, iz = z >= N && z < g.nz - N;
  float gx = 0.0f, gz = 0.0f, l = 0.0f;
  if (ix) {
    float v = 0.0f;
#pragma unroll
    for (int k = 1; k <= N; ++k)
      v = __fadd_rn(v, __fmul_rn(c.d1[k - 1], __fsub_rn(__ldg(f + p + k), __ldg(f + p - k))));
    gx = __fdiv_rn(v, h);
  }
  if (iz) {
    float v = 0.0f;
#pragma unroll
    for (int k = 1; k <= N; ++k)
      v = __fadd_rn(v, __fmul_rn(c.d1[k - 1], __fsub_rn(__ldg(f + p + k * s), __ldg(f + p - k * s))));
    gz = __fdiv_rn(v, h);
  }
  if (ix && iz) {
    const float fc = __ldg(f + p);
    float a = __fmul_rn(c.c0, fc), b = __fmul_rn(c.c0, fc);
#pragma unroll
    for (int k = 1; k <= N; ++k) {
      a = __fadd_rn(a, __fmul_rn(c.d2[k - 1], __fadd_rn(__ldg(f + p + k), __ldg(f + p - k))));
      b = __fadd_rn(b, __fmul_rn(c.d2[k - 1],
                                 __fadd_rn(__ldg(f + p + k * s), __ldg(f + p - k * s))));
    }
    l = __fmul_rn(__fadd_rn(a, b), ih2);
  }
  dx[p] = gx;
  dz[p] = gz;
  lap[p] = l;
}

// update_fields.jl:27-108 at (x, z): dP/dt and dS/dt of the next half step
// (before the boundary); non-interior cells keep their old values.  One fma
// per stencil term; the right-hand sides in this fixed order (the oracle's
// coupled_vel repeats it).
template <int N>
__device__ __forceinline__ void cp_vel_at(const Geo2& g, const CCoef& c, float dt, float ih,
                                          float ih2, const CpMat& m, const float* __restrict__ P,
                                          const float* __restrict__ S,
                                          const float* __restrict__ dP0,
                                          const float* __restrict__ dS0, int x, int z, float& uP,
                                          float& uS) {
  const long long p = (long long)z * g.ld + x;
  uP = __ldg(dP0 + p);
  uS = __ldg(dS0 + p);
  if (!interior2(g, x, z)) return;
  const long long s = g.ld;
  const float Pc = __ldg(P + p), Sc = __ldg(S + p);
  float dPx = 0.0f, dPz = 0.0f, dSx = 0.0f, dSz = 0.0f;
  float lPx = __fmul_rn(c.c0, Pc), lPz = lPx, lSx = __fmul_rn(c.c0, Sc), lSz = lSx;
#pragma unroll
  for (int l = 1; l <= N; ++l) {
    const float c1 = c.d1[l - 1], c2 = c.d2[l - 1];
    const float pxp = __ldg(P + p + l), pxm = __ldg(P + p - l);
    const float pzp = __ldg(P + p + l * s), pzm = __ldg(P + p - l * s);
    const float sxp = __ldg(S + p + l), sxm = __ldg(S + p - l);
    const float szp = __ldg(S + p + l * s), szm = __ldg(S + p - l * s);
    dPx = __fmaf_rn(c1, __fsub_rn(pxp, pxm), dPx);
    dPz = __fmaf_rn(c1, __fsub_rn(pzp, pzm), dPz);
    lPx = __fmaf_rn(c2, __fadd_rn(pxp, pxm), lPx);
    lPz = __fmaf_rn(c2, __fadd_rn(pzp, pzm), lPz);
    dSx = __fmaf_rn(c1, __fsub_rn(sxp, sxm), dSx);
    dSz = __fmaf_rn(c1, __fsub_rn(szp, szm), dSz);
    lSx = __fmaf_rn(c2, __fadd_rn(sxp, sxm), lSx);
    lSz = __fmaf_rn(c2, __fadd_rn(szp, szm), lSz);
  }
  dPx = __fmul_rn(dPx, ih);
  dPz = __fmul_rn(dPz, ih);
  dSx = __fmul_rn(dSx, ih);
  dSz = __fmul_rn(dSz, ih);
  const float lapP = __fmul_rn(__fadd_rn(lPx, lPz), ih2);
  const float lapS = __fmul_rn(__fadd_rn(lSx, lSz), ih2);
  const float ax = __ldg(m.ax + p), az = __ldg(m.az + p), bx = __ldg(m.bx + p),
              bz = __ldg(m.bz + p);
  float rP = __fmul_rn(Pc, __ldg(m.la + p));
  rP = __fmaf_rn(2.0f, __fmaf_rn(ax, dPx, __fmul_rn(az, dPz)), rP);
  rP = __fmaf_rn(__fmul_rn(-2.0f, Pc), __ldg(m.lb + p), rP);
  rP = __fmaf_rn(2.0f, __fmaf_rn(bx, dSz, -__fmul_rn(bz, dSx)), rP);
  rP = __fmaf_rn(__ldg(m.a + p), lapP, rP);
  float rS = __fmul_rn(2.0f, __fmaf_rn(bx, dSx, __fmul_rn(bz, dSz)));
  rS = __fmaf_rn(2.0f, __fmaf_rn(bz, dPx, -__fmul_rn(bx, dPz)), rS);
  rS = __fmaf_rn(__ldg(m.b + p), lapS, rS);
  uP = __fmaf_rn(dt, rP, uP);
  uS = __fmaf_rn(dt, rS, uS);
}

template <int N>
__global__ void __launch_bounds__(256, 6) k_cp_vel(Geo2 g, CCoef c, float dt, float ih, float ih2,
                                                HabcDev hp, HabcDev hs, CpMat m,
                                                const float* __restrict__ P,
                                                const float* __restrict__ S,
                                                const float* __restrict__ dP0,
                                                const float* __restrict__ dS0,
                                                float* __restrict__ dP1, float* __restrict__ dS1) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= g.nx || z >= g.nz) return;
  float uP, uS;
  cp_vel_at<N>(g, c, dt, ih, ih2, m, P, S, dP0, dS0, x, z, uP, uS);
  const long long p = (long long)z * g.ld + x;
  int sx, sz, dist;
  if (frame2(g, x, z, sx, sz, dist)) {
    const float w = habc_weight(hp, 0, dist);  // w_vx for both fields
    const float foP = __ldg(dP0 + p), foS = __ldg(dS0 + p);
    if (sx != 0 && sz != 0) {
      const long long px = p + sx, pz = p + (long long)sz * g.ld;
      float aP, aS, bP, bS;
      cp_vel_at<N>(g, c, dt, ih, ih2, m, P, S, dP0, dS0, x + sx, z, aP, aS);
      cp_vel_at<N>(g, c, dt, ih, ih2, m, P, S, dP0, dS0, x, z + sz, bP, bS);
      uP = higdon_corner(w, uP, higdon_side(hp, aP, foP, __ldg(dP0 + px)),
                         higdon_side(hp, bP, foP, __ldg(dP0 + pz)));
      uS = higdon_corner(w, uS, higdon_side(hs, aS, foS, __ldg(dS0 + px)),
                         higdon_side(hs, bS, foS, __ldg(dS0 + pz)));
    } else {
      const int xn = x + sx, zn = z + sz;
      const long long pn = (long long)zn * g.ld + xn;
      float nP, nS;
      cp_vel_at<N>(g, c, dt, ih, ih2, m, P, S, dP0, dS0, xn, zn, nP, nS);
      uP = higdon_edge(w, uP, higdon_side(hp, nP, foP, __ldg(dP0 + pn)));
      uS = higdon_edge(w, uS, higdon_side(hs, nS, foS, __ldg(dS0 + pn)));
    }
  }
  dP1[p] = uP;
  dS1[p] = uS;
}

// update_fields.jl:120-141 at (x, z): P, S of the next step before the boundary.
__device__ __forceinline__ void cp_pos_at(const Geo2& g, float dt, const float* __restrict__ P0,
                                          const float* __restrict__ S0,
                                          const float* __restrict__ dP1,
                                          const float* __restrict__ dS1, int x, int z, float& uP,
                                          float& uS) {
  const long long p = (long long)z * g.ld + x;
  uP = __ldg(P0 + p);
  uS = __ldg(S0 + p);
  if (!interior2(g, x, z)) return;
  uP = __fmaf_rn(dt, __ldg(dP1 + p), uP);
  uS = __fmaf_rn(dt, __ldg(dS1 + p), uS);
}

// j: the step's index within its chunk (step it = *it0 + j + 1).
__global__ void __launch_bounds__(256) k_cp_pos(Geo2 g, float dt, HabcDev hp, HabcDev hs,
                                                const float* __restrict__ P0,
                                                const float* __restrict__ S0,
                                                const float* __restrict__ dP1,
                                                const float* __restrict__ dS1,
                                                float* __restrict__ P1, float* __restrict__ S1,
                                                CellTags t, int j) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= g.nx || z >= g.nz) return;
  float uP, uS;
  cp_pos_at(g, dt, P0, S0, dP1, dS1, x, z, uP, uS);
  const long long p = (long long)z * g.ld + x;
  int sx, sz, dist;
  if (frame2(g, x, z, sx, sz, dist)) {
    const float w = habc_weight(hp, 2, dist);  // w_tau for both fields
    const float foP = __ldg(P0 + p), foS = __ldg(S0 + p);
    if (sx != 0 && sz != 0) {
      const long long px = p + sx, pz = p + (long long)sz * g.ld;
      float aP, aS, bP, bS;
      cp_pos_at(g, dt, P0, S0, dP1, dS1, x + sx, z, aP, aS);
      cp_pos_at(g, dt, P0, S0, dP1, dS1, x, z + sz, bP, bS);
      uP = higdon_corner(w, uP, higdon_side(hp, aP, foP, __ldg(P0 + px)),
                         higdon_side(hp, bP, foP, __ldg(P0 + pz)));
      uS = higdon_corner(w, uS, higdon_side(hs, aS, foS, __ldg(S0 + px)),
                         higdon_side(hs, bS, foS, __ldg(S0 + pz)));
    } else {
      const int xn = x + sx, zn = z + sz;
      const long long pn = (long long)zn * g.ld + xn;
      float nP, nS;
      cp_pos_at(g, dt, P0, S0, dP1, dS1, xn, zn, nP, nS);
      uP = higdon_edge(w, uP, higdon_side(hp, nP, foP, __ldg(P0 + pn)));
      uS = higdon_edge(w, uS, higdon_side(hs, nS, foS, __ldg(S0 + pn)));
    }
  }
  const int e = __ldg(t.tag + p);
  if (e >= 0) {  // injection into P, then recording of P and S (coupled2d.jl:239-250)
    const long long k = (long long)(*t.it0 + j);  // it - 1
    const int4 E = t.ent[e];
    uP = tag_inject(t, E, k, 0, uP);
    tag_record(t, E, k, 0, uP, uS, 0.0f);
  }
  P1[p] = uP;
  S1[p] = uS;
}

float min_pos(const float* v, long long n) {
  float m = INFINITY;
  for (long long k = 0; k < n; ++k)
    if (v[k] > 0.0f && v[k] < m) m = v[k];
  return m;
}

// Largest Gaussian radius the medium kernels accept (r = ceil(3 sigma)).
constexpr int kMaxSmoothRadius = 1024;

// Device medium: eight planes at d_med (plane stride `plane`), from host vp, vs.
int build_medium(fomo_ctx* ctx, cudaStream_t st, const Geo2& g, int nx, int nz, int pad, int N,
                 float dh, double sigma, const float* d_vp, const float* d_vs, float* d_med,
                 float* d_tmp, float* d_taps, const std::vector<float>& taps) {
  const long long pl = g.plane;
  float* a = d_med;
  float* b = d_med + pl;
  dim3 blk(32, 8), grd(cdiv(g.nx, 32), cdiv(g.nz, 8));
  k_cp_square<<<grd, blk, 0, st>>>(nx, nz, pad, g.nx, g.nz, g.ld, d_vp, d_vs, a, b);
  // smoothed alpha, beta in d_tmp[0], d_tmp[1]; d_tmp[2] holds the x pass
  float* as = d_tmp;
  float* bs = d_tmp + pl;
  float* t = d_tmp + 2 * pl;
  if (sigma > 0) {
    const int r = (int)(taps.size() - 1) / 2;
    k_cp_smooth<<<grd, blk, 0, st>>>(g.nx, g.nz, g.ld, 0, d_taps, r, a, t);
    k_cp_smooth<<<grd, blk, 0, st>>>(g.nx, g.nz, g.ld, 1, d_taps, r, t, as);
    k_cp_smooth<<<grd, blk, 0, st>>>(g.nx, g.nz, g.ld, 0, d_taps, r, b, t);
    k_cp_smooth<<<grd, blk, 0, st>>>(g.nx, g.nz, g.ld, 1, d_taps, r, t, bs);
  } else {
    FOMO_CU(ctx, cudaMemcpyAsync(as, a, sizeof(float) * pl, cudaMemcpyDeviceToDevice, st));
    FOMO_CU(ctx, cudaMemcpyAsync(bs, b, sizeof(float) * pl, cudaMemcpyDeviceToDevice, st));
  }
  CCoef c{};
  for (int l = 0; l < 5; ++l) {
    c.d1[l] = kD1[N][l];
    c.d2[l] = kD2[N][l];
  }
  c.c0 = kD2C0[N];
  const float h = dh, ih2 = 1.0f / (h * h);
#define FOMO_CPD_CASE(NN)                                                                      \
  case NN:                                                                                     \
    k_cp_derivs<NN><<<grd, blk, 0, st>>>(g, c, h, ih2, as, d_med + 2 * pl, d_med + 3 * pl,      \
                                         d_med + 6 * pl);                                      \
    k_cp_derivs<NN><<<grd, blk, 0, st>>>(g, c, h, ih2, bs, d_med + 4 * pl, d_med + 5 * pl,      \
                                         d_med + 7 * pl);                                      \
    break;
  switch (N) { FOMO_CPD_CASE(1) FOMO_CPD_CASE(2) FOMO_CPD_CASE(3) FOMO_CPD_CASE(4) FOMO_CPD_CASE(5) }
#undef FOMO_CPD_CASE
  FOMO_CU(ctx, cudaGetLastError());
  return FOMO_OK;
}

struct CpGrid {
  int N, pad;
  Geo2 g;
  std::vector<float> taps;
};

int cp_grid(fomo_ctx* ctx, int nx, int nz, int nbc, int fd_order, double sigma, CpGrid& G) {
  G.N = order_to_N(fd_order);
  if (G.N < 0) return fail(ctx, FOMO_EARG, "Unsupported FD order: " + std::to_string(fd_order));
  if (nx < 1 || nz < 1 || nbc < 0) return fail(ctx, FOMO_EARG, "invalid coupled2d grid");
  G.pad = nbc + G.N;
  if (G.pad < 2) return fail(ctx, FOMO_EARG, "nbc + fd_order/2 must be >= 2");
  if (!std::isfinite(sigma)) return fail(ctx, FOMO_EARG, "smooth_sigma must be finite");
  if (sigma > 0) {
    if (std::ceil(3.0 * sigma) > kMaxSmoothRadius)
      return fail(ctx, FOMO_EARG, "smooth_sigma above " + std::to_string(kMaxSmoothRadius / 3));
    G.taps = gaussian_taps(sigma);
  }
  G.g.nx = nx + 2 * G.pad;
  G.g.nz = nz + 2 * G.pad;
  G.g.ld = (G.g.nx + 31) & ~31;
  G.g.M = G.N;
  G.g.nbc = G.pad - 1;
  G.g.plane = (long long)G.g.ld * G.g.nz;
  if ((long long)G.g.nx * G.g.nz > (1LL << 31))
    return fail(ctx, FOMO_EARG, "padded grid exceeds 2^31 cells");
  return FOMO_OK;
}

}  // namespace
}  // namespace fomo

using namespace fomo;

extern "C" {

int fomo_coupled2d(fomo_ctx* ctx, const fomo_grid2d* gp, const float* vp, const float* vs,
                   float v_ref_s, double smooth_sigma, const fomo_acq* acq, int32_t snap_interval,
                   float* seis_P, float* seis_S, float* snaps_P, float* snaps_S,
                   const fomo_opts* opts, fomo_stats* stats) {
  if (!ctx) return FOMO_EARG;
  if (!gp || !acq || !vp || !vs)
    return fail(ctx, FOMO_EARG, "grid, acquisition and model arrays are required");
  if (opts && (opts->flags & (FOMO_F_DEVICE_PTRS | FOMO_F_SPONGE)))
    return fail(ctx, FOMO_EUNSUPPORTED, "coupled2d takes host arrays and the HABC boundary only");
  if (opts && opts->precision != FOMO_FP32)
    return fail(ctx, FOMO_EUNSUPPORTED, "coupled2d stores FP32 only");
  if (acq->n_shots != 1) return fail(ctx, FOMO_EARG, "coupled2d takes n_shots == 1");
  if (acq->n_src < 0 || acq->n_rec < 0 ||
      (acq->n_src > 0 && (!acq->sx || !acq->sz || !acq->wavelet)) ||
      (acq->n_rec > 0 && (!acq->rx || !acq->rz)))
    return fail(ctx, FOMO_EARG, "invalid acquisition");
  if (gp->nt < 1 || !(gp->dh > 0.0f) || !(gp->dt > 0.0f))
    return fail(ctx, FOMO_EARG, "nt, dh and dt must be positive");
  if (snap_interval < 0) return fail(ctx, FOMO_EARG, "snap_interval must be >= 0");
  CpGrid G;
  int rc = cp_grid(ctx, gp->nx, gp->nz, gp->nbc, gp->fd_order, smooth_sigma, G);
  if (rc) return rc;
  const int nx = gp->nx, nz = gp->nz, nt = gp->nt, pad = G.pad, N = G.N;
  const Geo2& g = G.g;
  const long long nint = (long long)nx * nz, pl = g.plane;
  for (int k = 0; k < acq->n_src; ++k)
    if (acq->sx[k] < 1 || acq->sx[k] > nx || acq->sz[k] < 1 || acq->sz[k] > nz)
      return fail(ctx, FOMO_EARG, "source index out of range");
  for (int k = 0; k < acq->n_rec; ++k)
    if (acq->rx[k] < 1 || acq->rx[k] > nx || acq->rz[k] < 1 || acq->rz[k] > nz)
      return fail(ctx, FOMO_EARG, "receiver index out of range");
  // v_ref_p / v_ref_s defaults: minimum of the positive velocities (coupled2d.jl:63-64)
  float vrp = gp->v_ref, vrs = v_ref_s;
  if (!(vrp > 0.0f)) vrp = min_pos(vp, nint);
  if (!(vrs > 0.0f)) vrs = min_pos(vs, nint);
  if (!std::isfinite(vrp) || !std::isfinite(vrs))
    return fail(ctx, FOMO_EARG, "vp and vs need a positive value for v_ref_p, v_ref_s");
  HabcHost hhp = make_habc(pad, vrp, gp->dt, gp->dh), hhs = make_habc(pad, vrs, gp->dt, gp->dh);
  // tagged cells: one entry per distinct source or receiver cell
  std::vector<int32_t> src_lin(acq->n_src), rec_lin(acq->n_rec);
  for (int k = 0; k < acq->n_src; ++k)
    src_lin[k] = (acq->sx[k] - 1 + pad) + g.ld * (acq->sz[k] - 1 + pad);
  for (int k = 0; k < acq->n_rec; ++k)
    rec_lin[k] = (acq->rx[k] - 1 + pad) + g.ld * (acq->rz[k] - 1 + pad);
  const CellTagHost tags = make_cell_tags(src_lin.data(), acq->n_src, rec_lin.data(), acq->n_rec);
  const int n_ent = (int)tags.lin.size();
  const int nsnap = snap_interval > 0 ? nt / snap_interval : 0;
  const long long seis_n = (long long)acq->n_rec * nt;

  FOMO_CU(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  Arena ar;
  const size_t o_model = ar.take<float>(2 * nint);
  const size_t o_med = ar.take<float>(8 * pl);
  const size_t o_tmp = ar.take<float>(3 * pl);
  const size_t o_state = ar.take<float>(8 * pl);
  const size_t o_taps = ar.take<float>(std::max<size_t>(G.taps.size(), 1));
  const size_t o_w = ar.take<float>(hhp.wtab.size());
  const size_t o_tag = ar.take<int32_t>(pl);
  const size_t o_ent = ar.take<int4>(std::max(n_ent, 1));
  const size_t o_elin = ar.take<int32_t>(std::max(n_ent, 1));
  const size_t o_list = ar.take<int32_t>(std::max<size_t>(tags.list.size(), 1));
  const size_t o_wav = ar.take<float>(std::max<long long>((long long)acq->n_src * nt, 1));
  const size_t o_seis = ar.take<float>(std::max<long long>(2 * seis_n, 1));
  const size_t o_snap = ar.take<float>(std::max<long long>(2LL * nsnap * nint, 1));
  const size_t o_it = ar.take<int>(1);  // device step index of replayed chunks
  if ((rc = ensure_workspace(ctx, ar.off))) return rc;
  float* d_model = ws_ptr<float>(ctx, o_model);
  float* d_med = ws_ptr<float>(ctx, o_med);
  float* d_state = ws_ptr<float>(ctx, o_state);
  float* d_taps = ws_ptr<float>(ctx, o_taps);
  float* d_w = ws_ptr<float>(ctx, o_w);
  int32_t* d_tag = ws_ptr<int32_t>(ctx, o_tag);
  int4* d_ent = ws_ptr<int4>(ctx, o_ent);
  int32_t* d_elin = ws_ptr<int32_t>(ctx, o_elin);
  int32_t* d_list = ws_ptr<int32_t>(ctx, o_list);
  float* d_wav = ws_ptr<float>(ctx, o_wav);
  float* d_seis = ws_ptr<float>(ctx, o_seis);
  float* d_snap = ws_ptr<float>(ctx, o_snap);
  FOMO_CU(ctx, cudaMemcpyAsync(d_model, vp, sizeof(float) * nint, cudaMemcpyHostToDevice, st));
  FOMO_CU(ctx, cudaMemcpyAsync(d_model + nint, vs, sizeof(float) * nint, cudaMemcpyHostToDevice, st));
  if (!G.taps.empty())
    FOMO_CU(ctx, cudaMemcpyAsync(d_taps, G.taps.data(), sizeof(float) * G.taps.size(),
                                 cudaMemcpyHostToDevice, st));
  FOMO_CU(ctx, cudaMemcpyAsync(d_w, hhp.wtab.data(), sizeof(float) * hhp.wtab.size(),
                               cudaMemcpyHostToDevice, st));
  if (acq->n_src)
    FOMO_CU(ctx, cudaMemcpyAsync(d_wav, acq->wavelet, sizeof(float) * acq->n_src * nt,
                                 cudaMemcpyHostToDevice, st));
  FOMO_CU(ctx, cudaMemsetAsync(d_tag, 0xFF, sizeof(int32_t) * pl, st));  // -1
  if (n_ent) {
    FOMO_CU(ctx, cudaMemcpyAsync(d_ent, tags.ent.data(), sizeof(int4) * n_ent,
                                 cudaMemcpyHostToDevice, st));
    FOMO_CU(ctx, cudaMemcpyAsync(d_elin, tags.lin.data(), sizeof(int32_t) * n_ent,
                                 cudaMemcpyHostToDevice, st));
    FOMO_CU(ctx, cudaMemcpyAsync(d_list, tags.list.data(), sizeof(int32_t) * tags.list.size(),
                                 cudaMemcpyHostToDevice, st));
    k_set_tags<<<cdiv(n_ent, 256), 256, 0, st>>>(d_tag, d_elin, n_ent);
  }
  if ((rc = build_medium(ctx, st, g, nx, nz, pad, N, gp->dh, smooth_sigma, d_model,
                         d_model + nint, d_med, ws_ptr<float>(ctx, o_tmp), d_taps, G.taps)))
    return rc;
  FOMO_CU(ctx, cudaMemsetAsync(d_state, 0, sizeof(float) * 8 * pl, st));
  FOMO_CU(ctx, cudaMemsetAsync(d_seis, 0, sizeof(float) * std::max<long long>(2 * seis_n, 1), st));

  CCoef c{};
  for (int l = 0; l < 5; ++l) {
    c.d1[l] = kD1[N][l];
    c.d2[l] = kD2[N][l];
  }
  c.c0 = kD2C0[N];
  const CpMat m{d_med, d_med + pl, d_med + 2 * pl, d_med + 3 * pl,
                d_med + 4 * pl, d_med + 5 * pl, d_med + 6 * pl, d_med + 7 * pl};
  const HabcDev hp{hhp.q, hhp.qt, hhp.qxt, hhp.nbc, hhp.wstride, d_w};
  const HabcDev hs{hhs.q, hhs.qt, hhs.qxt, hhs.nbc, hhs.wstride, d_w};  // same ramps
  const float dt = gp->dt, ih = 1.0f / gp->dh, ih2 = ih * ih;
  // set k: P, S, dP/dt, dS/dt
  auto field = [&](int set, int f) { return d_state + ((long long)set * 4 + f) * pl; };
  dim3 blk(32, 8), grd(cdiv(g.nx, 32), cdiv(g.nz, 8));
  int launches = 0;
  int A = 0, B = 1;
  // one step's two updates on stream `s`, set a -> set b
  int* d_it = ws_ptr<int>(ctx, o_it);
  FOMO_CU(ctx, cudaMemsetAsync(d_it, 0, sizeof(int), st));
  CellTags tg;
  tg.tag = d_tag;
  tg.ent = d_ent;
  tg.list = d_list;
  tg.wav = d_wav;
  tg.n_src = acq->n_src;
  tg.n_rec = acq->n_rec;
  tg.nt = nt;
  tg.s0 = d_seis;
  tg.s1 = d_seis + seis_n;
  tg.it0 = d_it;
  auto updates = [&](cudaStream_t s, int a, int b, int j) {
#define FOMO_CPV_CASE(NN)                                                                    \
  case NN:                                                                                   \
    k_cp_vel<NN><<<grd, blk, 0, s>>>(g, c, dt, ih, ih2, hp, hs, m, field(a, 0), field(a, 1),  \
                                     field(a, 2), field(a, 3), field(b, 2), field(b, 3));    \
    break;
    switch (N) { FOMO_CPV_CASE(1) FOMO_CPV_CASE(2) FOMO_CPV_CASE(3) FOMO_CPV_CASE(4) FOMO_CPV_CASE(5) }
#undef FOMO_CPV_CASE
    k_cp_pos<<<grd, blk, 0, s>>>(g, dt, hp, hs, field(a, 0), field(a, 1), field(b, 2),
                                 field(b, 3), field(b, 0), field(b, 1), tg, j);
  };
  FOMO_CU(ctx, cudaEventRecord(ctx->ev0, st));
  // Replayed chunks of K steps (K even: the ping-pong sets return to their
  // start; a multiple of snap_interval <= 256), captured once with a device
  // step index, as the acoustic solver does; the rest launch step by step
  // (FOMO_F_STEP_LAUNCH: every step), with identical results.
  int it_first = 1;
  // Snapshot frames of replayed chunk k are copied to the caller once chunk k
  // has run (an event per chunk, the context's copy stream), while later chunks
  // compute; copies into pageable memory return when done.
  struct Events {
    std::vector<cudaEvent_t> ev;
    ~Events() {
      for (auto e : ev) cudaEventDestroy(e);
    }
  } chunk_ev;
  int streamed_chunks = 0, frames_per_chunk = 0;
  cudaGraphExec_t exec = nullptr;
  struct ExecGuard {
    cudaGraphExec_t& e;
    cudaStream_t s;
    ~ExecGuard() {
      if (e) {
        cudaStreamSynchronize(s);
        cudaGraphExecDestroy(e);
      }
    }
  } exec_guard{exec, st};
  {
    const int si = nsnap ? snap_interval : 0;
    int K = 0;
    if (!(opts && (opts->flags & FOMO_F_STEP_LAUNCH))) {
      if (si == 0) {
        K = 64;
      } else if (si <= 256) {
        K = si * std::max(1, (64 + si / 2) / si);
        if (K % 2) K *= 2;
      }
    }
    const int nchunk = K > 0 ? nt / K : 0;
    if (nchunk >= 2) {
      const cudaStream_t cs = ctx->own_stream;  // the caller's stream may be uncapturable
      cudaGraph_t graph = nullptr;
      cudaError_t ce = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
      int nodes = 0;
      if (ce == cudaSuccess) {
        int a = A, b = B;
        for (int j = 0; j < K; ++j) {
          updates(cs, a, b, j);
          nodes += 2;
          if (si && (j + 1) % si == 0) {
            for (int f = 0; f < 2; ++f)
              k_snap_at<<<dim3(cdiv(nx, 128), nz), 128, 0, cs>>>(
                  d_it, j, si, field(b, f) + pad + (long long)pad * g.ld, g.ld, nx, nz,
                  d_snap + (long long)f * nsnap * nint);
            nodes += 2;
          }
          std::swap(a, b);
        }
        k_step_add<<<1, 1, 0, cs>>>(d_it, K);
        ++nodes;
        ce = cudaStreamEndCapture(cs, &graph);
      }
      if (ce == cudaSuccess) ce = cudaGraphInstantiate(&exec, graph, 0);
      if (graph) cudaGraphDestroy(graph);
      if (ce == cudaSuccess && si && (snaps_P || snaps_S)) {
        chunk_ev.ev.assign(nchunk, nullptr);
        for (auto& e : chunk_ev.ev)
          if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        frames_per_chunk = K / si;
      }
      for (int k = 0; ce == cudaSuccess && k < nchunk; ++k) {
        ce = cudaGraphLaunch(exec, st);
        if (ce == cudaSuccess && frames_per_chunk) ce = cudaEventRecord(chunk_ev.ev[k], st);
      }
      if (ce == cudaSuccess && frames_per_chunk) streamed_chunks = nchunk;
      if (ce != cudaSuccess)
        return fail(ctx, FOMO_ECUDA, std::string("replayed step chunk: ") + cudaGetErrorString(ce));
      launches += nchunk * nodes;
      it_first = nchunk * K + 1;
    }
  }
  for (int it = it_first; it <= nt; ++it) {
    updates(st, A, B, it - it_first);  // *d_it = it_first - 1 after the chunks
    launches += 2;
    if (nsnap && it % snap_interval == 0) {  // coupled2d.jl:252-258
      const long long k = it / snap_interval - 1;
      for (int f = 0; f < 2; ++f)
        FOMO_CU(ctx, cudaMemcpy2DAsync(d_snap + ((long long)f * nsnap + k) * nint,
                                       sizeof(float) * nx, field(B, f) + pad + (long long)pad * g.ld,
                                       sizeof(float) * g.ld, sizeof(float) * nx, nz,
                                       cudaMemcpyDeviceToDevice, st));
    }
    FOMO_CU(ctx, cudaGetLastError());
    std::swap(A, B);
  }
  FOMO_CU(ctx, cudaEventRecord(ctx->ev1, st));
  float* const snaps_out[2] = {snaps_P, snaps_S};
  for (int k = 0; k < streamed_chunks; ++k) {
    FOMO_CU(ctx, cudaStreamWaitEvent(ctx->copy_stream, chunk_ev.ev[k], 0));
    const long long f0 = (long long)k * frames_per_chunk;
    for (int f = 0; f < 2; ++f)
      if (snaps_out[f])
        FOMO_CU(ctx, cudaMemcpyAsync(snaps_out[f] + f0 * nint,
                                     d_snap + ((long long)f * nsnap + f0) * nint,
                                     sizeof(float) * frames_per_chunk * nint,
                                     cudaMemcpyDeviceToHost, ctx->copy_stream));
  }
  const long long streamed = (long long)streamed_chunks * frames_per_chunk;
  if (seis_n) {
    if (seis_P)
      FOMO_CU(ctx, cudaMemcpyAsync(seis_P, d_seis, sizeof(float) * seis_n, cudaMemcpyDeviceToHost, st));
    if (seis_S)
      FOMO_CU(ctx, cudaMemcpyAsync(seis_S, d_seis + seis_n, sizeof(float) * seis_n,
                                   cudaMemcpyDeviceToHost, st));
  }
  if (nsnap > streamed)
    for (int f = 0; f < 2; ++f)
      if (snaps_out[f])
        FOMO_CU(ctx, cudaMemcpyAsync(snaps_out[f] + streamed * nint,
                                     d_snap + ((long long)f * nsnap + streamed) * nint,
                                     sizeof(float) * (nsnap - streamed) * nint,
                                     cudaMemcpyDeviceToHost, st));
  FOMO_CU(ctx, cudaStreamSynchronize(st));
  if (streamed_chunks) FOMO_CU(ctx, cudaStreamSynchronize(ctx->copy_stream));
  float ms = 0.0f;
  FOMO_CU(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  if (stats) {
    *stats = fomo_stats{};
    stats->kernel_time_s = ms * 1e-3;
    const double cells = (double)g.nx * g.nz;
    stats->cell_updates = cells * nt;
    // per cell and step: velocity half step reads P, S, dP, dS and 8 medium
    // planes and writes dP, dS; position half step reads P, S, dP, dS, writes P, S
    stats->alg_bytes = 4.0 * cells * nt * (14.0 + 6.0);
    stats->n_shots = 1;
    stats->gpu_launches = launches;
    stats->kernel = FOMO_KERNEL_TWO_PHASE;
    stats->status = FOMO_OK;
  }
  return FOMO_OK;
}

int fomo_debug_coupled_medium(fomo_ctx* ctx, int32_t nx, int32_t nz, int32_t nbc,
                              int32_t fd_order, float dh, double smooth_sigma, const float* vp,
                              const float* vs, float* out) {
  if (!ctx) return FOMO_EARG;
  if (!vp || !vs || !out) return fail(ctx, FOMO_EARG, "vp, vs and out are required");
  if (!(dh > 0.0f)) return fail(ctx, FOMO_EARG, "dh must be > 0");
  CpGrid G;
  int rc = cp_grid(ctx, nx, nz, nbc, fd_order, smooth_sigma, G);
  if (rc) return rc;
  const Geo2& g = G.g;
  const long long nint = (long long)nx * nz, pl = g.plane;
  FOMO_CU(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  Arena ar;
  const size_t o_model = ar.take<float>(2 * nint);
  const size_t o_med = ar.take<float>(8 * pl);
  const size_t o_tmp = ar.take<float>(3 * pl);
  const size_t o_taps = ar.take<float>(std::max<size_t>(G.taps.size(), 1));
  if ((rc = ensure_workspace(ctx, ar.off))) return rc;
  float* d_model = ws_ptr<float>(ctx, o_model);
  float* d_med = ws_ptr<float>(ctx, o_med);
  float* d_taps = ws_ptr<float>(ctx, o_taps);
  FOMO_CU(ctx, cudaMemcpyAsync(d_model, vp, sizeof(float) * nint, cudaMemcpyHostToDevice, st));
  FOMO_CU(ctx, cudaMemcpyAsync(d_model + nint, vs, sizeof(float) * nint, cudaMemcpyHostToDevice, st));
  if (!G.taps.empty())
    FOMO_CU(ctx, cudaMemcpyAsync(d_taps, G.taps.data(), sizeof(float) * G.taps.size(),
                                 cudaMemcpyHostToDevice, st));
  if ((rc = build_medium(ctx, st, g, nx, nz, G.pad, G.N, dh, smooth_sigma, d_model, d_model + nint,
                         d_med, ws_ptr<float>(ctx, o_tmp), d_taps, G.taps)))
    return rc;
  const long long hp = (long long)g.nx * g.nz;
  for (int k = 0; k < 8; ++k)
    FOMO_CU(ctx, cudaMemcpy2DAsync(out + k * hp, sizeof(float) * g.nx, d_med + k * pl,
                                   sizeof(float) * g.ld, sizeof(float) * g.nx, g.nz,
                                   cudaMemcpyDeviceToHost, st));
  FOMO_CU(ctx, cudaStreamSynchronize(st));
  return FOMO_OK;
}

}  // extern "C"
