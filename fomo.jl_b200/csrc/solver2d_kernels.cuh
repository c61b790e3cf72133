// solver2d_kernels.cuh -- two-phase time-step kernels for the 2D solvers.
//
// One step = velocity sweep (A -> B) + stress/pressure sweep (A,B -> B) +
// inject/record, on ping-pong buffers A (time n) and B (time n+1).  The
// deterministic two-pass HABC of boundary/habc/kernels_det.jl:22-172 is fused
// into each sweep: a frame cell evaluates the Higdon value from the
// pre-correction field, recomputing the one inward neighbour's update from A
// (a pure function), so no scratch frame buffer and no second pass exist.
#pragma once
#include "fomo_internal.cuh"

namespace fomo {

// ---------------------------------------------------------------------------
// elastic2d velocity / stress updates (elastic2d/fused_kernels.jl:21-124,
// batch.jl:38-154).  Materials are shared by all shots; fields carry the
// shot offset already.
// ---------------------------------------------------------------------------
struct ElFields {
  const float* vx;
  const float* vz;
  const float* txx;
  const float* tzz;
  const float* txz;
};
struct ElOut {
  float* vx;
  float* vz;
  float* txx;
  float* tzz;
  float* txz;
};
struct ElMat {
  const float* bx;
  const float* bz;
  const float* lam;
  const float* l2m;
  const float* mut;
  // Padded, column-pair-interleaved copy of the five planes read by the lean
  // single sweep (layout in sweep2d.cuh); null where that kernel is not used.
  const float* pack = nullptr;
  int pack_pitch = 0;  // column pairs per pack row
  // Duplicated-value pack of the shot-pair sweep (PairPack in sweep2d.cuh).
  const float* ppack = nullptr;
  int ppack_pitch = 0;
};

// Source and receiver cells of a run, handled inside the step's last update
// kernel by the threads that own them: injection (each shot's sources in source
// order, as k_inject_record adds them), then recording.  One plane serves every
// shot of a batch: receivers are shared, and a source entry holds the index
// s * n_src + q of source q of shot s, which only shot s's threads apply.
struct CellTags {
  const int* tag = nullptr;   // pitched like the fields: -1, or an entry per distinct cell
  const int4* ent = nullptr;  // per entry: sources list[x, y), receivers list[z, w)
  const int* list = nullptr;
  const float* wav = nullptr;  // (n_src, nt), shared by the shots
  int n_src = 0, n_rec = 0, nt = 0;
  float* s0 = nullptr;  // seismograms (n_rec, nt, n_shots) (null: not recorded)
  float* s1 = nullptr;
  float* s2 = nullptr;
  const int* it0 = nullptr;  // steps completed before this launch's chunk
};

static __global__ void k_set_tags(int* __restrict__ tag, const int* __restrict__ lin, int n) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) tag[lin[e]] = e;
}

// u plus the wavelets of shot `shot`'s sources in the entry at 0-based step k,
// in source order.
__device__ __forceinline__ float tag_inject(const CellTags& t, const int4& E, long long k,
                                            int shot, float u) {
  for (int i = E.x; i < E.y; ++i) {
    const int e = t.list[i];
    const int s = e / t.n_src;  // an entry with sources implies n_src > 0
    if (s == shot) u = __fadd_rn(u, __ldg(t.wav + (e - s * t.n_src) + (long long)t.n_src * k));
  }
  return u;
}
__device__ __forceinline__ void tag_record(const CellTags& t, const int4& E, long long k,
                                           int shot, float r0, float r1, float r2) {
  const long long base = (long long)t.n_rec * (k + (long long)t.nt * shot);
  for (int i = E.z; i < E.w; ++i) {
    const long long o = t.list[i] + base;
    if (t.s0) t.s0[o] = r0;
    if (t.s1) t.s1[o] = r1;
    if (t.s2) t.s2[o] = r2;
  }
}

// Cerjan sponge (boundary/sponge.jl:30-78), fused into the sweep that produces
// the field: the updated value times damp[d], d = the cell's distance in cells
// to the nearest edge of the padded grid, for d < nbc.  In sponge mode HabcDev
// carries the user's nbc and the damping table (wtab[d], d < nbc).
__device__ __forceinline__ float sponge_damp(const Geo2& g, const HabcDev& h, int x, int z,
                                             float u) {
  const int d = min(min(x, g.nx - 1 - x), min(z, g.nz - 1 - z));
  return d < h.nbc ? __fmul_rn(u, __ldg(h.wtab + d)) : u;
}

template <int N>
__device__ __forceinline__ void el_vel_at(const Geo2& g, const Coef& c, float dtx, float dtz,
                                          const ElFields& a, const ElMat& m, int x, int z,
                                          float& ux, float& uz) {
  long long p = (long long)z * g.ld + x;
  float vx = __ldg(a.vx + p), vz = __ldg(a.vz + p);
  if (interior2(g, x, z)) {
    const long long sz = g.ld;
    float dxx = dm<N>(a.txx, p, 1, c);
    float dxzz = dm<N>(a.txz, p, sz, c);
    float dxzx = dp<N>(a.txz, p, 1, c);
    float dzz = dp<N>(a.tzz, p, sz, c);
    vx = __fmaf_rn(__ldg(m.bx + p), __fmaf_rn(dtx, dxx, __fmul_rn(dtz, dxzz)), vx);
    vz = __fmaf_rn(__ldg(m.bz + p), __fmaf_rn(dtx, dxzx, __fmul_rn(dtz, dzz)), vz);
  }
  ux = vx;
  uz = vz;
}

// SP: the sponge boundary instead of the fused HABC.
template <int N, bool SP = false>
__global__ void __launch_bounds__(256) k_el_vel(Geo2 g, Coef c, float dtx, float dtz, HabcDev h,
                                                ElFields a, ElMat m, float* __restrict__ vx1,
                                                float* __restrict__ vz1) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int z = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= g.nx || z >= g.nz) return;
  const long long so = (long long)blockIdx.z * g.plane;
  a.vx += so; a.vz += so; a.txx += so; a.tzz += so; a.txz += so;
  float ux, uz;
  el_vel_at<N>(g, c, dtx, dtz, a, m, x, z, ux, uz);
  long long p = (long long)z * g.ld + x;
  int sx, sz, dist;
  if constexpr (SP) {
    ux = sponge_damp(g, h, x, z, ux);
    uz = sponge_damp(g, h, x, z, uz);
  } else if (frame2(g, x, z, sx, sz, dist)) {
    float wx = habc_weight(h, 0, dist), wz = habc_weight(h, 1, dist);
    float fox = __ldg(a.vx + p), foz = __ldg(a.vz + p);
    if (sx != 0 && sz != 0) {
      long long px = p + sx, pz = p + (long long)sz * g.ld;
      float ax, az, bx, bz;
      el_vel_at<N>(g, c, dtx, dtz, a, m, x + sx, z, ax, az);
      el_vel_at<N>(g, c, dtx, dtz, a, m, x, z + sz, bx, bz);
      ux = higdon_corner(wx, ux, higdon_side(h, ax, fox, __ldg(a.vx + px)),
                         higdon_side(h, bx, fox, __ldg(a.vx + pz)));
      uz = higdon_corner(wz, uz, higdon_side(h, az, foz, __ldg(a.vz + px)),
                         higdon_side(h, bz, foz, __ldg(a.vz + pz)));
    } else {
      int nxp = x + sx, nzp = z + sz;
      long long pn = (long long)nzp * g.ld + nxp;
      float nx_, nz_;
      el_vel_at<N>(g, c, dtx, dtz, a, m, nxp, nzp, nx_, nz_);
      ux = higdon_edge(wx, ux, higdon_side(h, nx_, fox, __ldg(a.vx + pn)));
      uz = higdon_edge(wz, uz, higdon_side(h, nz_, foz, __ldg(a.vz + pn)));
    }
  }
  vx1[so + p] = ux;
  vz1[so + p] = uz;
}

template <int N>
__device__ __forceinline__ void el_str_at(const Geo2& g, const Coef& c, float dtx, float dtz,
                                          const float* __restrict__ vx, const float* __restrict__ vz,
                                          const ElFields& a, const ElMat& m, int x, int z,
                                          float& sxx, float& szz, float& sxz) {
  long long p = (long long)z * g.ld + x;
  sxx = __ldg(a.txx + p);
  szz = __ldg(a.tzz + p);
  sxz = __ldg(a.txz + p);
  if (interior2(g, x, z)) {
    const long long sz = g.ld;
    float dvxdx = dp<N>(vx, p, 1, c);
    float dvzdz = dm<N>(vz, p, sz, c);
    float dvxdz = dp<N>(vx, p, sz, c);
    float dvzdx = dm<N>(vz, p, 1, c);
    float lam = __ldg(m.lam + p), l2m = __ldg(m.l2m + p);
    float ex = __fmul_rn(dvxdx, dtx), ez = __fmul_rn(dvzdz, dtz);
    sxx = __fadd_rn(sxx, __fmaf_rn(l2m, ex, __fmul_rn(lam, ez)));
    szz = __fadd_rn(szz, __fmaf_rn(lam, ex, __fmul_rn(l2m, ez)));
    sxz = __fmaf_rn(__ldg(m.mut + p), __fmaf_rn(dvxdz, dtz, __fmul_rn(dvzdx, dtx)), sxz);
  }
}

// TG: inject into txx, tzz and record vx, vz on tagged cells (step *t.it0 + j + 1).
template <int N, bool SP = false, bool TG = false>
__global__ void __launch_bounds__(256) k_el_str(Geo2 g, Coef c, float dtx, float dtz, HabcDev h,
                                                ElFields a, const float* __restrict__ vx1,
                                                const float* __restrict__ vz1, ElMat m,
                                                float* __restrict__ txx1, float* __restrict__ tzz1,
                                                float* __restrict__ txz1,
                                                CellTags t = CellTags{}, int j = 0) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int z = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= g.nx || z >= g.nz) return;
  const long long so = (long long)blockIdx.z * g.plane;
  a.txx += so; a.tzz += so; a.txz += so;
  const float* vx = vx1 + so;
  const float* vz = vz1 + so;
  float sxx, szz, sxz;
  el_str_at<N>(g, c, dtx, dtz, vx, vz, a, m, x, z, sxx, szz, sxz);
  long long p = (long long)z * g.ld + x;
  int sx, sz, dist;
  if constexpr (SP) {
    sxx = sponge_damp(g, h, x, z, sxx);
    szz = sponge_damp(g, h, x, z, szz);
    sxz = sponge_damp(g, h, x, z, sxz);
  } else if (frame2(g, x, z, sx, sz, dist)) {
    float w = habc_weight(h, 2, dist);
    float o1 = __ldg(a.txx + p), o2 = __ldg(a.tzz + p), o3 = __ldg(a.txz + p);
    if (sx != 0 && sz != 0) {
      long long px = p + sx, pz = p + (long long)sz * g.ld;
      float a1, a2, a3, b1, b2, b3;
      el_str_at<N>(g, c, dtx, dtz, vx, vz, a, m, x + sx, z, a1, a2, a3);
      el_str_at<N>(g, c, dtx, dtz, vx, vz, a, m, x, z + sz, b1, b2, b3);
      sxx = higdon_corner(w, sxx, higdon_side(h, a1, o1, __ldg(a.txx + px)),
                          higdon_side(h, b1, o1, __ldg(a.txx + pz)));
      szz = higdon_corner(w, szz, higdon_side(h, a2, o2, __ldg(a.tzz + px)),
                          higdon_side(h, b2, o2, __ldg(a.tzz + pz)));
      sxz = higdon_corner(w, sxz, higdon_side(h, a3, o3, __ldg(a.txz + px)),
                          higdon_side(h, b3, o3, __ldg(a.txz + pz)));
    } else {
      int xn = x + sx, zn = z + sz;
      long long pn = (long long)zn * g.ld + xn;
      float n1, n2, n3;
      el_str_at<N>(g, c, dtx, dtz, vx, vz, a, m, xn, zn, n1, n2, n3);
      sxx = higdon_edge(w, sxx, higdon_side(h, n1, o1, __ldg(a.txx + pn)));
      szz = higdon_edge(w, szz, higdon_side(h, n2, o2, __ldg(a.tzz + pn)));
      sxz = higdon_edge(w, sxz, higdon_side(h, n3, o3, __ldg(a.txz + pn)));
    }
  }
  if constexpr (TG) {
    const int e = __ldg(t.tag + p);
    if (e >= 0) {
      const long long k = (long long)(*t.it0 + j);
      const int4 E = t.ent[e];
      sxx = tag_inject(t, E, k, blockIdx.z, sxx);
      szz = tag_inject(t, E, k, blockIdx.z, szz);
      tag_record(t, E, k, blockIdx.z, __ldg(vx + p), __ldg(vz + p), 0.0f);
    }
  }
  txx1[so + p] = sxx;
  tzz1[so + p] = szz;
  txz1[so + p] = sxz;
}

// ---------------------------------------------------------------------------
// acoustic2d velocity / pressure (acoustic2d/fused_kernels.jl:27-114,
// batch.jl:38-120)
// ---------------------------------------------------------------------------
template <int N>
__device__ __forceinline__ void ac_vel_at(const Geo2& g, const Coef& c, float dtx, float dtz,
                                          const float* __restrict__ pr, const float* __restrict__ vx0,
                                          const float* __restrict__ vz0, const float* __restrict__ bx,
                                          const float* __restrict__ bz, int x, int z, float& ux,
                                          float& uz) {
  long long p = (long long)z * g.ld + x;
  float vx = __ldg(vx0 + p), vz = __ldg(vz0 + p);
  if (interior2(g, x, z)) {
    float dpdx = dm<N>(pr, p, 1, c);
    float dpdz = dp<N>(pr, p, g.ld, c);
    vx = __fmaf_rn(__fmul_rn(__ldg(bx + p), dtx), dpdx, vx);
    vz = __fmaf_rn(__fmul_rn(__ldg(bz + p), dtz), dpdz, vz);
  }
  ux = vx;
  uz = vz;
}

// Velocity of time n+1 at (x, z) with the fused HABC (kernels_det.jl:22-57):
// the shared body of the uniform-batch and uneven-batch kernels.
template <int N>
__device__ __forceinline__ void ac_vel_cell(const Geo2& g, const Coef& c, float dtx, float dtz,
                                            const HabcDev& h, const float* __restrict__ p0,
                                            const float* __restrict__ vx0,
                                            const float* __restrict__ vz0,
                                            const float* __restrict__ bx,
                                            const float* __restrict__ bz, int x, int z, float& ux,
                                            float& uz) {
  ac_vel_at<N>(g, c, dtx, dtz, p0, vx0, vz0, bx, bz, x, z, ux, uz);
  long long p = (long long)z * g.ld + x;
  int sx, sz, dist;
  if (frame2(g, x, z, sx, sz, dist)) {
    float wx = habc_weight(h, 0, dist), wz = habc_weight(h, 1, dist);
    float fox = __ldg(vx0 + p), foz = __ldg(vz0 + p);
    if (sx != 0 && sz != 0) {
      long long px = p + sx, pz = p + (long long)sz * g.ld;
      float ax, az, bxv, bzv;
      ac_vel_at<N>(g, c, dtx, dtz, p0, vx0, vz0, bx, bz, x + sx, z, ax, az);
      ac_vel_at<N>(g, c, dtx, dtz, p0, vx0, vz0, bx, bz, x, z + sz, bxv, bzv);
      ux = higdon_corner(wx, ux, higdon_side(h, ax, fox, __ldg(vx0 + px)),
                         higdon_side(h, bxv, fox, __ldg(vx0 + pz)));
      uz = higdon_corner(wz, uz, higdon_side(h, az, foz, __ldg(vz0 + px)),
                         higdon_side(h, bzv, foz, __ldg(vz0 + pz)));
    } else {
      int xn = x + sx, zn = z + sz;
      long long pn = (long long)zn * g.ld + xn;
      float nx_, nz_;
      ac_vel_at<N>(g, c, dtx, dtz, p0, vx0, vz0, bx, bz, xn, zn, nx_, nz_);
      ux = higdon_edge(wx, ux, higdon_side(h, nx_, fox, __ldg(vx0 + pn)));
      uz = higdon_edge(wz, uz, higdon_side(h, nz_, foz, __ldg(vz0 + pn)));
    }
  }
}

// The acoustic velocity update comes in two occupancy forms with one body:
// k_ac_vel (no register bound; 40 registers, 6 blocks per SM) for the small,
// latency-bound tagged runs, and k_ac_vel8 (8 blocks per SM, 32 registers) for
// large grids.  The results are the same.
#define FOMO_AC_VEL_PARAMS                                                                 \
  Geo2 g, Coef c, float dtx, float dtz, HabcDev h, const float* __restrict__ p0,           \
      const float* __restrict__ vx0, const float* __restrict__ vz0,                        \
      const float* __restrict__ bx, const float* __restrict__ bz, float* __restrict__ vx1, \
      float* __restrict__ vz1
template <int N, bool SP>
__device__ __forceinline__ void ac_vel_body(FOMO_AC_VEL_PARAMS) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int z = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= g.nx || z >= g.nz) return;
  const long long so = (long long)blockIdx.z * g.plane;
  p0 += so; vx0 += so; vz0 += so;
  float ux, uz;
  if constexpr (SP) {
    ac_vel_at<N>(g, c, dtx, dtz, p0, vx0, vz0, bx, bz, x, z, ux, uz);
    ux = sponge_damp(g, h, x, z, ux);
    uz = sponge_damp(g, h, x, z, uz);
  } else {
    ac_vel_cell<N>(g, c, dtx, dtz, h, p0, vx0, vz0, bx, bz, x, z, ux, uz);
  }
  long long p = (long long)z * g.ld + x;
  vx1[so + p] = ux;
  vz1[so + p] = uz;
}
template <int N, bool SP = false>
__global__ void __launch_bounds__(256) k_ac_vel(FOMO_AC_VEL_PARAMS) {
  ac_vel_body<N, SP>(g, c, dtx, dtz, h, p0, vx0, vz0, bx, bz, vx1, vz1);
}
template <int N, bool SP = false>
__global__ void __launch_bounds__(256, 8) k_ac_vel8(FOMO_AC_VEL_PARAMS) {
  ac_vel_body<N, SP>(g, c, dtx, dtz, h, p0, vx0, vz0, bx, bz, vx1, vz1);
}
#undef FOMO_AC_VEL_PARAMS

template <int N>
__device__ __forceinline__ float ac_prs_at(const Geo2& g, const Coef& c, float dtx, float dtz,
                                           const float* __restrict__ vx, const float* __restrict__ vz,
                                           const float* __restrict__ p0,
                                           const float* __restrict__ kappa, int x, int z) {
  long long p = (long long)z * g.ld + x;
  float v = __ldg(p0 + p);
  if (interior2(g, x, z)) {
    float dvxdx = dp<N>(vx, p, 1, c);
    float dvzdz = dm<N>(vz, p, g.ld, c);
    v = __fmaf_rn(__ldg(kappa + p), __fmaf_rn(dvxdx, dtx, __fmul_rn(dvzdz, dtz)), v);
  }
  return v;
}

// Pressure of time n+1 at (x, z) with the fused HABC.
template <int N>
__device__ __forceinline__ float ac_prs_cell(const Geo2& g, const Coef& c, float dtx, float dtz,
                                             const HabcDev& h, const float* __restrict__ p0,
                                             const float* __restrict__ vx,
                                             const float* __restrict__ vz,
                                             const float* __restrict__ kappa, int x, int z) {
  float u = ac_prs_at<N>(g, c, dtx, dtz, vx, vz, p0, kappa, x, z);
  long long p = (long long)z * g.ld + x;
  int sx, sz, dist;
  if (frame2(g, x, z, sx, sz, dist)) {
    float w = habc_weight(h, 2, dist);
    float fo = __ldg(p0 + p);
    if (sx != 0 && sz != 0) {
      long long px = p + sx, pz = p + (long long)sz * g.ld;
      float a = ac_prs_at<N>(g, c, dtx, dtz, vx, vz, p0, kappa, x + sx, z);
      float b = ac_prs_at<N>(g, c, dtx, dtz, vx, vz, p0, kappa, x, z + sz);
      u = higdon_corner(w, u, higdon_side(h, a, fo, __ldg(p0 + px)),
                        higdon_side(h, b, fo, __ldg(p0 + pz)));
    } else {
      int xn = x + sx, zn = z + sz;
      long long pn = (long long)zn * g.ld + xn;
      float a = ac_prs_at<N>(g, c, dtx, dtz, vx, vz, p0, kappa, xn, zn);
      u = higdon_edge(w, u, higdon_side(h, a, fo, __ldg(p0 + pn)));
    }
  }
  return u;
}

// TG: inject into p and record p, vx, vz on tagged cells.  k_ac_prs (no register
// bound) serves the small tagged runs, k_ac_prs8 (8 blocks per SM) large grids,
// as for the velocity update.
#define FOMO_AC_PRS_PARAMS                                                                  \
  Geo2 g, Coef c, float dtx, float dtz, HabcDev h, const float* __restrict__ p0,            \
      const float* __restrict__ vx1, const float* __restrict__ vz1,                         \
      const float* __restrict__ kappa, float* __restrict__ p1, CellTags t, int j
template <int N, bool SP, bool TG>
__device__ __forceinline__ void ac_prs_body(FOMO_AC_PRS_PARAMS) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int z = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= g.nx || z >= g.nz) return;
  const long long so = (long long)blockIdx.z * g.plane;
  float u;
  if constexpr (SP)
    u = sponge_damp(g, h, x, z,
                    ac_prs_at<N>(g, c, dtx, dtz, vx1 + so, vz1 + so, p0 + so, kappa, x, z));
  else
    u = ac_prs_cell<N>(g, c, dtx, dtz, h, p0 + so, vx1 + so, vz1 + so, kappa, x, z);
  if constexpr (TG) {
    const long long p = (long long)z * g.ld + x;
    const int e = __ldg(t.tag + p);
    if (e >= 0) {
      const long long k = (long long)(*t.it0 + j);
      const int4 E = t.ent[e];
      u = tag_inject(t, E, k, blockIdx.z, u);
      tag_record(t, E, k, blockIdx.z, u, __ldg(vx1 + so + p), __ldg(vz1 + so + p));
    }
  }
  p1[so + (long long)z * g.ld + x] = u;
}
template <int N, bool SP = false, bool TG = false>
__global__ void __launch_bounds__(256) k_ac_prs(FOMO_AC_PRS_PARAMS) {
  ac_prs_body<N, SP, TG>(g, c, dtx, dtz, h, p0, vx1, vz1, kappa, p1, t, j);
}
template <int N, bool SP = false>
__global__ void __launch_bounds__(256, 8) k_ac_prs8(FOMO_AC_PRS_PARAMS) {
  ac_prs_body<N, SP, false>(g, c, dtx, dtz, h, p0, vx1, vz1, kappa, p1, t, j);
}
#undef FOMO_AC_PRS_PARAMS

// ---------------------------------------------------------------------------
// scalar2d leapfrog (scalar2d/scalar2d.jl:29-84): u2 = update(u1, u0), then
// HABC with f_old = u1; three rotating buffers keep every read race-free.
// ---------------------------------------------------------------------------
struct D2Coef {
  float two_c0;
  float d[5];
};

template <int N>
__device__ __forceinline__ float sc_at(const Geo2& g, const D2Coef& c, const float* __restrict__ u1,
                                       const float* __restrict__ u0, const float* __restrict__ c2,
                                       int x, int z) {
  long long p = (long long)z * g.ld + x;
  float uc = __ldg(u1 + p);
  if (!interior2(g, x, z)) return uc;
  float lap = __fmul_rn(c.two_c0, uc);
  const long long s = g.ld;
#pragma unroll
  for (int l = 1; l <= N; ++l) {
    float nb = __fadd_rn(__fadd_rn(__fadd_rn(__ldg(u1 + p + l), __ldg(u1 + p - l)),
                                   __ldg(u1 + p + l * s)),
                         __ldg(u1 + p - l * s));
    lap = __fmaf_rn(c.d[l - 1], nb, lap);
  }
  return __fmaf_rn(__ldg(c2 + p), lap, __fsub_rn(__fmul_rn(2.0f, uc), __ldg(u0 + p)));
}

// TG: inject into u and record it on tagged cells (step *t.it0 + j + 1).  Tagged
// (small, latency-bound) runs take 6 blocks per SM, untagged (large) ones 8.
template <int N, bool TG = false>
__global__ void __launch_bounds__(256, TG ? 6 : 8) k_sc_step(Geo2 g, D2Coef c, HabcDev h,
                                                 const float* __restrict__ u1,
                                                 const float* __restrict__ u0,
                                                 const float* __restrict__ c2,
                                                 float* __restrict__ u2,
                                                 CellTags t = CellTags{}, int j = 0) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int z = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= g.nx || z >= g.nz) return;
  float u = sc_at<N>(g, c, u1, u0, c2, x, z);
  long long p = (long long)z * g.ld + x;
  int sx, sz, dist;
  if (frame2(g, x, z, sx, sz, dist)) {
    float w = habc_weight(h, 2, dist);
    float fo = __ldg(u1 + p);
    if (sx != 0 && sz != 0) {
      long long px = p + sx, pz = p + (long long)sz * g.ld;
      float a = sc_at<N>(g, c, u1, u0, c2, x + sx, z);
      float b = sc_at<N>(g, c, u1, u0, c2, x, z + sz);
      u = higdon_corner(w, u, higdon_side(h, a, fo, __ldg(u1 + px)),
                        higdon_side(h, b, fo, __ldg(u1 + pz)));
    } else {
      int xn = x + sx, zn = z + sz;
      long long pn = (long long)zn * g.ld + xn;
      float a = sc_at<N>(g, c, u1, u0, c2, xn, zn);
      u = higdon_edge(w, u, higdon_side(h, a, fo, __ldg(u1 + pn)));
    }
  }
  if constexpr (TG) {
    const int e = __ldg(t.tag + p);
    if (e >= 0) {
      const long long k = (long long)(*t.it0 + j);
      const int4 E = t.ent[e];
      u = tag_inject(t, E, k, 0, u);
      tag_record(t, E, k, 0, u, 0.0f, 0.0f);
    }
  }
  u2[p] = u;
}

// ---------------------------------------------------------------------------
// Injection then recording, one block per shot (inject_source.jl:4-24,
// batch_acq.jl:40-130, record_receiver.jl:3-18).  Sources are added by one
// thread in source order, so coincident sources sum deterministically (the
// reference's concurrent `+=` races there); recording follows a barrier so a
// receiver on a source cell sees the injected value, as the reference's
// launch order does.
//   inj0/inj1: fields receiving the wavelet (acoustic p; elastic txx,tzz;
//              scalar u).  rec0..2: recorded fields (null = skip).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void inject_record_body(int it, int nt, long long plane, int n_src,
                                                   const int* __restrict__ src_lin,
                                                   const float* __restrict__ wav, float* inj0,
                                                   float* inj1, int n_rec,
                                                   const int* __restrict__ rec_lin,
                                                   const float* rec0, const float* rec1,
                                                   const float* rec2, float* __restrict__ s0,
                                                   float* __restrict__ s1, float* __restrict__ s2);

static __global__ void k_inject_record(int it, int nt, long long plane, int n_src,
                                const int* __restrict__ src_lin, const float* __restrict__ wav,
                                float* inj0, float* inj1, int n_rec,
                                const int* __restrict__ rec_lin, const float* rec0,
                                const float* rec1, const float* rec2, float* __restrict__ s0,
                                float* __restrict__ s1, float* __restrict__ s2) {
  inject_record_body(it, nt, plane, n_src, src_lin, wav, inj0, inj1, n_rec, rec_lin, rec0, rec1,
                     rec2, s0, s1, s2);
}

// The same for step *it0 + j + 1: inside a captured chunk of steps the step
// index lives in device memory (it0 = steps completed before the chunk).
static __global__ void k_inject_record_at(const int* __restrict__ it0, int j, int nt,
                                          long long plane, int n_src,
                                          const int* __restrict__ src_lin,
                                          const float* __restrict__ wav, float* inj0, float* inj1,
                                          int n_rec, const int* __restrict__ rec_lin,
                                          const float* rec0, const float* rec1, const float* rec2,
                                          float* __restrict__ s0, float* __restrict__ s1,
                                          float* __restrict__ s2) {
  inject_record_body(*it0 + j + 1, nt, plane, n_src, src_lin, wav, inj0, inj1, n_rec, rec_lin,
                     rec0, rec1, rec2, s0, s1, s2);
}

// Interior snapshot (nx x nz, x fastest) of step *it0 + j + 1 when that step
// is a multiple of snap_interval (fused_kernels.jl:192-195).
static __global__ void k_snap_at(const int* __restrict__ it0, int j, int snap_interval,
                                 const float* __restrict__ src, long long ld, int nx, int nz,
                                 float* __restrict__ snaps) {
  const int it = *it0 + j + 1;
  if (it % snap_interval) return;
  float* dst = snaps + (long long)(it / snap_interval - 1) * nx * nz;
  const int z = blockIdx.y;
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < nx; x += gridDim.x * blockDim.x)
    dst[(long long)z * nx + x] = src[(long long)z * ld + x];
}

// Advances the device step index by the chunk length.
static __global__ void k_step_add(int* it0, int k) { *it0 += k; }

__device__ __forceinline__ void inject_record_body(int it, int nt, long long plane, int n_src,
                                                   const int* __restrict__ src_lin,
                                                   const float* __restrict__ wav, float* inj0,
                                                   float* inj1, int n_rec,
                                                   const int* __restrict__ rec_lin,
                                                   const float* rec0, const float* rec1,
                                                   const float* rec2, float* __restrict__ s0,
                                                   float* __restrict__ s1, float* __restrict__ s2) {
  const int s = blockIdx.x;
  const long long so = (long long)s * plane;
  if (threadIdx.x == 0) {
    for (int q = 0; q < n_src; ++q) {
      long long p = so + src_lin[(long long)s * n_src + q];
      float w = wav[(long long)(it - 1) * n_src + q];
      inj0[p] = __fadd_rn(inj0[p], w);
      if (inj1) inj1[p] = __fadd_rn(inj1[p], w);
    }
  }
  __syncthreads();
  const long long ob = (long long)n_rec * ((long long)(it - 1) + (long long)nt * s);
  for (int r = threadIdx.x; r < n_rec; r += blockDim.x) {
    long long p = so + rec_lin[r];
    if (rec0) s0[ob + r] = rec0[p];
    if (rec1) s1[ob + r] = rec1[p];
    if (rec2) s2[ob + r] = rec2[p];
  }
}

}  // namespace fomo
