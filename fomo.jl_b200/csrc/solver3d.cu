// solver3d.cu -- acoustic3d and elastic3d (equations/acoustic3d, equations/elastic3d).
//
// One step = velocity update (all cells, A -> B) + two-pass HABC on the
// velocity frame + stress/pressure update (A,B -> B) + two-pass HABC on the
// stress frame + inject/record.  The reference's 3D Higdon kernel
// (boundary/habc/kernels_3d.jl:117-193) updates in place and races between
// neighbouring frame cells; here pass 1 evaluates every frame cell from the
// read-only pre-correction field into a frame-indexed scratch and pass 2
// writes it back, so results are deterministic (the same two-pass form as the
// reference's 2D det-HABC, kernels_det.jl).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "fomo_internal.cuh"
#include "sweep3d.cuh"

namespace fomo {

// Injection and recording of one 3D step (linear indices; a negative index
// is a point another z-slab holds, skipped here).  The injected fields (p, or
// txx/tyy/tzz) are never the recorded ones (vx, vy, vz), so the recording
// needs no ordering after the injection and runs over all blocks; block 0
// injects.
__global__ void k_inject_record3(int it, int nt, int n_src, const int* __restrict__ src_lin,
                                 const float* __restrict__ wav, float* inj0, float* inj1,
                                 float* inj2, int n_rec, const int* __restrict__ rec_lin,
                                 const float* rec0, const float* rec1, const float* rec2,
                                 float* __restrict__ s0, float* __restrict__ s1,
                                 float* __restrict__ s2) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    for (int q = 0; q < n_src; ++q) {
      const long long p = src_lin[q];
      if (p < 0) continue;
      const float w = wav[(long long)(it - 1) * n_src + q];
      inj0[p] = __fadd_rn(inj0[p], w);
      if (inj1) inj1[p] = __fadd_rn(inj1[p], w);
      if (inj2) inj2[p] = __fadd_rn(inj2[p], w);
    }
  }
  const long long ob = (long long)n_rec * (it - 1);
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n_rec; r += gridDim.x * blockDim.x) {
    const long long p = rec_lin[r];
    if (p < 0) continue;
    s0[ob + r] = rec0[p];
    s1[ob + r] = rec1[p];
    s2[ob + r] = rec2[p];
  }
}

namespace {

__device__ __forceinline__ bool interior3(const Geo3& g, int x, int y, int z) {
  return x >= g.M && x < g.nx - g.M && y >= g.M && y < g.ny - g.M && z >= g.M && z < g.nz - g.M;
}

template <int N>
__device__ __forceinline__ float dmS(const float* __restrict__ f, long long p, long long s,
                                     const Coef& c) {
  return dm<N>(f, p, s, c);
}

// ---------------------------------------------------------------------------
// acoustic3d updates (acoustic3d/update_velocity.jl:16-53, update_pressure.jl:16-50)
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(256) k_ac3_vel(Geo3 g, Coef c, float dtdh,
                                                 const float* __restrict__ p,
                                                 const float* __restrict__ vx0,
                                                 const float* __restrict__ vy0,
                                                 const float* __restrict__ vz0,
                                                 const float* __restrict__ bx,
                                                 const float* __restrict__ by,
                                                 const float* __restrict__ bz, float* vx1,
                                                 float* vy1, float* vz1) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= g.nx || y >= g.ny || z >= g.nz) return;
  const long long q = x + g.sy * y + g.sz * z;
  float ux = __ldg(vx0 + q), uy = __ldg(vy0 + q), uz = __ldg(vz0 + q);
  if (interior3(g, x, y, z)) {
    const float dx = dm<N>(p, q, 1, c), dy = dm<N>(p, q, g.sy, c), dz = dp<N>(p, q, g.sz, c);
    ux = __fmaf_rn(__fmul_rn(__ldg(bx + q), dtdh), dx, ux);
    uy = __fmaf_rn(__fmul_rn(__ldg(by + q), dtdh), dy, uy);
    uz = __fmaf_rn(__fmul_rn(__ldg(bz + q), dtdh), dz, uz);
  }
  vx1[q] = ux;
  vy1[q] = uy;
  vz1[q] = uz;
}

template <int N>
__global__ void __launch_bounds__(256) k_ac3_prs(Geo3 g, Coef c, float dtdh,
                                                 const float* __restrict__ p0,
                                                 const float* __restrict__ vx,
                                                 const float* __restrict__ vy,
                                                 const float* __restrict__ vz,
                                                 const float* __restrict__ kap, float* p1) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= g.nx || y >= g.ny || z >= g.nz) return;
  const long long q = x + g.sy * y + g.sz * z;
  float u = __ldg(p0 + q);
  if (interior3(g, x, y, z)) {
    const float dx = dp<N>(vx, q, 1, c), dy = dp<N>(vy, q, g.sy, c), dz = dm<N>(vz, q, g.sz, c);
    u = __fmaf_rn(__fmul_rn(__ldg(kap + q), dtdh), __fadd_rn(__fadd_rn(dx, dy), dz), u);
  }
  p1[q] = u;
}

// ---------------------------------------------------------------------------
// elastic3d updates (elastic3d/update_velocity.jl:17-84, update_stress.jl:21-94)
// ---------------------------------------------------------------------------
struct El3 {
  const float* f[9];  // vx vy vz txx tyy tzz txy txz tyz
};
struct El3Out {
  float* f[9];
};
struct El3Mat {
  const float *bx, *by, *bz, *lam, *l2m, *mxy, *mxz, *myz;
};

template <int N>
__global__ void __launch_bounds__(256) k_el3_vel(Geo3 g, Coef c, float dtdh, El3 a, El3Mat m,
                                                 El3Out o) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= g.nx || y >= g.ny || z >= g.nz) return;
  const long long q = x + g.sy * y + g.sz * z;
  float ux = __ldg(a.f[0] + q), uy = __ldg(a.f[1] + q), uz = __ldg(a.f[2] + q);
  if (interior3(g, x, y, z)) {
    const float* txx = a.f[3];
    const float* tyy = a.f[4];
    const float* tzz = a.f[5];
    const float* txy = a.f[6];
    const float* txz = a.f[7];
    const float* tyz = a.f[8];
    const float a1 = dm<N>(txx, q, 1, c), a2 = dp<N>(txy, q, g.sy, c), a3 = dm<N>(txz, q, g.sz, c);
    const float b1 = dp<N>(txy, q, 1, c), b2 = dm<N>(tyy, q, g.sy, c), b3 = dm<N>(tyz, q, g.sz, c);
    const float c1 = dp<N>(txz, q, 1, c), c2 = dp<N>(tyz, q, g.sy, c), c3 = dp<N>(tzz, q, g.sz, c);
    ux = __fmaf_rn(__fmul_rn(__ldg(m.bx + q), dtdh), __fadd_rn(__fadd_rn(a1, a2), a3), ux);
    uy = __fmaf_rn(__fmul_rn(__ldg(m.by + q), dtdh), __fadd_rn(__fadd_rn(b1, b2), b3), uy);
    uz = __fmaf_rn(__fmul_rn(__ldg(m.bz + q), dtdh), __fadd_rn(__fadd_rn(c1, c2), c3), uz);
  }
  o.f[0][q] = ux;
  o.f[1][q] = uy;
  o.f[2][q] = uz;
}

template <int N>
__global__ void __launch_bounds__(256) k_el3_str(Geo3 g, Coef c, float dtdh, El3 a,
                                                 const float* __restrict__ vx,
                                                 const float* __restrict__ vy,
                                                 const float* __restrict__ vz, El3Mat m,
                                                 El3Out o) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= g.nx || y >= g.ny || z >= g.nz) return;
  const long long q = x + g.sy * y + g.sz * z;
  float s[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) s[f] = __ldg(a.f[3 + f] + q);
  if (interior3(g, x, y, z)) {
    const float dxx = dp<N>(vx, q, 1, c), dyy = dp<N>(vy, q, g.sy, c), dzz = dm<N>(vz, q, g.sz, c);
    const float dxy = dm<N>(vx, q, g.sy, c), dyx = dm<N>(vy, q, 1, c);
    const float dxz = dp<N>(vx, q, g.sz, c), dzx = dm<N>(vz, q, 1, c);
    const float dyz = dp<N>(vy, q, g.sz, c), dzy = dm<N>(vz, q, g.sy, c);
    const float lm = __ldg(m.lam + q), l2 = __ldg(m.l2m + q);
    s[0] = __fmaf_rn(__fmaf_rn(lm, dzz, __fmaf_rn(lm, dyy, __fmul_rn(l2, dxx))), dtdh, s[0]);
    s[1] = __fmaf_rn(__fmaf_rn(lm, dzz, __fmaf_rn(l2, dyy, __fmul_rn(lm, dxx))), dtdh, s[1]);
    s[2] = __fmaf_rn(__fmaf_rn(l2, dzz, __fmaf_rn(lm, dyy, __fmul_rn(lm, dxx))), dtdh, s[2]);
    s[3] = __fmaf_rn(__fmul_rn(__ldg(m.mxy + q), __fadd_rn(dxy, dyx)), dtdh, s[3]);
    s[4] = __fmaf_rn(__fmul_rn(__ldg(m.mxz + q), __fadd_rn(dxz, dzx)), dtdh, s[4]);
    s[5] = __fmaf_rn(__fmul_rn(__ldg(m.myz + q), __fadd_rn(dyz, dzy)), dtdh, s[5]);
  }
#pragma unroll
  for (int f = 0; f < 6; ++f) o.f[3 + f][q] = s[f];
}

// ---------------------------------------------------------------------------
// z-marching forms of the elastic3d updates: the same per-cell arithmetic as
// k_el3_vel / k_el3_str (bit-identical).  A 32x8 thread tile marches down a
// range of z planes.  The z-derivative inputs of a thread's own column sit in
// register windows (w[k] = plane z - N + k, k = 0..2N); the x/y neighbours of
// plane z come from shared-memory tiles with N-wide halos.  Each input is read
// from HBM about once per step, against the per-cell kernels' 2N re-reads of
// every z-derivative input.  Persistent blocks take (tile, z-chunk) items.
// ---------------------------------------------------------------------------
constexpr int kZmX = 32, kZmY = 8;

struct ZmPlan {
  int ntx, nty;  // tiles in x and y
  int zch;       // planes per z-chunk
  int items;     // ntx * nty * chunks
};

// staggered sums over shared memory (f at the cell, s = element stride)
template <int N>
__device__ __forceinline__ float sdm(const float* f, int s, const Coef& c) {
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l)
    acc = __fmaf_rn(c.a[l - 1], __fsub_rn(f[(l - 1) * s], f[-l * s]), acc);
  return acc;
}
template <int N>
__device__ __forceinline__ float sdp(const float* f, int s, const Coef& c) {
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l)
    acc = __fmaf_rn(c.a[l - 1], __fsub_rn(f[l * s], f[-(l - 1) * s]), acc);
  return acc;
}
// ... over a register window w[k] = plane z - N + k
template <int N>
__device__ __forceinline__ float wdm(const float (&w)[2 * N + 1], const Coef& c) {
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l) acc = __fmaf_rn(c.a[l - 1], __fsub_rn(w[N + l - 1], w[N - l]), acc);
  return acc;
}
template <int N>
__device__ __forceinline__ float wdp(const float (&w)[2 * N + 1], const Coef& c) {
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l) acc = __fmaf_rn(c.a[l - 1], __fsub_rn(w[N + l], w[N - l + 1]), acc);
  return acc;
}

// zero outside the padded grid
__device__ __forceinline__ float ld3(const Geo3& g, const float* __restrict__ f, int x, int y,
                                     int z) {
  return (x >= 0 && x < g.nx && y >= 0 && y < g.ny && z >= 0 && z < g.nz)
             ? __ldg(f + x + g.sy * y + g.sz * z)
             : 0.0f;
}

template <int N>
__global__ void __launch_bounds__(kZmX * kZmY, 3) k_el3_vel_zm(Geo3 g, Coef c, float dtdh, El3 a,
                                                            El3Mat m, El3Out o, ZmPlan zp) {
  constexpr int H = N, TX = kZmX, TY = kZmY, WX = TX + 2 * H, WY = TY + 2 * H;
  __shared__ float s_xx[TY][WX], s_xy[WY][WX], s_yy[WY][TX], s_xz[TY][WX], s_yz[WY][TX];
  const int tx = threadIdx.x, ty = threadIdx.y;
  // halo cells this thread loads: one x side (TX >= 2H), and the top and/or
  // bottom y side (both when H > TY / 2)
  const bool hxl = tx < H, hxr = tx >= TX - H, hyl = ty < H, hyr = ty >= TY - H;
  const int hx = hxl ? -H : H;
  const float *txx = a.f[3], *tyy = a.f[4], *tzz = a.f[5], *txy = a.f[6], *txz = a.f[7],
              *tyz = a.f[8];
  for (int item = blockIdx.x; item < zp.items; item += gridDim.x) {
    const int tile = item % (zp.ntx * zp.nty), chunk = item / (zp.ntx * zp.nty);
    const int x = (tile % zp.ntx) * TX + tx, y = (tile / zp.ntx) * TY + ty;
    const int z0 = chunk * zp.zch, z1 = min(g.nz, z0 + zp.zch);
    const bool own = x < g.nx && y < g.ny;
    const long long col = x + g.sy * y;
    float wxz[2 * N + 1], wyz[2 * N + 1], wzz[2 * N + 1];
#pragma unroll
    for (int k = 0; k < 2 * N; ++k) {
      wxz[k] = ld3(g, txz, x, y, z0 - N + k);
      wyz[k] = ld3(g, tyz, x, y, z0 - N + k);
      wzz[k] = ld3(g, tzz, x, y, z0 - N + k);
    }
    // values of the next plane, loaded one iteration ahead: tile centres, this
    // thread's x / y halo cells, and the window planes z + N
    float p_xx, p_xy, p_yy, h_xx, h_xy, h_xz, n_xz, n_yz, n_zz;
    float t_xy, t_yy, t_yz, b_xy, b_yy, b_yz;
    auto fetch = [&](int zz) {
      p_xx = ld3(g, txx, x, y, zz);
      p_xy = ld3(g, txy, x, y, zz);
      p_yy = ld3(g, tyy, x, y, zz);
      if (hxl || hxr) {
        h_xx = ld3(g, txx, x + hx, y, zz);
        h_xy = ld3(g, txy, x + hx, y, zz);
        h_xz = ld3(g, txz, x + hx, y, zz);
      }
      if (hyl) {
        t_xy = ld3(g, txy, x, y - H, zz);
        t_yy = ld3(g, tyy, x, y - H, zz);
        t_yz = ld3(g, tyz, x, y - H, zz);
      }
      if (hyr) {
        b_xy = ld3(g, txy, x, y + H, zz);
        b_yy = ld3(g, tyy, x, y + H, zz);
        b_yz = ld3(g, tyz, x, y + H, zz);
      }
      n_xz = ld3(g, txz, x, y, zz + N);
      n_yz = ld3(g, tyz, x, y, zz + N);
      n_zz = ld3(g, tzz, x, y, zz + N);
    };
    fetch(z0);
    for (int z = z0; z < z1; ++z) {
      wxz[2 * N] = n_xz;
      wyz[2 * N] = n_yz;
      wzz[2 * N] = n_zz;
      __syncthreads();  // the previous plane's readers are done
      s_xx[ty][tx + H] = p_xx;
      s_xy[ty + H][tx + H] = p_xy;
      s_yy[ty + H][tx] = p_yy;
      s_xz[ty][tx + H] = wxz[N];
      s_yz[ty + H][tx] = wyz[N];
      if (hxl || hxr) {
        const int cx = hxl ? tx : tx + 2 * H;
        s_xx[ty][cx] = h_xx;
        s_xy[ty + H][cx] = h_xy;
        s_xz[ty][cx] = h_xz;
      }
      if (hyl) {
        s_xy[ty][tx + H] = t_xy;
        s_yy[ty][tx] = t_yy;
        s_yz[ty][tx] = t_yz;
      }
      if (hyr) {
        s_xy[ty + 2 * H][tx + H] = b_xy;
        s_yy[ty + 2 * H][tx] = b_yy;
        s_yz[ty + 2 * H][tx] = b_yz;
      }
      if (z + 1 < z1) fetch(z + 1);
      __syncthreads();
      if (own) {
        const long long q = col + g.sz * z;
        float ux = __ldg(a.f[0] + q), uy = __ldg(a.f[1] + q), uz = __ldg(a.f[2] + q);
        if (interior3(g, x, y, z)) {
          const float a1 = sdm<N>(&s_xx[ty][tx + H], 1, c);
          const float a2 = sdp<N>(&s_xy[ty + H][tx + H], WX, c);
          const float a3 = wdm<N>(wxz, c);
          const float b1 = sdp<N>(&s_xy[ty + H][tx + H], 1, c);
          const float b2 = sdm<N>(&s_yy[ty + H][tx], TX, c);
          const float b3 = wdm<N>(wyz, c);
          const float c1 = sdp<N>(&s_xz[ty][tx + H], 1, c);
          const float c2 = sdp<N>(&s_yz[ty + H][tx], TX, c);
          const float c3 = wdp<N>(wzz, c);
          ux = __fmaf_rn(__fmul_rn(__ldg(m.bx + q), dtdh), __fadd_rn(__fadd_rn(a1, a2), a3), ux);
          uy = __fmaf_rn(__fmul_rn(__ldg(m.by + q), dtdh), __fadd_rn(__fadd_rn(b1, b2), b3), uy);
          uz = __fmaf_rn(__fmul_rn(__ldg(m.bz + q), dtdh), __fadd_rn(__fadd_rn(c1, c2), c3), uz);
        }
        o.f[0][q] = ux;
        o.f[1][q] = uy;
        o.f[2][q] = uz;
      }
#pragma unroll
      for (int k = 0; k < 2 * N; ++k) {
        wxz[k] = wxz[k + 1];
        wyz[k] = wyz[k + 1];
        wzz[k] = wzz[k + 1];
      }
    }
  }
}

template <int N>
__global__ void __launch_bounds__(kZmX * kZmY, 3) k_el3_str_zm(Geo3 g, Coef c, float dtdh, El3 a,
                                                            const float* __restrict__ vx,
                                                            const float* __restrict__ vy,
                                                            const float* __restrict__ vz,
                                                            El3Mat m, El3Out o, ZmPlan zp) {
  constexpr int H = N, TX = kZmX, TY = kZmY, WX = TX + 2 * H, WY = TY + 2 * H;
  __shared__ float s_vx[WY][WX], s_vy[WY][WX], s_vz[WY][WX];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const bool hxl = tx < H, hxr = tx >= TX - H, hyl = ty < H, hyr = ty >= TY - H;
  const int hx = hxl ? -H : H;
  for (int item = blockIdx.x; item < zp.items; item += gridDim.x) {
    const int tile = item % (zp.ntx * zp.nty), chunk = item / (zp.ntx * zp.nty);
    const int x = (tile % zp.ntx) * TX + tx, y = (tile / zp.ntx) * TY + ty;
    const int z0 = chunk * zp.zch, z1 = min(g.nz, z0 + zp.zch);
    const bool own = x < g.nx && y < g.ny;
    const long long col = x + g.sy * y;
    float wx[2 * N + 1], wy[2 * N + 1], wz[2 * N + 1];
#pragma unroll
    for (int k = 0; k < 2 * N; ++k) {
      wx[k] = ld3(g, vx, x, y, z0 - N + k);
      wy[k] = ld3(g, vy, x, y, z0 - N + k);
      wz[k] = ld3(g, vz, x, y, z0 - N + k);
    }
    // next plane's halo cells and window planes z + N, loaded one iteration ahead
    float h_x, h_y, h_z, n_x, n_y, n_z, t_x, t_y, t_z, b_x, b_y, b_z;
    auto fetch = [&](int zz) {
      if (hxl || hxr) {
        h_x = ld3(g, vx, x + hx, y, zz);
        h_y = ld3(g, vy, x + hx, y, zz);
        h_z = ld3(g, vz, x + hx, y, zz);
      }
      if (hyl) {
        t_x = ld3(g, vx, x, y - H, zz);
        t_y = ld3(g, vy, x, y - H, zz);
        t_z = ld3(g, vz, x, y - H, zz);
      }
      if (hyr) {
        b_x = ld3(g, vx, x, y + H, zz);
        b_y = ld3(g, vy, x, y + H, zz);
        b_z = ld3(g, vz, x, y + H, zz);
      }
      n_x = ld3(g, vx, x, y, zz + N);
      n_y = ld3(g, vy, x, y, zz + N);
      n_z = ld3(g, vz, x, y, zz + N);
    };
    fetch(z0);
    for (int z = z0; z < z1; ++z) {
      wx[2 * N] = n_x;
      wy[2 * N] = n_y;
      wz[2 * N] = n_z;
      __syncthreads();  // the previous plane's readers are done
      s_vx[ty + H][tx + H] = wx[N];
      s_vy[ty + H][tx + H] = wy[N];
      s_vz[ty + H][tx + H] = wz[N];
      if (hxl || hxr) {
        const int cx = hxl ? tx : tx + 2 * H;
        s_vx[ty + H][cx] = h_x;
        s_vy[ty + H][cx] = h_y;
        s_vz[ty + H][cx] = h_z;
      }
      if (hyl) {
        s_vx[ty][tx + H] = t_x;
        s_vy[ty][tx + H] = t_y;
        s_vz[ty][tx + H] = t_z;
      }
      if (hyr) {
        s_vx[ty + 2 * H][tx + H] = b_x;
        s_vy[ty + 2 * H][tx + H] = b_y;
        s_vz[ty + 2 * H][tx + H] = b_z;
      }
      if (z + 1 < z1) fetch(z + 1);
      __syncthreads();
      if (own) {
        const long long q = col + g.sz * z;
        float s[6];
#pragma unroll
        for (int f = 0; f < 6; ++f) s[f] = __ldg(a.f[3 + f] + q);
        if (interior3(g, x, y, z)) {
          const float* px = &s_vx[ty + H][tx + H];
          const float* py = &s_vy[ty + H][tx + H];
          const float* pz = &s_vz[ty + H][tx + H];
          const float dxx = sdp<N>(px, 1, c), dyy = sdp<N>(py, WX, c), dzz = wdm<N>(wz, c);
          const float dxy = sdm<N>(px, WX, c), dyx = sdm<N>(py, 1, c);
          const float dxz = wdp<N>(wx, c), dzx = sdm<N>(pz, 1, c);
          const float dyz = wdp<N>(wy, c), dzy = sdm<N>(pz, WX, c);
          const float lm = __ldg(m.lam + q), l2 = __ldg(m.l2m + q);
          s[0] = __fmaf_rn(__fmaf_rn(lm, dzz, __fmaf_rn(lm, dyy, __fmul_rn(l2, dxx))), dtdh, s[0]);
          s[1] = __fmaf_rn(__fmaf_rn(lm, dzz, __fmaf_rn(l2, dyy, __fmul_rn(lm, dxx))), dtdh, s[1]);
          s[2] = __fmaf_rn(__fmaf_rn(l2, dzz, __fmaf_rn(lm, dyy, __fmul_rn(lm, dxx))), dtdh, s[2]);
          s[3] = __fmaf_rn(__fmul_rn(__ldg(m.mxy + q), __fadd_rn(dxy, dyx)), dtdh, s[3]);
          s[4] = __fmaf_rn(__fmul_rn(__ldg(m.mxz + q), __fadd_rn(dxz, dzx)), dtdh, s[4]);
          s[5] = __fmaf_rn(__fmul_rn(__ldg(m.myz + q), __fadd_rn(dyz, dzy)), dtdh, s[5]);
        }
#pragma unroll
        for (int f = 0; f < 6; ++f) o.f[3 + f][q] = s[f];
      }
#pragma unroll
      for (int k = 0; k < 2 * N; ++k) {
        wx[k] = wx[k + 1];
        wy[k] = wy[k + 1];
        wz[k] = wz[k + 1];
      }
    }
  }
}

template <int N>
int zm_resident() {
  int nv = 0, ns = 0, dev = 0, nsm = 148;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nv, k_el3_vel_zm<N>, kZmX * kZmY, 0) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ns, k_el3_str_zm<N>, kZmX * kZmY, 0) !=
          cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return std::max(1, std::min(nv, ns)) * nsm;
}

// Tiles of 32x8 columns; the z range of each tile is cut into chunks so that
// the persistent grid gets about four items per resident block (a chunk
// re-reads 2N planes to fill its windows).
inline ZmPlan make_zm_plan(const Geo3& g, int N, int resident, unsigned& grid) {
  ZmPlan zp;
  zp.ntx = (int)cdiv(g.nx, kZmX);
  zp.nty = (int)cdiv(g.ny, kZmY);
  const long long tiles = (long long)zp.ntx * zp.nty;
  const long long want = 4LL * std::max(1, resident);
  int nchunk = (int)std::max(1LL, std::min<long long>((want + tiles - 1) / tiles, g.nz / (4 * N)));
  zp.zch = (g.nz + nchunk - 1) / nchunk;
  nchunk = (g.nz + zp.zch - 1) / zp.zch;
  zp.items = (int)(tiles * nchunk);
  grid = (unsigned)std::max(1, std::min(zp.items, std::max(1, resident)));
  return zp;
}

// ---------------------------------------------------------------------------
// 3D frame: 1<=x<=nx-2 (etc.) within nbc of some face, enumerated slab by slab
// (z bands over the full xy interior, then per middle z the 2D xy frame).
// ---------------------------------------------------------------------------
struct Frame3 {
  long long slab;   // (nx-2)(ny-2)nbc cells in each z band
  long long ring;   // 2D xy frame size of one middle z plane
  long long total;
  int Wx, Wy, Hy;   // nx-2, ny-2, ny-2-2nbc
};

inline Frame3 make_frame3(const Geo3& g) {
  Frame3 f;
  f.Wx = g.nx - 2;
  f.Wy = g.ny - 2;
  f.Hy = g.ny - 2 - 2 * g.nbc;
  f.slab = (long long)f.Wx * f.Wy * g.nbc;
  f.ring = 2LL * f.Wx * g.nbc + 2LL * g.nbc * f.Hy;
  const long long nmid = g.nz - 2 - 2LL * g.nbc;
  f.total = 2 * f.slab + std::max(0LL, nmid) * f.ring;
  return f;
}

// idx -> (x, y, z) in 32-bit arithmetic (the host keeps frames below 2^31 cells)
__device__ __forceinline__ void frame3_xyz(const Geo3& g, const Frame3& fr, long long idx_, int& x,
                                           int& y, int& z) {
  const unsigned idx = (unsigned)idx_;
  const unsigned slab = (unsigned)fr.slab, wx = (unsigned)fr.Wx;
  if (idx < 2u * slab) {
    const unsigned t = idx < slab ? idx : idx - slab;
    const unsigned plane = wx * (unsigned)fr.Wy;
    const unsigned kz = t / plane;
    const unsigned r = t - kz * plane;
    const unsigned jy = r / wx;
    y = 1 + (int)jy;
    x = 1 + (int)(r - jy * wx);
    z = idx < slab ? 1 + (int)kz : g.nz - 1 - g.nbc + (int)kz;
    return;
  }
  const unsigned t = idx - 2u * slab;
  const unsigned ring = (unsigned)fr.ring;
  const unsigned kz = t / ring;
  const unsigned r = t - kz * ring;
  z = g.nbc + 1 + (int)kz;
  const unsigned band = wx * (unsigned)g.nbc;
  if (r < 2u * band) {  // y bands
    const unsigned u = r < band ? r : r - band;
    const unsigned jy = u / wx;
    x = 1 + (int)(u - jy * wx);
    y = r < band ? 1 + (int)jy : g.ny - 1 - g.nbc + (int)jy;
  } else {  // x bands of the middle y rows
    const unsigned u = r - 2u * band;
    const unsigned nb2 = 2u * (unsigned)g.nbc;
    const unsigned jy = u / nb2;
    const unsigned ix = u - jy * nb2;
    y = g.nbc + 1 + (int)jy;
    x = ix < (unsigned)g.nbc ? 1 + (int)ix : g.nx - 1 - g.nbc + ((int)ix - g.nbc);
  }
}

struct FieldSet3 {
  const float* f[6];
  const float* fo[6];
  int kind[6];
  int n;
};
struct FieldOut3 {
  float* f[6];
};

// Pass 1: the Higdon value of every frame cell of NF fields into scratch --
// kernels_3d.jl:151-193 evaluated from read-only inputs: the mean of the
// active directions' side terms, blended with the weight ramp.  The cell's
// sides, distance and neighbour offsets are shared by its fields.
template <int NF>
__global__ void __launch_bounds__(256) k_habc3_pass1(Geo3 g, Frame3 fr, HabcDev h, FieldSet3 fs,
                                                     float* __restrict__ scr) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= fr.total) return;
  int x, y, z;
  frame3_xyz(g, fr, idx, x, y, z);
  const long long q = x + g.sy * y + g.sz * z;
  const int sx = x <= g.nbc ? 1 : (x >= g.nx - 1 - g.nbc ? -1 : 0);
  const int sy = y <= g.nbc ? 1 : (y >= g.ny - 1 - g.nbc ? -1 : 0);
  const int sz = z <= g.nbc ? 1 : (z >= g.nz - 1 - g.nbc ? -1 : 0);
  const int nd = (sx != 0) + (sy != 0) + (sz != 0);
  const long long nbx = q + sx, nby = q + sy * g.sy, nbz = q + sz * g.sz;
  const int dist = min(min(min(x, g.nx - 1 - x), min(y, g.ny - 1 - y)), min(z, g.nz - 1 - z));
#pragma unroll
  for (int k = 0; k < NF; ++k) {
    const float* f = fs.f[k];
    const float* fo = fs.fo[k];
    const float fop = __ldg(fo + q);
    float sum = 0.0f;
    if (sx) sum = __fadd_rn(sum, higdon_side(h, __ldg(f + nbx), fop, __ldg(fo + nbx)));
    if (sy) sum = __fadd_rn(sum, higdon_side(h, __ldg(f + nby), fop, __ldg(fo + nby)));
    if (sz) sum = __fadd_rn(sum, higdon_side(h, __ldg(f + nbz), fop, __ldg(fo + nbz)));
    const float w = habc_weight(h, fs.kind[k], dist);
    scr[k * fr.total + idx] =
        __fmaf_rn(w, __ldg(f + q), __fdiv_rn(__fmul_rn(__fsub_rn(1.0f, w), sum), (float)nd));
  }
}

// Pass 2: scratch back into the NF fields.
template <int NF>
__global__ void __launch_bounds__(256) k_habc3_pass2(Geo3 g, Frame3 fr, FieldOut3 fo,
                                                     const float* __restrict__ scr) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= fr.total) return;
  int x, y, z;
  frame3_xyz(g, fr, idx, x, y, z);
  const long long q = x + g.sy * y + g.sz * z;
#pragma unroll
  for (int k = 0; k < NF; ++k) fo.f[k][q] = scr[k * fr.total + idx];
}

// Both passes for NF = 1, 3 or 6 fields.
inline void habc3_passes(cudaStream_t st, unsigned fblocks, const Geo3& g, const Frame3& fr,
                         const HabcDev& h, const FieldSet3& fs, const FieldOut3& fo, float* scr) {
  switch (fs.n) {
    case 1:
      k_habc3_pass1<1><<<fblocks, 256, 0, st>>>(g, fr, h, fs, scr);
      k_habc3_pass2<1><<<fblocks, 256, 0, st>>>(g, fr, fo, scr);
      break;
    case 3:
      k_habc3_pass1<3><<<fblocks, 256, 0, st>>>(g, fr, h, fs, scr);
      k_habc3_pass2<3><<<fblocks, 256, 0, st>>>(g, fr, fo, scr);
      break;
    default:
      k_habc3_pass1<6><<<fblocks, 256, 0, st>>>(g, fr, h, fs, scr);
      k_habc3_pass2<6><<<fblocks, 256, 0, st>>>(g, fr, fo, scr);
      break;
  }
}

// ---------------------------------------------------------------------------
// device medium preparation (pad_array_3d.jl, elastic3d/medium.jl, acoustic3d/medium.jl)
// ---------------------------------------------------------------------------
// A raw (unpadded) model read through the edge-replicating padding; `a`
// holds its planes from kz0 on (a z-slab may upload only the planes it needs).
struct Raw3 {
  const float* a;
  int nx, ny, nz, pad;
  int kz0;
  __device__ __forceinline__ float at(int x, int y, int z) const {
    const int ii = min(max(x - pad, 0), nx - 1), jj = min(max(y - pad, 0), ny - 1),
              kk = min(max(z - pad, 0), nz - 1);
    return __ldg(a + ii + (long long)nx * (jj + (long long)ny * (kk - kz0)));
  }
};

__device__ __forceinline__ float harm2d(float r1, float r2) {
  if (r1 == 0.0f && r2 == 0.0f) return 0.0f;
  if (r1 == 0.0f) return __fdiv_rn(2.0f, r2);
  if (r2 == 0.0f) return __fdiv_rn(2.0f, r1);
  return __fdiv_rn(2.0f, __fadd_rn(r1, r2));
}
__device__ __forceinline__ float harm4d(float m1, float m2, float m3, float m4) {
  if (m1 == 0.0f || m2 == 0.0f || m3 == 0.0f || m4 == 0.0f) return 0.0f;
  return __fdiv_rn(4.0f, __fadd_rn(__fadd_rn(__fadd_rn(__frcp_rn(m1), __frcp_rn(m2)), __frcp_rn(m3)),
                                   __frcp_rn(m4)));
}

// Local plane zl of the volume is global padded plane z = zl + g.z0.
__global__ void k_medium3d(int kind, Geo3 g, Raw3 vp, Raw3 vs, Raw3 rho, float* o0, float* o1,
                           float* o2, float* o3, float* o4, float* o5, float* o6, float* o7) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int zl = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= g.nx || y >= g.ny || zl >= g.nz) return;
  const long long q = x + g.sy * y + g.sz * zl;
  const int z = zl + g.z0;
  const int xb = max(x, 1), yb = max(y, 1), zb = min(z, g.gnz - 2);
  o0[q] = harm2d(rho.at(xb - 1, y, z), rho.at(xb, y, z));
  o1[q] = harm2d(rho.at(x, yb - 1, z), rho.at(x, yb, z));
  o2[q] = harm2d(rho.at(x, y, zb), rho.at(x, y, zb + 1));
  const float r = rho.at(x, y, z), v = vp.at(x, y, z);
  const float rv2 = __fmul_rn(r, __fmul_rn(v, v));
  if (kind == 1) {
    o3[q] = rv2;  // kappa (acoustic3d/medium.jl:55)
    return;
  }
  auto mu = [&](int i, int j, int k) {
    const float s = vs.at(i, j, k);
    return __fmul_rn(rho.at(i, j, k), __fmul_rn(s, s));
  };
  const float m = mu(x, y, z), two_m = __fmul_rn(2.0f, m);
  const float lam = __fsub_rn(rv2, two_m);
  o3[q] = lam;
  o4[q] = __fadd_rn(lam, two_m);
  // mu_txy: x>=2,y>=2 (1-based) then row 1 <- 2 in x, then in y
  o5[q] = harm4d(mu(xb - 1, yb - 1, z), mu(xb, yb - 1, z), mu(xb - 1, yb, z), mu(xb, yb, z));
  // mu_txz: x>=2, z<=nz-1 then x row 1 <- 2, z plane nz <- nz-1
  o6[q] = harm4d(mu(xb - 1, y, zb), mu(xb, y, zb), mu(xb - 1, y, zb + 1), mu(xb, y, zb + 1));
  // mu_tyz: y>=2, z<=nz-1
  o7[q] = harm4d(mu(x, yb - 1, zb), mu(x, yb, zb), mu(x, yb - 1, zb + 1), mu(x, yb, zb + 1));
}

// plane snapshot: dst[a + na*b] = src[base + a*sa + b*sb]
__global__ void k_gather_plane(const float* __restrict__ src, long long base, long long sa,
                               long long sb, int na, int nb, float* __restrict__ dst) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (a >= na || b >= nb) return;
  dst[a + (long long)na * b] = src[base + a * sa + b * sb];
}

// ---------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------
int check3(fomo_ctx* ctx, const char* what, const int32_t* a, const int32_t* b, const int32_t* c,
           int n, int nx, int ny, int nz) {
  for (int k = 0; k < n; ++k)
    if (a[k] < 1 || a[k] > nx || b[k] < 1 || b[k] > ny || c[k] < 1 || c[k] > nz)
      return fail(ctx, FOMO_EARG, std::string(what) + " index out of range");
  return FOMO_OK;
}

template <class T>
int hcopy(fomo_ctx* ctx, const T* src, long long n, bool dev, std::vector<T>& out) {
  out.resize((size_t)std::max(n, 0LL));
  if (n <= 0) return FOMO_OK;
  if (dev) FOMO_CU(ctx, cudaMemcpy(out.data(), src, sizeof(T) * n, cudaMemcpyDeviceToHost));
  else std::memcpy(out.data(), src, sizeof(T) * n);
  return FOMO_OK;
}

int run3d(fomo_ctx* ctx, bool elastic, const fomo_grid3d* gp, const float* vp, const float* vs,
          const float* rho, const fomo_acq3d* acq, int snap_interval, int snap_plane,
          int snap_index, float* svx, float* svy, float* svz, float* snaps, const fomo_opts* opts,
          fomo_stats* stats) {
  if (!ctx) return FOMO_EARG;
  if (!gp || !acq || !vp || !rho || (elastic && !vs))
    return fail(ctx, FOMO_EARG, "grid, acquisition and model arrays are required");
  const int N = order_to_N(gp->fd_order);
  if (N < 0) return fail(ctx, FOMO_EARG, "Unsupported FD order: " + std::to_string(gp->fd_order));
  if (gp->nx < 1 || gp->ny < 1 || gp->nz < 1 || gp->nt < 1 || gp->nbc < 0 || !(gp->dh > 0.0f) ||
      !(gp->dt > 0.0f))
    return fail(ctx, FOMO_EARG, "invalid 3D grid");
  if (acq->n_src < 0 || acq->n_rec < 0 || (acq->n_src > 0 && (!acq->sx || !acq->sy || !acq->sz ||
                                                               !acq->wavelet)) ||
      (acq->n_rec > 0 && (!acq->rx || !acq->ry || !acq->rz)))
    return fail(ctx, FOMO_EARG, "invalid 3D acquisition");
  if (snap_interval < 0 || snap_plane < 0 || snap_plane > 2)
    return fail(ctx, FOMO_EARG, "snap_plane must be :xz, :xy or :yz");
  if (opts && opts->precision != FOMO_FP32)
    return fail(ctx, FOMO_EUNSUPPORTED, "3D solvers store FP32 only");
  const bool dev = opts && (opts->flags & FOMO_F_DEVICE_PTRS);
  FOMO_CU(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const int M = N, pad = gp->nbc + M;
  if (pad < 2) return fail(ctx, FOMO_EARG, "nbc + fd_order/2 must be >= 2");
  const int nx = gp->nx, ny = gp->ny, nz = gp->nz, nt = gp->nt;
  Geo3 g;
  g.nx = nx + 2 * pad;
  g.ny = ny + 2 * pad;
  g.nz = nz + 2 * pad;
  g.ld = (g.nx + 31) & ~31;
  g.sy = g.ld;
  g.sz = (long long)g.ld * g.ny;
  g.vol = g.sz * g.nz;
  g.M = M;
  g.nbc = pad - 1;
  g.gnz = g.nz;
  g.zhi = g.nz;
  if (g.vol > (1LL << 31) - 1) return fail(ctx, FOMO_EARG, "padded volume exceeds 2^31 cells");
  const long long nint = (long long)nx * ny * nz;
  const int si = (snap_index > 0 ? snap_index : ny / 2) + pad - 1;  // 0-based padded index
  const int limit = snap_plane == 0 ? g.ny : (snap_plane == 1 ? g.nz : g.nx);
  if (snap_interval > 0 && snaps && (si < 0 || si >= limit))
    return fail(ctx, FOMO_EARG, "snap_index out of range");

  std::vector<int32_t> hx, hy, hz, rx, ry, rz;
  int rc;
  if ((rc = hcopy(ctx, acq->sx, acq->n_src, dev, hx)) || (rc = hcopy(ctx, acq->sy, acq->n_src, dev, hy)) ||
      (rc = hcopy(ctx, acq->sz, acq->n_src, dev, hz)) || (rc = hcopy(ctx, acq->rx, acq->n_rec, dev, rx)) ||
      (rc = hcopy(ctx, acq->ry, acq->n_rec, dev, ry)) || (rc = hcopy(ctx, acq->rz, acq->n_rec, dev, rz)))
    return rc;
  if ((rc = check3(ctx, "source", hx.data(), hy.data(), hz.data(), acq->n_src, nx, ny, nz)) ||
      (rc = check3(ctx, "receiver", rx.data(), ry.data(), rz.data(), acq->n_rec, nx, ny, nz)))
    return rc;
  std::vector<int32_t> src_lin(acq->n_src), rec_lin(acq->n_rec);
  auto lin = [&](int a, int b, int c) {
    return (int32_t)((a - 1 + pad) + g.sy * (b - 1 + pad) + g.sz * (c - 1 + pad));
  };
  for (int k = 0; k < acq->n_src; ++k) src_lin[k] = lin(hx[k], hy[k], hz[k]);
  for (int k = 0; k < acq->n_rec; ++k) rec_lin[k] = lin(rx[k], ry[k], rz[k]);
  float v_ref = gp->v_ref;
  if (!(v_ref > 0.0f)) {
    std::vector<float> hvp;
    if ((rc = hcopy(ctx, vp, nint, dev, hvp))) return rc;
    v_ref = INFINITY;
    for (float v : hvp)
      if (v > 0.0f && v < v_ref) v_ref = v;
    if (!std::isfinite(v_ref)) return fail(ctx, FOMO_EARG, "vp has no positive value for v_ref");
  }
  // weight ramps for offsets 0, .25, .5, .75 (habc_3d.jl:40-43)
  HabcHost hh = make_habc(pad, v_ref, gp->dt, gp->dh);
  const std::vector<float> wt3 = habc3_ramps(pad, hh.wstride);

  const int nfield = elastic ? 9 : 4;  // vx vy vz (txx tyy tzz txy txz tyz | p)
  const int nmat = elastic ? 8 : 4;
  const Frame3 fr = make_frame3(g);
  if (fr.total >= (1LL << 31))  // the frame enumeration uses 32-bit indices
    return fail(ctx, FOMO_EARG, "3D grid too large: the HABC frame exceeds 2^31 cells");
  const int nphase_max = elastic ? 6 : 3;
  const long long seis_n = (long long)acq->n_rec * nt;
  const long long snap_sz = snap_plane == 0 ? (long long)nx * nz
                                            : (snap_plane == 1 ? (long long)nx * ny : (long long)ny * nz);
  const int nsnap = snap_interval > 0 ? nt / snap_interval : 0;
  Arena ar;
  size_t o_model = dev ? 0 : ar.take<float>(3 * nint);
  size_t o_mat = ar.take<float>(nmat * g.vol);
  size_t o_state = ar.take<float>(2LL * nfield * g.vol);
  size_t o_scr = ar.take<float>(std::max(1LL, nphase_max * fr.total));
  size_t o_bnd = ar.take<char>(fused3_table_bytes(g));
  size_t o_w = ar.take<float>(wt3.size());
  size_t o_src = ar.take<int32_t>(std::max(acq->n_src, 1));
  size_t o_rec = ar.take<int32_t>(std::max(acq->n_rec, 1));
  size_t o_wav = dev ? 0 : ar.take<float>(std::max(1LL, (long long)acq->n_src * nt));
  size_t o_seis = dev ? 0 : ar.take<float>(std::max(1LL, 3 * seis_n));
  size_t o_snap = (!dev && snaps && nsnap) ? ar.take<float>(nsnap * snap_sz) : 0;
  if ((rc = ensure_workspace(ctx, ar.off))) return rc;

  const float* d_vp = vp;
  const float* d_vs = vs;
  const float* d_rho = rho;
  const float* d_wav = acq->wavelet;
  if (!dev) {
    float* m = ws_ptr<float>(ctx, o_model);
    FOMO_CU(ctx, cudaMemcpyAsync(m, vp, 4 * nint, cudaMemcpyHostToDevice, st));
    FOMO_CU(ctx, cudaMemcpyAsync(m + 2 * nint, rho, 4 * nint, cudaMemcpyHostToDevice, st));
    d_vp = m;
    d_rho = m + 2 * nint;
    if (elastic) {
      FOMO_CU(ctx, cudaMemcpyAsync(m + nint, vs, 4 * nint, cudaMemcpyHostToDevice, st));
      d_vs = m + nint;
    }
    if (acq->n_src) {
      float* w = ws_ptr<float>(ctx, o_wav);
      FOMO_CU(ctx, cudaMemcpyAsync(w, acq->wavelet, 4LL * acq->n_src * nt, cudaMemcpyHostToDevice, st));
      d_wav = w;
    }
  }
  float* d_mat = ws_ptr<float>(ctx, o_mat);
  float* d_state = ws_ptr<float>(ctx, o_state);
  float* d_scr = ws_ptr<float>(ctx, o_scr);
  float* d_w = ws_ptr<float>(ctx, o_w);
  int32_t* d_src = ws_ptr<int32_t>(ctx, o_src);
  int32_t* d_rec = ws_ptr<int32_t>(ctx, o_rec);
  FOMO_CU(ctx, cudaMemcpyAsync(d_w, wt3.data(), 4 * wt3.size(), cudaMemcpyHostToDevice, st));
  if (acq->n_src)
    FOMO_CU(ctx, cudaMemcpyAsync(d_src, src_lin.data(), 4LL * acq->n_src, cudaMemcpyHostToDevice, st));
  if (acq->n_rec)
    FOMO_CU(ctx, cudaMemcpyAsync(d_rec, rec_lin.data(), 4LL * acq->n_rec, cudaMemcpyHostToDevice, st));
  float* d_seis[3];
  for (int k = 0; k < 3; ++k) {
    float* out = k == 0 ? svx : (k == 1 ? svy : svz);
    d_seis[k] = dev ? out : ws_ptr<float>(ctx, o_seis) + k * seis_n;
  }
  float* d_snap = dev ? snaps : (o_snap ? ws_ptr<float>(ctx, o_snap) : nullptr);
  if (!snaps) d_snap = nullptr;

  dim3 blk(32, 4, 2), grd(cdiv(g.nx, 32), cdiv(g.ny, 4), cdiv(g.nz, 2));
  {
    Raw3 a{d_vp, nx, ny, nz, pad, 0}, s{elastic ? d_vs : d_vp, nx, ny, nz, pad, 0},
        r{d_rho, nx, ny, nz, pad, 0};
    float* o[8];
    for (int k = 0; k < 8; ++k) o[k] = k < nmat ? d_mat + k * g.vol : nullptr;
    k_medium3d<<<grd, blk, 0, st>>>(elastic ? 0 : 1, g, a, s, r, o[0], o[1], o[2], o[3], o[4], o[5],
                                    o[6], o[7]);
    FOMO_CU(ctx, cudaGetLastError());
  }
  FOMO_CU(ctx, cudaMemsetAsync(d_state, 0, 4 * 2LL * nfield * g.vol, st));
  auto field = [&](int set, int f) { return d_state + ((long long)set * nfield + f) * g.vol; };
  Coef c;
  for (int l = 0; l < 5; ++l) c.a[l] = kFD[N][l];
  HabcDev h{hh.q, hh.qt, hh.qxt, hh.nbc, hh.wstride, d_w};
  const float dtdh = gp->dt / gp->dh;
  const unsigned fblocks = (unsigned)std::max<long long>(1, (fr.total + 255) / 256);
  const unsigned rec_blocks = (unsigned)std::min(1184, std::max(1, (acq->n_rec + 255) / 256));
  // Elastic updates.  Measured on 488x488x388 (order 8): the z-marching
  // velocity update beats the per-cell one (1.85 vs 2.05 ms), the z-marching
  // stress update loses (2.65 vs 2.15 ms).  AUTO takes the faster of each;
  // ZMARCH and TWO_PHASE select one form for both (identical results).
  // The fused TMA half steps (sweep3d.cu: update and Higdon boundary in one
  // pass each) are the default wherever they run; SINGLE_SWEEP requests them.
  const int kreq = opts ? opts->kernel : FOMO_KERNEL_AUTO;
  const bool fused = (kreq == FOMO_KERNEL_AUTO || kreq == FOMO_KERNEL_SINGLE_SWEEP) &&
                     fused3_supported(N);
  if (kreq == FOMO_KERNEL_SINGLE_SWEEP && !fused)
    return fail(ctx, FOMO_EUNSUPPORTED, "fused 3D half steps need the TMA tensor-map encoder");
  const bool zm_vel = elastic && !fused && kreq != FOMO_KERNEL_TWO_PHASE;
  const bool zm_str = elastic && !fused && kreq == FOMO_KERNEL_ZMARCH;
  const bool zmarch = zm_vel || zm_str;
  unsigned zgrid = 1;
  ZmPlan zp{};
  if (zmarch) {
    int resident = 0;
    switch (N) {
      case 1: resident = zm_resident<1>(); break;
      case 2: resident = zm_resident<2>(); break;
      case 3: resident = zm_resident<3>(); break;
      case 4: resident = zm_resident<4>(); break;
      default: resident = zm_resident<5>(); break;
    }
    if (resident < 1) return fail(ctx, FOMO_ECUDA, "z-marching 3D kernels do not fit an SM");
    zp = make_zm_plan(g, N, resident, zgrid);
  }
  Fused3Plan fp;
  if (fused) {
    FOMO_CU(ctx, fused3_make_plan(fp, g, N, elastic, d_state, d_mat, ws_ptr<char>(ctx, o_bnd), st));
    FOMO_CU(ctx, cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), st));
  }
  int A = 0, B = 1, launches = 0;
  FOMO_CU(ctx, cudaEventRecord(ctx->ev0, st));
  for (int it = 1; it <= nt; ++it) {
    // velocity phase
    if (fused) {
      FOMO_CU(ctx, fused3_velocity(st, fp, g, d_state, A, B, c, dtdh, h, ctx->d_flag));
    } else if (elastic) {
      El3 a;
      El3Out o;
      for (int f = 0; f < 9; ++f) {
        a.f[f] = field(A, f);
        o.f[f] = field(B, f);
      }
      El3Mat m{d_mat, d_mat + g.vol, d_mat + 2 * g.vol, d_mat + 3 * g.vol, d_mat + 4 * g.vol,
               d_mat + 5 * g.vol, d_mat + 6 * g.vol, d_mat + 7 * g.vol};
#define FOMO_EL3V(NN)                                                            \
  case NN:                                                                       \
    if (zm_vel)                                                                  \
      k_el3_vel_zm<NN><<<zgrid, dim3(kZmX, kZmY), 0, st>>>(g, c, dtdh, a, m, o, zp); \
    else                                                                         \
      k_el3_vel<NN><<<grd, blk, 0, st>>>(g, c, dtdh, a, m, o);                   \
    break;
      switch (N) { FOMO_EL3V(1) FOMO_EL3V(2) FOMO_EL3V(3) FOMO_EL3V(4) FOMO_EL3V(5) }
#undef FOMO_EL3V
    } else {
#define FOMO_AC3V(NN)                                                                              \
  case NN:                                                                                         \
    k_ac3_vel<NN><<<grd, blk, 0, st>>>(g, c, dtdh, field(A, 3), field(A, 0), field(A, 1),          \
                                       field(A, 2), d_mat, d_mat + g.vol, d_mat + 2 * g.vol,       \
                                       field(B, 0), field(B, 1), field(B, 2));                     \
    break;
      switch (N) { FOMO_AC3V(1) FOMO_AC3V(2) FOMO_AC3V(3) FOMO_AC3V(4) FOMO_AC3V(5) }
#undef FOMO_AC3V
    }
    if (fr.total > 0 && !fused) {
      FieldSet3 fs;
      FieldOut3 fo;
      fs.n = 3;
      for (int k = 0; k < 3; ++k) {
        fs.f[k] = field(B, k);
        fs.fo[k] = field(A, k);
        fs.kind[k] = k;
        fo.f[k] = field(B, k);
      }
      habc3_passes(st, fblocks, g, fr, h, fs, fo, d_scr);
    }
    // stress / pressure phase
    if (fused) {
      FOMO_CU(ctx, fused3_stress(st, fp, g, d_state, A, B, c, dtdh, h, ctx->d_flag));
    } else if (elastic) {
      El3 a;
      El3Out o;
      for (int f = 0; f < 9; ++f) {
        a.f[f] = field(A, f);
        o.f[f] = field(B, f);
      }
      El3Mat m{d_mat, d_mat + g.vol, d_mat + 2 * g.vol, d_mat + 3 * g.vol, d_mat + 4 * g.vol,
               d_mat + 5 * g.vol, d_mat + 6 * g.vol, d_mat + 7 * g.vol};
#define FOMO_EL3S(NN)                                                                          \
  case NN:                                                                                     \
    if (zm_str)                                                                                \
      k_el3_str_zm<NN><<<zgrid, dim3(kZmX, kZmY), 0, st>>>(g, c, dtdh, a, field(B, 0),        \
                                                           field(B, 1), field(B, 2), m, o, zp); \
    else                                                                                       \
      k_el3_str<NN><<<grd, blk, 0, st>>>(g, c, dtdh, a, field(B, 0), field(B, 1), field(B, 2), \
                                         m, o);                                                \
    break;
      switch (N) { FOMO_EL3S(1) FOMO_EL3S(2) FOMO_EL3S(3) FOMO_EL3S(4) FOMO_EL3S(5) }
#undef FOMO_EL3S
    } else {
#define FOMO_AC3P(NN)                                                                           \
  case NN:                                                                                      \
    k_ac3_prs<NN><<<grd, blk, 0, st>>>(g, c, dtdh, field(A, 3), field(B, 0), field(B, 1),       \
                                       field(B, 2), d_mat + 3 * g.vol, field(B, 3));            \
    break;
      switch (N) { FOMO_AC3P(1) FOMO_AC3P(2) FOMO_AC3P(3) FOMO_AC3P(4) FOMO_AC3P(5) }
#undef FOMO_AC3P
    }
    if (fr.total > 0 && !fused) {
      FieldSet3 fs;
      FieldOut3 fo;
      fs.n = elastic ? 6 : 1;
      for (int k = 0; k < fs.n; ++k) {
        fs.f[k] = field(B, 3 + k);
        fs.fo[k] = field(A, 3 + k);
        fs.kind[k] = 3;
        fo.f[k] = field(B, 3 + k);
      }
      habc3_passes(st, fblocks, g, fr, h, fs, fo, d_scr);
    }
    // inject (p | txx,tyy,tzz), record vx vy vz (acoustic3d.jl:171-176, elastic3d.jl:139-147)
    k_inject_record3<<<rec_blocks, 256, 0, st>>>(it, nt, acq->n_src, d_src, d_wav, field(B, 3),
                                        elastic ? field(B, 4) : nullptr,
                                        elastic ? field(B, 5) : nullptr, acq->n_rec, d_rec,
                                        field(B, 0), field(B, 1), field(B, 2), d_seis[0],
                                        d_seis[1], d_seis[2]);
    launches += (fr.total > 0 && !fused) ? 7 : 3;
    FOMO_CU(ctx, cudaGetLastError());
    if (d_snap && snap_interval > 0 && it % snap_interval == 0) {
      // snapshot of p (acoustic) / vz (elastic) on the plane (acoustic3d.jl:177-184)
      const float* f = elastic ? field(B, 2) : field(B, 3);
      float* dst = d_snap + (long long)(it / snap_interval - 1) * snap_sz;
      long long base, sa, sb;
      int na, nb;
      if (snap_plane == 0) {
        base = pad + g.sy * si + g.sz * pad; sa = 1; sb = g.sz; na = nx; nb = nz;
      } else if (snap_plane == 1) {
        base = pad + g.sy * pad + g.sz * si; sa = 1; sb = g.sy; na = nx; nb = ny;
      } else {
        base = si + g.sy * pad + g.sz * pad; sa = g.sy; sb = g.sz; na = ny; nb = nz;
      }
      k_gather_plane<<<dim3(cdiv(na, 128), nb), 128, 0, st>>>(f, base, sa, sb, na, nb, dst);
    }
    std::swap(A, B);
  }
  FOMO_CU(ctx, cudaEventRecord(ctx->ev1, st));
  if (!dev) {
    if (seis_n)
      for (int k = 0; k < 3; ++k) {
        float* out = k == 0 ? svx : (k == 1 ? svy : svz);
        if (out) FOMO_CU(ctx, cudaMemcpyAsync(out, d_seis[k], 4 * seis_n, cudaMemcpyDeviceToHost, st));
      }
    if (d_snap && nsnap)
      FOMO_CU(ctx, cudaMemcpyAsync(snaps, d_snap, 4LL * nsnap * snap_sz, cudaMemcpyDeviceToHost, st));
  }
  if (opts && opts->final_state) {
    // (nxp, nyp, nzp, nfield) unpitched host layout
    const long long hp = (long long)g.nx * g.ny * g.nz;
    for (int f = 0; f < nfield; ++f)
      FOMO_CU(ctx, cudaMemcpy2DAsync(opts->final_state + f * hp, 4 * (size_t)g.nx, field(A, f),
                                     4 * (size_t)g.ld, 4 * (size_t)g.nx, (size_t)g.ny * g.nz,
                                     cudaMemcpyDeviceToHost, st));
  }
  FOMO_CU(ctx, cudaStreamSynchronize(st));
  if (fused) {
    int hflag = 0;
    FOMO_CU(ctx, cudaMemcpy(&hflag, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (hflag) return fail(ctx, FOMO_ECUDA, "fused 3D half step: a bounded TMA wait timed out");
  }
  float ms = 0.0f;
  FOMO_CU(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  if (stats) {
    std::memset(stats, 0, sizeof *stats);
    stats->kernel_time_s = ms * 1e-3;
    stats->cell_updates = (double)g.nx * g.ny * g.nz * nt;
    stats->alg_bytes = 4.0 * (double)g.nx * g.ny * g.nz * nt * (2.0 * nfield + nmat);
    stats->n_shots = 1;
    stats->gpu_launches = launches;
    stats->kernel = fused ? FOMO_KERNEL_SINGLE_SWEEP
                          : (zm_str ? FOMO_KERNEL_ZMARCH
                                    : (zm_vel ? FOMO_KERNEL_AUTO : FOMO_KERNEL_TWO_PHASE));
  }
  return FOMO_OK;
}

}  // namespace

cudaError_t medium3d(cudaStream_t st, bool elastic, const Geo3& g, const float* vp,
                     const float* vs, const float* rho, int nx, int ny, int nz, int pad, int kz0,
                     float* mat) {
  dim3 blk(32, 4, 2), grd(cdiv(g.nx, 32), cdiv(g.ny, 4), cdiv(g.nz, 2));
  Raw3 a{vp, nx, ny, nz, pad, kz0}, s{elastic ? vs : vp, nx, ny, nz, pad, kz0},
      r{rho, nx, ny, nz, pad, kz0};
  const int nmat = elastic ? 8 : 4;
  float* o[8];
  for (int k = 0; k < 8; ++k) o[k] = k < nmat ? mat + k * g.vol : nullptr;
  k_medium3d<<<grd, blk, 0, st>>>(elastic ? 0 : 1, g, a, s, r, o[0], o[1], o[2], o[3], o[4], o[5],
                                  o[6], o[7]);
  return cudaGetLastError();
}

cudaError_t inject_record3(cudaStream_t st, bool elastic, const Geo3& g, float* state, int B,
                           int it, int nt, int n_src, const int* src_lin, const float* wav,
                           int n_rec, const int* rec_lin, float* s0, float* s1, float* s2) {
  const int nfield = elastic ? 9 : 4;
  auto field = [&](int f) { return state + ((long long)B * nfield + f) * g.vol; };
  const unsigned rec_blocks = (unsigned)std::min(1184, std::max(1, (n_rec + 255) / 256));
  k_inject_record3<<<rec_blocks, 256, 0, st>>>(it, nt, n_src, src_lin, wav, field(3),
                                               elastic ? field(4) : nullptr,
                                               elastic ? field(5) : nullptr, n_rec, rec_lin,
                                               field(0), field(1), field(2), s0, s1, s2);
  return cudaGetLastError();
}

}  // namespace fomo

using namespace fomo;

extern "C" {

int fomo_acoustic3d(fomo_ctx* ctx, const fomo_grid3d* g, const float* vp, const float* rho,
                    const fomo_acq3d* acq, int32_t snap_interval, int32_t snap_plane,
                    int32_t snap_index, float* seis_vx, float* seis_vy, float* seis_vz,
                    float* snaps, const fomo_opts* opts, fomo_stats* stats) {
  return run3d(ctx, false, g, vp, nullptr, rho, acq, snap_interval, snap_plane, snap_index,
               seis_vx, seis_vy, seis_vz, snaps, opts, stats);
}

int fomo_elastic3d(fomo_ctx* ctx, const fomo_grid3d* g, const float* vp, const float* vs,
                   const float* rho, const fomo_acq3d* acq, int32_t snap_interval,
                   int32_t snap_plane, int32_t snap_index, float* seis_vx, float* seis_vy,
                   float* seis_vz, float* snaps, const fomo_opts* opts, fomo_stats* stats) {
  return run3d(ctx, true, g, vp, vs, rho, acq, snap_interval, snap_plane, snap_index, seis_vx,
               seis_vy, seis_vz, snaps, opts, stats);
}

}  // extern "C"
