// mixed2d.cuh -- elastic2d with FP16 wavefield storage (no reference counterpart).
//
// Wavefields are stored in IEEE binary16 except within kFp16Band cells of the
// padded grid's edge, where they stay FP32; all arithmetic is FP32 with the
// same canonical sequence as the FP32 kernels.  Why the band: the reference's
// elastic Higdon zone carries a slowly growing mode seeded by rounding noise;
// with FP16 noise it overflows binary16 within a few thousand steps, while in
// FP32 storage it stays confined to the outer cells.  Stored values are scaled
// by powers of two, velocities by kFp16Sv and stresses by kFp16St, so that the
// physical amplitudes sit in binary16's normal range; the scales are folded
// into the materials (b * Sv/St, lambda, lambda + 2mu, mu * St/Sv) and the
// wavelet (* St), and removed at the receivers (/ Sv), which is exact.
// A stored value is the FP32 result rounded to nearest even.
#pragma once
#include <cuda_fp16.h>

#include "solver2d_kernels.cuh"

namespace fomo {

struct HField {  // one wavefield of one ping-pong set, all shots (shot offset = shot * plane)
  float* f32;    // cells of the band
  __half* f16;   // other cells
};
struct HSet {
  HField f[5];  // vx, vz, txx, tzz, txz
};

__device__ __forceinline__ bool in_band(const Geo2& g, int x, int z) {
  return min(min(x, g.nx - 1 - x), min(z, g.nz - 1 - z)) < kFp16Band;
}
// BAND = false: the caller knows (x, z) lies outside the FP32 band.
template <bool BAND = true>
__device__ __forceinline__ float hld(const HField& f, const Geo2& g, long long so, int x, int z) {
  const long long p = so + (long long)z * g.ld + x;
  if (!BAND) return __half2float(f.f16[p]);
  return in_band(g, x, z) ? __ldg(f.f32 + p) : __half2float(f.f16[p]);
}
template <bool BAND = true>
__device__ __forceinline__ void hst(const HField& f, const Geo2& g, long long so, int x, int z,
                                    float v) {
  const long long p = so + (long long)z * g.ld + x;
  if (BAND && in_band(g, x, z)) f.f32[p] = v;
  else f.f16[p] = __float2half_rn(v);
}
// Does a block of bw x bh cells at (x0, z0), with a reach of r cells around
// it, stay clear of the FP32 band?
__device__ __forceinline__ bool block_clear(const Geo2& g, int x0, int z0, int bw, int bh, int r) {
  return x0 - r >= kFp16Band && x0 + bw - 1 + r <= g.nx - 1 - kFp16Band && z0 - r >= kFp16Band &&
         z0 + bh - 1 + r <= g.nz - 1 - kFp16Band;
}

// Staggered derivative sums (canonical order l = 1..N, one fma per term).
template <int N, bool BAND = true>
__device__ __forceinline__ float hdmx(const HField& f, const Geo2& g, long long so, int x, int z,
                                      const Coef& c) {
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l)
    acc = __fmaf_rn(c.a[l - 1], __fsub_rn(hld<BAND>(f, g, so, x + l - 1, z), hld<BAND>(f, g, so, x - l, z)), acc);
  return acc;
}
template <int N, bool BAND = true>
__device__ __forceinline__ float hdpx(const HField& f, const Geo2& g, long long so, int x, int z,
                                      const Coef& c) {
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l)
    acc = __fmaf_rn(c.a[l - 1], __fsub_rn(hld<BAND>(f, g, so, x + l, z), hld<BAND>(f, g, so, x - l + 1, z)), acc);
  return acc;
}
template <int N, bool BAND = true>
__device__ __forceinline__ float hdmz(const HField& f, const Geo2& g, long long so, int x, int z,
                                      const Coef& c) {
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l)
    acc = __fmaf_rn(c.a[l - 1], __fsub_rn(hld<BAND>(f, g, so, x, z + l - 1), hld<BAND>(f, g, so, x, z - l)), acc);
  return acc;
}
template <int N, bool BAND = true>
__device__ __forceinline__ float hdpz(const HField& f, const Geo2& g, long long so, int x, int z,
                                      const Coef& c) {
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l)
    acc = __fmaf_rn(c.a[l - 1], __fsub_rn(hld<BAND>(f, g, so, x, z + l), hld<BAND>(f, g, so, x, z - l + 1)), acc);
  return acc;
}

template <int N, bool BAND>
__device__ __forceinline__ void elh_vel_at(const Geo2& g, const Coef& c, float dtx, float dtz,
                                           const HSet& a, long long so, const ElMat& m, int x,
                                           int z, float& ux, float& uz) {
  float vx = hld<BAND>(a.f[0], g, so, x, z), vz = hld<BAND>(a.f[1], g, so, x, z);
  if (interior2(g, x, z)) {
    const long long p = (long long)z * g.ld + x;
    const float dxx = hdmx<N, BAND>(a.f[2], g, so, x, z, c);
    const float dxzz = hdmz<N, BAND>(a.f[4], g, so, x, z, c);
    const float dxzx = hdpx<N, BAND>(a.f[4], g, so, x, z, c);
    const float dzz = hdpz<N, BAND>(a.f[3], g, so, x, z, c);
    vx = __fmaf_rn(__ldg(m.bx + p), __fmaf_rn(dtx, dxx, __fmul_rn(dtz, dxzz)), vx);
    vz = __fmaf_rn(__ldg(m.bz + p), __fmaf_rn(dtx, dxzx, __fmul_rn(dtz, dzz)), vz);
  }
  ux = vx;
  uz = vz;
}

// k_el_vel with binary16/FP32-band storage (same per-cell arithmetic).
// Blocks whose cells, stencils and HABC neighbours all stay clear of the band
// read and write binary16 without per-cell band tests (BAND = false); the
// Higdon frame (pad - 1 cells) can be wider than the band, so it is applied
// on both paths.
template <int N, bool BAND>
__device__ __forceinline__ void elh_vel_cell(const Geo2& g, const Coef& c, float dtx, float dtz,
                                             const HabcDev& h, const HSet& a, long long so,
                                             const ElMat& m, int x, int z, float& ux, float& uz) {
  elh_vel_at<N, BAND>(g, c, dtx, dtz, a, so, m, x, z, ux, uz);
  int sx, sz, dist;
  if (frame2(g, x, z, sx, sz, dist)) {
    const float wx = habc_weight(h, 0, dist), wz = habc_weight(h, 1, dist);
    const float fox = hld<BAND>(a.f[0], g, so, x, z), foz = hld<BAND>(a.f[1], g, so, x, z);
    if (sx != 0 && sz != 0) {
      float ax, az, bx, bz;
      elh_vel_at<N, BAND>(g, c, dtx, dtz, a, so, m, x + sx, z, ax, az);
      elh_vel_at<N, BAND>(g, c, dtx, dtz, a, so, m, x, z + sz, bx, bz);
      ux = higdon_corner(wx, ux, higdon_side(h, ax, fox, hld<BAND>(a.f[0], g, so, x + sx, z)),
                         higdon_side(h, bx, fox, hld<BAND>(a.f[0], g, so, x, z + sz)));
      uz = higdon_corner(wz, uz, higdon_side(h, az, foz, hld<BAND>(a.f[1], g, so, x + sx, z)),
                         higdon_side(h, bz, foz, hld<BAND>(a.f[1], g, so, x, z + sz)));
    } else {
      const int xn = x + sx, zn = z + sz;
      float nx_, nz_;
      elh_vel_at<N, BAND>(g, c, dtx, dtz, a, so, m, xn, zn, nx_, nz_);
      ux = higdon_edge(wx, ux, higdon_side(h, nx_, fox, hld<BAND>(a.f[0], g, so, xn, zn)));
      uz = higdon_edge(wz, uz, higdon_side(h, nz_, foz, hld<BAND>(a.f[1], g, so, xn, zn)));
    }
  }
}

template <int N>
__global__ void __launch_bounds__(256) k_elh_vel(Geo2 g, Coef c, float dtx, float dtz, HabcDev h,
                                                 HSet a, ElMat m, HField ox, HField oz) {
  const int x0 = blockIdx.x * blockDim.x, z0 = blockIdx.y * blockDim.y;
  const int x = x0 + threadIdx.x, z = z0 + threadIdx.y;
  if (x >= g.nx || z >= g.nz) return;
  const long long so = (long long)blockIdx.z * g.plane;
  float ux, uz;
  // reach: the stencil (N) around a Higdon neighbour (1)
  if (block_clear(g, x0, z0, blockDim.x, blockDim.y, N + 1)) {
    elh_vel_cell<N, false>(g, c, dtx, dtz, h, a, so, m, x, z, ux, uz);
    hst<false>(ox, g, so, x, z, ux);
    hst<false>(oz, g, so, x, z, uz);
  } else {
    elh_vel_cell<N, true>(g, c, dtx, dtz, h, a, so, m, x, z, ux, uz);
    hst(ox, g, so, x, z, ux);
    hst(oz, g, so, x, z, uz);
  }
}

template <int N, bool BAND>
__device__ __forceinline__ void elh_str_at(const Geo2& g, const Coef& c, float dtx, float dtz,
                                           const HField& vx, const HField& vz, const HSet& a,
                                           long long so, const ElMat& m, int x, int z, float& sxx,
                                           float& szz, float& sxz) {
  sxx = hld<BAND>(a.f[2], g, so, x, z);
  szz = hld<BAND>(a.f[3], g, so, x, z);
  sxz = hld<BAND>(a.f[4], g, so, x, z);
  if (interior2(g, x, z)) {
    const long long p = (long long)z * g.ld + x;
    const float dvxdx = hdpx<N, BAND>(vx, g, so, x, z, c);
    const float dvzdz = hdmz<N, BAND>(vz, g, so, x, z, c);
    const float dvxdz = hdpz<N, BAND>(vx, g, so, x, z, c);
    const float dvzdx = hdmx<N, BAND>(vz, g, so, x, z, c);
    const float lam = __ldg(m.lam + p), l2m = __ldg(m.l2m + p);
    const float ex = __fmul_rn(dvxdx, dtx), ez = __fmul_rn(dvzdz, dtz);
    sxx = __fadd_rn(sxx, __fmaf_rn(l2m, ex, __fmul_rn(lam, ez)));
    szz = __fadd_rn(szz, __fmaf_rn(lam, ex, __fmul_rn(l2m, ez)));
    sxz = __fmaf_rn(__ldg(m.mut + p), __fmaf_rn(dvxdz, dtz, __fmul_rn(dvzdx, dtx)), sxz);
  }
}

template <int N, bool BAND>
__device__ __forceinline__ void elh_str_cell(const Geo2& g, const Coef& c, float dtx, float dtz,
                                             const HabcDev& h, const HSet& a, const HField& vx,
                                             const HField& vz, long long so, const ElMat& m, int x,
                                             int z, float& sxx, float& szz, float& sxz) {
  elh_str_at<N, BAND>(g, c, dtx, dtz, vx, vz, a, so, m, x, z, sxx, szz, sxz);
  int sx, sz, dist;
  if (frame2(g, x, z, sx, sz, dist)) {
    const float w = habc_weight(h, 2, dist);
    const float o1 = hld<BAND>(a.f[2], g, so, x, z), o2 = hld<BAND>(a.f[3], g, so, x, z),
                o3 = hld<BAND>(a.f[4], g, so, x, z);
    if (sx != 0 && sz != 0) {
      float a1, a2, a3, b1, b2, b3;
      elh_str_at<N, BAND>(g, c, dtx, dtz, vx, vz, a, so, m, x + sx, z, a1, a2, a3);
      elh_str_at<N, BAND>(g, c, dtx, dtz, vx, vz, a, so, m, x, z + sz, b1, b2, b3);
      sxx = higdon_corner(w, sxx, higdon_side(h, a1, o1, hld<BAND>(a.f[2], g, so, x + sx, z)),
                          higdon_side(h, b1, o1, hld<BAND>(a.f[2], g, so, x, z + sz)));
      szz = higdon_corner(w, szz, higdon_side(h, a2, o2, hld<BAND>(a.f[3], g, so, x + sx, z)),
                          higdon_side(h, b2, o2, hld<BAND>(a.f[3], g, so, x, z + sz)));
      sxz = higdon_corner(w, sxz, higdon_side(h, a3, o3, hld<BAND>(a.f[4], g, so, x + sx, z)),
                          higdon_side(h, b3, o3, hld<BAND>(a.f[4], g, so, x, z + sz)));
    } else {
      const int xn = x + sx, zn = z + sz;
      float n1, n2, n3;
      elh_str_at<N, BAND>(g, c, dtx, dtz, vx, vz, a, so, m, xn, zn, n1, n2, n3);
      sxx = higdon_edge(w, sxx, higdon_side(h, n1, o1, hld<BAND>(a.f[2], g, so, xn, zn)));
      szz = higdon_edge(w, szz, higdon_side(h, n2, o2, hld<BAND>(a.f[3], g, so, xn, zn)));
      sxz = higdon_edge(w, sxz, higdon_side(h, n3, o3, hld<BAND>(a.f[4], g, so, xn, zn)));
    }
  }
}

template <int N>
__global__ void __launch_bounds__(256) k_elh_str(Geo2 g, Coef c, float dtx, float dtz, HabcDev h,
                                                 HSet a, HField vx, HField vz, ElMat m,
                                                 HField oxx, HField ozz, HField oxz) {
  const int x0 = blockIdx.x * blockDim.x, z0 = blockIdx.y * blockDim.y;
  const int x = x0 + threadIdx.x, z = z0 + threadIdx.y;
  if (x >= g.nx || z >= g.nz) return;
  const long long so = (long long)blockIdx.z * g.plane;
  float sxx, szz, sxz;
  if (block_clear(g, x0, z0, blockDim.x, blockDim.y, N + 1)) {
    elh_str_cell<N, false>(g, c, dtx, dtz, h, a, vx, vz, so, m, x, z, sxx, szz, sxz);
    hst<false>(oxx, g, so, x, z, sxx);
    hst<false>(ozz, g, so, x, z, szz);
    hst<false>(oxz, g, so, x, z, sxz);
  } else {
    elh_str_cell<N, true>(g, c, dtx, dtz, h, a, vx, vz, so, m, x, z, sxx, szz, sxz);
    hst(oxx, g, so, x, z, sxx);
    hst(ozz, g, so, x, z, szz);
    hst(oxz, g, so, x, z, sxz);
  }
}

// Injection (w * St into txx and tzz, stored back) then recording of vx, vz
// (/ Sv), one block per shot; linear indices are padded-grid cells.
static __global__ void k_elh_inject_record(int it, int nt, Geo2 g, int n_src,
                                           const int* __restrict__ src_lin,
                                           const float* __restrict__ wav, HField txx, HField tzz,
                                           int n_rec, const int* __restrict__ rec_lin, HField vx,
                                           HField vz, float* __restrict__ s0,
                                           float* __restrict__ s1) {
  const int s = blockIdx.x;
  const long long so = (long long)s * g.plane;
  if (threadIdx.x == 0)
    for (int q = 0; q < n_src; ++q) {
      const int p = src_lin[(long long)s * n_src + q];
      const int x = p % g.ld, z = p / g.ld;
      const float w = __fmul_rn(wav[(long long)(it - 1) * n_src + q], kFp16St);
      hst(txx, g, so, x, z, __fadd_rn(hld(txx, g, so, x, z), w));
      hst(tzz, g, so, x, z, __fadd_rn(hld(tzz, g, so, x, z), w));
    }
  __syncthreads();
  const long long ob = (long long)n_rec * ((long long)(it - 1) + (long long)nt * s);
  for (int r = threadIdx.x; r < n_rec; r += blockDim.x) {
    const int p = rec_lin[r];
    const int x = p % g.ld, z = p / g.ld;
    s0[ob + r] = __fdiv_rn(hld(vx, g, so, x, z), kFp16Sv);
    s1[ob + r] = __fdiv_rn(hld(vz, g, so, x, z), kFp16Sv);
  }
}

// Unscaled FP32 copy of a stored field (snapshots, final state):
// dst[x + nxo * z] = field(x0 + x, z0 + z) / scale for one shot.
static __global__ void k_elh_unpack(Geo2 g, HField f, long long so, int x0, int z0, int nxo,
                                    int nzo, float scale, float* __restrict__ dst) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y;
  if (x >= nxo || z >= nzo) return;
  dst[x + (long long)nxo * z] = __fdiv_rn(hld(f, g, so, x0 + x, z0 + z), scale);
}

static __global__ void k_scale(float* __restrict__ a, long long n, float s) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    a[i] = __fmul_rn(a[i], s);
}

}  // namespace fomo
