// sweep2d.cu -- single-sweep elastic time step (one launch per step).
//
// The two-phase kernels read every wavefield twice per step (velocity sweep,
// then stress sweep: 60 B per shot-cell).  This kernel does the whole step in
// one pass over HBM -- read A (time n) once, write B (time n+1) once, 40 B per
// shot-cell -- by marching each CTA down a column strip of one shot:
//
//   TMA ring (stress of time n, rows zfirst.., 3 fields, x-halo HS)
//     -> v'  = velocity update            rows h-M   .. (smem rows VP)
//     -> v'' = det-HABC(v')               rows h-M-1 .. (smem rows VV, -> B.v)
//     -> s'  = stress update from v''     rows h-2M-2.. (smem rows SP)
//     -> s'' = det-HABC(s')               rows h-2M-3.. (-> B.stress)
//
// where h is the first row of the chunk just landed.  Each stage reads only
// rows/columns the previous stages already produced, with x-halos of M+2
// (v'), M+1 (v''), 1 (s') around the TX output columns, so every value equals
// the two-phase / oracle value bit for bit (same canonical arithmetic).
//
// Rows outside the padded grid come from TMA's out-of-bounds zero fill and
// only ever feed results that are discarded (warm-up rows above zA, columns
// outside [0, nx)).  mbarrier waits are bounded: on timeout the CTA records
// an error in *err and stops waiting (the host reports it).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <vector>
#include <climits>
#include <cstring>
#include <mutex>

#include "sweep2d.cuh"
#include "tma.cuh"

namespace fomo {
namespace {

// The shared mbarrier / TMA primitives (tma.cuh), bounded waits included.
using tma::fence_proxy_async;
using tma::mbar_expect_tx;
using tma::mbar_init;
using tma::mbar_wait_bounded;
__device__ __forceinline__ void tma_load_3d(float* dst, const CUtensorMap* map, int x, int y,
                                            int z, uint64_t* bar) {
  tma::load_3d(dst, map, x, y, z, bar);
}

constexpr int halo_x(int M) { return (2 * M + 2 + 3) & ~3; }  // stress x-halo, 16-byte aligned

template <int N, int R, int P>
struct SweepShape {
  static constexpr int M = N;
  static constexpr int HS = halo_x(M);
  // TMA ring: the v' stage reads rows hz-2M .. hz+R-1; chunk j+P is issued
  // once iteration j's v' stage is done, into the slot of chunk j+P-NSLOT.
  static constexpr int NSLOT = P + (2 * M + R - 1) / R;
  static constexpr int SR = NSLOT * R;
  static constexpr int SVP = R + 2;          // v'  rows hz-M-2 .. hz-M+R-1
  static constexpr int SVV = 2 * M + R + 1;  // v'' rows hz-3M-2 .. hz-M-2+R
  static constexpr int SSP = R + 2;          // s'  rows hz-2M-4 .. hz-2M-3+R
};

// (b + d) mod n for d in (-n, n), b in [0, n)
__device__ __forceinline__ int wrap(int b, int d, int n) {
  int t = b + d;
  if (d < 0) t += (t < 0) ? n : 0;
  else t -= (t >= n) ? n : 0;
  return t;
}

template <int N, int NT, int R, int P>
__global__ void __launch_bounds__(NT) k_el_sweep(const __grid_constant__ CUtensorMap tm_xx,
                                                 const __grid_constant__ CUtensorMap tm_zz,
                                                 const __grid_constant__ CUtensorMap tm_xz,
                                                 SweepGeom gm, Coef c, float dtx, float dtz,
                                                 HabcDev h, ElFields A, ElMat m, ElOut o,
                                                 const long long* __restrict__ bounds,
                                                 int* __restrict__ err) {
  using S = SweepShape<N, R, P>;
  constexpr int M = S::M, HS = S::HS, SR = S::SR, SVP = S::SVP, SVV = S::SVV, SSP = S::SSP;
  constexpr int NSLOT = S::NSLOT;
  const int TX = gm.TX, W = gm.W;
  extern __shared__ __align__(128) float sm[];
  float* ring = sm;                  // [3][SR][W]   txx, tzz, txz of time n
  float* rvp = ring + 3 * SR * W;    // [2][SVP][NT] v'
  float* rvv = rvp + 2 * SVP * NT;   // [2][SVV][NT] v''
  float* rsp = rvv + 2 * SVV * NT;   // [3][SSP][NT] s'
  float* rvo = rsp + 3 * SSP * NT;   // [2][SVP][NT] A.v on the v' rows (Higdon old values)
  float* rso = rvo + 2 * SVP * NT;   // [3][SSP][NT] A.stress on the s' rows
  float* swt = rso + 3 * SSP * NT;   // [3][h.wstride] HABC weight ramps
  const int nfl = 3 * SR * W + (4 * SVP + 2 * SVV + 6 * SSP) * NT + 3 * h.wstride;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + ((nfl + 1) & ~1));  // [NSLOT]

  // ---- persistent work split: this CTA owns rows [r_lo, r_hi) of the
  // flattened (strip + nstrip*shot, z) space, i.e. one or a few z-segments ----
  const long long r_lo = bounds[blockIdx.x];
  const long long r_hi = bounds[blockIdx.x + 1];

  // ---- thread -> column offset co (relative to x0); stage membership ----
  const int t = threadIdx.x;
  int co;
  if (t < TX + 2) co = t - 1;
  else if (t < TX + 2 + M) co = -2 - (t - (TX + 2));
  else if (t < TX + 2 + 2 * M) co = TX + 1 + (t - (TX + 2 + M));
  else if (t == TX + 2 + 2 * M) co = -M - 2;
  else co = TX + M + 1;  // t == TX + 3 + 2M, or idle beyond
  const bool do_v1 = t < TX + 2 * M + 4;
  const bool do_v2 = t < TX + 2 + 2 * M;
  const bool do_s1 = t < TX + 2;
  const bool do_s2 = t >= 1 && t <= TX;
  const int ci = co + M + 2;  // column slot in v'/v''/s' rows
  const int cr = co + HS;     // column slot in ring rows

  for (int k = t; k < nfl; k += NT) sm[k] = 0.0f;
  __syncthreads();
  for (int k = t; k < 3 * h.wstride; k += NT) swt[k] = __ldg(h.wtab + k);
  auto wsm = [&](int kind, int dist) { return dist < h.wstride ? swt[kind * h.wstride + dist] : 1.0f; };
  if (t == 0) {
    for (int k = 0; k < NSLOT; ++k) mbar_init(&bars[k], 1);
    tma::mbar_init_fence();
  }
  __syncthreads();

  const uint32_t chunk_bytes = 3u * (uint32_t)R * (uint32_t)W * 4u;
  int gc = 0;  // chunks consumed so far by this CTA (slot = gc % NSLOT)
  bool live = true;
  for (long long r = r_lo; r < r_hi;) {
    const long long item = r / gm.nz;
    const int zA = (int)(r - item * gm.nz);
    const int zB = (int)min((long long)gm.nz, zA + (r_hi - r));
    r += zB - zA;
    const int strip = (int)(item % gm.nstrip);
    const int shot = (int)(item / gm.nstrip);
    const int x0 = strip * TX;
    const long long so = (long long)shot * gm.plane;
    const int x = x0 + co;
    // column predicates (fixed per segment): valid, interior, frame side, distance
    const bool xin = x >= 0 && x < gm.nx;
    const bool xint = x >= M && x < gm.nx - M;
    const bool xfr = x >= 1 && x <= gm.nx - 2;
    const int sxc = x <= gm.nbc ? 1 : (x >= gm.nx - 1 - gm.nbc ? -1 : 0);
    const int dxc = min(x, gm.nx - 1 - x);

    const int zfirst = zA - 2 * M - 2 - R;  // first ring row of this segment
    const int J = (zB + 2 * M + 3 - R - zfirst + R - 1) / R + 1;
    auto issue = [&](int jj) {  // segment-local chunk jj -> ring slot (gc + jj) % NSLOT
      const int g = gc + jj;
      uint64_t* b = &bars[g % NSLOT];
      float* dst = ring + (g % NSLOT) * R * W;
      const int zr = zfirst + jj * R;
      mbar_expect_tx(b, chunk_bytes);
      tma_load_3d(dst, &tm_xx, x0 - HS, zr, shot, b);
      tma_load_3d(dst + SR * W, &tm_zz, x0 - HS, zr, shot, b);
      tma_load_3d(dst + 2 * SR * W, &tm_xz, x0 - HS, zr, shot, b);
    };
    __syncthreads();  // the previous segment's readers of the ring are done
    if (t == 0 && live) {
      fence_proxy_async();
      for (int jj = 0; jj < P && jj < J; ++jj) issue(jj);
    }
    int p1 = 0, b2 = 0, s3 = 0;
    for (int j = 0; j < J; ++j) {
    const int hz = zfirst + j * R;  // first row of the chunk landing this iteration
    // Prefetch what does not depend on the chunk: A.v + buoyancy of the v'
    // rows, old stress + Lame parameters of the s' rows.
    float pax[R], paz[R], pbx[R], pbz[R], pxx[R], pzz[R], pxz[R], plam[R], pl2m[R], pmut[R];
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
      const int z = hz - M + rr, zs = hz - 2 * M - 2 + rr;
      pax[rr] = paz[rr] = pbx[rr] = pbz[rr] = 0.0f;
      pxx[rr] = pzz[rr] = pxz[rr] = plam[rr] = pl2m[rr] = pmut[rr] = 0.0f;
      if (do_v1 && xin && z >= 0 && z < gm.nz) {
        const long long pm = (long long)z * gm.ld + x;
        pax[rr] = __ldg(A.vx + so + pm);
        paz[rr] = __ldg(A.vz + so + pm);
        pbx[rr] = __ldg(m.bx + pm);
        pbz[rr] = __ldg(m.bz + pm);
      }
      if (do_s1 && xin && zs >= 0 && zs < gm.nz) {
        const long long pm = (long long)zs * gm.ld + x;
        pxx[rr] = __ldg(A.txx + so + pm);
        pzz[rr] = __ldg(A.tzz + so + pm);
        pxz[rr] = __ldg(A.txz + so + pm);
        plam[rr] = __ldg(m.lam + pm);
        pl2m[rr] = __ldg(m.l2m + pm);
        pmut[rr] = __ldg(m.mut + pm);
      }
    }
    const int rb = ((gc + j) % NSLOT) * R;  // ring row of hz
    if (live)
      live = mbar_wait_bounded(&bars[(gc + j) % NSLOT], (uint32_t)(((gc + j) / NSLOT) & 1), err);

    // ---- v' rows hz-M+rr: z-window of txz/tzz in registers, rows interleaved ----
    if (do_v1) {
      constexpr int WN = 2 * M + R;  // window rows hz-2M .. hz+R-1
      float wxz[WN], wzz[WN];
#pragma unroll
      for (int k = 0; k < WN; ++k) {
        const int off = wrap(rb, k - 2 * M, SR) * W + cr;
        wxz[k] = ring[2 * SR * W + off];
        wzz[k] = ring[SR * W + off];
      }
      const float* rxx[R];
      const float* rxz[R];
      float dxx[R], dxzx[R], dxzz[R], dzz[R];
#pragma unroll
      for (int rr = 0; rr < R; ++rr) {
        const int off = wrap(rb, rr - M, SR) * W + cr;
        rxx[rr] = ring + off;
        rxz[rr] = ring + 2 * SR * W + off;
        dxx[rr] = dxzx[rr] = dxzz[rr] = dzz[rr] = 0.0f;
      }
#pragma unroll
      for (int l = 1; l <= N; ++l) {
        const float a = c.a[l - 1];
#pragma unroll
        for (int rr = 0; rr < R; ++rr) {
          const int k0 = M + rr;  // window index of row hz-M+rr
          dxx[rr] = __fmaf_rn(a, __fsub_rn(rxx[rr][l - 1], rxx[rr][-l]), dxx[rr]);
          dxzz[rr] = __fmaf_rn(a, __fsub_rn(wxz[k0 + l - 1], wxz[k0 - l]), dxzz[rr]);
          dxzx[rr] = __fmaf_rn(a, __fsub_rn(rxz[rr][l], rxz[rr][-(l - 1)]), dxzx[rr]);
          dzz[rr] = __fmaf_rn(a, __fsub_rn(wzz[k0 + l], wzz[k0 - l + 1]), dzz[rr]);
        }
      }
#pragma unroll
      for (int rr = 0; rr < R; ++rr) {
        const int z = hz - M + rr;
        float ux = pax[rr], uz = paz[rr];
        if (xint && z >= M && z < gm.nz - M) {
          ux = __fmaf_rn(pbx[rr], __fmaf_rn(dtx, dxx[rr], __fmul_rn(dtz, dxzz[rr])), ux);
          uz = __fmaf_rn(pbz[rr], __fmaf_rn(dtx, dxzx[rr], __fmul_rn(dtz, dzz[rr])), uz);
        }
        const int rv = wrap(p1, rr, SVP);
        rvp[rv * NT + ci] = ux;
        rvp[(SVP + rv) * NT + ci] = uz;
        rvo[rv * NT + ci] = pax[rr];
        rvo[(SVP + rv) * NT + ci] = paz[rr];
      }
    }
    __syncthreads();
    // the v' stage was the last reader of the ring slot chunk j+P now refills
    if (t == 0 && live && j + P < J) {
      fence_proxy_async();
      issue(j + P);
    }

    // ---- v'' rows hz-M-1+rr: Higdon on frame cells, then B.v ----
    if (do_v2) {
#pragma unroll
      for (int rr = 0; rr < R; ++rr) {
        const int z = hz - M - 1 + rr;
        const int rv = wrap(p1, rr - 1, SVP);
        float ux = rvp[rv * NT + ci], uz = rvp[(SVP + rv) * NT + ci];
        const int szr = z <= gm.nbc ? 1 : (z >= gm.nz - 1 - gm.nbc ? -1 : 0);
        if (xfr && z >= 1 && z <= gm.nz - 2 && (sxc != 0 || szr != 0)) {
          const int dist = min(dxc, min(z, gm.nz - 1 - z));
          const float wx = wsm(0, dist), wz = wsm(1, dist);
          const float fox = rvo[rv * NT + ci], foz = rvo[(SVP + rv) * NT + ci];
          if (sxc != 0 && szr != 0) {
            const int rz = wrap(p1, rr - 1 + szr, SVP);
            ux = higdon_corner(wx, ux,
                               higdon_side(h, rvp[rv * NT + ci + sxc], fox, rvo[rv * NT + ci + sxc]),
                               higdon_side(h, rvp[rz * NT + ci], fox, rvo[rz * NT + ci]));
            uz = higdon_corner(wz, uz,
                               higdon_side(h, rvp[(SVP + rv) * NT + ci + sxc], foz,
                                           rvo[(SVP + rv) * NT + ci + sxc]),
                               higdon_side(h, rvp[(SVP + rz) * NT + ci], foz, rvo[(SVP + rz) * NT + ci]));
          } else if (sxc != 0) {
            ux = higdon_edge(wx, ux,
                             higdon_side(h, rvp[rv * NT + ci + sxc], fox, rvo[rv * NT + ci + sxc]));
            uz = higdon_edge(wz, uz,
                             higdon_side(h, rvp[(SVP + rv) * NT + ci + sxc], foz,
                                         rvo[(SVP + rv) * NT + ci + sxc]));
          } else {
            const int rz = wrap(p1, rr - 1 + szr, SVP);
            ux = higdon_edge(wx, ux, higdon_side(h, rvp[rz * NT + ci], fox, rvo[rz * NT + ci]));
            uz = higdon_edge(wz, uz,
                             higdon_side(h, rvp[(SVP + rz) * NT + ci], foz, rvo[(SVP + rz) * NT + ci]));
          }
        }
        const int rw = wrap(b2, M + 1 + rr, SVV);
        rvv[rw * NT + ci] = ux;
        rvv[(SVV + rw) * NT + ci] = uz;
        if (co >= 0 && co < TX && xin && z >= zA && z < zB) {
          const long long p = so + (long long)z * gm.ld + x;
          o.vx[p] = ux;
          o.vz[p] = uz;
        }
      }
    }
    __syncthreads();

    // ---- s' rows hz-2M-2+rr from v'': z-window of v'' in registers ----
    if (do_s1) {
      constexpr int WN = 2 * M + R;  // v'' rows hz-3M-2 .. hz-M-3+R
      float wvx[WN], wvz[WN];
#pragma unroll
      for (int k = 0; k < WN; ++k) {
        const int rw = wrap(b2, k - M, SVV);
        wvx[k] = rvv[rw * NT + ci];
        wvz[k] = rvv[(SVV + rw) * NT + ci];
      }
      const float* vxr[R];
      const float* vzr[R];
      float dvxdx[R], dvzdz[R], dvxdz[R], dvzdx[R];
#pragma unroll
      for (int rr = 0; rr < R; ++rr) {
        const int rw = wrap(b2, rr, SVV);
        vxr[rr] = rvv + rw * NT + ci;
        vzr[rr] = rvv + (SVV + rw) * NT + ci;
        dvxdx[rr] = dvzdz[rr] = dvxdz[rr] = dvzdx[rr] = 0.0f;
      }
#pragma unroll
      for (int l = 1; l <= N; ++l) {
        const float a = c.a[l - 1];
#pragma unroll
        for (int rr = 0; rr < R; ++rr) {
          const int k0 = M + rr;  // window index of row hz-2M-2+rr
          dvxdx[rr] = __fmaf_rn(a, __fsub_rn(vxr[rr][l], vxr[rr][-(l - 1)]), dvxdx[rr]);
          dvzdz[rr] = __fmaf_rn(a, __fsub_rn(wvz[k0 + l - 1], wvz[k0 - l]), dvzdz[rr]);
          dvxdz[rr] = __fmaf_rn(a, __fsub_rn(wvx[k0 + l], wvx[k0 - l + 1]), dvxdz[rr]);
          dvzdx[rr] = __fmaf_rn(a, __fsub_rn(vzr[rr][l - 1], vzr[rr][-l]), dvzdx[rr]);
        }
      }
#pragma unroll
      for (int rr = 0; rr < R; ++rr) {
        const int z = hz - 2 * M - 2 + rr;
        float sxx = pxx[rr], szz = pzz[rr], sxz = pxz[rr];
        if (xint && z >= M && z < gm.nz - M) {
          const float ex = __fmul_rn(dvxdx[rr], dtx), ez = __fmul_rn(dvzdz[rr], dtz);
          sxx = __fadd_rn(sxx, __fmaf_rn(pl2m[rr], ex, __fmul_rn(plam[rr], ez)));
          szz = __fadd_rn(szz, __fmaf_rn(plam[rr], ex, __fmul_rn(pl2m[rr], ez)));
          sxz = __fmaf_rn(pmut[rr], __fmaf_rn(dvxdz[rr], dtz, __fmul_rn(dvzdx[rr], dtx)), sxz);
        }
        const int rs = wrap(s3, rr, SSP);
        rsp[rs * NT + ci] = sxx;
        rsp[(SSP + rs) * NT + ci] = szz;
        rsp[(2 * SSP + rs) * NT + ci] = sxz;
        rso[rs * NT + ci] = pxx[rr];
        rso[(SSP + rs) * NT + ci] = pzz[rr];
        rso[(2 * SSP + rs) * NT + ci] = pxz[rr];
      }
    }
    __syncthreads();

    // ---- s'' rows hz-2M-3+rr: Higdon on frame cells, then B.stress ----
    if (do_s2 && xin) {
      float* out[3] = {o.txx + so, o.tzz + so, o.txz + so};
#pragma unroll
      for (int rr = 0; rr < R; ++rr) {
        const int z = hz - 2 * M - 3 + rr;
        if (z < zA || z >= zB) continue;
        const int rs = wrap(s3, rr - 1, SSP);
        float v[3] = {rsp[rs * NT + ci], rsp[(SSP + rs) * NT + ci], rsp[(2 * SSP + rs) * NT + ci]};
        const int szr = z <= gm.nbc ? 1 : (z >= gm.nz - 1 - gm.nbc ? -1 : 0);
        const long long p = (long long)z * gm.ld + x;
        if (xfr && z >= 1 && z <= gm.nz - 2 && (sxc != 0 || szr != 0)) {
          const int dist = min(dxc, min(z, gm.nz - 1 - z));
          const float w = wsm(2, dist);
          const int rz = wrap(s3, rr - 1 + szr, SSP);
#pragma unroll
          for (int f = 0; f < 3; ++f) {
            const float* sp_ = rsp + f * SSP * NT;
            const float* so_ = rso + f * SSP * NT;
            const float fo = so_[rs * NT + ci];
            if (sxc != 0 && szr != 0) {
              v[f] = higdon_corner(w, v[f], higdon_side(h, sp_[rs * NT + ci + sxc], fo, so_[rs * NT + ci + sxc]),
                                   higdon_side(h, sp_[rz * NT + ci], fo, so_[rz * NT + ci]));
            } else if (sxc != 0) {
              v[f] = higdon_edge(w, v[f], higdon_side(h, sp_[rs * NT + ci + sxc], fo, so_[rs * NT + ci + sxc]));
            } else {
              v[f] = higdon_edge(w, v[f], higdon_side(h, sp_[rz * NT + ci], fo, so_[rz * NT + ci]));
            }
          }
        }
        out[0][p] = v[0];
        out[1][p] = v[1];
        out[2][p] = v[2];
      }
    }
    p1 = wrap(p1, R, SVP);
    b2 = wrap(b2, R, SVV);
    s3 = wrap(s3, R, SSP);
    }
    gc += J;
  }
  // After a timed-out wait, drain (bounded) the copies this CTA may still have
  // in flight before its shared memory is released.
  if (!live && t == 0)
    for (int g = gc > NSLOT ? gc - NSLOT : 0; g < gc; ++g)
      mbar_wait_bounded(&bars[g % NSLOT], (uint32_t)((g / NSLOT) & 1), err);
}

// ===========================================================================
// Pair-blocked single sweep (the "x2" variants).
//
// 256 threads = two row halves of 128; a thread owns two adjacent columns and
// every iteration advances two rows, half hh taking row +hh of each stage.
// Iteration i of a segment (v' rows zv = zv0 + 2i, zv + 1):
//   stage A:  v'(zv+hh)      from the tau ring (stress of time n)
//             s'(zv-3-M+hh)  from the v'' ring
//   stage B:  v''(zv-1+hh)   = HABC(v')  -> v'' ring, B.v
//             s''(zv-4-M+hh) = HABC(s')  -> B.stress
// The stress of time n (3 fields) and A.v (2 fields) arrive by TMA in boxes
// of 2 rows x 256 columns into shared rings; the materials come from L2 (they
// are shared by every shot).  Each cell is computed with the canonical
// arithmetic of the two-phase kernels, so results are bit-identical to them.
//
// Columns (relative to the strip's first output column X0):
//   s''  [0, TX)                 outputs
//   s'   [-2, TX+2)              HABC of s'' needs s' at +-1
//   v''  [-2-M, TX+2+M)          stress derivatives need v'' at +-M
//   v'   [-HV, TX+HV), HV>=M+3   HABC of v'' needs v' at +-1
//   tau  [-HV-TN, -HV-TN+256)    v' derivatives need tau at +-M
// ===========================================================================
constexpr int kX2Threads = 256;
constexpr int kX2W = 256;  // ring row pitch = TMA box width (floats)
__host__ __device__ constexpr int x2_hv(int N) { return (N + 3 + 3) & ~3; }
__host__ __device__ constexpr int x2_tn(int N) { return (N + 3) & ~3; }
__host__ __device__ constexpr int x2_txmax(int N) {
  return (kX2W - x2_tn(N) - N - 2 * x2_hv(N)) & ~3;
}

template <int N, int P>
struct X2Shape {
  static constexpr int TN = x2_tn(N), HV = x2_hv(N);
  // tau pairs live at iteration i: i-3 .. i+N (s'' old rows .. v' window), + P prefetched
  static constexpr int NPT = N + 4 + P;
  static constexpr int NPV = 2 + P;   // A.v pairs i-1, i, + P prefetched
  static constexpr int NPVV = N + 2;  // v'' rows zv-3-2N .. zv
  static constexpr int LRT = 2 * NPT, LRV = 2 * NPV, LRVV = 2 * NPVV;
  static constexpr int O_TAU = 0;                            // [3][LRT][W]
  static constexpr int O_VO = O_TAU + 3 * LRT * kX2W;        // [2][LRV][W]
  static constexpr int O_VP = O_VO + 2 * LRV * kX2W;         // [2][4][W]
  static constexpr int O_VV = O_VP + 2 * 4 * kX2W;           // [2][LRVV][W]
  static constexpr int O_SP = O_VV + 2 * LRVV * kX2W;        // [3][4][W]
  static constexpr int O_WT = O_SP + 3 * 4 * kX2W;           // [3][wstride]
};

__device__ __forceinline__ int pmod(int x, int n) {
  const int r = x % n;
  return r < 0 ? r + n : r;
}

// x-derivative windows: xv[j] holds column c - 2E + j of a ring row, j < 4E+2
template <int N>
__device__ __forceinline__ void load_xwin(const float* row, int c, float* xv) {
  constexpr int E = (N + 1) / 2;
#pragma unroll
  for (int j = 0; j <= 2 * E; ++j) {
    const float2 v = *reinterpret_cast<const float2*>(row + c - 2 * E + 2 * j);
    xv[2 * j] = v.x;
    xv[2 * j + 1] = v.y;
  }
}
// backward-staggered x derivative at cell c+e:  sum a_l (f[c+e+l-1] - f[c+e-l])
template <int N>
__device__ __forceinline__ float xdm(const float* xv, int e, const Coef& c) {
  constexpr int E = (N + 1) / 2;
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l)
    acc = __fmaf_rn(c.a[l - 1], __fsub_rn(xv[2 * E + e + l - 1], xv[2 * E + e - l]), acc);
  return acc;
}
// forward-staggered x derivative at cell c+e:  sum a_l (f[c+e+l] - f[c+e-l+1])
template <int N>
__device__ __forceinline__ float xdp(const float* xv, int e, const Coef& c) {
  constexpr int E = (N + 1) / 2;
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l)
    acc = __fmaf_rn(c.a[l - 1], __fsub_rn(xv[2 * E + e + l], xv[2 * E + e - l + 1]), acc);
  return acc;
}

template <int N, int P>
__global__ void __launch_bounds__(kX2Threads, 1)
    k_el_sweep_x2(const __grid_constant__ CUtensorMap tm_xx, const __grid_constant__ CUtensorMap tm_zz,
                  const __grid_constant__ CUtensorMap tm_xz, const __grid_constant__ CUtensorMap tm_vx,
                  const __grid_constant__ CUtensorMap tm_vz, SweepGeom gm, Coef c, float dtx,
                  float dtz, HabcDev h, ElMat m, ElOut o, const long long* __restrict__ bounds,
                  int* __restrict__ err) {
  using S = X2Shape<N, P>;
  constexpr int W = kX2W, M = N, TN = S::TN, HV = S::HV;
  constexpr int NPT = S::NPT, NPV = S::NPV, LRT = S::LRT, LRV = S::LRV, LRVV = S::LRVV;
  extern __shared__ __align__(128) float sm[];
  float* s_tau = sm + S::O_TAU;
  float* s_vo = sm + S::O_VO;
  float* s_vp = sm + S::O_VP;
  float* s_vv = sm + S::O_VV;
  float* s_sp = sm + S::O_SP;
  float* s_wt = sm + S::O_WT;
  const int nwt = (3 * h.wstride + 31) & ~31;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + S::O_WT + nwt);  // [NPT]

  const int tid = threadIdx.x, hh = tid >> 7, sc = 2 * (tid & 127);
  const int TX = gm.TX, WV = TX + 2 * HV;
  const Geo2 g2{gm.nx, gm.nz, gm.ld, M, gm.nbc, gm.plane};

  for (int k = tid; k < S::O_WT; k += kX2Threads) sm[k] = 0.0f;
  for (int k = tid; k < 3 * h.wstride; k += kX2Threads) s_wt[k] = __ldg(h.wtab + k);
  if (tid == 0) {
    for (int k = 0; k < NPT; ++k) mbar_init(&bars[k], 1);
    tma::mbar_init_fence();
  }
  __syncthreads();
  auto wsm = [&](int kind, int dist) {
    return dist < h.wstride ? s_wt[kind * h.wstride + dist] : 1.0f;
  };
  auto interior = [&](int x, int z) { return x >= M && x < gm.nx - M && z >= M && z < gm.nz - M; };

  const long long r_lo = bounds[blockIdx.x];
  const long long r_hi = bounds[blockIdx.x + 1];
  int gt = 0, gv = 0;  // tau / A.v pairs this CTA has consumed (ring slot bases)
  bool live = true;
  for (long long r = r_lo; r < r_hi;) {
    const long long item = r / gm.nz;
    const int za = (int)(r - item * gm.nz);
    const int zb = (int)min((long long)gm.nz, za + (r_hi - r));
    r += zb - za;
    const int strip = (int)(item % gm.nstrip);
    const int shot = (int)(item / gm.nstrip);
    const long long so = (long long)shot * gm.plane;
    const int X0 = strip * TX, XV = X0 - HV, XT = XV - TN;
    const int zv0 = za - 2 - M;  // first v' row: v'' from za-1-M feeds s' from za-1
    // iterations until s''(zb-1) (row zv0+2i-3-M at hh=1)
    const int I = (zb - za + 4 + 2 * M + 1) / 2 + 1;
    const int KT = I + M;  // tau pairs 0 .. I-1+M (pair k: rows zv0-M+2k, +1)
    const int tbase = (2 * gt) % LRT, vbase = (2 * gv) % LRV;
    auto issue = [&](int k) {  // tau pair k, plus A.v pair k-M (rows zv0+2(k-M), +1)
      const int slot = (gt + k) % NPT;
      uint64_t* bar = &bars[slot];
      const bool wv = k >= M;
      mbar_expect_tx(bar, (uint32_t)((wv ? 5 : 3) * 2 * W * 4));
      const int zt = zv0 - M + 2 * k;
      tma_load_3d(s_tau + (0 * LRT + 2 * slot) * W, &tm_xx, XT, zt, shot, bar);
      tma_load_3d(s_tau + (1 * LRT + 2 * slot) * W, &tm_zz, XT, zt, shot, bar);
      tma_load_3d(s_tau + (2 * LRT + 2 * slot) * W, &tm_xz, XT, zt, shot, bar);
      if (wv) {
        const int vs = (gv + k - M) % NPV;
        const int zw = zv0 + 2 * (k - M);
        tma_load_3d(s_vo + (0 * LRV + 2 * vs) * W, &tm_vx, XV, zw, shot, bar);
        tma_load_3d(s_vo + (1 * LRV + 2 * vs) * W, &tm_vz, XV, zw, shot, bar);
      }
    };
    __syncthreads();  // the previous segment's readers are done with every ring
    if (tid == 0 && live) {
      fence_proxy_async();
      for (int k = 0; k <= M + P && k < KT; ++k) issue(k);
    }
    const int xc = XV + sc;  // global column of the thread's first cell
    for (int i = 0; i < I; ++i) {
      const int zv = zv0 + 2 * i;
      if (live)
        for (int k = (i == 0 ? 0 : i + M); k <= i + M; ++k) {
          const int gk = gt + k;
          live = mbar_wait_bounded(&bars[gk % NPT], (uint32_t)((gk / NPT) & 1), err) && live;
        }

      // ================= stage A =================
      // ---- v' at row zr ----
      if (sc < WV) {
        const int zr = zv + hh;
        const int tb = pmod(tbase + 2 * i + hh + M, LRT);  // tau ring row of zr
        const int ct = sc + TN;                             // tau column of the first cell
        const float* txx = s_tau;
        const float* tzz = s_tau + LRT * W;
        const float* txz = s_tau + 2 * LRT * W;
        float xw[4 * ((N + 1) / 2) + 2];
        float dxx[2], dxzx[2], dxzz[2], dzz[2];
        load_xwin<N>(txx + tb * W, ct, xw);
        dxx[0] = xdm<N>(xw, 0, c);
        dxx[1] = xdm<N>(xw, 1, c);
        load_xwin<N>(txz + tb * W, ct, xw);
        dxzx[0] = xdp<N>(xw, 0, c);
        dxzx[1] = xdp<N>(xw, 1, c);
        dxzz[0] = dxzz[1] = dzz[0] = dzz[1] = 0.0f;
#pragma unroll
        for (int l = 1; l <= N; ++l) {
          const float a = c.a[l - 1];
          const float2 p0 = *reinterpret_cast<const float2*>(txz + wrap(tb, l - 1, LRT) * W + ct);
          const float2 p1 = *reinterpret_cast<const float2*>(txz + wrap(tb, -l, LRT) * W + ct);
          dxzz[0] = __fmaf_rn(a, __fsub_rn(p0.x, p1.x), dxzz[0]);
          dxzz[1] = __fmaf_rn(a, __fsub_rn(p0.y, p1.y), dxzz[1]);
          const float2 q0 = *reinterpret_cast<const float2*>(tzz + wrap(tb, l, LRT) * W + ct);
          const float2 q1 = *reinterpret_cast<const float2*>(tzz + wrap(tb, 1 - l, LRT) * W + ct);
          dzz[0] = __fmaf_rn(a, __fsub_rn(q0.x, q1.x), dzz[0]);
          dzz[1] = __fmaf_rn(a, __fsub_rn(q0.y, q1.y), dzz[1]);
        }
        const int vr = pmod(vbase + 2 * i + hh, LRV);  // A.v ring row of zr
        const float2 ox = *reinterpret_cast<const float2*>(s_vo + vr * W + sc);
        const float2 oz = *reinterpret_cast<const float2*>(s_vo + (LRV + vr) * W + sc);
        float ux[2] = {ox.x, ox.y}, uz[2] = {oz.x, oz.y};
        float bx[2] = {0.0f, 0.0f}, bz[2] = {0.0f, 0.0f};
        if (zr >= 0 && zr < gm.nz) {
          const long long pm = (long long)zr * gm.ld + xc;
          if (xc >= 0 && xc + 1 < gm.nx) {
            const float2 b0 = __ldg(reinterpret_cast<const float2*>(m.bx + pm));
            const float2 b1 = __ldg(reinterpret_cast<const float2*>(m.bz + pm));
            bx[0] = b0.x; bx[1] = b0.y; bz[0] = b1.x; bz[1] = b1.y;
          } else {
#pragma unroll
            for (int e = 0; e < 2; ++e)
              if (xc + e >= 0 && xc + e < gm.nx) {
                bx[e] = __ldg(m.bx + pm + e);
                bz[e] = __ldg(m.bz + pm + e);
              }
          }
        }
#pragma unroll
        for (int e = 0; e < 2; ++e)
          if (interior(xc + e, zr)) {
            ux[e] = __fmaf_rn(bx[e], __fmaf_rn(dtx, dxx[e], __fmul_rn(dtz, dxzz[e])), ux[e]);
            uz[e] = __fmaf_rn(bz[e], __fmaf_rn(dtx, dxzx[e], __fmul_rn(dtz, dzz[e])), uz[e]);
          }
        const int pr = (2 * i + hh) & 3;  // v' ring row of zr
        *reinterpret_cast<float2*>(s_vp + pr * W + sc) = make_float2(ux[0], ux[1]);
        *reinterpret_cast<float2*>(s_vp + (4 + pr) * W + sc) = make_float2(uz[0], uz[1]);
      }
      // ---- s' at row q ----
      if (sc >= HV - 2 && sc < HV + TX + 2) {
        const int q = zv - 3 - M + hh;
        const int vb = pmod(2 * i - 2 - M + hh, LRVV);  // v'' ring row of q
        const float* vvx = s_vv;
        const float* vvz = s_vv + LRVV * W;
        float xw[4 * ((N + 1) / 2) + 2];
        float dvxdx[2], dvzdx[2], dvxdz[2], dvzdz[2];
        load_xwin<N>(vvx + vb * W, sc, xw);
        dvxdx[0] = xdp<N>(xw, 0, c);
        dvxdx[1] = xdp<N>(xw, 1, c);
        load_xwin<N>(vvz + vb * W, sc, xw);
        dvzdx[0] = xdm<N>(xw, 0, c);
        dvzdx[1] = xdm<N>(xw, 1, c);
        dvxdz[0] = dvxdz[1] = dvzdz[0] = dvzdz[1] = 0.0f;
#pragma unroll
        for (int l = 1; l <= N; ++l) {
          const float a = c.a[l - 1];
          const float2 p0 = *reinterpret_cast<const float2*>(vvx + wrap(vb, l, LRVV) * W + sc);
          const float2 p1 = *reinterpret_cast<const float2*>(vvx + wrap(vb, 1 - l, LRVV) * W + sc);
          dvxdz[0] = __fmaf_rn(a, __fsub_rn(p0.x, p1.x), dvxdz[0]);
          dvxdz[1] = __fmaf_rn(a, __fsub_rn(p0.y, p1.y), dvxdz[1]);
          const float2 q0 = *reinterpret_cast<const float2*>(vvz + wrap(vb, l - 1, LRVV) * W + sc);
          const float2 q1 = *reinterpret_cast<const float2*>(vvz + wrap(vb, -l, LRVV) * W + sc);
          dvzdz[0] = __fmaf_rn(a, __fsub_rn(q0.x, q1.x), dvzdz[0]);
          dvzdz[1] = __fmaf_rn(a, __fsub_rn(q0.y, q1.y), dvzdz[1]);
        }
        const int tq = pmod(tbase + 2 * i - 3 + hh, LRT);  // tau ring row of q
        const float2 oxx = *reinterpret_cast<const float2*>(s_tau + tq * W + sc + TN);
        const float2 ozz = *reinterpret_cast<const float2*>(s_tau + (LRT + tq) * W + sc + TN);
        const float2 oxz = *reinterpret_cast<const float2*>(s_tau + (2 * LRT + tq) * W + sc + TN);
        float sxx[2] = {oxx.x, oxx.y}, szz[2] = {ozz.x, ozz.y}, sxz[2] = {oxz.x, oxz.y};
        float lam[2] = {0.0f, 0.0f}, l2m[2] = {0.0f, 0.0f}, mut[2] = {0.0f, 0.0f};
        if (q >= 0 && q < gm.nz) {
          const long long pm = (long long)q * gm.ld + xc;
          if (xc >= 0 && xc + 1 < gm.nx) {
            const float2 a0 = __ldg(reinterpret_cast<const float2*>(m.lam + pm));
            const float2 a1 = __ldg(reinterpret_cast<const float2*>(m.l2m + pm));
            const float2 a2 = __ldg(reinterpret_cast<const float2*>(m.mut + pm));
            lam[0] = a0.x; lam[1] = a0.y; l2m[0] = a1.x; l2m[1] = a1.y; mut[0] = a2.x; mut[1] = a2.y;
          } else {
#pragma unroll
            for (int e = 0; e < 2; ++e)
              if (xc + e >= 0 && xc + e < gm.nx) {
                lam[e] = __ldg(m.lam + pm + e);
                l2m[e] = __ldg(m.l2m + pm + e);
                mut[e] = __ldg(m.mut + pm + e);
              }
          }
        }
#pragma unroll
        for (int e = 0; e < 2; ++e)
          if (interior(xc + e, q)) {
            const float ex = __fmul_rn(dvxdx[e], dtx), ez = __fmul_rn(dvzdz[e], dtz);
            sxx[e] = __fadd_rn(sxx[e], __fmaf_rn(l2m[e], ex, __fmul_rn(lam[e], ez)));
            szz[e] = __fadd_rn(szz[e], __fmaf_rn(lam[e], ex, __fmul_rn(l2m[e], ez)));
            sxz[e] = __fmaf_rn(mut[e], __fmaf_rn(dvxdz[e], dtz, __fmul_rn(dvzdx[e], dtx)), sxz[e]);
          }
        const int sr = (2 * i + hh) & 3;  // s' ring row of q
        *reinterpret_cast<float2*>(s_sp + sr * W + sc) = make_float2(sxx[0], sxx[1]);
        *reinterpret_cast<float2*>(s_sp + (4 + sr) * W + sc) = make_float2(szz[0], szz[1]);
        *reinterpret_cast<float2*>(s_sp + (8 + sr) * W + sc) = make_float2(sxz[0], sxz[1]);
      }
      __syncthreads();

      // ================= stage B =================
      // ---- v'' at row qv: Higdon on frame cells; -> v'' ring, B.v ----
      if (sc < WV) {
        const int qv = zv - 1 + hh;
        const int pr = (2 * i - 1 + hh) & 3;           // v' ring row of qv
        const int orow = pmod(vbase + 2 * i - 1 + hh, LRV);  // A.v ring row of qv
        float v[2][2];  // [field][cell]
        {
          const float2 fx = *reinterpret_cast<const float2*>(s_vp + pr * W + sc);
          const float2 fz = *reinterpret_cast<const float2*>(s_vp + (4 + pr) * W + sc);
          v[0][0] = fx.x; v[0][1] = fx.y; v[1][0] = fz.x; v[1][1] = fz.y;
        }
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          int sx, sz, dist;
          if (!frame2(g2, xc + e, qv, sx, sz, dist)) continue;
          const int col = sc + e;
          const int coln = min(max(col + sx, 0), W - 1);
          const int prn = (2 * i - 1 + hh + sz) & 3;
          const int orn = pmod(vbase + 2 * i - 1 + hh + sz, LRV);
#pragma unroll
          for (int f = 0; f < 2; ++f) {
            const float* fp = s_vp + f * 4 * W;
            const float* fo = s_vo + f * LRV * W;
            const float w = wsm(f, dist);
            const float fop = fo[orow * W + col];
            if (sx != 0 && sz != 0)
              v[f][e] = higdon_corner(w, v[f][e],
                                      higdon_side(h, fp[pr * W + coln], fop, fo[orow * W + coln]),
                                      higdon_side(h, fp[prn * W + col], fop, fo[orn * W + col]));
            else if (sx != 0)
              v[f][e] = higdon_edge(w, v[f][e],
                                    higdon_side(h, fp[pr * W + coln], fop, fo[orow * W + coln]));
            else
              v[f][e] = higdon_edge(w, v[f][e],
                                    higdon_side(h, fp[prn * W + col], fop, fo[orn * W + col]));
          }
        }
        const int vw = (2 * i + hh) % LRVV;  // v'' ring row of qv
        *reinterpret_cast<float2*>(s_vv + vw * W + sc) = make_float2(v[0][0], v[0][1]);
        *reinterpret_cast<float2*>(s_vv + (LRVV + vw) * W + sc) = make_float2(v[1][0], v[1][1]);
        if (qv >= za && qv < zb && sc >= HV && sc < HV + TX && xc < gm.nx) {
          const long long p = so + (long long)qv * gm.ld + xc;
          if (xc + 1 < gm.nx) {
            *reinterpret_cast<float2*>(o.vx + p) = make_float2(v[0][0], v[0][1]);
            *reinterpret_cast<float2*>(o.vz + p) = make_float2(v[1][0], v[1][1]);
          } else {
            o.vx[p] = v[0][0];
            o.vz[p] = v[1][0];
          }
        }
      }
      // ---- s'' at row qs: Higdon on frame cells -> B.stress ----
      {
        const int qs = zv - 4 - M + hh;
        if (qs >= za && qs < zb && sc >= HV && sc < HV + TX && xc < gm.nx) {
          const int sr = (2 * i - 1 + hh) & 3;  // s' ring row of qs
          float v[3][2];
#pragma unroll
          for (int f = 0; f < 3; ++f) {
            const float2 t2 = *reinterpret_cast<const float2*>(s_sp + (4 * f + sr) * W + sc);
            v[f][0] = t2.x;
            v[f][1] = t2.y;
          }
          const int trow = pmod(tbase + 2 * i - 4 + hh, LRT);  // tau ring row of qs
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            int sx, sz, dist;
            if (!frame2(g2, xc + e, qs, sx, sz, dist)) continue;
            const int col = sc + e;
            const int coln = min(max(col + sx, 0), W - 1);
            const int srn = (2 * i - 1 + hh + sz) & 3;
            const int trn = pmod(tbase + 2 * i - 4 + hh + sz, LRT);
            const float w = wsm(2, dist);
#pragma unroll
            for (int f = 0; f < 3; ++f) {
              const float* fp = s_sp + 4 * f * W;
              const float* fo = s_tau + f * LRT * W + TN;
              const float fop = fo[trow * W + col];
              if (sx != 0 && sz != 0)
                v[f][e] = higdon_corner(w, v[f][e],
                                        higdon_side(h, fp[sr * W + coln], fop, fo[trow * W + coln]),
                                        higdon_side(h, fp[srn * W + col], fop, fo[trn * W + col]));
              else if (sx != 0)
                v[f][e] = higdon_edge(w, v[f][e],
                                      higdon_side(h, fp[sr * W + coln], fop, fo[trow * W + coln]));
              else
                v[f][e] = higdon_edge(w, v[f][e],
                                      higdon_side(h, fp[srn * W + col], fop, fo[trn * W + col]));
            }
          }
          const long long p = so + (long long)qs * gm.ld + xc;
          float* out[3] = {o.txx, o.tzz, o.txz};
#pragma unroll
          for (int f = 0; f < 3; ++f) {
            if (xc + 1 < gm.nx)
              *reinterpret_cast<float2*>(out[f] + p) = make_float2(v[f][0], v[f][1]);
            else
              out[f][p] = v[f][0];
          }
        }
      }
      __syncthreads();
      // tau pair i-3 and A.v pair i-1 are dead: refill their slots
      if (tid == 0 && live && i + M + 1 + P < KT) {
        fence_proxy_async();
        issue(i + M + 1 + P);
      }
    }
    gt += KT;
    gv += I;
  }
}

// ===========================================================================
// Register-window single sweep (the "rw" variants).
//
// 128 threads; thread t owns the column pair XV + 2t, +1 and takes two rows
// per iteration through all four stages, so it keeps both z-derivative
// windows in registers: txz/tzz rows zv-M .. zv+M+1 for v', and v''x/v''z rows
// q-M .. q+M+1 for s' (q = zv-3-M).  Shared memory holds only what crosses
// columns: the x-derivative rows and the Higdon x-neighbours.  The stress of
// time n arrives by TMA in three small streams of 2-row boxes (rows zv+M for
// the window, rows zv for the x-derivatives, rows q for the old values), so a
// CTA needs about 100 KB and two fit on an SM.  Materials are read from L2
// one iteration ahead.  Per iteration i (zv = zv0 + 2i):
//   A: v'(zv, zv+1)        s'(q, q+1)
//   B: v''(zv-1, zv)       s''(q-1, q)      (Higdon on frame cells; outputs)
// Same canonical per-cell arithmetic as every other kernel (bit-identical).
// ===========================================================================
constexpr int kRWThreads = 128;

template <int N, int P>
struct RWShape {
  static constexpr int TN = x2_tn(N), HV = x2_hv(N);
  static constexpr int NZ = P + 1;                  // z / x stream slots
  static constexpr int NO = P + 2;                  // old-stress / A.v stream slots (and barriers)
  static constexpr int LVV = (N + 2 + 1) & ~1;      // v'' rows kept for the s' x-derivatives
  static constexpr int O_Z = 0;                          // [NZ][txz, tzz][2][W]   rows zv+M, +1
  static constexpr int O_X = O_Z + NZ * 4 * kX2W;        // [NZ][txx, txz][2][W]   rows zv, zv+1
  static constexpr int O_O = O_X + NZ * 4 * kX2W;        // [NO][txx, tzz, txz][2][W] rows q, q+1
  static constexpr int O_V = O_O + NO * 6 * kX2W;        // [NO][vx, vz][2][W]     rows zv, zv+1
  static constexpr int O_VP = O_V + NO * 4 * kX2W;       // [vx, vz][4][W]  v'
  static constexpr int O_VV = O_VP + 8 * kX2W;           // [vx, vz][LVV][W] v''
  static constexpr int O_SP = O_VV + 2 * LVV * kX2W;     // [xx, zz, xz][4][W] s'
  static constexpr int O_WT = O_SP + 12 * kX2W;          // [3][wstride] weights
};

template <int N, int P>
__global__ void __launch_bounds__(kRWThreads, 2)
    k_el_sweep_rw(const __grid_constant__ CUtensorMap tm_xx, const __grid_constant__ CUtensorMap tm_zz,
                  const __grid_constant__ CUtensorMap tm_xz, const __grid_constant__ CUtensorMap tm_vx,
                  const __grid_constant__ CUtensorMap tm_vz, SweepGeom gm, Coef c, float dtx,
                  float dtz, HabcDev h, ElMat m, ElOut o, const long long* __restrict__ bounds,
                  int* __restrict__ err) {
  using S = RWShape<N, P>;
  constexpr int W = kX2W, M = N, TN = S::TN, HV = S::HV;
  constexpr int NZ = S::NZ, NO = S::NO, LVV = S::LVV;
  constexpr int WN = 2 * M + 2;  // window rows
  extern __shared__ __align__(128) float sm[];
  float* s_z = sm + S::O_Z;
  float* s_x = sm + S::O_X;
  float* s_o = sm + S::O_O;
  float* s_v = sm + S::O_V;
  float* s_vp = sm + S::O_VP;
  float* s_vv = sm + S::O_VV;
  float* s_sp = sm + S::O_SP;
  float* s_wt = sm + S::O_WT;
  const int nwt = (3 * h.wstride + 31) & ~31;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + S::O_WT + nwt);  // [NO]

  const int tid = threadIdx.x, sc = 2 * tid;
  const int TX = gm.TX, WV = TX + 2 * HV;
  const Geo2 g2{gm.nx, gm.nz, gm.ld, M, gm.nbc, gm.plane};
  for (int k = tid; k < S::O_WT; k += kRWThreads) sm[k] = 0.0f;
  for (int k = tid; k < 3 * h.wstride; k += kRWThreads) s_wt[k] = __ldg(h.wtab + k);
  if (tid == 0) {
    for (int k = 0; k < NO; ++k) mbar_init(&bars[k], 1);
    tma::mbar_init_fence();
  }
  __syncthreads();
  auto wsm = [&](int kind, int dist) {
    return dist < h.wstride ? s_wt[kind * h.wstride + dist] : 1.0f;
  };
  auto interior = [&](int x, int z) { return x >= M && x < gm.nx - M && z >= M && z < gm.nz - M; };
  const bool do_v = sc < WV;
  const bool do_s = sc >= HV - 2 && sc < HV + TX + 2;
  const bool do_o = sc >= HV && sc < HV + TX;

  const long long r_lo = bounds[blockIdx.x];
  const long long r_hi = bounds[blockIdx.x + 1];
  int gb = 0;  // batches this CTA has consumed (ring slot / barrier phase base)
  bool live = true;
  for (long long r = r_lo; r < r_hi;) {
    const long long item = r / gm.nz;
    const int za = (int)(r - item * gm.nz);
    const int zb = (int)min((long long)gm.nz, za + (r_hi - r));
    r += zb - za;
    const int strip = (int)(item % gm.nstrip);
    const int shot = (int)(item / gm.nstrip);
    const long long so = (long long)shot * gm.plane;
    const int X0 = strip * TX, XV = X0 - HV, XT = XV - TN;
    const int xc = XV + sc;
    // M warm-up iterations fill the txz/tzz window before the first needed v' row
    const int zv0 = za - 2 - 3 * M;
    const int I = (zb - za + 4 + 4 * M + 1) / 2 + 1;
    auto issue = [&](int k) {
      const int gk = gb + k, zs = gk % NZ, os = gk % NO;
      uint64_t* bar = &bars[os];
      mbar_expect_tx(bar, 9u * 2u * W * 4u);
      const int zr = zv0 + 2 * k;
      tma_load_3d(s_z + (zs * 2 + 0) * 2 * W, &tm_xz, XT, zr + M, shot, bar);
      tma_load_3d(s_z + (zs * 2 + 1) * 2 * W, &tm_zz, XT, zr + M, shot, bar);
      tma_load_3d(s_x + (zs * 2 + 0) * 2 * W, &tm_xx, XT, zr, shot, bar);
      tma_load_3d(s_x + (zs * 2 + 1) * 2 * W, &tm_xz, XT, zr, shot, bar);
      tma_load_3d(s_o + (os * 3 + 0) * 2 * W, &tm_xx, XT, zr - 3 - M, shot, bar);
      tma_load_3d(s_o + (os * 3 + 1) * 2 * W, &tm_zz, XT, zr - 3 - M, shot, bar);
      tma_load_3d(s_o + (os * 3 + 2) * 2 * W, &tm_xz, XT, zr - 3 - M, shot, bar);
      tma_load_3d(s_v + (os * 2 + 0) * 2 * W, &tm_vx, XV, zr, shot, bar);
      tma_load_3d(s_v + (os * 2 + 1) * 2 * W, &tm_vz, XV, zr, shot, bar);
    };
    __syncthreads();  // the previous segment's readers are done with every ring
    if (tid == 0 && live) {
      fence_proxy_async();
      for (int k = 0; k <= P && k < I; ++k) issue(k);
    }
    // register state
    float wxz[WN][2], wzz[WN][2], wvx[WN][2], wvz[WN][2];
#pragma unroll
    for (int k = 0; k < WN; ++k)
#pragma unroll
      for (int e = 0; e < 2; ++e) wxz[k][e] = wzz[k][e] = wvx[k][e] = wvz[k][e] = 0.0f;
    float vpp[2][2][2], spp[3][2][2];  // previous iteration's v' / s' rows [field][row][cell]
#pragma unroll
    for (int f = 0; f < 2; ++f)
#pragma unroll
      for (int k = 0; k < 4; ++k) vpp[f][k >> 1][k & 1] = 0.0f;
#pragma unroll
    for (int f = 0; f < 3; ++f)
#pragma unroll
      for (int k = 0; k < 4; ++k) spp[f][k >> 1][k & 1] = 0.0f;
    // materials of iteration i, loaded during iteration i-1
    float mbx[2][2], mbz[2][2], mla[2][2], ml2[2][2], mmu[2][2];
    auto load_mat = [&](int zv) {
#pragma unroll
      for (int rr = 0; rr < 2; ++rr) {
        const int zr = zv + rr, zq = zv - 3 - M + rr;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int x = xc + e;
          const bool xin = x >= 0 && x < gm.nx;
          const bool vin = do_v && xin && zr >= 0 && zr < gm.nz;
          const bool sin_ = do_s && xin && zq >= 0 && zq < gm.nz;
          const long long pv = (long long)zr * gm.ld + x, ps = (long long)zq * gm.ld + x;
          mbx[rr][e] = vin ? __ldg(m.bx + pv) : 0.0f;
          mbz[rr][e] = vin ? __ldg(m.bz + pv) : 0.0f;
          mla[rr][e] = sin_ ? __ldg(m.lam + ps) : 0.0f;
          ml2[rr][e] = sin_ ? __ldg(m.l2m + ps) : 0.0f;
          mmu[rr][e] = sin_ ? __ldg(m.mut + ps) : 0.0f;
        }
      }
    };
    load_mat(zv0);

    for (int i = 0; i < I; ++i) {
      const int zv = zv0 + 2 * i, q = zv - 3 - M;
      const int gi = gb + i, zs = gi % NZ, os = gi % NO, osp = (gi + NO - 1) % NO;
      if (live)
        live = mbar_wait_bounded(&bars[os], (uint32_t)((gi / NO) & 1), err) && live;
      // ---------------- stage A ----------------
      // new window rows zv+M, zv+M+1 of txz and tzz
#pragma unroll
      for (int rr = 0; rr < 2; ++rr) {
        const float2 a = *reinterpret_cast<const float2*>(s_z + ((zs * 2 + 0) * 2 + rr) * W + sc + TN);
        const float2 b = *reinterpret_cast<const float2*>(s_z + ((zs * 2 + 1) * 2 + rr) * W + sc + TN);
        wxz[2 * M + rr][0] = a.x;
        wxz[2 * M + rr][1] = a.y;
        wzz[2 * M + rr][0] = b.x;
        wzz[2 * M + rr][1] = b.y;
      }
      float vpc[2][2][2];  // v' rows zv, zv+1 [field][row][cell]
      if (do_v) {
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
          const int zr = zv + rr;
          float xw[4 * ((N + 1) / 2) + 2];
          float dxx[2], dxzx[2];
          load_xwin<N>(s_x + ((zs * 2 + 0) * 2 + rr) * W, sc + TN, xw);
          dxx[0] = xdm<N>(xw, 0, c);
          dxx[1] = xdm<N>(xw, 1, c);
          load_xwin<N>(s_x + ((zs * 2 + 1) * 2 + rr) * W, sc + TN, xw);
          dxzx[0] = xdp<N>(xw, 0, c);
          dxzx[1] = xdp<N>(xw, 1, c);
          const float2 ox = *reinterpret_cast<const float2*>(s_v + ((os * 2 + 0) * 2 + rr) * W + sc);
          const float2 oz = *reinterpret_cast<const float2*>(s_v + ((os * 2 + 1) * 2 + rr) * W + sc);
          const float vo[2][2] = {{ox.x, ox.y}, {oz.x, oz.y}};
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            float dxzz = 0.0f, dzz = 0.0f;
#pragma unroll
            for (int l = 1; l <= N; ++l) {
              dxzz = __fmaf_rn(c.a[l - 1], __fsub_rn(wxz[rr + M + l - 1][e], wxz[rr + M - l][e]), dxzz);
              dzz = __fmaf_rn(c.a[l - 1], __fsub_rn(wzz[rr + M + l][e], wzz[rr + M - l + 1][e]), dzz);
            }
            float ux = vo[0][e], uz = vo[1][e];
            if (interior(xc + e, zr)) {
              ux = __fmaf_rn(mbx[rr][e], __fmaf_rn(dtx, dxx[e], __fmul_rn(dtz, dxzz)), ux);
              uz = __fmaf_rn(mbz[rr][e], __fmaf_rn(dtx, dxzx[e], __fmul_rn(dtz, dzz)), uz);
            }
            vpc[0][rr][e] = ux;
            vpc[1][rr][e] = uz;
          }
          const int pr = (2 * i + rr) & 3;  // v' ring row of zr
          *reinterpret_cast<float2*>(s_vp + pr * W + sc) = make_float2(vpc[0][rr][0], vpc[0][rr][1]);
          *reinterpret_cast<float2*>(s_vp + (4 + pr) * W + sc) =
              make_float2(vpc[1][rr][0], vpc[1][rr][1]);
        }
      }
      // shift the txz / tzz window by two rows for the next iteration
#pragma unroll
      for (int k = 0; k < 2 * M; ++k)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          wxz[k][e] = wxz[k + 2][e];
          wzz[k][e] = wzz[k + 2][e];
        }
      float spc[3][2][2];  // s' rows q, q+1 [field][row][cell]
      if (do_s) {
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
          const int zq = q + rr;
          const int vb = (2 * i - 2 - M + rr + 2 * LVV) % LVV;  // v'' ring row of zq
          float xw[4 * ((N + 1) / 2) + 2];
          float dvxdx[2], dvzdx[2];
          load_xwin<N>(s_vv + vb * W, sc, xw);
          dvxdx[0] = xdp<N>(xw, 0, c);
          dvxdx[1] = xdp<N>(xw, 1, c);
          load_xwin<N>(s_vv + (LVV + vb) * W, sc, xw);
          dvzdx[0] = xdm<N>(xw, 0, c);
          dvzdx[1] = xdm<N>(xw, 1, c);
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            float dvxdz = 0.0f, dvzdz = 0.0f;
#pragma unroll
            for (int l = 1; l <= N; ++l) {
              dvxdz = __fmaf_rn(c.a[l - 1], __fsub_rn(wvx[rr + M + l][e], wvx[rr + M - l + 1][e]), dvxdz);
              dvzdz = __fmaf_rn(c.a[l - 1], __fsub_rn(wvz[rr + M + l - 1][e], wvz[rr + M - l][e]), dvzdz);
            }
            float sxx = s_o[((os * 3 + 0) * 2 + rr) * W + sc + TN + e];
            float szz = s_o[((os * 3 + 1) * 2 + rr) * W + sc + TN + e];
            float sxz = s_o[((os * 3 + 2) * 2 + rr) * W + sc + TN + e];
            if (interior(xc + e, zq)) {
              const float ex = __fmul_rn(dvxdx[e], dtx), ez = __fmul_rn(dvzdz, dtz);
              sxx = __fadd_rn(sxx, __fmaf_rn(ml2[rr][e], ex, __fmul_rn(mla[rr][e], ez)));
              szz = __fadd_rn(szz, __fmaf_rn(mla[rr][e], ex, __fmul_rn(ml2[rr][e], ez)));
              sxz = __fmaf_rn(mmu[rr][e], __fmaf_rn(dvxdz, dtz, __fmul_rn(dvzdx[e], dtx)), sxz);
            }
            spc[0][rr][e] = sxx;
            spc[1][rr][e] = szz;
            spc[2][rr][e] = sxz;
          }
          const int sr = (2 * i + rr) & 3;  // s' ring row of zq
#pragma unroll
          for (int f = 0; f < 3; ++f)
            *reinterpret_cast<float2*>(s_sp + (4 * f + sr) * W + sc) =
                make_float2(spc[f][rr][0], spc[f][rr][1]);
        }
      }
      __syncthreads();

      // ---------------- stage B ----------------
      // v'' rows zv-1 (rr = 0) and zv (rr = 1); v' rows zv-2 .. zv+1 are in vpp / vpc
      float vvn[2][2][2];
      if (do_v) {
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
          const int qv = zv - 1 + rr;
#pragma unroll
          for (int e = 0; e < 2; ++e) {
#pragma unroll
            for (int f = 0; f < 2; ++f) vvn[f][rr][e] = rr ? vpc[f][0][e] : vpp[f][1][e];
            int sx, sz, dist;
            if (!frame2(g2, xc + e, qv, sx, sz, dist)) continue;
            const int col = sc + e;
            const int coln = min(max(col + sx, 0), W - 1);
            // A.v rows zv-2, zv-1 (previous pair slot) and zv, zv+1 (this pair); row qv:
            const int orow = rr ? 0 : 1;
            const int prow = (2 * i - 1 + rr) & 3;  // v' ring row of qv
            // z-neighbour row qv + sz: A.v and v'
            // row qv + sz: zv-2 / zv-1 sit in the previous pair's slot, zv / zv+1 in this one
            const bool up = sz > 0;
            const int ozs = up ? os : osp;
            const int ozr = rr;
#pragma unroll
            for (int f = 0; f < 2; ++f) {
              const float* fo = s_v + (((rr ? os : osp) * 2 + f) * 2 + orow) * W;
              const float fop = fo[col];
              const float w = wsm(f, dist);
              const float* fzo = s_v + ((ozs * 2 + f) * 2 + ozr) * W;
              const float vz_n = rr ? (up ? vpc[f][1][e] : vpp[f][1][e]) : (up ? vpc[f][0][e] : vpp[f][0][e]);
              const float vx_n = s_vp[(4 * f + prow) * W + coln];
              if (sx != 0 && sz != 0)
                vvn[f][rr][e] = higdon_corner(w, vvn[f][rr][e], higdon_side(h, vx_n, fop, fo[coln]),
                                              higdon_side(h, vz_n, fop, fzo[col]));
              else if (sx != 0)
                vvn[f][rr][e] = higdon_edge(w, vvn[f][rr][e], higdon_side(h, vx_n, fop, fo[coln]));
              else
                vvn[f][rr][e] = higdon_edge(w, vvn[f][rr][e], higdon_side(h, vz_n, fop, fzo[col]));
            }
          }
          const int vw = (2 * i + rr) % LVV;  // v'' ring row of qv
          *reinterpret_cast<float2*>(s_vv + vw * W + sc) = make_float2(vvn[0][rr][0], vvn[0][rr][1]);
          *reinterpret_cast<float2*>(s_vv + (LVV + vw) * W + sc) =
              make_float2(vvn[1][rr][0], vvn[1][rr][1]);
          if (do_o && qv >= za && qv < zb && xc < gm.nx) {
            const long long p = so + (long long)qv * gm.ld + xc;
            if (xc + 1 < gm.nx) {
              *reinterpret_cast<float2*>(o.vx + p) = make_float2(vvn[0][rr][0], vvn[0][rr][1]);
              *reinterpret_cast<float2*>(o.vz + p) = make_float2(vvn[1][rr][0], vvn[1][rr][1]);
            } else {
              o.vx[p] = vvn[0][rr][0];
              o.vz[p] = vvn[1][rr][0];
            }
          }
        }
      }
      // the v'' window advances: rows q-M+2 .. q+M+1, then the new rows zv-1, zv
#pragma unroll
      for (int k = 0; k < 2 * M; ++k)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          wvx[k][e] = wvx[k + 2][e];
          wvz[k][e] = wvz[k + 2][e];
        }
#pragma unroll
      for (int rr = 0; rr < 2; ++rr)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          wvx[2 * M + rr][e] = do_v ? vvn[0][rr][e] : 0.0f;
          wvz[2 * M + rr][e] = do_v ? vvn[1][rr][e] : 0.0f;
        }
      // s'' rows q-1 (rr = 0) and q (rr = 1); s' rows q-2 .. q+1 are in spp / spc
      if (do_o) {
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
          const int qs = q - 1 + rr;
          if (qs < za || qs >= zb || xc >= gm.nx) continue;
          float v[3][2];
#pragma unroll
          for (int e = 0; e < 2; ++e) {
#pragma unroll
            for (int f = 0; f < 3; ++f) v[f][e] = rr ? spc[f][0][e] : spp[f][1][e];
            int sx, sz, dist;
            if (!frame2(g2, xc + e, qs, sx, sz, dist)) continue;
            const int col = sc + e;
            const int coln = min(max(col + sx, 0), W - 1);
            const int srow = (2 * i - 1 + rr) & 3;  // s' ring row of qs
            const bool up = sz > 0;
            // old stress rows: q-2, q-1 in the previous pair slot, q, q+1 in this one
            const int oso = rr ? os : osp, oro = rr ? 0 : 1;  // row qs
            const int osz = up ? os : osp, orz = rr;         // row qs + sz
            const float w = wsm(2, dist);
#pragma unroll
            for (int f = 0; f < 3; ++f) {
              const float* fo = s_o + ((oso * 3 + f) * 2 + oro) * W + TN;
              const float* fzo = s_o + ((osz * 3 + f) * 2 + orz) * W + TN;
              const float fop = fo[col];
              const float sz_n = rr ? (up ? spc[f][1][e] : spp[f][1][e]) : (up ? spc[f][0][e] : spp[f][0][e]);
              const float sx_n = s_sp[(4 * f + srow) * W + coln];
              if (sx != 0 && sz != 0)
                v[f][e] = higdon_corner(w, v[f][e], higdon_side(h, sx_n, fop, fo[coln]),
                                        higdon_side(h, sz_n, fop, fzo[col]));
              else if (sx != 0)
                v[f][e] = higdon_edge(w, v[f][e], higdon_side(h, sx_n, fop, fo[coln]));
              else
                v[f][e] = higdon_edge(w, v[f][e], higdon_side(h, sz_n, fop, fzo[col]));
            }
          }
          const long long p = so + (long long)qs * gm.ld + xc;
          float* out[3] = {o.txx, o.tzz, o.txz};
#pragma unroll
          for (int f = 0; f < 3; ++f) {
            if (xc + 1 < gm.nx)
              *reinterpret_cast<float2*>(out[f] + p) = make_float2(v[f][0], v[f][1]);
            else
              out[f][p] = v[f][0];
          }
        }
      }
#pragma unroll
      for (int f = 0; f < 2; ++f)
#pragma unroll
        for (int k = 0; k < 4; ++k) vpp[f][k >> 1][k & 1] = do_v ? vpc[f][k >> 1][k & 1] : 0.0f;
#pragma unroll
      for (int f = 0; f < 3; ++f)
#pragma unroll
        for (int k = 0; k < 4; ++k) spp[f][k >> 1][k & 1] = do_s ? spc[f][k >> 1][k & 1] : 0.0f;
      load_mat(zv + 2);
      __syncthreads();
      if (tid == 0 && live && i + 1 + P < I) {
        fence_proxy_async();
        issue(i + 1 + P);
      }
    }
    gb += I;
  }
}

// ===========================================================================
// Lean register-window sweep (the "rl" variants).
//
// The same two-stage march as k_el_sweep_rw (2x2 cells per thread, both
// z-derivative windows in registers, three TMA stress streams, same canonical
// arithmetic, bit-identical results), with the per-cell bookkeeping moved out
// of the inner loop:
//   - the HABC frame and interior tests split into per-column constants of the
//     thread (computed once per segment) and per-row values that are the same
//     for the whole CTA (computed once per row);
//   - materials come from a padded, column-pair-interleaved pack (six vector
//     loads per row pair, no bounds tests, pointers advanced by two rows);
//   - ring slots advance by counters instead of divisions;
//   - NT threads (64 or 128; 256 / NT CTAs per SM keep two warps on each
//     scheduler) and a TMA row of W = 2 (NT + TN) floats (at most 256), so
//     narrower CTAs can cover a grid with fewer idle lanes.
// ===========================================================================
// TMA row width: 2 (NT + TN) rounded up to 16 floats (every ring row pair
// then starts on a 128-byte boundary), at most 256 (the TMA box limit).
__host__ __device__ constexpr int rl_w(int N, int NT) {
  return ((2 * (NT + x2_tn(N)) + 15) & ~15) < 256 ? ((2 * (NT + x2_tn(N)) + 15) & ~15) : 256;
}
__host__ __device__ constexpr int rl_txmax(int N, int NT) {
  // v' columns [0, TX + 2HV) on the threads; tau columns [-TN, W - TN) cover them +- N
  return ((2 * NT - 2 * x2_hv(N)) < (rl_w(N, NT) - x2_tn(N) - N - 2 * x2_hv(N))
              ? (2 * NT - 2 * x2_hv(N))
              : (rl_w(N, NT) - x2_tn(N) - N - 2 * x2_hv(N))) &
         ~3;
}

// binary16 form: 8-column halos so that every TMA x coordinate of a binary16
// row is a multiple of 8 elements (16 bytes)
__host__ __device__ constexpr int rl_w16(int NT) {
  return ((2 * (NT + 8) + 15) & ~15) < 256 ? ((2 * (NT + 8) + 15) & ~15) : 256;
}
__host__ __device__ constexpr int rl_txmax16(int N, int NT) {
  return ((2 * NT - 16) < (rl_w16(NT) - 8 - N - 16) ? (2 * NT - 16) : (rl_w16(NT) - 8 - N - 16)) &
         ~7;
}

template <int N, int NT, int P, int LV = (N + 2 <= 4 ? 4 : 8), bool H16 = false>
struct RLShape {
  static constexpr int W = H16 ? rl_w16(NT) : rl_w(N, NT);
  static constexpr int TN = H16 ? 8 : x2_tn(N), HV = H16 ? 8 : x2_hv(N);
  static constexpr int NZ = P + 1;                 // z / x stream slots
  static constexpr int NO = P + 2;                 // old-stress / A.v stream slots (and barriers)
  static constexpr int LVV = LV;                   // v'' ring rows (a power of two >= N + 2)
  static constexpr int O_Z = 0;                    // [NZ][txz, tzz][2][W]   rows zv+M, +1
  static constexpr int O_X = O_Z + NZ * 4 * W;     // [NZ][txx, txz][2][W]   rows zv, zv+1
  static constexpr int O_O = O_X + NZ * 4 * W;     // [NO][txx, tzz, txz][2][W] rows q, q+1
  static constexpr int O_V = O_O + NO * 6 * W;     // [NO][vx, vz][2][W]     rows zv, zv+1
  static constexpr int O_VP = O_V + NO * 4 * W;    // [vx, vz][4][W]  v'
  static constexpr int O_VV = O_VP + 8 * W;        // [vx, vz][LVV][W] v''
  static constexpr int O_SP = O_VV + 2 * LVV * W;  // [xx, zz, xz][4][W] s'
  // binary16 staging boxes (2 rows of W halves, each box on a 128-byte boundary):
  // z [NZ][txz, tzz], x [NZ][txx, txz], o [NO][txx, tzz, txz], v [NO][vx, vz]
  static constexpr int NB16 = H16 ? 4 * NZ + 5 * NO : 0;
  static constexpr int HB = ((4 * W + 127) & ~127) / 4;  // floats per staging box
  static constexpr int O_H = O_SP + 12 * W;
  static constexpr int O_WT = O_H + NB16 * HB;     // [3][wstride] weights
};

template <int N, int NT, int P>
__global__ void __launch_bounds__(NT, 256 / NT)
    k_el_sweep_rl(const __grid_constant__ CUtensorMap tm_xx, const __grid_constant__ CUtensorMap tm_zz,
                  const __grid_constant__ CUtensorMap tm_xz, const __grid_constant__ CUtensorMap tm_vx,
                  const __grid_constant__ CUtensorMap tm_vz, SweepGeom gm, Coef c, float dtx,
                  float dtz, HabcDev h, MatPack mp, ElOut o, const long long* __restrict__ bounds,
                  int* __restrict__ err) {
  using S = RLShape<N, NT, P>;
  constexpr int W = S::W, M = N, TN = S::TN, HV = S::HV;
  constexpr int NZ = S::NZ, NO = S::NO, LVV = S::LVV;
  constexpr int WN = 2 * M + 2;  // window rows
  extern __shared__ __align__(128) float sm[];
  float* s_z = sm + S::O_Z;
  float* s_x = sm + S::O_X;
  float* s_o = sm + S::O_O;
  float* s_v = sm + S::O_V;
  float* s_vp = sm + S::O_VP;
  float* s_vv = sm + S::O_VV;
  float* s_sp = sm + S::O_SP;
  float* s_wt = sm + S::O_WT;
  const int nwt = (3 * h.wstride + 31) & ~31;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + S::O_WT + nwt);  // [NO]

  const int tid = threadIdx.x, sc = 2 * tid;
  const int TX = gm.TX, WV = TX + 2 * HV;
  const int nx = gm.nx, nz = gm.nz, nbc = gm.nbc;
  for (int k = tid; k < S::O_WT; k += NT) sm[k] = 0.0f;
  for (int k = tid; k < 3 * h.wstride; k += NT) s_wt[k] = __ldg(h.wtab + k);
  if (tid == 0) {
    for (int k = 0; k < NO; ++k) mbar_init(&bars[k], 1);
    tma::mbar_init_fence();
  }
  __syncthreads();
  auto wsm = [&](int kind, int dist) {
    return dist < h.wstride ? s_wt[kind * h.wstride + dist] : 1.0f;
  };
  // Row classification (kernels_fused.jl:28-52, interior of fused_kernels.jl:48):
  // frame rows 1..nz-2; Higdon side +1 (top band) / -1 (bottom band) / 0.
  auto zside = [&](int z) { return z <= nbc ? 1 : (z >= nz - 1 - nbc ? -1 : 0); };
  auto zframe = [&](int z) { return z >= 1 && z <= nz - 2; };
  auto zinner = [&](int z) { return z >= M && z < nz - M; };
  auto zdist = [&](int z) { return min(z, nz - 1 - z); };
  const bool do_v = sc < WV;
  const bool do_s = sc >= HV - 2 && sc < HV + TX + 2;
  const bool do_o = sc >= HV && sc < HV + TX;
  const long long mrow = 2LL * mp.pitch;  // pack step per iteration (two rows)

  const long long r_lo = bounds[blockIdx.x];
  const long long r_hi = bounds[blockIdx.x + 1];
  int gb = 0;  // batches this CTA has consumed (ring slot / barrier phase base)
  bool live = true;
  for (long long r = r_lo; r < r_hi;) {
    const long long item = r / nz;
    const int za = (int)(r - item * nz);
    const int zb = (int)min((long long)nz, za + (r_hi - r));
    r += zb - za;
    const int strip = (int)(item % gm.nstrip);
    const int shot = (int)(item / gm.nstrip);
    const int X0 = strip * TX, XV = X0 - HV, XT = XV - TN;
    const int xc = XV + sc;
    // per-column constants of this thread's two cells
    bool xin[2], xfr[2];
    int xsd[2], xds[2], xcn[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int x = xc + e;
      xin[e] = x >= M && x < nx - M;
      xsd[e] = x <= nbc ? 1 : (x >= nx - 1 - nbc ? -1 : 0);
      xfr[e] = x >= 1 && x <= nx - 2;
      xds[e] = min(x, nx - 1 - x);
      xcn[e] = min(max(sc + e + xsd[e], 0), W - 1);
    }
    // a cell of this thread lies in a left/right Higdon band on every frame row
    const bool xband = (xfr[0] && xsd[0] != 0) || (xfr[1] && xsd[1] != 0);
    const bool o_any = do_o && xc < nx, o_pair = xc + 1 < nx;
    float* const ob[5] = {o.vx, o.vz, o.txx, o.tzz, o.txz};
    const long long obase = (long long)shot * gm.plane + xc;
    // M warm-up iterations fill the txz/tzz window before the first needed v' row
    const int zv0 = za - 2 - 3 * M;
    const int I = (zb - za + 4 + 4 * M + 1) / 2 + 1;
    auto issue = [&](int k) {
      const int gk = gb + k, zs = gk % NZ, os = gk % NO;
      uint64_t* bar = &bars[os];
      mbar_expect_tx(bar, 9u * 2u * W * 4u);
      const int zr = zv0 + 2 * k;
      tma_load_3d(s_z + (zs * 4 + 0) * W, &tm_xz, XT, zr + M, shot, bar);
      tma_load_3d(s_z + (zs * 4 + 2) * W, &tm_zz, XT, zr + M, shot, bar);
      tma_load_3d(s_x + (zs * 4 + 0) * W, &tm_xx, XT, zr, shot, bar);
      tma_load_3d(s_x + (zs * 4 + 2) * W, &tm_xz, XT, zr, shot, bar);
      tma_load_3d(s_o + (os * 6 + 0) * W, &tm_xx, XT, zr - 3 - M, shot, bar);
      tma_load_3d(s_o + (os * 6 + 2) * W, &tm_zz, XT, zr - 3 - M, shot, bar);
      tma_load_3d(s_o + (os * 6 + 4) * W, &tm_xz, XT, zr - 3 - M, shot, bar);
      tma_load_3d(s_v + (os * 4 + 0) * W, &tm_vx, XV, zr, shot, bar);
      tma_load_3d(s_v + (os * 4 + 2) * W, &tm_vz, XV, zr, shot, bar);
    };
    __syncthreads();  // the previous segment's readers are done with every ring
    if (tid == 0 && live) {
      fence_proxy_async();
      for (int k = 0; k <= P && k < I; ++k) issue(k);
    }
    // register state
    float wxz[WN][2], wzz[WN][2], wvx[WN][2], wvz[WN][2];
#pragma unroll
    for (int k = 0; k < WN; ++k)
#pragma unroll
      for (int e = 0; e < 2; ++e) wxz[k][e] = wzz[k][e] = wvx[k][e] = wvz[k][e] = 0.0f;
    float vpp[2][2][2], spp[3][2][2];  // previous iteration's v' / s' rows [field][row][cell]
#pragma unroll
    for (int f = 0; f < 2; ++f)
#pragma unroll
      for (int k = 0; k < 4; ++k) vpp[f][k >> 1][k & 1] = 0.0f;
#pragma unroll
    for (int f = 0; f < 3; ++f)
#pragma unroll
      for (int k = 0; k < 4; ++k) spp[f][k >> 1][k & 1] = 0.0f;
    // materials of iteration i (rows zv, zv+1 for v'; q, q+1 for s'), loaded during i-1
    const long long pcol = (xc >> 1) + kPackColPad / 2;
    const float4* pv = mp.v + (long long)(zv0 + kPackRowPad) * mp.pitch + pcol;
    const float4* pl = mp.l + (long long)(zv0 - 3 - M + kPackRowPad) * mp.pitch + pcol;
    const float2* pu = mp.mu + (long long)(zv0 - 3 - M + kPackRowPad) * mp.pitch + pcol;
    float4 mv[2], ml[2];
    float2 mu[2];
    auto load_mat = [&]() {
#pragma unroll
      for (int rr = 0; rr < 2; ++rr) {
        mv[rr] = __ldg(pv + rr * mp.pitch);
        ml[rr] = __ldg(pl + rr * mp.pitch);
        mu[rr] = __ldg(pu + rr * mp.pitch);
      }
      pv += mrow;
      pl += mrow;
      pu += mrow;
    };
    load_mat();
    // ring slots of iteration i: zs = (gb+i) % NZ, os = (gb+i) % NO, osp = (gb+i-1) % NO
    int zs = gb % NZ, os = gb % NO, osp = (gb + NO - 1) % NO;
    uint32_t ph = (uint32_t)((gb / NO) & 1);

    for (int i = 0; i < I; ++i) {
      const int zv = zv0 + 2 * i, q = zv - 3 - M;
      if (live) live = mbar_wait_bounded(&bars[os], ph, err) && live;
      const float bxv[2][2] = {{mv[0].x, mv[0].y}, {mv[1].x, mv[1].y}};
      const float bzv[2][2] = {{mv[0].z, mv[0].w}, {mv[1].z, mv[1].w}};
      const float lav[2][2] = {{ml[0].x, ml[0].y}, {ml[1].x, ml[1].y}};
      const float l2v[2][2] = {{ml[0].z, ml[0].w}, {ml[1].z, ml[1].w}};
      const float muv[2][2] = {{mu[0].x, mu[0].y}, {mu[1].x, mu[1].y}};
      // ---------------- stage A ----------------
      // new window rows zv+M, zv+M+1 of txz and tzz
#pragma unroll
      for (int rr = 0; rr < 2; ++rr) {
        const float2 a = *reinterpret_cast<const float2*>(s_z + (zs * 4 + rr) * W + sc + TN);
        const float2 b = *reinterpret_cast<const float2*>(s_z + (zs * 4 + 2 + rr) * W + sc + TN);
        wxz[2 * M + rr][0] = a.x;
        wxz[2 * M + rr][1] = a.y;
        wzz[2 * M + rr][0] = b.x;
        wzz[2 * M + rr][1] = b.y;
      }
      float vpc[2][2][2];  // v' rows zv, zv+1 [field][row][cell]
      if (do_v) {
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
          const bool zin = zinner(zv + rr);
          float xw[4 * ((N + 1) / 2) + 2];
          float dxx[2], dxzx[2];
          load_xwin<N>(s_x + (zs * 4 + rr) * W, sc + TN, xw);
          dxx[0] = xdm<N>(xw, 0, c);
          dxx[1] = xdm<N>(xw, 1, c);
          load_xwin<N>(s_x + (zs * 4 + 2 + rr) * W, sc + TN, xw);
          dxzx[0] = xdp<N>(xw, 0, c);
          dxzx[1] = xdp<N>(xw, 1, c);
          const float2 ox = *reinterpret_cast<const float2*>(s_v + (os * 4 + rr) * W + sc);
          const float2 oz = *reinterpret_cast<const float2*>(s_v + (os * 4 + 2 + rr) * W + sc);
          const float vo[2][2] = {{ox.x, ox.y}, {oz.x, oz.y}};
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            float dxzz = 0.0f, dzz = 0.0f;
#pragma unroll
            for (int l = 1; l <= N; ++l) {
              dxzz = __fmaf_rn(c.a[l - 1], __fsub_rn(wxz[rr + M + l - 1][e], wxz[rr + M - l][e]), dxzz);
              dzz = __fmaf_rn(c.a[l - 1], __fsub_rn(wzz[rr + M + l][e], wzz[rr + M - l + 1][e]), dzz);
            }
            float ux = vo[0][e], uz = vo[1][e];
            if (zin && xin[e]) {
              ux = __fmaf_rn(bxv[rr][e], __fmaf_rn(dtx, dxx[e], __fmul_rn(dtz, dxzz)), ux);
              uz = __fmaf_rn(bzv[rr][e], __fmaf_rn(dtx, dxzx[e], __fmul_rn(dtz, dzz)), uz);
            }
            vpc[0][rr][e] = ux;
            vpc[1][rr][e] = uz;
          }
          const int pr = (2 * i + rr) & 3;  // v' ring row of zv + rr
          *reinterpret_cast<float2*>(s_vp + pr * W + sc) = make_float2(vpc[0][rr][0], vpc[0][rr][1]);
          *reinterpret_cast<float2*>(s_vp + (4 + pr) * W + sc) =
              make_float2(vpc[1][rr][0], vpc[1][rr][1]);
        }
      }
      // shift the txz / tzz window by two rows for the next iteration
#pragma unroll
      for (int k = 0; k < 2 * M; ++k)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          wxz[k][e] = wxz[k + 2][e];
          wzz[k][e] = wzz[k + 2][e];
        }
      float spc[3][2][2];  // s' rows q, q+1 [field][row][cell]
      if (do_s) {
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
          const bool zin = zinner(q + rr);
          const int vb = (2 * i - 2 - M + rr) & (LVV - 1);  // v'' ring row of q + rr
          float xw[4 * ((N + 1) / 2) + 2];
          float dvxdx[2], dvzdx[2];
          load_xwin<N>(s_vv + vb * W, sc, xw);
          dvxdx[0] = xdp<N>(xw, 0, c);
          dvxdx[1] = xdp<N>(xw, 1, c);
          load_xwin<N>(s_vv + (LVV + vb) * W, sc, xw);
          dvzdx[0] = xdm<N>(xw, 0, c);
          dvzdx[1] = xdm<N>(xw, 1, c);
          const float2 oxx = *reinterpret_cast<const float2*>(s_o + (os * 6 + 0 + rr) * W + sc + TN);
          const float2 ozz = *reinterpret_cast<const float2*>(s_o + (os * 6 + 2 + rr) * W + sc + TN);
          const float2 oxz = *reinterpret_cast<const float2*>(s_o + (os * 6 + 4 + rr) * W + sc + TN);
          const float so_[3][2] = {{oxx.x, oxx.y}, {ozz.x, ozz.y}, {oxz.x, oxz.y}};
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            float dvxdz = 0.0f, dvzdz = 0.0f;
#pragma unroll
            for (int l = 1; l <= N; ++l) {
              dvxdz = __fmaf_rn(c.a[l - 1], __fsub_rn(wvx[rr + M + l][e], wvx[rr + M - l + 1][e]), dvxdz);
              dvzdz = __fmaf_rn(c.a[l - 1], __fsub_rn(wvz[rr + M + l - 1][e], wvz[rr + M - l][e]), dvzdz);
            }
            float sxx = so_[0][e], szz = so_[1][e], sxz = so_[2][e];
            if (zin && xin[e]) {
              const float ex = __fmul_rn(dvxdx[e], dtx), ez = __fmul_rn(dvzdz, dtz);
              sxx = __fadd_rn(sxx, __fmaf_rn(l2v[rr][e], ex, __fmul_rn(lav[rr][e], ez)));
              szz = __fadd_rn(szz, __fmaf_rn(lav[rr][e], ex, __fmul_rn(l2v[rr][e], ez)));
              sxz = __fmaf_rn(muv[rr][e], __fmaf_rn(dvxdz, dtz, __fmul_rn(dvzdx[e], dtx)), sxz);
            }
            spc[0][rr][e] = sxx;
            spc[1][rr][e] = szz;
            spc[2][rr][e] = sxz;
          }
          const int sr = (2 * i + rr) & 3;  // s' ring row of q + rr
#pragma unroll
          for (int f = 0; f < 3; ++f)
            *reinterpret_cast<float2*>(s_sp + (4 * f + sr) * W + sc) =
                make_float2(spc[f][rr][0], spc[f][rr][1]);
        }
      }
      __syncthreads();

      // ---------------- stage B ----------------
      // v'' rows zv-1 (rr = 0) and zv (rr = 1); v' rows zv-2 .. zv+1 are in vpp / vpc
      float vvn[2][2][2];
      if (do_v) {
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
          const int qv = zv - 1 + rr;
#pragma unroll
          for (int f = 0; f < 2; ++f)
#pragma unroll
            for (int e = 0; e < 2; ++e) vvn[f][rr][e] = rr ? vpc[f][0][e] : vpp[f][1][e];
          const int zsd = zside(qv);
          if (zframe(qv) && (zsd != 0 || xband)) {
            const int zd = zdist(qv);
            const int prow = (2 * i - 1 + rr) & 3;  // v' ring row of qv
            // A.v rows zv-2, zv-1 sit in the previous pair's slot, zv, zv+1 in this one
            const int orow = rr ? 0 : 1;
            const int oslot = rr ? os : osp;
            const int zslot = zsd > 0 ? os : osp;  // slot of row qv + zsd (row index rr)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              if (!xfr[e] || (xsd[e] == 0 && zsd == 0)) continue;
              const int col = sc + e, coln = xcn[e];
              const int dist = min(xds[e], zd);
#pragma unroll
              for (int f = 0; f < 2; ++f) {
                const float* fo = s_v + (oslot * 4 + 2 * f + orow) * W;
                const float fop = fo[col];
                const float w = wsm(f, dist);
                const float vz_n = rr ? (zsd > 0 ? vpc[f][1][e] : vpp[f][1][e])
                                      : (zsd > 0 ? vpc[f][0][e] : vpp[f][0][e]);
                if (xsd[e] != 0 && zsd != 0)
                  vvn[f][rr][e] = higdon_corner(
                      w, vvn[f][rr][e],
                      higdon_side(h, s_vp[(4 * f + prow) * W + coln], fop, fo[coln]),
                      higdon_side(h, vz_n, fop, s_v[(zslot * 4 + 2 * f + rr) * W + col]));
                else if (xsd[e] != 0)
                  vvn[f][rr][e] = higdon_edge(
                      w, vvn[f][rr][e],
                      higdon_side(h, s_vp[(4 * f + prow) * W + coln], fop, fo[coln]));
                else
                  vvn[f][rr][e] = higdon_edge(
                      w, vvn[f][rr][e],
                      higdon_side(h, vz_n, fop, s_v[(zslot * 4 + 2 * f + rr) * W + col]));
              }
            }
          }
          const int vw = (2 * i + rr) & (LVV - 1);  // v'' ring row of qv
          *reinterpret_cast<float2*>(s_vv + vw * W + sc) = make_float2(vvn[0][rr][0], vvn[0][rr][1]);
          *reinterpret_cast<float2*>(s_vv + (LVV + vw) * W + sc) =
              make_float2(vvn[1][rr][0], vvn[1][rr][1]);
          if (o_any && qv >= za && qv < zb) {
            const long long p = obase + (long long)qv * gm.ld;
            if (o_pair) {
              *reinterpret_cast<float2*>(ob[0] + p) = make_float2(vvn[0][rr][0], vvn[0][rr][1]);
              *reinterpret_cast<float2*>(ob[1] + p) = make_float2(vvn[1][rr][0], vvn[1][rr][1]);
            } else {
              ob[0][p] = vvn[0][rr][0];
              ob[1][p] = vvn[1][rr][0];
            }
          }
        }
      }
      // the v'' window advances: rows q-M+2 .. q+M+1, then the new rows zv-1, zv
#pragma unroll
      for (int k = 0; k < 2 * M; ++k)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          wvx[k][e] = wvx[k + 2][e];
          wvz[k][e] = wvz[k + 2][e];
        }
#pragma unroll
      for (int rr = 0; rr < 2; ++rr)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          wvx[2 * M + rr][e] = vvn[0][rr][e];
          wvz[2 * M + rr][e] = vvn[1][rr][e];
        }
      // s'' rows q-1 (rr = 0) and q (rr = 1); s' rows q-2 .. q+1 are in spp / spc
      if (o_any) {
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
          const int qs = q - 1 + rr;
          if (qs < za || qs >= zb) continue;
          float v[3][2];
#pragma unroll
          for (int f = 0; f < 3; ++f)
#pragma unroll
            for (int e = 0; e < 2; ++e) v[f][e] = rr ? spc[f][0][e] : spp[f][1][e];
          const int zsd = zside(qs);
          if (zframe(qs) && (zsd != 0 || xband)) {
            const int zd = zdist(qs);
            const int srow = (2 * i - 1 + rr) & 3;  // s' ring row of qs
            // old stress rows: q-2, q-1 in the previous pair slot, q, q+1 in this one
            const int oso = rr ? os : osp, oro = rr ? 0 : 1;  // row qs
            const int osz = zsd > 0 ? os : osp;              // row qs + zsd (row index rr)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              if (!xfr[e] || (xsd[e] == 0 && zsd == 0)) continue;
              const int col = sc + e, coln = xcn[e];
              const float w = wsm(2, min(xds[e], zd));
#pragma unroll
              for (int f = 0; f < 3; ++f) {
                const float* fo = s_o + (oso * 6 + 2 * f + oro) * W + TN;
                const float fop = fo[col];
                const float sz_n = rr ? (zsd > 0 ? spc[f][1][e] : spp[f][1][e])
                                      : (zsd > 0 ? spc[f][0][e] : spp[f][0][e]);
                if (xsd[e] != 0 && zsd != 0)
                  v[f][e] = higdon_corner(
                      w, v[f][e], higdon_side(h, s_sp[(4 * f + srow) * W + coln], fop, fo[coln]),
                      higdon_side(h, sz_n, fop, s_o[(osz * 6 + 2 * f + rr) * W + TN + col]));
                else if (xsd[e] != 0)
                  v[f][e] = higdon_edge(
                      w, v[f][e], higdon_side(h, s_sp[(4 * f + srow) * W + coln], fop, fo[coln]));
                else
                  v[f][e] = higdon_edge(
                      w, v[f][e],
                      higdon_side(h, sz_n, fop, s_o[(osz * 6 + 2 * f + rr) * W + TN + col]));
              }
            }
          }
          const long long p = obase + (long long)qs * gm.ld;
#pragma unroll
          for (int f = 0; f < 3; ++f) {
            if (o_pair)
              *reinterpret_cast<float2*>(ob[2 + f] + p) = make_float2(v[f][0], v[f][1]);
            else
              ob[2 + f][p] = v[f][0];
          }
        }
      }
#pragma unroll
      for (int f = 0; f < 2; ++f)
#pragma unroll
        for (int k = 0; k < 4; ++k) vpp[f][k >> 1][k & 1] = vpc[f][k >> 1][k & 1];
#pragma unroll
      for (int f = 0; f < 3; ++f)
#pragma unroll
        for (int k = 0; k < 4; ++k) spp[f][k >> 1][k & 1] = spc[f][k >> 1][k & 1];
      load_mat();
      __syncthreads();
      if (tid == 0 && live && i + 1 + P < I) {
        fence_proxy_async();
        issue(i + 1 + P);
      }
      zs = zs + 1 == NZ ? 0 : zs + 1;
      osp = os;
      os = os + 1 == NO ? 0 : os + 1;
      ph ^= os == 0 ? 1u : 0u;
    }
    gb += I;
  }
}

// ===========================================================================
// Warp-specialized register-window sweep (the "ws" variants).
//
// The lean sweep's work split by role: NV "velocity" threads hold the txz/tzz
// z-windows and produce v', v'' (HABC, B.v); NV "stress" threads hold the
// v''x/v''z z-windows and produce s', s'' (HABC, B.stress).  Each role runs
// its own loop, so a thread keeps only its role's state (about half the
// registers of k_el_sweep_rl) and more warps fit on an SM to hide the latency
// of the dependent FMA chains.  The roles meet at a named CTA barrier twice per
// row pair, in the same sequence in both loops; the v'' rows a stress thread
// needs in its window come from the shared v'' ring, written one iteration
// earlier by the velocity threads of the same columns.  Same canonical
// arithmetic, bit-identical results.
// ===========================================================================
__device__ __forceinline__ void cta_bar(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
// v'' ring depth of the warp-specialized sweep.  With SPLIT the ring is deep
// enough (>= N + 4 rows) that the rows the stress role reads in stage A never
// share a slot with the rows the velocity role writes in stage B of the same
// iteration, so the mid-iteration barrier only has to order each role with
// itself.
__host__ __device__ constexpr int ws_lvv(int N, bool split) {
  return split ? (N + 4 <= 8 ? 8 : 16) : (N + 2 <= 4 ? 4 : 8);
}

template <int N, int NV, int P, int MINB, bool SPLIT, bool H16>
__global__ void __launch_bounds__(2 * NV, MINB)
    k_el_sweep_ws(const __grid_constant__ CUtensorMap tm_xx, const __grid_constant__ CUtensorMap tm_zz,
                  const __grid_constant__ CUtensorMap tm_xz, const __grid_constant__ CUtensorMap tm_vx,
                  const __grid_constant__ CUtensorMap tm_vz, const __grid_constant__ CUtensorMap th_xx,
                  const __grid_constant__ CUtensorMap th_zz, const __grid_constant__ CUtensorMap th_xz,
                  const __grid_constant__ CUtensorMap th_vx, const __grid_constant__ CUtensorMap th_vz,
                  SweepGeom gm, Coef c, float dtx, float dtz, HabcDev h, MatPack mp, ElOut o,
                  ElOut16 o16, const long long* __restrict__ bounds, int* __restrict__ err) {
  static_assert(NV % 32 == 0, "each role is whole warps: named barriers count whole warps");
  // H16: binary16 storage outside the kFp16Band-wide FP32 band (th_* map the
  // binary16 arrays, o16 receives them); TMA brings the binary16 rows into
  // staging boxes (and the FP32 rows where the band reaches), each role widens
  // the rows it reads into the FP32 rings, and stored values are rounded to
  // binary16 outside the band -- the velocities the stress role reads included,
  // as they would be read back from storage.
  using S = RLShape<N, NV, P, ws_lvv(N, SPLIT), H16>;
  static_assert(!H16 || (S::TN % 8 == 0 && S::HV % 8 == 0), "binary16 TMA x must be 8-aligned");
  constexpr int NT = 2 * NV;
  // mid-iteration barrier: per role (ids 2, 3) when SPLIT, else the whole CTA (id 1)
  const int mid_id = SPLIT ? (threadIdx.x < NV ? 2 : 3) : 1;
  constexpr int mid_n = SPLIT ? NV : NT;
  constexpr int W = S::W, M = N, TN = S::TN, HV = S::HV;
  constexpr int NZ = S::NZ, NO = S::NO, LVV = S::LVV;
  constexpr int WN = 2 * M + 2;  // window rows
  extern __shared__ __align__(128) float sm[];
  float* s_z = sm + S::O_Z;
  float* s_x = sm + S::O_X;
  float* s_o = sm + S::O_O;
  float* s_v = sm + S::O_V;
  float* s_vp = sm + S::O_VP;
  float* s_vv = sm + S::O_VV;
  float* s_sp = sm + S::O_SP;
  float* s_wt = sm + S::O_WT;
  const int nwt = (3 * h.wstride + 31) & ~31;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + S::O_WT + nwt);  // [NO]
  float* s_h = sm + S::O_H;  // binary16 staging boxes
  auto hbox = [&](int b) { return s_h + b * S::HB; };

  const int tid = threadIdx.x;
  const bool vel = tid < NV;  // warp-uniform role
  const int sc = 2 * (vel ? tid : tid - NV);
  const int TX = gm.TX, WV = TX + 2 * HV;
  const int nx = gm.nx, nz = gm.nz, nbc = gm.nbc;
  for (int k = tid; k < S::O_WT; k += NT) sm[k] = 0.0f;
  for (int k = tid; k < 3 * h.wstride; k += NT) s_wt[k] = __ldg(h.wtab + k);
  if (tid == 0) {
    for (int k = 0; k < NO; ++k) mbar_init(&bars[k], 1);
    tma::mbar_init_fence();
  }
  __syncthreads();
  auto wsm = [&](int kind, int dist) {
    return dist < h.wstride ? s_wt[kind * h.wstride + dist] : 1.0f;
  };
  // Row classification (kernels_fused.jl:28-52, interior of fused_kernels.jl:48)
  auto zside = [&](int z) { return z <= nbc ? 1 : (z >= nz - 1 - nbc ? -1 : 0); };
  auto zframe = [&](int z) { return z >= 1 && z <= nz - 2; };
  auto zinner = [&](int z) { return z >= M && z < nz - M; };
  auto zdist = [&](int z) { return min(z, nz - 1 - z); };
  // FP32 band of the binary16 storage: rows (and columns) within kFp16Band of
  // the edge; rows outside the grid count as band (TMA fills them with zeros)
  auto zband16 = [&](int z) { return z < kFp16Band || z >= nz - kFp16Band; };
  auto xband16 = [&](int x) { return x < kFp16Band || x >= nx - kFp16Band; };
  // Widens binary16 rows y0, y0+1 of a staging box into the FP32 rows at dst
  // (columns x0 + c) outside the band; every thread of the role takes column
  // pairs c = 2t, 2t + 2 NV, ...
  auto widen = [&](float* dst, const float* box, int x0, int y0) {
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
      if (zband16(y0 + rr)) continue;
      const __half* src = reinterpret_cast<const __half*>(box) + rr * W;
      float* d = dst + rr * W;
#pragma unroll
      for (int c0 = 0; c0 < W; c0 += 2 * NV) {
        const int cc = c0 + sc;
        if (cc < W) {
          const float2 v = __half22float2(*reinterpret_cast<const __half2*>(src + cc));
          const bool b0 = xband16(x0 + cc), b1 = xband16(x0 + cc + 1);
          if (!b0 && !b1) *reinterpret_cast<float2*>(d + cc) = v;
          else {
            if (!b0) d[cc] = v.x;
            if (!b1) d[cc + 1] = v.y;
          }
        }
      }
    }
  };
  // the value as stored: rounded to binary16 outside the band
  auto stored = [&](float v, bool band) {
    return (H16 && !band) ? __half2float(__float2half_rn(v)) : v;
  };
  const bool do_v = sc < WV;
  const bool do_s = sc >= HV - 2 && sc < HV + TX + 2;
  const bool do_o = sc >= HV && sc < HV + TX;
  const long long mrow = 2LL * mp.pitch;  // pack step per iteration (two rows)
  const long long r_lo = bounds[blockIdx.x];
  const long long r_hi = bounds[blockIdx.x + 1];

  // One segment = a run of rows [za, zb) of one (shot, strip); both roles walk
  // the same segments and iterations.
  struct Seg {
    int za, zb, shot, XV, XT, xc, zv0, I;
    bool xin[2], xfr[2], xband, o_any, o_pair;
    bool xedge[2];  // frame cell of a left/right band (on rows outside the z bands)
    int xsd[2], xds[2], xcn[2];
    long long obase;
  };
  auto segment = [&](long long& r, Seg& g) {
    const long long item = r / nz;
    g.za = (int)(r - item * nz);
    g.zb = (int)min((long long)nz, g.za + (r_hi - r));
    r += g.zb - g.za;
    const int strip = (int)(item % gm.nstrip);
    g.shot = (int)(item / gm.nstrip);
    g.XV = strip * TX - HV;
    g.XT = g.XV - TN;
    g.xc = g.XV + sc;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int x = g.xc + e;
      g.xin[e] = x >= M && x < nx - M;
      g.xsd[e] = x <= nbc ? 1 : (x >= nx - 1 - nbc ? -1 : 0);
      g.xfr[e] = x >= 1 && x <= nx - 2;
      g.xds[e] = min(x, nx - 1 - x);
      g.xcn[e] = min(max(sc + e + g.xsd[e], 0), W - 1);
    }
    g.xedge[0] = g.xfr[0] && g.xsd[0] != 0;
    g.xedge[1] = g.xfr[1] && g.xsd[1] != 0;
    g.xband = g.xedge[0] || g.xedge[1];
    g.o_any = do_o && g.xc < nx;
    g.o_pair = g.xc + 1 < nx;
    g.obase = (long long)g.shot * gm.plane + g.xc;
    g.zv0 = g.za - 2 - 3 * M;  // M warm-up iterations fill the windows
    g.I = (g.zb - g.za + 4 + 4 * M + 1) / 2 + 1;
  };

  if (vel) {
    // ======================= velocity role =======================
    int gb = 0;
    bool live = true;
    for (long long r = r_lo; r < r_hi;) {
      Seg g;
      segment(r, g);
      auto issue = [&](int k) {
        const int gk = gb + k, zs = gk % NZ, os = gk % NO;
        uint64_t* bar = &bars[os];
        const int zr = g.zv0 + 2 * k;
        if constexpr (!H16) {
          mbar_expect_tx(bar, 9u * 2u * W * 4u);
          tma_load_3d(s_z + (zs * 4 + 0) * W, &tm_xz, g.XT, zr + M, g.shot, bar);
          tma_load_3d(s_z + (zs * 4 + 2) * W, &tm_zz, g.XT, zr + M, g.shot, bar);
          tma_load_3d(s_x + (zs * 4 + 0) * W, &tm_xx, g.XT, zr, g.shot, bar);
          tma_load_3d(s_x + (zs * 4 + 2) * W, &tm_xz, g.XT, zr, g.shot, bar);
          tma_load_3d(s_o + (os * 6 + 0) * W, &tm_xx, g.XT, zr - 3 - M, g.shot, bar);
          tma_load_3d(s_o + (os * 6 + 2) * W, &tm_zz, g.XT, zr - 3 - M, g.shot, bar);
          tma_load_3d(s_o + (os * 6 + 4) * W, &tm_xz, g.XT, zr - 3 - M, g.shot, bar);
          tma_load_3d(s_v + (os * 4 + 0) * W, &tm_vx, g.XV, zr, g.shot, bar);
          tma_load_3d(s_v + (os * 4 + 2) * W, &tm_vz, g.XV, zr, g.shot, bar);
        } else {
          // per stream (z, x, o, v): binary16 rows unless both rows are band
          // rows; FP32 rows where a row or a column of the box is band
          const int ys[4] = {zr + M, zr, zr - 3 - M, zr};
          const bool xt = xband16(g.XT) || xband16(g.XT + W - 1);
          const bool xv = xband16(g.XV) || xband16(g.XV + W - 1);
          bool n16[4], n32[4];
          uint32_t bytes = 0;
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const bool b0 = zband16(ys[t]), b1 = zband16(ys[t] + 1);
            n16[t] = !(b0 && b1);
            n32[t] = (t == 3 ? xv : xt) || b0 || b1;
            const uint32_t nf = t == 2 ? 3u : 2u;
            bytes += nf * ((n16[t] ? 4u * W : 0u) + (n32[t] ? 8u * W : 0u));
          }
          mbar_expect_tx(bar, bytes);
          if (n32[0]) {
            tma_load_3d(s_z + (zs * 4 + 0) * W, &tm_xz, g.XT, ys[0], g.shot, bar);
            tma_load_3d(s_z + (zs * 4 + 2) * W, &tm_zz, g.XT, ys[0], g.shot, bar);
          }
          if (n16[0]) {
            tma_load_3d(hbox(zs * 2 + 0), &th_xz, g.XT, ys[0], g.shot, bar);
            tma_load_3d(hbox(zs * 2 + 1), &th_zz, g.XT, ys[0], g.shot, bar);
          }
          if (n32[1]) {
            tma_load_3d(s_x + (zs * 4 + 0) * W, &tm_xx, g.XT, ys[1], g.shot, bar);
            tma_load_3d(s_x + (zs * 4 + 2) * W, &tm_xz, g.XT, ys[1], g.shot, bar);
          }
          if (n16[1]) {
            tma_load_3d(hbox(2 * NZ + zs * 2 + 0), &th_xx, g.XT, ys[1], g.shot, bar);
            tma_load_3d(hbox(2 * NZ + zs * 2 + 1), &th_xz, g.XT, ys[1], g.shot, bar);
          }
          if (n32[2]) {
            tma_load_3d(s_o + (os * 6 + 0) * W, &tm_xx, g.XT, ys[2], g.shot, bar);
            tma_load_3d(s_o + (os * 6 + 2) * W, &tm_zz, g.XT, ys[2], g.shot, bar);
            tma_load_3d(s_o + (os * 6 + 4) * W, &tm_xz, g.XT, ys[2], g.shot, bar);
          }
          if (n16[2]) {
            tma_load_3d(hbox(4 * NZ + os * 3 + 0), &th_xx, g.XT, ys[2], g.shot, bar);
            tma_load_3d(hbox(4 * NZ + os * 3 + 1), &th_zz, g.XT, ys[2], g.shot, bar);
            tma_load_3d(hbox(4 * NZ + os * 3 + 2), &th_xz, g.XT, ys[2], g.shot, bar);
          }
          if (n32[3]) {
            tma_load_3d(s_v + (os * 4 + 0) * W, &tm_vx, g.XV, ys[3], g.shot, bar);
            tma_load_3d(s_v + (os * 4 + 2) * W, &tm_vz, g.XV, ys[3], g.shot, bar);
          }
          if (n16[3]) {
            tma_load_3d(hbox(4 * NZ + 3 * NO + os * 2 + 0), &th_vx, g.XV, ys[3], g.shot, bar);
            tma_load_3d(hbox(4 * NZ + 3 * NO + os * 2 + 1), &th_vz, g.XV, ys[3], g.shot, bar);
          }
        }
      };
      cta_bar(1, NT);  // the previous segment's readers are done with every ring
      if (tid == 0 && live) {
        fence_proxy_async();
        for (int k = 0; k <= P && k < g.I; ++k) issue(k);
      }
      float wxz[WN][2], wzz[WN][2];
#pragma unroll
      for (int k = 0; k < WN; ++k)
#pragma unroll
        for (int e = 0; e < 2; ++e) wxz[k][e] = wzz[k][e] = 0.0f;
      // HABC weights of the x-band cells on rows outside the z bands (dist = xds there)
      float wxb[2][2];
#pragma unroll
      for (int f = 0; f < 2; ++f)
#pragma unroll
        for (int e = 0; e < 2; ++e) wxb[f][e] = wsm(f, g.xds[e]);
      // output rows zv-1 (iteration 0) onwards, advanced two rows per iteration
      float* ovx = o.vx + g.obase + (long long)(g.zv0 - 1) * gm.ld;
      float* ovz = o.vz + g.obase + (long long)(g.zv0 - 1) * gm.ld;
      float vpp[2][2][2];  // previous iteration's v' rows [field][row][cell]
#pragma unroll
      for (int f = 0; f < 2; ++f)
#pragma unroll
        for (int k = 0; k < 4; ++k) vpp[f][k >> 1][k & 1] = 0.0f;
      const long long pcol = (g.xc >> 1) + kPackColPad / 2;
      const float4* pv = mp.v + (long long)(g.zv0 + kPackRowPad) * mp.pitch + pcol;
      float4 mv[2];
      mv[0] = __ldg(pv);
      mv[1] = __ldg(pv + mp.pitch);
      pv += mrow;
      int zs = gb % NZ, os = gb % NO, osp = (gb + NO - 1) % NO;
      uint32_t ph = (uint32_t)((gb / NO) & 1);
      for (int i = 0; i < g.I; ++i) {
        const int zv = g.zv0 + 2 * i;
        if (live) live = mbar_wait_bounded(&bars[os], ph, err) && live;
        if constexpr (H16) {
          widen(s_z + (zs * 4 + 0) * W, hbox(zs * 2 + 0), g.XT, zv + M);
          widen(s_z + (zs * 4 + 2) * W, hbox(zs * 2 + 1), g.XT, zv + M);
          widen(s_x + (zs * 4 + 0) * W, hbox(2 * NZ + zs * 2 + 0), g.XT, zv);
          widen(s_x + (zs * 4 + 2) * W, hbox(2 * NZ + zs * 2 + 1), g.XT, zv);
          widen(s_v + (os * 4 + 0) * W, hbox(4 * NZ + 3 * NO + os * 2 + 0), g.XV, zv);
          widen(s_v + (os * 4 + 2) * W, hbox(4 * NZ + 3 * NO + os * 2 + 1), g.XV, zv);
          cta_bar(4, NV);  // the role's widened rows are complete
        }
        const float bxv[2][2] = {{mv[0].x, mv[0].y}, {mv[1].x, mv[1].y}};
        const float bzv[2][2] = {{mv[0].z, mv[0].w}, {mv[1].z, mv[1].w}};
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
          const float2 a = *reinterpret_cast<const float2*>(s_z + (zs * 4 + rr) * W + sc + TN);
          const float2 b = *reinterpret_cast<const float2*>(s_z + (zs * 4 + 2 + rr) * W + sc + TN);
          wxz[2 * M + rr][0] = a.x;
          wxz[2 * M + rr][1] = a.y;
          wzz[2 * M + rr][0] = b.x;
          wzz[2 * M + rr][1] = b.y;
        }
        float vpc[2][2][2];  // v' rows zv, zv+1 [field][row][cell]
        if (do_v) {
#pragma unroll
          for (int rr = 0; rr < 2; ++rr) {
            const bool zin = zinner(zv + rr);
            constexpr int E = (N + 1) / 2;
            float xa[4 * E + 2], xb[4 * E + 2];  // txx and txz rows zv + rr around the pair
            load_xwin<N>(s_x + (zs * 4 + rr) * W, sc + TN, xa);
            load_xwin<N>(s_x + (zs * 4 + 2 + rr) * W, sc + TN, xb);
            const float2 ox = *reinterpret_cast<const float2*>(s_v + (os * 4 + rr) * W + sc);
            const float2 oz = *reinterpret_cast<const float2*>(s_v + (os * 4 + 2 + rr) * W + sc);
            const float vo[2][2] = {{ox.x, ox.y}, {oz.x, oz.y}};
            // the eight derivative sums of the row pair, advanced together term by term
            // (each sum keeps the canonical order l = 1..N)
            float dxx[2] = {0.0f, 0.0f}, dxzx[2] = {0.0f, 0.0f};
            float dxzz[2] = {0.0f, 0.0f}, dzz[2] = {0.0f, 0.0f};
#pragma unroll
            for (int l = 1; l <= N; ++l) {
              const float a = c.a[l - 1];
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                dxx[e] = __fmaf_rn(a, __fsub_rn(xa[2 * E + e + l - 1], xa[2 * E + e - l]), dxx[e]);
                dxzx[e] = __fmaf_rn(a, __fsub_rn(xb[2 * E + e + l], xb[2 * E + e - l + 1]), dxzx[e]);
                dxzz[e] = __fmaf_rn(a, __fsub_rn(wxz[rr + M + l - 1][e], wxz[rr + M - l][e]), dxzz[e]);
                dzz[e] = __fmaf_rn(a, __fsub_rn(wzz[rr + M + l][e], wzz[rr + M - l + 1][e]), dzz[e]);
              }
            }
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              float ux = vo[0][e], uz = vo[1][e];
              if (zin && g.xin[e]) {
                ux = __fmaf_rn(bxv[rr][e], __fmaf_rn(dtx, dxx[e], __fmul_rn(dtz, dxzz[e])), ux);
                uz = __fmaf_rn(bzv[rr][e], __fmaf_rn(dtx, dxzx[e], __fmul_rn(dtz, dzz[e])), uz);
              }
              vpc[0][rr][e] = ux;
              vpc[1][rr][e] = uz;
            }
            const int pr = (2 * i + rr) & 3;  // v' ring row of zv + rr
            *reinterpret_cast<float2*>(s_vp + pr * W + sc) = make_float2(vpc[0][rr][0], vpc[0][rr][1]);
            *reinterpret_cast<float2*>(s_vp + (4 + pr) * W + sc) =
                make_float2(vpc[1][rr][0], vpc[1][rr][1]);
          }
        }
#pragma unroll
        for (int k = 0; k < 2 * M; ++k)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            wxz[k][e] = wxz[k + 2][e];
            wzz[k][e] = wzz[k + 2][e];
          }
        cta_bar(mid_id, mid_n);
        // v'' rows zv-1 (rr = 0) and zv (rr = 1); v' rows zv-2 .. zv+1 are in vpp / vpc
        if (do_v) {
#pragma unroll
          for (int rr = 0; rr < 2; ++rr) {
            const int qv = zv - 1 + rr;
            float vvn[2][2];
#pragma unroll
            for (int f = 0; f < 2; ++f)
#pragma unroll
              for (int e = 0; e < 2; ++e) vvn[f][e] = rr ? vpc[f][0][e] : vpp[f][1][e];
            const int zsd = zside(qv);
            const bool zfr = zframe(qv);
            if (zfr && zsd != 0 && !g.xband) {
              // z band, no x band on this thread: z-side edge on its frame cells
              const int zd = zdist(qv);
              const float* vo_r = s_v + ((rr ? os : osp) * 4 + (rr ? 0 : 1)) * W + sc;
              const float* vz_r = s_v + ((zsd > 0 ? os : osp) * 4 + rr) * W + sc;
#pragma unroll
              for (int f = 0; f < 2; ++f) {
                const float w = wsm(f, zd);
                const float2 fo = *reinterpret_cast<const float2*>(vo_r + f * 2 * W);
                const float2 fz = *reinterpret_cast<const float2*>(vz_r + f * 2 * W);
                const float fo_[2] = {fo.x, fo.y}, fz_[2] = {fz.x, fz.y};
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                  const float vz_n = rr ? (zsd > 0 ? vpc[f][1][e] : vpp[f][1][e])
                                        : (zsd > 0 ? vpc[f][0][e] : vpp[f][0][e]);
                  const float res = higdon_edge(w, vvn[f][e], higdon_side(h, vz_n, fo_[e], fz_[e]));
                  vvn[f][e] = g.xfr[e] ? res : vvn[f][e];
                }
              }
            } else if (zfr && zsd == 0 && g.xband) {
              // x band outside the z bands: x-side edge on the band cells
              const float* vo_r = s_v + ((rr ? os : osp) * 4 + (rr ? 0 : 1)) * W;
              const float* vp_r = s_vp + ((2 * i - 1 + rr) & 3) * W;
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                const int col = sc + e, coln = g.xcn[e];
#pragma unroll
                for (int f = 0; f < 2; ++f) {
                  const float fop = vo_r[f * 2 * W + col];
                  const float res = higdon_edge(
                      wxb[f][e], vvn[f][e],
                      higdon_side(h, vp_r[f * 4 * W + coln], fop, vo_r[f * 2 * W + coln]));
                  vvn[f][e] = g.xedge[e] ? res : vvn[f][e];
                }
              }
            } else if (zfr && zsd != 0) {
              // z band and x band: corners, edges of both kinds
              const int zd = zdist(qv);
              // row bases (field f at + f * stride): A.v row qv (rows zv-2, zv-1 sit in
              // the previous pair's slot, zv, zv+1 in this one), A.v row qv + zsd, v' row qv
              const float* vo_r = s_v + ((rr ? os : osp) * 4 + (rr ? 0 : 1)) * W;
              const float* vz_r = s_v + ((zsd > 0 ? os : osp) * 4 + rr) * W;
              const float* vp_r = s_vp + ((2 * i - 1 + rr) & 3) * W;
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                const bool fr = g.xfr[e];
                const bool corner = g.xsd[e] != 0, xs = g.xsd[e] != 0;
                const int col = sc + e, coln = g.xcn[e];
                const int dist = min(g.xds[e], zd);
#pragma unroll
                for (int f = 0; f < 2; ++f) {
                  const float w = wsm(f, dist);
                  const float fop = vo_r[f * 2 * W + col];
                  const float vz_n = rr ? (zsd > 0 ? vpc[f][1][e] : vpp[f][1][e])
                                        : (zsd > 0 ? vpc[f][0][e] : vpp[f][0][e]);
                  const float hx = higdon_side(h, vp_r[f * 4 * W + coln], fop, vo_r[f * 2 * W + coln]);
                  const float hz = higdon_side(h, vz_n, fop, vz_r[f * 2 * W + col]);
                  const float res = corner ? higdon_corner(w, vvn[f][e], hx, hz)
                                           : higdon_edge(w, vvn[f][e], xs ? hx : hz);
                  vvn[f][e] = fr ? res : vvn[f][e];
                }
              }
            }
            bool bnd[2] = {true, true};
            if constexpr (H16) {
              const bool zb16 = zband16(qv);
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                bnd[e] = zb16 || xband16(g.xc + e);
#pragma unroll
                for (int f = 0; f < 2; ++f) vvn[f][e] = stored(vvn[f][e], bnd[e]);
              }
            }
            const int vw = (2 * i + rr) & (LVV - 1);  // v'' ring row of qv
            *reinterpret_cast<float2*>(s_vv + vw * W + sc) = make_float2(vvn[0][0], vvn[0][1]);
            *reinterpret_cast<float2*>(s_vv + (LVV + vw) * W + sc) = make_float2(vvn[1][0], vvn[1][1]);
            if (g.o_any && qv >= g.za && qv < g.zb) {
              float* px = rr ? ovx + gm.ld : ovx;
              float* pz = rr ? ovz + gm.ld : ovz;
              if constexpr (!H16) {
                if (g.o_pair) {
                  *reinterpret_cast<float2*>(px) = make_float2(vvn[0][0], vvn[0][1]);
                  *reinterpret_cast<float2*>(pz) = make_float2(vvn[1][0], vvn[1][1]);
                } else {
                  *px = vvn[0][0];
                  *pz = vvn[1][0];
                }
              } else {
                // the binary16 arrays run parallel to the FP32 ones (same index)
                __half* hx = o16.vx + (px - o.vx);
                __half* hz = o16.vz + (pz - o.vz);
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                  if (e == 1 && !g.o_pair) break;
                  if (bnd[e]) {
                    px[e] = vvn[0][e];
                    pz[e] = vvn[1][e];
                  } else {
                    hx[e] = __float2half_rn(vvn[0][e]);
                    hz[e] = __float2half_rn(vvn[1][e]);
                  }
                }
              }
            }
          }
        }
        ovx += 2 * gm.ld;
        ovz += 2 * gm.ld;
#pragma unroll
        for (int f = 0; f < 2; ++f)
#pragma unroll
          for (int k = 0; k < 4; ++k) vpp[f][k >> 1][k & 1] = vpc[f][k >> 1][k & 1];
        mv[0] = __ldg(pv);
        mv[1] = __ldg(pv + mp.pitch);
        pv += mrow;
        cta_bar(1, NT);
        if (tid == 0 && live && i + 1 + P < g.I) {
          fence_proxy_async();
          issue(i + 1 + P);
        }
        zs = zs + 1 == NZ ? 0 : zs + 1;
        osp = os;
        os = os + 1 == NO ? 0 : os + 1;
        ph ^= os == 0 ? 1u : 0u;
      }
      gb += g.I;
    }
  } else {
    // ======================== stress role ========================
    int gb = 0;
    bool live = true;
    for (long long r = r_lo; r < r_hi;) {
      Seg g;
      segment(r, g);
      cta_bar(1, NT);  // pairs with the velocity role's segment barrier
      float wvx[WN][2], wvz[WN][2];
#pragma unroll
      for (int k = 0; k < WN; ++k)
#pragma unroll
        for (int e = 0; e < 2; ++e) wvx[k][e] = wvz[k][e] = 0.0f;
      float wxb[2];  // HABC weights of the x-band cells outside the z bands
#pragma unroll
      for (int e = 0; e < 2; ++e) wxb[e] = wsm(2, g.xds[e]);
      // output rows q-1 (iteration 0) onwards, advanced two rows per iteration
      float* ot[3];
      ot[0] = o.txx + g.obase + (long long)(g.zv0 - 4 - M) * gm.ld;
      ot[1] = o.tzz + g.obase + (long long)(g.zv0 - 4 - M) * gm.ld;
      ot[2] = o.txz + g.obase + (long long)(g.zv0 - 4 - M) * gm.ld;
      float spp[3][2][2];  // previous iteration's s' rows [field][row][cell]
#pragma unroll
      for (int f = 0; f < 3; ++f)
#pragma unroll
        for (int k = 0; k < 4; ++k) spp[f][k >> 1][k & 1] = 0.0f;
      const long long pcol = (g.xc >> 1) + kPackColPad / 2;
      const long long prow0 = (long long)(g.zv0 - 3 - M + kPackRowPad) * mp.pitch + pcol;
      const float4* pl = mp.l + prow0;
      const float2* pu = mp.mu + prow0;
      float4 ml[2];
      float2 mu[2];
      ml[0] = __ldg(pl);
      ml[1] = __ldg(pl + mp.pitch);
      mu[0] = __ldg(pu);
      mu[1] = __ldg(pu + mp.pitch);
      pl += mrow;
      pu += mrow;
      int os = gb % NO, osp = (gb + NO - 1) % NO;
      uint32_t ph = (uint32_t)((gb / NO) & 1);
      for (int i = 0; i < g.I; ++i) {
        const int zv = g.zv0 + 2 * i, q = zv - 3 - M;
        if (live) live = mbar_wait_bounded(&bars[os], ph, err) && live;
        if constexpr (H16) {
          widen(s_o + (os * 6 + 0) * W, hbox(4 * NZ + os * 3 + 0), g.XT, q);
          widen(s_o + (os * 6 + 2) * W, hbox(4 * NZ + os * 3 + 1), g.XT, q);
          widen(s_o + (os * 6 + 4) * W, hbox(4 * NZ + os * 3 + 2), g.XT, q);
          cta_bar(5, NV);  // the role's widened rows are complete
        }
        const float lav[2][2] = {{ml[0].x, ml[0].y}, {ml[1].x, ml[1].y}};
        const float l2v[2][2] = {{ml[0].z, ml[0].w}, {ml[1].z, ml[1].w}};
        const float muv[2][2] = {{mu[0].x, mu[0].y}, {mu[1].x, mu[1].y}};
        // the v'' window advances by two rows: rows q-M .. q+M-1 move down, and
        // v'' rows q+M, q+M+1 (= zv-3, zv-2, written by the velocity role in
        // the previous iteration) enter at the top

        if (i > 0) {
#pragma unroll
          for (int k = 0; k < 2 * M; ++k)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              wvx[k][e] = wvx[k + 2][e];
              wvz[k][e] = wvz[k + 2][e];
            }
#pragma unroll
          for (int rr = 0; rr < 2; ++rr) {
            const int vr = (2 * i - 2 + rr) & (LVV - 1);
            const float2 a = *reinterpret_cast<const float2*>(s_vv + vr * W + sc);
            const float2 b = *reinterpret_cast<const float2*>(s_vv + (LVV + vr) * W + sc);
            wvx[2 * M + rr][0] = a.x;
            wvx[2 * M + rr][1] = a.y;
            wvz[2 * M + rr][0] = b.x;
            wvz[2 * M + rr][1] = b.y;
          }
        }
        float spc[3][2][2];  // s' rows q, q+1 [field][row][cell]
        if (do_s) {
#pragma unroll
          for (int rr = 0; rr < 2; ++rr) {
            const bool zin = zinner(q + rr);
            const int vb = (2 * i - 2 - M + rr) & (LVV - 1);  // v'' ring row of q + rr
            constexpr int E = (N + 1) / 2;
            float xa[4 * E + 2], xb[4 * E + 2];  // v''x and v''z rows q + rr around the pair
            load_xwin<N>(s_vv + vb * W, sc, xa);
            load_xwin<N>(s_vv + (LVV + vb) * W, sc, xb);
            const float2 oxx = *reinterpret_cast<const float2*>(s_o + (os * 6 + 0 + rr) * W + sc + TN);
            const float2 ozz = *reinterpret_cast<const float2*>(s_o + (os * 6 + 2 + rr) * W + sc + TN);
            const float2 oxz = *reinterpret_cast<const float2*>(s_o + (os * 6 + 4 + rr) * W + sc + TN);
            const float so_[3][2] = {{oxx.x, oxx.y}, {ozz.x, ozz.y}, {oxz.x, oxz.y}};
            // the eight derivative sums of the row pair, advanced together term by term
            // (each sum keeps the canonical order l = 1..N)
            float dvxdx[2] = {0.0f, 0.0f}, dvzdx[2] = {0.0f, 0.0f};
            float dvxdz[2] = {0.0f, 0.0f}, dvzdz[2] = {0.0f, 0.0f};
#pragma unroll
            for (int l = 1; l <= N; ++l) {
              const float a = c.a[l - 1];
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                dvxdx[e] = __fmaf_rn(a, __fsub_rn(xa[2 * E + e + l], xa[2 * E + e - l + 1]), dvxdx[e]);
                dvzdx[e] = __fmaf_rn(a, __fsub_rn(xb[2 * E + e + l - 1], xb[2 * E + e - l]), dvzdx[e]);
                dvxdz[e] = __fmaf_rn(a, __fsub_rn(wvx[rr + M + l][e], wvx[rr + M - l + 1][e]), dvxdz[e]);
                dvzdz[e] = __fmaf_rn(a, __fsub_rn(wvz[rr + M + l - 1][e], wvz[rr + M - l][e]), dvzdz[e]);
              }
            }
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              float sxx = so_[0][e], szz = so_[1][e], sxz = so_[2][e];
              if (zin && g.xin[e]) {
                const float ex = __fmul_rn(dvxdx[e], dtx), ez = __fmul_rn(dvzdz[e], dtz);
                sxx = __fadd_rn(sxx, __fmaf_rn(l2v[rr][e], ex, __fmul_rn(lav[rr][e], ez)));
                szz = __fadd_rn(szz, __fmaf_rn(lav[rr][e], ex, __fmul_rn(l2v[rr][e], ez)));
                sxz = __fmaf_rn(muv[rr][e], __fmaf_rn(dvxdz[e], dtz, __fmul_rn(dvzdx[e], dtx)), sxz);
              }
              spc[0][rr][e] = sxx;
              spc[1][rr][e] = szz;
              spc[2][rr][e] = sxz;
            }
            const int sr = (2 * i + rr) & 3;  // s' ring row of q + rr
#pragma unroll
            for (int f = 0; f < 3; ++f)
              *reinterpret_cast<float2*>(s_sp + (4 * f + sr) * W + sc) =
                  make_float2(spc[f][rr][0], spc[f][rr][1]);
          }
        }
        cta_bar(mid_id, mid_n);
        // s'' rows q-1 (rr = 0) and q (rr = 1); s' rows q-2 .. q+1 are in spp / spc
        if (g.o_any) {
#pragma unroll
          for (int rr = 0; rr < 2; ++rr) {
            const int qs = q - 1 + rr;
            if (qs < g.za || qs >= g.zb) continue;
            float v[3][2];
#pragma unroll
            for (int f = 0; f < 3; ++f)
#pragma unroll
              for (int e = 0; e < 2; ++e) v[f][e] = rr ? spc[f][0][e] : spp[f][1][e];
            const int zsd = zside(qs);
            const bool zfr = zframe(qs);
            if (zfr && zsd != 0 && !g.xband) {
              // z band, no x band on this thread: z-side edge on its frame cells
              const float w = wsm(2, zdist(qs));
              const float* so_r = s_o + ((rr ? os : osp) * 6 + (rr ? 0 : 1)) * W + TN + sc;
              const float* sz_r = s_o + ((zsd > 0 ? os : osp) * 6 + rr) * W + TN + sc;
#pragma unroll
              for (int f = 0; f < 3; ++f) {
                const float2 fo = *reinterpret_cast<const float2*>(so_r + f * 2 * W);
                const float2 fz = *reinterpret_cast<const float2*>(sz_r + f * 2 * W);
                const float fo_[2] = {fo.x, fo.y}, fz_[2] = {fz.x, fz.y};
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                  const float sz_n = rr ? (zsd > 0 ? spc[f][1][e] : spp[f][1][e])
                                        : (zsd > 0 ? spc[f][0][e] : spp[f][0][e]);
                  const float res = higdon_edge(w, v[f][e], higdon_side(h, sz_n, fo_[e], fz_[e]));
                  v[f][e] = g.xfr[e] ? res : v[f][e];
                }
              }
            } else if (zfr && zsd == 0 && g.xband) {
              // x band outside the z bands: x-side edge on the band cells
              const float* so_r = s_o + ((rr ? os : osp) * 6 + (rr ? 0 : 1)) * W + TN;
              const float* sp_r = s_sp + ((2 * i - 1 + rr) & 3) * W;
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                const int col = sc + e, coln = g.xcn[e];
#pragma unroll
                for (int f = 0; f < 3; ++f) {
                  const float fop = so_r[f * 2 * W + col];
                  const float res = higdon_edge(
                      wxb[e], v[f][e],
                      higdon_side(h, sp_r[f * 4 * W + coln], fop, so_r[f * 2 * W + coln]));
                  v[f][e] = g.xedge[e] ? res : v[f][e];
                }
              }
            } else if (zfr && zsd != 0) {
              // z band and x band: corners, edges of both kinds
              const int zd = zdist(qs);
              // row bases (field f at + f * stride): old stress row qs (rows q-2, q-1 in
              // the previous pair slot, q, q+1 in this one), row qs + zsd, s' row qs
              const float* so_r = s_o + ((rr ? os : osp) * 6 + (rr ? 0 : 1)) * W + TN;
              const float* sz_r = s_o + ((zsd > 0 ? os : osp) * 6 + rr) * W + TN;
              const float* sp_r = s_sp + ((2 * i - 1 + rr) & 3) * W;
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                const bool fr = g.xfr[e];
                const bool corner = g.xsd[e] != 0, xs = g.xsd[e] != 0;
                const int col = sc + e, coln = g.xcn[e];
                const float w = wsm(2, min(g.xds[e], zd));
#pragma unroll
                for (int f = 0; f < 3; ++f) {
                  const float fop = so_r[f * 2 * W + col];
                  const float sz_n = rr ? (zsd > 0 ? spc[f][1][e] : spp[f][1][e])
                                        : (zsd > 0 ? spc[f][0][e] : spp[f][0][e]);
                  const float hx = higdon_side(h, sp_r[f * 4 * W + coln], fop, so_r[f * 2 * W + coln]);
                  const float hz = higdon_side(h, sz_n, fop, sz_r[f * 2 * W + col]);
                  const float res = corner ? higdon_corner(w, v[f][e], hx, hz)
                                           : higdon_edge(w, v[f][e], xs ? hx : hz);
                  v[f][e] = fr ? res : v[f][e];
                }
              }
            }
            if constexpr (!H16) {
#pragma unroll
              for (int f = 0; f < 3; ++f) {
                float* pt = rr ? ot[f] + gm.ld : ot[f];
                if (g.o_pair)
                  *reinterpret_cast<float2*>(pt) = make_float2(v[f][0], v[f][1]);
                else
                  *pt = v[f][0];
              }
            } else {
              __half* const oh[3] = {o16.txx, o16.tzz, o16.txz};
              float* const of[3] = {o.txx, o.tzz, o.txz};
              const bool zb16 = zband16(qs);
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                if (e == 1 && !g.o_pair) break;
                const bool bnd = zb16 || xband16(g.xc + e);
#pragma unroll
                for (int f = 0; f < 3; ++f) {
                  float* pt = (rr ? ot[f] + gm.ld : ot[f]) + e;
                  if (bnd) *pt = v[f][e];
                  else oh[f][pt - of[f]] = __float2half_rn(v[f][e]);
                }
              }
            }
          }
        }
#pragma unroll
        for (int f = 0; f < 3; ++f) ot[f] += 2 * gm.ld;
#pragma unroll
        for (int f = 0; f < 3; ++f)
#pragma unroll
          for (int k = 0; k < 4; ++k) spp[f][k >> 1][k & 1] = spc[f][k >> 1][k & 1];
        ml[0] = __ldg(pl);
        ml[1] = __ldg(pl + mp.pitch);
        mu[0] = __ldg(pu);
        mu[1] = __ldg(pu + mp.pitch);
        pl += mrow;
        pu += mrow;
        cta_bar(1, NT);
        osp = os;
        os = os + 1 == NO ? 0 : os + 1;
        ph ^= os == 0 ? 1u : 0u;
      }
      gb += g.I;
    }
  }
}

// ---- host side --------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
  std::call_once(g_encode_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    else
      cudaGetLastError();
  });
  return g_encode;
}

template <int N, int NT, int R, int P>
size_t smem_bytes(int W, int wstride) {
  using S = SweepShape<N, R, P>;
  size_t floats = (size_t)3 * S::SR * W + (size_t)(4 * S::SVP + 2 * S::SVV + 6 * S::SSP) * NT +
                  3 * (size_t)wstride;
  floats = (floats + 1) & ~size_t(1);
  return floats * 4 + sizeof(uint64_t) * S::NSLOT;
}

constexpr int kMaxDynSmem = 227 * 1024;

template <int N, int P>
size_t x2_smem_bytes(int wstride) {
  using S = X2Shape<N, P>;
  return (size_t)(S::O_WT + ((3 * wstride + 31) & ~31)) * 4 + sizeof(uint64_t) * S::NPT;
}
// pair-blocked variants: prefetch depth in row pairs
constexpr int kX2P[] = {1, 2, 3};
constexpr int kNumX2 = sizeof(kX2P) / sizeof(kX2P[0]);
#define FOMO_X2_VARIANTS(X, NN) X(0, NN, 1) X(1, NN, 2) X(2, NN, 3)
// register-window variants: prefetch depth in row pairs
constexpr int kRWP[] = {1, 2};
constexpr int kNumRW = sizeof(kRWP) / sizeof(kRWP[0]);
#define FOMO_RW_VARIANTS(X, NN) X(0, NN, 1) X(1, NN, 2)

// lean register-window variants: (threads, prefetch depth in row pairs)
constexpr int kRLNT[] = {128, 128, 64, 64};
constexpr int kRLP[] = {1, 2, 1, 2};
constexpr int kNumRL = sizeof(kRLP) / sizeof(kRLP[0]);
#define FOMO_RL_VARIANTS(X, NN) X(0, NN, 128, 1) X(1, NN, 128, 2) X(2, NN, 64, 1) X(3, NN, 64, 2)

template <int N, int NT, int P, int LV = (N + 2 <= 4 ? 4 : 8), bool H16 = false>
size_t rl_smem_bytes(int wstride) {
  using S = RLShape<N, NT, P, LV, H16>;
  return (size_t)(S::O_WT + ((3 * wstride + 31) & ~31)) * 4 + sizeof(uint64_t) * S::NO;
}

// warp-specialized variants: (threads per role, prefetch depth, CTAs per SM)
// (threads per role, prefetch depth, CTAs per SM, role-local mid-iteration barrier)
constexpr int kWSNV[] = {128, 64, 64, 64, 64, 64};
constexpr int kWSP[] = {1, 1, 1, 2, 1, 1};
constexpr bool kWSH16[] = {false, false, false, false, true, true};  // binary16 storage form
constexpr int kNumWS = sizeof(kWSP) / sizeof(kWSP[0]);
#define FOMO_WS_VARIANTS(X, NN)                                                           \
  X(0, NN, 128, 1, 2, true, false) X(1, NN, 64, 1, 4, false, false)                      \
  X(2, NN, 64, 1, 3, true, false) X(3, NN, 64, 2, 3, true, false) X(4, NN, 64, 1, 3, true, \
                                                                      true)                \
  X(5, NN, 64, 1, 2, true, true)

template <int N, int P>
size_t rw_smem_bytes(int wstride) {
  using S = RWShape<N, P>;
  return (size_t)(S::O_WT + ((3 * wstride + 31) & ~31)) * 4 + sizeof(uint64_t) * S::NO;
}

struct Variant {
  int NT, R, P;
};
constexpr Variant kVariants[] = {{128, 4, 2}, {160, 4, 2}, {96, 4, 2}, {128, 2, 3}};
// Dispatch a templated call on the variant index (threads, rows/chunk, prefetch).
#define FOMO_SWEEP_VARIANTS(X, NN) \
  X(0, NN, 128, 4, 2) X(1, NN, 160, 4, 2) X(2, NN, 96, 4, 2) X(3, NN, 128, 2, 3)
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

template <int N, int NT, int R, int P>
cudaError_t launch_v(cudaStream_t st, const SweepPlan& sp, int set, const Coef& c, float dtx,
                     float dtz, const HabcDev& h, const ElFields& a, const ElMat& m,
                     const ElOut& o, int* err) {
  auto kern = k_el_sweep<N, NT, R, P>;
  const size_t smem = sp.smem;
  static std::atomic<int> attr_set{0};  // opt in to the large dynamic smem once
  if (!attr_set.load(std::memory_order_acquire)) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kMaxDynSmem);
    if (e != cudaSuccess) return e;
    attr_set.store(1, std::memory_order_release);
  }
  if (smem > (size_t)kMaxDynSmem) return cudaErrorInvalidValue;
  const unsigned grid = (unsigned)sp.grid;
  kern<<<grid, NT, smem, st>>>(sp.tm[set][0], sp.tm[set][1], sp.tm[set][2], sp.gm, c, dtx, dtz, h,
                               a, m, o, sp.d_bounds, err);
  return cudaGetLastError();
}

template <int N>
cudaError_t launch_n(cudaStream_t st, const SweepPlan& sp, int set, const Coef& c, float dtx,
                     float dtz, const HabcDev& h, const ElFields& a, const ElMat& m,
                     const ElOut& o, int* err) {
#define FOMO_LAUNCH_V(V, NN, NT, R, P) \
  case V: return launch_v<NN, NT, R, P>(st, sp, set, c, dtx, dtz, h, a, m, o, err);
  switch (sp.variant) { FOMO_SWEEP_VARIANTS(FOMO_LAUNCH_V, N) }
#undef FOMO_LAUNCH_V
  return cudaErrorInvalidValue;
}

template <int N, int P>
cudaError_t launch_x2(cudaStream_t st, const SweepPlan& sp, int set, const Coef& c, float dtx,
                      float dtz, const HabcDev& h, const ElMat& m, const ElOut& o, int* err) {
  auto kern = k_el_sweep_x2<N, P>;
  static std::atomic<int> attr_set{0};
  if (!attr_set.load(std::memory_order_acquire)) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kMaxDynSmem);
    if (e != cudaSuccess) return e;
    attr_set.store(1, std::memory_order_release);
  }
  if (sp.smem > (size_t)kMaxDynSmem) return cudaErrorInvalidValue;
  kern<<<(unsigned)sp.grid, kX2Threads, sp.smem, st>>>(sp.tm[set][0], sp.tm[set][1], sp.tm[set][2],
                                                        sp.tm[set][3], sp.tm[set][4], sp.gm, c, dtx,
                                                        dtz, h, m, o, sp.d_bounds, err);
  return cudaGetLastError();
}

template <int N>
cudaError_t launch_x2_n(cudaStream_t st, const SweepPlan& sp, int set, const Coef& c, float dtx,
                        float dtz, const HabcDev& h, const ElMat& m, const ElOut& o, int* err) {
#define FOMO_LAUNCH_X2(V, NN, PP) \
  case V: return launch_x2<NN, PP>(st, sp, set, c, dtx, dtz, h, m, o, err);
  switch (sp.variant - kNumVariants) { FOMO_X2_VARIANTS(FOMO_LAUNCH_X2, N) }
#undef FOMO_LAUNCH_X2
  return cudaErrorInvalidValue;
}

template <int N, int P>
cudaError_t launch_rw(cudaStream_t st, const SweepPlan& sp, int set, const Coef& c, float dtx,
                      float dtz, const HabcDev& h, const ElMat& m, const ElOut& o, int* err) {
  auto kern = k_el_sweep_rw<N, P>;
  static std::atomic<int> attr_set{0};
  if (!attr_set.load(std::memory_order_acquire)) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kMaxDynSmem);
    if (e != cudaSuccess) return e;
    attr_set.store(1, std::memory_order_release);
  }
  if (sp.smem > (size_t)kMaxDynSmem) return cudaErrorInvalidValue;
  kern<<<(unsigned)sp.grid, kRWThreads, sp.smem, st>>>(sp.tm[set][0], sp.tm[set][1], sp.tm[set][2],
                                                        sp.tm[set][3], sp.tm[set][4], sp.gm, c, dtx,
                                                        dtz, h, m, o, sp.d_bounds, err);
  return cudaGetLastError();
}

template <int N>
cudaError_t launch_rw_n(cudaStream_t st, const SweepPlan& sp, int set, const Coef& c, float dtx,
                        float dtz, const HabcDev& h, const ElMat& m, const ElOut& o, int* err) {
#define FOMO_LAUNCH_RW(V, NN, PP) \
  case V: return launch_rw<NN, PP>(st, sp, set, c, dtx, dtz, h, m, o, err);
  switch (sp.variant - kNumVariants - kNumX2) { FOMO_RW_VARIANTS(FOMO_LAUNCH_RW, N) }
#undef FOMO_LAUNCH_RW
  return cudaErrorInvalidValue;
}

template <int N, int NT, int P>
cudaError_t launch_rl(cudaStream_t st, const SweepPlan& sp, int set, const Coef& c, float dtx,
                      float dtz, const HabcDev& h, const ElMat& m, const ElOut& o, int* err) {
  auto kern = k_el_sweep_rl<N, NT, P>;
  static std::atomic<int> attr_set{0};
  if (!attr_set.load(std::memory_order_acquire)) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kMaxDynSmem);
    if (e != cudaSuccess) return e;
    attr_set.store(1, std::memory_order_release);
  }
  if (sp.smem > (size_t)kMaxDynSmem || !m.pack || m.pack_pitch < 1) return cudaErrorInvalidValue;
  const long long cells = (long long)(sp.gm.nz + 2 * kPackRowPad) * m.pack_pitch;
  const MatPack mp{reinterpret_cast<const float4*>(m.pack),
                   reinterpret_cast<const float4*>(m.pack) + cells,
                   reinterpret_cast<const float2*>(m.pack + 8 * cells), m.pack_pitch};
  kern<<<(unsigned)sp.grid, NT, sp.smem, st>>>(sp.tm[set][0], sp.tm[set][1], sp.tm[set][2],
                                                sp.tm[set][3], sp.tm[set][4], sp.gm, c, dtx, dtz, h,
                                                mp, o, sp.d_bounds, err);
  return cudaGetLastError();
}

template <int N>
cudaError_t launch_rl_n(cudaStream_t st, const SweepPlan& sp, int set, const Coef& c, float dtx,
                        float dtz, const HabcDev& h, const ElMat& m, const ElOut& o, int* err) {
#define FOMO_LAUNCH_RL(V, NN, NT, PP) \
  case V: return launch_rl<NN, NT, PP>(st, sp, set, c, dtx, dtz, h, m, o, err);
  switch (sp.variant - kNumVariants - kNumX2 - kNumRW) { FOMO_RL_VARIANTS(FOMO_LAUNCH_RL, N) }
#undef FOMO_LAUNCH_RL
  return cudaErrorInvalidValue;
}

template <int N, int NV, int P, int MINB, bool SPLIT, bool H16>
cudaError_t launch_ws(cudaStream_t st, const SweepPlan& sp, int set, const Coef& c, float dtx,
                      float dtz, const HabcDev& h, const ElMat& m, const ElOut& o,
                      const ElOut16* o16, int* err) {
  auto kern = k_el_sweep_ws<N, NV, P, MINB, SPLIT, H16>;
  static std::atomic<int> attr_set{0};
  if (!attr_set.load(std::memory_order_acquire)) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kMaxDynSmem);
    if (e != cudaSuccess) return e;
    attr_set.store(1, std::memory_order_release);
  }
  if (sp.smem > (size_t)kMaxDynSmem || !m.pack || m.pack_pitch < 1) return cudaErrorInvalidValue;
  if (H16 && (!sp.h16 || !o16)) return cudaErrorInvalidValue;
  const long long cells = (long long)(sp.gm.nz + 2 * kPackRowPad) * m.pack_pitch;
  const MatPack mp{reinterpret_cast<const float4*>(m.pack),
                   reinterpret_cast<const float4*>(m.pack) + cells,
                   reinterpret_cast<const float2*>(m.pack + 8 * cells), m.pack_pitch};
  const CUtensorMap* th = H16 ? sp.tm16[set] : sp.tm[set];  // unused by the FP32 form
  const ElOut16 oh = o16 ? *o16 : ElOut16{};
  kern<<<(unsigned)sp.grid, 2 * NV, sp.smem, st>>>(sp.tm[set][0], sp.tm[set][1], sp.tm[set][2],
                                                    sp.tm[set][3], sp.tm[set][4], th[0], th[1],
                                                    th[2], th[3], th[4], sp.gm, c, dtx, dtz, h, mp,
                                                    o, oh, sp.d_bounds, err);
  return cudaGetLastError();
}

template <int N>
cudaError_t launch_ws_n(cudaStream_t st, const SweepPlan& sp, int set, const Coef& c, float dtx,
                        float dtz, const HabcDev& h, const ElMat& m, const ElOut& o,
                        const ElOut16* o16, int* err) {
#define FOMO_LAUNCH_WS(V, NN, NV, PP, MB, SP, HH) \
  case V: return launch_ws<NN, NV, PP, MB, SP, HH>(st, sp, set, c, dtx, dtz, h, m, o, o16, err);
  switch (sp.variant - kNumVariants - kNumX2 - kNumRW - kNumRL) {
    FOMO_WS_VARIANTS(FOMO_LAUNCH_WS, N)
  }
#undef FOMO_LAUNCH_WS
  return cudaErrorInvalidValue;
}

size_t ws_smem_for(int N, int v, int wstride) {
#define FOMO_SMEM_WS(V, NN, NV, PP, MB, SP, HH) \
  case V: return rl_smem_bytes<NN, NV, PP, ws_lvv(NN, SP), HH>(wstride);
#define FOMO_SMEM_WSN(NN)                              \
  case NN:                                             \
    switch (v) { FOMO_WS_VARIANTS(FOMO_SMEM_WS, NN) }  \
    break;
  switch (N) { FOMO_SMEM_WSN(1) FOMO_SMEM_WSN(2) FOMO_SMEM_WSN(3) FOMO_SMEM_WSN(4) FOMO_SMEM_WSN(5) }
#undef FOMO_SMEM_WSN
#undef FOMO_SMEM_WS
  return 0;
}

size_t rl_smem_for(int N, int v, int wstride) {
#define FOMO_SMEM_RL(V, NN, NT, PP) \
  case V: return rl_smem_bytes<NN, NT, PP>(wstride);
#define FOMO_SMEM_RLN(NN)                              \
  case NN:                                             \
    switch (v) { FOMO_RL_VARIANTS(FOMO_SMEM_RL, NN) }  \
    break;
  switch (N) { FOMO_SMEM_RLN(1) FOMO_SMEM_RLN(2) FOMO_SMEM_RLN(3) FOMO_SMEM_RLN(4) FOMO_SMEM_RLN(5) }
#undef FOMO_SMEM_RLN
#undef FOMO_SMEM_RL
  return 0;
}

// Copies the five elastic planes into the lean sweep's material pack.
__global__ void k_sweep_pack(int nx, int nz, int ld, ElMat m, float4* pv, float4* pl, float2* pu,
                             int pitch, long long cells) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < cells;
       k += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(k / pitch) - kPackRowPad;
    const int x = 2 * ((int)(k % pitch) - kPackColPad / 2);
    auto at = [&](const float* a, int xx) {
      return z >= 0 && z < nz && xx >= 0 && xx < nx ? a[(long long)z * ld + xx] : 0.0f;
    };
    pv[k] = make_float4(at(m.bx, x), at(m.bx, x + 1), at(m.bz, x), at(m.bz, x + 1));
    pl[k] = make_float4(at(m.lam, x), at(m.lam, x + 1), at(m.l2m, x), at(m.l2m, x + 1));
    pu[k] = make_float2(at(m.mut, x), at(m.mut, x + 1));
  }
}

size_t rw_smem_for(int N, int v, int wstride) {
#define FOMO_SMEM_RW(V, NN, PP) \
  case V: return rw_smem_bytes<NN, PP>(wstride);
#define FOMO_SMEM_RWN(NN)                              \
  case NN:                                             \
    switch (v) { FOMO_RW_VARIANTS(FOMO_SMEM_RW, NN) }  \
    break;
  switch (N) { FOMO_SMEM_RWN(1) FOMO_SMEM_RWN(2) FOMO_SMEM_RWN(3) FOMO_SMEM_RWN(4) FOMO_SMEM_RWN(5) }
#undef FOMO_SMEM_RWN
#undef FOMO_SMEM_RW
  return 0;
}

size_t x2_smem_for(int N, int v2, int wstride) {
#define FOMO_SMEM_X2(V, NN, PP) \
  case V: return x2_smem_bytes<NN, PP>(wstride);
#define FOMO_SMEM_X2N(NN)                                  \
  case NN:                                                 \
    switch (v2) { FOMO_X2_VARIANTS(FOMO_SMEM_X2, NN) }     \
    break;
  switch (N) { FOMO_SMEM_X2N(1) FOMO_SMEM_X2N(2) FOMO_SMEM_X2N(3) FOMO_SMEM_X2N(4) FOMO_SMEM_X2N(5) }
#undef FOMO_SMEM_X2N
#undef FOMO_SMEM_X2
  return 0;
}

size_t smem_for(int N, int variant, int W, int wstride) {
#define FOMO_SMEM_V(V, NN, NT, R, P) \
  case V: return smem_bytes<NN, NT, R, P>(W, wstride);
#define FOMO_SMEM_N(NN)                                  \
  case NN:                                               \
    switch (variant) { FOMO_SWEEP_VARIANTS(FOMO_SMEM_V, NN) } \
    break;
  switch (N) { FOMO_SMEM_N(1) FOMO_SMEM_N(2) FOMO_SMEM_N(3) FOMO_SMEM_N(4) FOMO_SMEM_N(5) }
#undef FOMO_SMEM_N
#undef FOMO_SMEM_V
  return 0;
}

}  // namespace

// The single sweep pays off on large batches; a small problem gives each CTA
// only a few rows, and the z-segment warm-up then dominates.  Measured (order
// 8, one shot): 240x200 two-phase 61 k vs sweep 36 k steps/s, 1000x800 24.9 k vs
// 22.6 k; the 32-shot 1170x670 batch (25 M cell-shots) 0.49 vs 1.0 ms per step
// for the sweep.
int pick_kernel_2d(int phys, int N, int nxp, int nzp, int ns) {
  (void)N;
  const double work = (double)nxp * nzp * ns;  // cell-updates per step
  return phys == 1 && encoder() && work >= 4.0e6 ? FOMO_KERNEL_SINGLE_SWEEP
                                                  : FOMO_KERNEL_TWO_PHASE;
}

bool sweep2d_supported(int phys, int N) { return phys == 1 && N >= 1 && N <= 5 && encoder(); }

constexpr int kWSBase = kNumVariants + kNumX2 + kNumRW + kNumRL;
constexpr int kPairBase = kWSBase + kNumWS;  // the shot-pair variants (sweep2d_pair.cu)

int sweep_num_variants() { return kPairBase + pair_num_variants(); }

bool sweep_variant_ws(int variant) { return variant >= kWSBase && variant < kPairBase; }

bool sweep_variant_pair(int variant) {
  return variant >= kPairBase && variant < kPairBase + pair_num_variants();
}

int sweep_pack_pitch(int nx) { return ((nx + 2 * 128 + kPackColPad) / 2 + 16) & ~15; }

size_t sweep_pack_floats(int nx, int nz) {
  return (size_t)(nz + 2 * kPackRowPad) * sweep_pack_pitch(nx) * 10;
}

cudaError_t build_sweep_pack(cudaStream_t st, const Geo2& g, ElMat& m, float* dst) {
  if (!dst || (reinterpret_cast<uintptr_t>(dst) & 15)) return cudaErrorInvalidValue;
  const int pitch = sweep_pack_pitch(g.nx);
  const long long cells = (long long)(g.nz + 2 * kPackRowPad) * pitch;
  float4* pv = reinterpret_cast<float4*>(dst);
  k_sweep_pack<<<1184, 256, 0, st>>>(g.nx, g.nz, g.ld, m, pv, pv + cells,
                                     reinterpret_cast<float2*>(dst + 8 * cells), pitch, cells);
  m.pack = dst;
  m.pack_pitch = pitch;
  return cudaGetLastError();
}

// Builds the work decomposition and the six tensor maps (3 stress fields x 2
// ping-pong sets).  variant selects (threads, rows per chunk, prefetch depth);
// TX is the strip width (multiple of 4).
bool sweep_variant_h16(int variant) {
  const int v = variant - kWSBase;
  return v >= 0 && v < kNumWS && kWSH16[v];
}

cudaError_t make_sweep_plan(SweepPlan& sp, int N, int variant, int TX, int per_sm, const Geo2& g,
                            int ns, float* const sets[2][5], float frame_weight,
                            long long* d_bounds, cudaStream_t st, __half* const* sets16) {
  auto enc = encoder();
  if (!enc) return cudaErrorNotSupported;
  if (variant < 0 || variant >= sweep_num_variants() || per_sm < 1) return cudaErrorInvalidValue;
  const bool pr = sweep_variant_pair(variant);
  const bool ws = !pr && variant >= kWSBase;
  const bool rl = !ws && variant >= kNumVariants + kNumX2 + kNumRW;
  const bool rw = !ws && !rl && variant >= kNumVariants + kNumX2;
  const bool x2 = variant >= kNumVariants;  // the 2-row TMA-box families
  int W = 0, R = 2;
  sp.h16 = false;
  // a shot-pair plan walks (pair, strip) items; gm.ns holds the pair count
  const int items_ns = pr ? (ns + 1) / 2 : ns;
  if (pr) {
    const int v = variant - kPairBase;
    if (sets16 || TX < 8 || TX > pair_txmax(N, v) || (TX & 1)) 
      return cudaErrorInvalidValue;
    W = pair_box_width(N, v);
    sp.family = 5;
    sp.P = 1;
  } else if (ws) {
    const int v = variant - kNumVariants - kNumX2 - kNumRW - kNumRL;
    if (kWSH16[v]) {
      // binary16 rows: every TMA x coordinate (strip * TX - 8 - 8, strip * TX - 8)
      // must be a multiple of 8 elements
      if (!sets16 || TX < 8 || TX > rl_txmax16(N, kWSNV[v]) || (TX & 7))
        return cudaErrorInvalidValue;
      W = rl_w16(kWSNV[v]);
      sp.h16 = true;
    } else {
      if (sets16 || TX < 8 || TX > rl_txmax(N, kWSNV[v]) || (TX & 3)) return cudaErrorInvalidValue;
      W = rl_w(N, kWSNV[v]);
    }
    sp.family = 4;
    sp.P = kWSP[v];
  } else if (rl) {
    if (sets16) return cudaErrorInvalidValue;
    const int v = variant - kNumVariants - kNumX2 - kNumRW;
    if (TX < 8 || TX > rl_txmax(N, kRLNT[v]) || (TX & 3)) return cudaErrorInvalidValue;
    W = rl_w(N, kRLNT[v]);
    sp.family = 3;
    sp.P = kRLP[v];
  } else if (x2) {
    if (sets16 || TX < 8 || TX > x2_txmax(N) || (TX & 3)) return cudaErrorInvalidValue;
    W = kX2W;
    sp.family = rw ? 2 : 1;
    sp.P = rw ? kRWP[variant - kNumVariants - kNumX2] : kX2P[variant - kNumVariants];
  } else {
    if (sets16) return cudaErrorInvalidValue;
    const int NT = kVariants[variant].NT;
    R = kVariants[variant].R;
    const int M = N, HS = halo_x(M);
    if (TX < 8 || TX + 2 * M + 4 > NT || (TX & 3)) return cudaErrorInvalidValue;
    const int walign = 32 / R;  // R rows of W floats = a multiple of 128 bytes (TMA destination)
    W = (TX + 2 * HS + walign - 1) / walign * walign;
    if (W > 256) return cudaErrorInvalidValue;
    sp.family = 0;
    sp.P = 0;
  }
  sp.variant = variant;
  sp.N = N;
  sp.gm.nx = g.nx;
  sp.gm.nz = g.nz;
  sp.gm.ld = g.ld;
  sp.gm.plane = g.plane;
  sp.gm.nbc = g.nbc;
  sp.gm.TX = TX;
  sp.gm.W = W;
  sp.gm.nstrip = (g.nx + TX - 1) / TX;
  sp.gm.ns = items_ns;
  sp.smem = pr   ? pair_smem(N, variant - kPairBase, g.nbc + 3)
             : ws   ? ws_smem_for(N, variant - kNumVariants - kNumX2 - kNumRW - kNumRL, g.nbc + 3)
             : rl ? rl_smem_for(N, variant - kNumVariants - kNumX2 - kNumRW, g.nbc + 3)
             : rw ? rw_smem_for(N, variant - kNumVariants - kNumX2, g.nbc + 3)
             : x2 ? x2_smem_for(N, variant - kNumVariants, g.nbc + 3)
                  : smem_for(N, variant, W, g.nbc + 3);
  const int bps = sweep_blocks_per_sm(sp);
  if (bps < 1) return cudaErrorInvalidConfiguration;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  sp.per_sm = std::min(per_sm, bps);
  const long long rows = (long long)sp.gm.nstrip * items_ns * g.nz;
  sp.grid = (int)std::max(1LL, std::min({(long long)sp.per_sm * nsm, rows, (long long)kMaxGrid}));
  sp.frame_weight = frame_weight;
  // Cost-balanced split of the flattened (strip, shot, row) space.  A row costs
  // 1 + frame_weight * (b + s + b * s), b = 1 on a z-band row, s = 1 in a strip
  // that holds x-band columns (every warp of such a strip takes the Higdon
  // path); every z-segment a CTA starts (its first row, and each new (shot,
  // strip) item inside its range) costs the warm-up rows that fill the
  // register windows.  (Fitted to per-CTA timings of the warp-specialized
  // sweep at order 10: 1.13 / 1.20 / 1.52 for b, s, both, and 31 rows per
  // segment.)  The smallest per-CTA budget whose greedy split needs at most
  // `grid` CTAs is found by bisection.
  {
    std::vector<double> strip_frac(sp.gm.nstrip);
    for (int k = 0; k < sp.gm.nstrip; ++k) {
      int nf = 0;
      for (int x = k * TX; x < std::min(g.nx, (k + 1) * TX); ++x)
        nf += (x >= 1 && x <= g.nx - 2 && (x <= g.nbc || x >= g.nx - 1 - g.nbc)) ? 1 : 0;
      strip_frac[k] = (double)nf / TX;
    }
    // cost of each row of each strip, and the prefix sums along z
    std::vector<double> pre((size_t)sp.gm.nstrip * (g.nz + 1), 0.0);
    for (int k = 0; k < sp.gm.nstrip; ++k)
      for (int z = 0; z < g.nz; ++z) {
        const bool band = z >= 1 && z <= g.nz - 2 && (z <= g.nbc || z >= g.nz - 1 - g.nbc);
        const double xs = strip_frac[k] > 0.0 ? 1.0 : 0.0, zb = band ? 1.0 : 0.0;
        const double c = 1.0 + frame_weight * (zb + xs + zb * xs);
        pre[(size_t)k * (g.nz + 1) + z + 1] = pre[(size_t)k * (g.nz + 1) + z] + c;
      }
    const double warm = x2 ? 4.0 * N + 11.0 : 2.0 * N + 2.0;
    auto cost = [&](long long r0, long long r1) {  // rows [r0, r1) of one item
      const long long item = r0 / g.nz;
      const int k = (int)(item % sp.gm.nstrip);
      const double* pk = pre.data() + (size_t)k * (g.nz + 1);
      return pk[r1 - item * g.nz] - pk[r0 - item * g.nz];
    };
    // greedy split under budget B; fills b when given, returns the CTAs used
    auto split = [&](double B, std::vector<long long>* b) {
      long long r = 0;
      int used = 0;
      while (r < rows) {
        if (b && used < (int)b->size() - 1) (*b)[used] = r;
        ++used;
        double acc = 0.0;
        bool first = true;
        while (r < rows) {
          const long long item_end = (r / g.nz + 1) * g.nz;
          const double seg = warm + cost(r, item_end);
          if (acc + seg <= B) {  // the rest of this item fits
            acc += seg;
            r = item_end;
            first = false;
            continue;
          }
          // take as many rows of this item as fit (at least one for a fresh CTA)
          long long lo = r, hi = item_end;  // largest e in (r, item_end] with warm + cost <= B - acc
          while (hi - lo > 1) {
            const long long mid = (lo + hi) / 2;
            if (acc + warm + cost(r, mid) <= B) lo = mid;
            else hi = mid;
          }
          if (lo == r && first) lo = r + 1;
          r = lo;
          break;
        }
      }
      return used;
    };
    double total = 0.0;
    for (long long it = 0; it < rows / g.nz; ++it) total += warm + cost(it * g.nz, (it + 1) * g.nz);
    double lo = total / sp.grid, hi = total + warm;
    for (int k = 0; k < 40 && hi - lo > 1e-3 * lo; ++k) {
      const double mid = 0.5 * (lo + hi);
      if (split(mid, nullptr) <= sp.grid) hi = mid;
      else lo = mid;
    }
    std::vector<long long> b(sp.grid + 1, rows);
    split(hi, &b);
    b[sp.grid] = rows;
    cudaError_t e = cudaMemcpyAsync(d_bounds, b.data(), sizeof(long long) * b.size(),
                                    cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    // the host vector dies with this scope: the copy above must have finished
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    sp.d_bounds = d_bounds;
  }
  if (pr) {
    // pair-interleaved fields: one 8-byte element {shot 2p, shot 2p+1} per cell
    for (int s = 0; s < 2; ++s)
      for (int f = 0; f < 5; ++f) {
        cuuint64_t dims[3] = {(cuuint64_t)g.nx, (cuuint64_t)g.nz, (cuuint64_t)items_ns};
        cuuint64_t strides[2] = {(cuuint64_t)g.ld * 8, (cuuint64_t)g.plane * 8};
        cuuint32_t box[3] = {(cuuint32_t)W, 2, 1};
        cuuint32_t es[3] = {1, 1, 1};
        CUresult r = enc(&sp.tm[s][f], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, sets[s][f], dims,
                         strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
      }
    return cudaSuccess;
  }
  for (int s = 0; s < 2; ++s)
    for (int f = 0; f < (x2 ? 5 : 3); ++f) {
      cuuint64_t dims[3] = {(cuuint64_t)g.nx, (cuuint64_t)g.nz, (cuuint64_t)ns};
      cuuint64_t strides[2] = {(cuuint64_t)g.ld * 4, (cuuint64_t)g.plane * 4};
      cuuint32_t box[3] = {(cuuint32_t)W, (cuuint32_t)R, 1};
      cuuint32_t es[3] = {1, 1, 1};
      CUresult r = enc(&sp.tm[s][f], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, sets[s][f], dims,
                       strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                       CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
      if (sp.h16) {
        cuuint64_t strides16[2] = {(cuuint64_t)g.ld * 2, (cuuint64_t)g.plane * 2};
        r = enc(&sp.tm16[s][f], CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, sets16[s * 5 + f], dims,
                strides16, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
      }
    }
  return cudaSuccess;
}

int sweep_tx_candidates(int variant, int N, int nx, int* out, int max_out) {
  int n = 0;
  if (sweep_variant_pair(variant)) {
    // the widest strip, and the narrowest (even) strip with the same strip count
    const int tmax = pair_txmax(N, variant - kPairBase);
    if (tmax >= 8 && n < max_out) out[n++] = tmax;
    const int ns = (nx + tmax - 1) / tmax;
    const int tbal = (((nx + ns - 1) / ns) + 1) & ~1;
    if (tbal >= 8 && tbal < tmax && n < max_out) out[n++] = tbal;
    return n;
  }
  if (variant >= kNumVariants) {
    // the widest strip, and the narrowest strip with the same strip count
    const int v = variant - kNumVariants - kNumX2 - kNumRW;
    const bool h16 = v >= kNumRL && kWSH16[v - kNumRL];
    const int tmax = h16           ? rl_txmax16(N, kWSNV[v - kNumRL])
                     : v >= kNumRL ? rl_txmax(N, kWSNV[v - kNumRL])
                     : v >= 0      ? rl_txmax(N, kRLNT[v])
                                   : x2_txmax(N);
    if (h16) {  // strip widths of binary16 rows are multiples of 8
      if (tmax >= 8 && n < max_out) out[n++] = tmax;
      const int ns = (nx + tmax - 1) / tmax;
      const int tbal = (((nx + ns - 1) / ns) + 7) & ~7;
      if (tbal >= 8 && tbal < tmax && n < max_out) out[n++] = tbal;
      return n;
    }
    if (tmax >= 8 && n < max_out) out[n++] = tmax;
    const int ns = (nx + tmax - 1) / tmax;
    const int tbal = (((nx + ns - 1) / ns) + 3) & ~3;
    if (tbal >= 8 && tbal < tmax && n < max_out) out[n++] = tbal;
    return n;
  }
  // the widest strip whose v' columns (TX + 2M + 4) fill the CTA's threads
  const int tmax = (kVariants[variant].NT - 2 * N - 4) & ~3;
  if (tmax >= 8 && n < max_out) out[n++] = tmax;
  return n;
}

template <int N, int NT, int R, int P>
int occ_v(const SweepPlan& sp) {
  int nb = 0;
  cudaFuncSetAttribute(k_el_sweep<N, NT, R, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kMaxDynSmem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_el_sweep<N, NT, R, P>, NT, sp.smem) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nb;
}

template <int N, int P>
int occ_x2(const SweepPlan& sp) {
  int nb = 0;
  cudaFuncSetAttribute(k_el_sweep_x2<N, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kMaxDynSmem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_el_sweep_x2<N, P>, kX2Threads,
                                                    sp.smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nb;
}

template <int N, int P>
int occ_rw(const SweepPlan& sp) {
  int nb = 0;
  cudaFuncSetAttribute(k_el_sweep_rw<N, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kMaxDynSmem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_el_sweep_rw<N, P>, kRWThreads,
                                                    sp.smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nb;
}

template <int N, int NT, int P>
int occ_rl(const SweepPlan& sp) {
  int nb = 0;
  cudaFuncSetAttribute(k_el_sweep_rl<N, NT, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kMaxDynSmem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_el_sweep_rl<N, NT, P>, NT, sp.smem) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nb;
}

template <int N, int NV, int P, int MINB, bool SPLIT, bool H16>
int occ_ws(const SweepPlan& sp) {
  int nb = 0;
  auto kern = k_el_sweep_ws<N, NV, P, MINB, SPLIT, H16>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 2 * NV, sp.smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nb;
}

int sweep_blocks_per_sm(const SweepPlan& sp) {
  if (sp.family == 5) return pair_blocks_per_sm(sp.N, sp.variant - kPairBase, sp.smem);
  if (sp.family == 4) {
#define FOMO_OCC_WS(V, NN, NV, PP, MB, SP, HH) \
  case V: return occ_ws<NN, NV, PP, MB, SP, HH>(sp);
#define FOMO_OCC_WSN(NN)                                                         \
  case NN:                                                                       \
    switch (sp.variant - kNumVariants - kNumX2 - kNumRW - kNumRL) {              \
      FOMO_WS_VARIANTS(FOMO_OCC_WS, NN)                                          \
    }                                                                            \
    break;
    switch (sp.N) { FOMO_OCC_WSN(1) FOMO_OCC_WSN(2) FOMO_OCC_WSN(3) FOMO_OCC_WSN(4) FOMO_OCC_WSN(5) }
#undef FOMO_OCC_WSN
#undef FOMO_OCC_WS
    return 0;
  }
  if (sp.family == 3) {
#define FOMO_OCC_RL(V, NN, NT, PP) \
  case V: return occ_rl<NN, NT, PP>(sp);
#define FOMO_OCC_RLN(NN)                                                                        \
  case NN:                                                                                      \
    switch (sp.variant - kNumVariants - kNumX2 - kNumRW) { FOMO_RL_VARIANTS(FOMO_OCC_RL, NN) } \
    break;
    switch (sp.N) { FOMO_OCC_RLN(1) FOMO_OCC_RLN(2) FOMO_OCC_RLN(3) FOMO_OCC_RLN(4) FOMO_OCC_RLN(5) }
#undef FOMO_OCC_RLN
#undef FOMO_OCC_RL
    return 0;
  }
  if (sp.family == 2) {
#define FOMO_OCC_RW(V, NN, PP) \
  case V: return occ_rw<NN, PP>(sp);
#define FOMO_OCC_RWN(NN)                                                              \
  case NN:                                                                            \
    switch (sp.variant - kNumVariants - kNumX2) { FOMO_RW_VARIANTS(FOMO_OCC_RW, NN) } \
    break;
    switch (sp.N) { FOMO_OCC_RWN(1) FOMO_OCC_RWN(2) FOMO_OCC_RWN(3) FOMO_OCC_RWN(4) FOMO_OCC_RWN(5) }
#undef FOMO_OCC_RWN
#undef FOMO_OCC_RW
    return 0;
  }
  if (sp.family == 1) {
#define FOMO_OCC_X2(V, NN, PP) \
  case V: return occ_x2<NN, PP>(sp);
#define FOMO_OCC_X2N(NN)                                                     \
  case NN:                                                                   \
    switch (sp.variant - kNumVariants) { FOMO_X2_VARIANTS(FOMO_OCC_X2, NN) } \
    break;
    switch (sp.N) { FOMO_OCC_X2N(1) FOMO_OCC_X2N(2) FOMO_OCC_X2N(3) FOMO_OCC_X2N(4) FOMO_OCC_X2N(5) }
#undef FOMO_OCC_X2N
#undef FOMO_OCC_X2
    return 0;
  }
#define FOMO_OCC_V(V, NN, NT, R, P) \
  case V: return occ_v<NN, NT, R, P>(sp);
#define FOMO_OCC_N(NN)                                     \
  case NN:                                                 \
    switch (sp.variant) { FOMO_SWEEP_VARIANTS(FOMO_OCC_V, NN) } \
    break;
  switch (sp.N) { FOMO_OCC_N(1) FOMO_OCC_N(2) FOMO_OCC_N(3) FOMO_OCC_N(4) FOMO_OCC_N(5) }
#undef FOMO_OCC_N
#undef FOMO_OCC_V
  return 0;
}

cudaError_t launch_sweep_elastic(cudaStream_t st, const SweepPlan& sp, int set, const Coef& c,
                                 float dtx, float dtz, const HabcDev& h, const ElFields& a,
                                 const ElMat& m, const ElOut& o, int* err, const ElOut16* o16) {
  if (sp.h16 != (o16 != nullptr)) return cudaErrorInvalidValue;
  if (sp.family == 5) {
    const PairPack mp{reinterpret_cast<const float4*>(m.ppack),
                      reinterpret_cast<const float4*>(m.ppack) +
                          (long long)(sp.gm.nz + 2 * kPairRowPad) * m.ppack_pitch,
                      reinterpret_cast<const float2*>(m.ppack +
                                                      8LL * (sp.gm.nz + 2 * kPairRowPad) *
                                                          m.ppack_pitch),
                      m.ppack_pitch};
    const PairOut po{reinterpret_cast<float2*>(o.vx), reinterpret_cast<float2*>(o.vz),
                     reinterpret_cast<float2*>(o.txx), reinterpret_cast<float2*>(o.tzz),
                     reinterpret_cast<float2*>(o.txz)};
    if (!m.ppack) return cudaErrorInvalidValue;
    return launch_pair_elastic(st, sp, sp.variant - kPairBase, set,
                               make_pair_coef(c, dtx, dtz, h), h, mp, po, err);
  }
  if (sp.family == 4) {
    switch (sp.N) {
      case 1: return launch_ws_n<1>(st, sp, set, c, dtx, dtz, h, m, o, o16, err);
      case 2: return launch_ws_n<2>(st, sp, set, c, dtx, dtz, h, m, o, o16, err);
      case 3: return launch_ws_n<3>(st, sp, set, c, dtx, dtz, h, m, o, o16, err);
      case 4: return launch_ws_n<4>(st, sp, set, c, dtx, dtz, h, m, o, o16, err);
      case 5: return launch_ws_n<5>(st, sp, set, c, dtx, dtz, h, m, o, o16, err);
    }
    return cudaErrorInvalidValue;
  }
  if (sp.family == 3) {
    switch (sp.N) {
      case 1: return launch_rl_n<1>(st, sp, set, c, dtx, dtz, h, m, o, err);
      case 2: return launch_rl_n<2>(st, sp, set, c, dtx, dtz, h, m, o, err);
      case 3: return launch_rl_n<3>(st, sp, set, c, dtx, dtz, h, m, o, err);
      case 4: return launch_rl_n<4>(st, sp, set, c, dtx, dtz, h, m, o, err);
      case 5: return launch_rl_n<5>(st, sp, set, c, dtx, dtz, h, m, o, err);
    }
    return cudaErrorInvalidValue;
  }
  if (sp.family == 2) {
    switch (sp.N) {
      case 1: return launch_rw_n<1>(st, sp, set, c, dtx, dtz, h, m, o, err);
      case 2: return launch_rw_n<2>(st, sp, set, c, dtx, dtz, h, m, o, err);
      case 3: return launch_rw_n<3>(st, sp, set, c, dtx, dtz, h, m, o, err);
      case 4: return launch_rw_n<4>(st, sp, set, c, dtx, dtz, h, m, o, err);
      case 5: return launch_rw_n<5>(st, sp, set, c, dtx, dtz, h, m, o, err);
    }
    return cudaErrorInvalidValue;
  }
  if (sp.family == 1) {
    switch (sp.N) {
      case 1: return launch_x2_n<1>(st, sp, set, c, dtx, dtz, h, m, o, err);
      case 2: return launch_x2_n<2>(st, sp, set, c, dtx, dtz, h, m, o, err);
      case 3: return launch_x2_n<3>(st, sp, set, c, dtx, dtz, h, m, o, err);
      case 4: return launch_x2_n<4>(st, sp, set, c, dtx, dtz, h, m, o, err);
      case 5: return launch_x2_n<5>(st, sp, set, c, dtx, dtz, h, m, o, err);
    }
    return cudaErrorInvalidValue;
  }
  switch (sp.N) {
    case 1: return launch_n<1>(st, sp, set, c, dtx, dtz, h, a, m, o, err);
    case 2: return launch_n<2>(st, sp, set, c, dtx, dtz, h, a, m, o, err);
    case 3: return launch_n<3>(st, sp, set, c, dtx, dtz, h, a, m, o, err);
    case 4: return launch_n<4>(st, sp, set, c, dtx, dtz, h, a, m, o, err);
    case 5: return launch_n<5>(st, sp, set, c, dtx, dtz, h, a, m, o, err);
  }
  return cudaErrorInvalidValue;
}

}  // namespace fomo
