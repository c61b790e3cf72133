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

namespace fomo {
namespace {

__device__ __forceinline__ uint32_t s_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(s_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(s_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tma_load_3d(float* dst, const CUtensorMap* map, int x, int y,
                                            int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(s_addr(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(s_addr(bar))
      : "memory");
}

// Bounded wait: gives up after 2^22 polls (about a second), records the failure.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err) {
  for (int spin = 0; spin < (1 << 22); ++spin)
    if (mbar_try_wait(bar, parity)) return true;
  atomicOr(err, 1);
  return false;
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
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
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

int pick_kernel_2d(int phys, int N, int nxp, int nzp, int ns) {
  (void)N;
  (void)nxp;
  (void)nzp;
  (void)ns;
  return phys == 1 && encoder() ? FOMO_KERNEL_SINGLE_SWEEP : FOMO_KERNEL_TWO_PHASE;
}

bool sweep2d_supported(int phys, int N) { return phys == 1 && N >= 1 && N <= 5 && encoder(); }

int sweep_num_variants() { return kNumVariants; }

// Builds the work decomposition and the six tensor maps (3 stress fields x 2
// ping-pong sets).  variant selects (threads, rows per chunk, prefetch depth);
// TX is the strip width (multiple of 4).
cudaError_t make_sweep_plan(SweepPlan& sp, int N, int variant, int TX, int per_sm, const Geo2& g,
                            int ns, float* const stress_sets[2][3], float frame_weight,
                            long long* d_bounds, cudaStream_t st) {
  auto enc = encoder();
  if (!enc) return cudaErrorNotSupported;
  if (variant < 0 || variant >= kNumVariants || per_sm < 1) return cudaErrorInvalidValue;
  const int NT = kVariants[variant].NT, R = kVariants[variant].R;
  const int M = N, HS = halo_x(M);
  if (TX < 8 || TX + 2 * M + 4 > NT || (TX & 3)) return cudaErrorInvalidValue;
  const int walign = 32 / R;  // R rows of W floats = a multiple of 128 bytes (TMA destination)
  int W = (TX + 2 * HS + walign - 1) / walign * walign;
  if (W > 256) return cudaErrorInvalidValue;
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
  sp.gm.ns = ns;
  sp.smem = smem_for(N, variant, W, g.nbc + 3);
  const int bps = sweep_blocks_per_sm(sp);
  if (bps < 1) return cudaErrorInvalidConfiguration;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  sp.per_sm = std::min(per_sm, bps);
  const long long rows = (long long)sp.gm.nstrip * ns * g.nz;
  sp.grid = (int)std::max(1LL, std::min({(long long)sp.per_sm * nsm, rows, (long long)kMaxGrid}));
  sp.frame_weight = frame_weight;
  // Cost-balanced split of the flattened (strip, shot, row) space: a row of a
  // strip costs 1 + frame_weight * (fraction of its cells in the HABC frame).
  {
    std::vector<double> strip_frac(sp.gm.nstrip);
    for (int k = 0; k < sp.gm.nstrip; ++k) {
      int nf = 0;
      for (int x = k * TX; x < std::min(g.nx, (k + 1) * TX); ++x)
        nf += (x >= 1 && x <= g.nx - 2 && (x <= g.nbc || x >= g.nx - 1 - g.nbc)) ? 1 : 0;
      strip_frac[k] = (double)nf / TX;
    }
    auto row_cost = [&](int strip, int z) {
      const bool band = z >= 1 && z <= g.nz - 2 && (z <= g.nbc || z >= g.nz - 1 - g.nbc);
      return 1.0 + frame_weight * (band ? 1.0 : strip_frac[strip]);
    };
    double shot_cost = 0.0;
    for (int k = 0; k < sp.gm.nstrip; ++k)
      for (int z = 0; z < g.nz; ++z) shot_cost += row_cost(k, z);
    const double total = shot_cost * ns;
    std::vector<long long> b(sp.grid + 1, rows);
    b[0] = 0;
    double acc = 0.0;
    int next = 1;
    for (long long r = 0; r < rows && next < sp.grid; ++r) {
      const long long item = r / g.nz;
      acc += row_cost((int)(item % sp.gm.nstrip), (int)(r - item * g.nz));
      while (next < sp.grid && acc >= total * next / sp.grid) b[next++] = r + 1;
    }
    cudaError_t e = cudaMemcpyAsync(d_bounds, b.data(), sizeof(long long) * b.size(),
                                    cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    // the host vector dies with this scope: the copy above must have finished
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    sp.d_bounds = d_bounds;
  }
  for (int s = 0; s < 2; ++s)
    for (int f = 0; f < 3; ++f) {
      cuuint64_t dims[3] = {(cuuint64_t)g.nx, (cuuint64_t)g.nz, (cuuint64_t)ns};
      cuuint64_t strides[2] = {(cuuint64_t)g.ld * 4, (cuuint64_t)g.plane * 4};
      cuuint32_t box[3] = {(cuuint32_t)W, (cuuint32_t)R, 1};
      cuuint32_t es[3] = {1, 1, 1};
      CUresult r = enc(&sp.tm[s][f], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, stress_sets[s][f], dims,
                       strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                       CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    }
  return cudaSuccess;
}

int sweep_tx_candidates(int variant, int N, int* out, int max_out) {
  // the widest strip whose v' columns (TX + 2M + 4) fill the CTA's threads
  int n = 0;
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

int sweep_blocks_per_sm(const SweepPlan& sp) {
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
                                 const ElMat& m, const ElOut& o, int* err) {
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
