// sweep2d_pair.cu -- single-sweep elastic time step over PAIRS of shots, in
// Blackwell's packed FP32 instructions (the "pair" variants of the sweep).
//
// The shots of elastic2d_batch share one model, so two shots advance together:
// each wavefield is stored shot-pair-interleaved -- element (x, z) of pair p is
// the float2 {shot 2p, shot 2p+1} -- and every stencil term, update and Higdon
// operation is one add/sub/mul/fma.rn.f32x2 on both shots.  Those round each
// lane to nearest like the scalar instruction, so each lane is the canonical
// scalar sequence of the oracle, bit for bit.  The materials, the HABC
// classification, the weights and every address are shared by the two shots:
// per shot-cell the thread issues about half the instructions of the one-shot
// sweep, and the two lanes never need shuffling (the operands of a pair are
// always one 8-byte element).
//
// March (elastic2d/batch.jl:38-154, fused_kernels.jl:21-124; kernels_det.jl:
// 22-57 for the Higdon values).  A CTA owns a strip of TX columns of one pair
// and a range of rows, and walks down z two rows per iteration with two roles
// of NV threads, one column each:
//   velocity threads hold the txz / tzz z-windows in registers, read txx / txz
//     x-windows from TMA-staged rows, and produce v' (update) and v'' (HABC),
//     which goes to HBM (B.v) and to a shared v'' ring;
//   stress threads hold the v''x / v''z z-windows, read v'' x-windows from the
//     ring, and produce s' and s'' (HABC) -> B.stress.
// The A-set rows come by TMA into rings guarded by mbarriers (bounded waits);
// the roles meet once per iteration at a CTA barrier (plus one role-local
// barrier for the v' / s' rows the x-band Higdon reads from neighbour columns).
// Persistent CTAs take contiguous ranges of the flattened (pair, strip, row)
// space, as the one-shot sweeps do.  Rows outside the grid come from TMA's
// zero fill and only feed discarded results (window warm-up rows, halo
// columns).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>

#include "sweep2d.cuh"
#include "tma.cuh"

namespace fomo {
namespace {

// ---- packed FP32 pair arithmetic (round to nearest even per lane) ----------
__device__ __forceinline__ float2 p_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 p_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 p_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b as fma(-1, b, a): -1 * b is exact, so the fma rounds a - b once, as
// sub.rn.f32x2 does (signed zeros included).  m1 = {-1, -1}, kept in a
// register pair by the caller.
__device__ __forceinline__ float2 p_sub(float2 m1, float2 a, float2 b) {
  return __ffma2_rn(m1, b, a);
}
__device__ __forceinline__ float2 lo2(const float4& v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4& v) { return make_float2(v.z, v.w); }

// Higdon terms (kernels_det.jl:22-57), the canonical sequence of
// higdon_side / higdon_edge / higdon_corner on both lanes.  wt = {w, w, 1-w, 1-w}.
__device__ __forceinline__ float2 ph_side(const PairCoef& k, float2 f_nb, float2 fo_p, float2 fo_nb) {
  float2 s = p_mul(k.nq, f_nb);
  s = p_fma(k.nqt, fo_p, s);
  return p_fma(k.nqxt, fo_nb, s);
}
__device__ __forceinline__ float2 ph_edge(const float4& wt, float2 fc, float2 s) {
  return p_fma(lo2(wt), fc, p_mul(hi2(wt), s));
}
__device__ __forceinline__ float2 ph_corner(const float4& wt, float2 fc, float2 sx, float2 sz) {
  return p_fma(lo2(wt), fc, p_mul(p_mul(hi2(wt), make_float2(0.5f, 0.5f)), p_add(sx, sz)));
}

// The value as the result of an (empty) asm statement: the compiler keeps a
// duplicated constant pair in registers instead of rebuilding it from the
// constant bank before every packed instruction that reads it.
__device__ __forceinline__ float2 pinned(float2 v) {
  asm volatile("" : "+f"(v.x), "+f"(v.y));
  return v;
}

// (a + d) mod n for a in [0, n), 0 <= d < n
__device__ __forceinline__ int ring(int a, int d, int n) {
  const int t = a + d;
  return t >= n ? t - n : t;
}

}  // namespace

// Shared-memory layout and strip geometry of a pair variant (units: float2).
template <int N, int NV, int P>
struct PairShape {
  static constexpr int M = N;
  static constexpr int HV = (N + 3) & ~1;            // v' halo >= N + 2, even (TMA x alignment)
  static constexpr int TN = 2 * N + 2 - HV;          // extra stress halo left of the v' window
  static constexpr int TXMAX = (NV - HV - N - 2) & ~1;
  static constexpr int W = (TN + HV + TXMAX + 2 * N + 2 + 7) & ~7;  // TMA box width
  static constexpr int NZ = P + 1;      // z-entry / x-window stream slots
  static constexpr int NO = P + 2;      // old-stress / A.v stream slots (and mbarriers)
  static constexpr int LVV = M + 4;     // v'' ring rows: rows q .. zv live at once
  static constexpr int O_Z = 0;                    // [NZ][txz, tzz][2][W]       rows zv+M, +1
  static constexpr int O_X = O_Z + NZ * 4 * W;     // [NZ][txx, txz][2][W]       rows zv, zv+1
  static constexpr int O_O = O_X + NZ * 4 * W;     // [NO][txx, tzz, txz][2][W]  rows q, q+1
  static constexpr int O_V = O_O + NO * 6 * W;     // [NO][vx, vz][2][W]         rows zv, zv+1
  static constexpr int O_VP = O_V + NO * 4 * W;    // [vx, vz][4][W]   v'
  static constexpr int O_VV = O_VP + 8 * W;        // [vx, vz][LVV][W] v''
  static constexpr int O_SP = O_VV + 2 * LVV * W;  // [xx, zz, xz][4][W] s'
  static constexpr int O_WT = O_SP + 12 * W;       // [3][wstride] float4 {w, w, 1-w, 1-w}
  static_assert(W <= 256, "TMA box width");
  static_assert((2 * W * 8) % 128 == 0, "two-row boxes keep 128-byte alignment");
};

template <int N, int NV, int P, int MINB>
__global__ void __launch_bounds__(2 * NV, MINB)
    k_el_pair(const __grid_constant__ CUtensorMap tm_xx, const __grid_constant__ CUtensorMap tm_zz,
              const __grid_constant__ CUtensorMap tm_xz, const __grid_constant__ CUtensorMap tm_vx,
              const __grid_constant__ CUtensorMap tm_vz, SweepGeom gm, PairCoef kp, HabcDev h,
              PairPack mp, PairOut o, const long long* __restrict__ bounds,
              int* __restrict__ err) {
  using S = PairShape<N, NV, P>;
  static_assert(NV % 32 == 0, "each role is whole warps: named barriers count whole warps");
  PairCoef k;
#pragma unroll
  for (int l = 0; l < 5; ++l) k.a[l] = pinned(kp.a[l]);
  k.dtx = pinned(kp.dtx);
  k.dtz = pinned(kp.dtz);
  k.nq = pinned(kp.nq);
  k.nqt = pinned(kp.nqt);
  k.nqxt = pinned(kp.nqxt);
  const float2 m1 = pinned(make_float2(-1.0f, -1.0f));
  constexpr int NT = 2 * NV;
  constexpr int W = S::W, M = N, TN = S::TN, HV = S::HV;
  constexpr int NZ = S::NZ, NO = S::NO, LVV = S::LVV;
  constexpr int WN = 2 * M + 2;  // z-window rows
  extern __shared__ __align__(128) float2 sm2[];
  float2* s_z = sm2 + S::O_Z;
  float2* s_x = sm2 + S::O_X;
  float2* s_o = sm2 + S::O_O;
  float2* s_v = sm2 + S::O_V;
  float2* s_vp = sm2 + S::O_VP;
  float2* s_vv = sm2 + S::O_VV;
  float2* s_sp = sm2 + S::O_SP;
  float4* s_wt = reinterpret_cast<float4*>(sm2 + S::O_WT);
  const int nwt = 3 * h.wstride;
  uint64_t* bars = reinterpret_cast<uint64_t*>(s_wt + nwt);  // [NO]

  const int tid = threadIdx.x;
  const bool vel = tid < NV;  // warp-uniform role
  const int c = vel ? tid : tid - NV;  // the thread's column in the window
  const int TX = gm.TX;
  const int nx = gm.nx, nz = gm.nz, nbc = gm.nbc;
  for (int q = tid; q < S::O_WT; q += NT) sm2[q] = make_float2(0.0f, 0.0f);
  for (int q = tid; q < nwt; q += NT) {
    const float w = __ldg(h.wtab + q);
    const float om = __fsub_rn(1.0f, w);
    s_wt[q] = make_float4(w, w, om, om);
  }
  if (tid == 0) {
    for (int q = 0; q < NO; ++q) tma::mbar_init(&bars[q], 1);
    tma::mbar_init_fence();
  }
  __syncthreads();
  // Row classification (kernels_fused.jl:28-52; interior of fused_kernels.jl:48).
  // Frame cells lie within nbc of an edge, so dist <= nbc < wstride: every
  // weight lookup below is in the table.
  auto zside = [&](int z) { return z <= nbc ? 1 : (z >= nz - 1 - nbc ? -1 : 0); };
  auto zframe = [&](int z) { return z >= 1 && z <= nz - 2; };
  auto zinner = [&](int z) { return z >= M && z < nz - M; };
  auto zdist = [&](int z) { return min(z, nz - 1 - z); };
  const bool do_v = c >= HV - N - 2 && c < HV + TX + N + 2;  // v' columns
  const bool do_s = c >= HV - 1 && c < HV + TX + 1;          // s' columns
  const bool do_o = c >= HV && c < HV + TX;                  // output columns
  const long long r_lo = bounds[blockIdx.x];
  const long long r_hi = bounds[blockIdx.x + 1];

  // One segment = a run of rows [za, zb) of one (pair, strip); both roles walk
  // the same segments and iterations.
  struct Seg {
    int za, zb, pair, XV, XT, x, zv0, I, xsd, xds, cn;
    bool xin, xfr, o_any, hbx;
    long long obase;
  };
  auto segment = [&](long long& r, Seg& g) {
    const long long item = r / nz;
    g.za = (int)(r - item * nz);
    g.zb = (int)min((long long)nz, g.za + (r_hi - r));
    r += g.zb - g.za;
    const int strip = (int)(item % gm.nstrip);
    g.pair = (int)(item / gm.nstrip);
    g.XV = strip * TX - HV;
    g.XT = g.XV - TN;
    g.x = g.XV + c;
    g.xin = g.x >= M && g.x < nx - M;
    g.xsd = g.x <= nbc ? 1 : (g.x >= nx - 1 - nbc ? -1 : 0);
    g.xfr = g.x >= 1 && g.x <= nx - 2;
    g.xds = min(g.x, nx - 1 - g.x);
    g.cn = min(max(c + g.xsd, 0), W - 1);
    g.o_any = do_o && g.x < nx;
    // the window reaches an x-band: only then do threads read neighbour columns'
    // v' / s' rows (x-side Higdon), which need the shared rows and the
    // role-local barrier (CTA-uniform per segment)
    g.hbx = g.XV <= nbc || g.XV + NV - 1 >= nx - 1 - nbc;
    g.obase = (long long)g.pair * gm.plane + g.x;
    g.zv0 = g.za - 2 - 3 * M;  // M warm-up iterations fill the windows
    g.I = (g.zb - g.za + 4 + 4 * M + 1) / 2 + 1;
  };
  const long long pcol = (long long)kPairColPad + c;  // + XV per segment

  if (vel) {
    // ======================= velocity role =======================
    int gb = 0;
    bool live = true;
    for (long long r = r_lo; r < r_hi;) {
      Seg g;
      segment(r, g);
      auto issue = [&](int q) {
        const int gq = gb + q, zs = gq % NZ, os = gq % NO;
        uint64_t* bar = &bars[os];
        const int zr = g.zv0 + 2 * q;
        tma::mbar_expect_tx(bar, 9u * 2u * W * 8u);
        tma::load_3d(s_z + (zs * 4 + 0) * W, &tm_xz, g.XT, zr + M, g.pair, bar);
        tma::load_3d(s_z + (zs * 4 + 2) * W, &tm_zz, g.XT, zr + M, g.pair, bar);
        tma::load_3d(s_x + (zs * 4 + 0) * W, &tm_xx, g.XT, zr, g.pair, bar);
        tma::load_3d(s_x + (zs * 4 + 2) * W, &tm_xz, g.XT, zr, g.pair, bar);
        tma::load_3d(s_o + (os * 6 + 0) * W, &tm_xx, g.XT, zr - 3 - M, g.pair, bar);
        tma::load_3d(s_o + (os * 6 + 2) * W, &tm_zz, g.XT, zr - 3 - M, g.pair, bar);
        tma::load_3d(s_o + (os * 6 + 4) * W, &tm_xz, g.XT, zr - 3 - M, g.pair, bar);
        tma::load_3d(s_v + (os * 4 + 0) * W, &tm_vx, g.XV, zr, g.pair, bar);
        tma::load_3d(s_v + (os * 4 + 2) * W, &tm_vz, g.XV, zr, g.pair, bar);
      };
      tma::bar_sync(1, NT);  // the previous segment's readers are done with every ring
      if (tid == 0 && live) {
        tma::fence_proxy_async();
        for (int q = 0; q <= P && q < g.I; ++q) issue(q);
      }
      float2 wxz[WN], wzz[WN];
#pragma unroll
      for (int q = 0; q < WN; ++q) wxz[q] = wzz[q] = make_float2(0.0f, 0.0f);
      float2* ovx = o.vx + g.obase + (long long)(g.zv0 - 1) * gm.ld;
      float2* ovz = o.vz + g.obase + (long long)(g.zv0 - 1) * gm.ld;
      float2 vpp[2][2];  // previous iteration's v' rows [field][row]
#pragma unroll
      for (int f = 0; f < 2; ++f) vpp[f][0] = vpp[f][1] = make_float2(0.0f, 0.0f);
      const float4* pv = mp.v + (long long)(g.zv0 + kPairRowPad) * mp.pitch + pcol + g.XV;
      float4 mv0 = __ldg(pv), mv1 = __ldg(pv + mp.pitch);
      pv += 2 * mp.pitch;
      int zs = gb % NZ, os = gb % NO, osp = (gb + NO - 1) % NO;
      uint32_t ph = (uint32_t)((gb / NO) & 1);
      int vw = 0;  // v'' ring row of row zv - 1
      for (int i = 0; i < g.I; ++i) {
        const int zv = g.zv0 + 2 * i;
        if (live) live = tma::mbar_wait_bounded(&bars[os], ph, err) && live;
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
          wxz[2 * M + rr] = s_z[(zs * 4 + rr) * W + c + TN];
          wzz[2 * M + rr] = s_z[(zs * 4 + 2 + rr) * W + c + TN];
        }
        float2 vpc[2][2];  // v' rows zv, zv+1 [field][row]
        if (do_v) {
#pragma unroll
          for (int rr = 0; rr < 2; ++rr) {
            const float2* rxx = s_x + (zs * 4 + rr) * W + c + TN;
            const float2* rxz = s_x + (zs * 4 + 2 + rr) * W + c + TN;
            float2 dxx = make_float2(0.0f, 0.0f), dxzx = dxx, dxzz = dxx, dzz = dxx;
#pragma unroll
            for (int l = 1; l <= N; ++l) {
              const float2 a = k.a[l - 1];
              dxx = p_fma(a, p_sub(m1, rxx[l - 1], rxx[-l]), dxx);
              dxzx = p_fma(a, p_sub(m1, rxz[l], rxz[1 - l]), dxzx);
              dxzz = p_fma(a, p_sub(m1, wxz[rr + M + l - 1], wxz[rr + M - l]), dxzz);
              dzz = p_fma(a, p_sub(m1, wzz[rr + M + l], wzz[rr + M - l + 1]), dzz);
            }
            float2 ux = s_v[(os * 4 + rr) * W + c];
            float2 uz = s_v[(os * 4 + 2 + rr) * W + c];
            if (zinner(zv + rr) && g.xin) {
              const float4 mv = rr ? mv1 : mv0;
              ux = p_fma(lo2(mv), p_fma(k.dtx, dxx, p_mul(k.dtz, dxzz)), ux);
              uz = p_fma(hi2(mv), p_fma(k.dtx, dxzx, p_mul(k.dtz, dzz)), uz);
            }
            vpc[0][rr] = ux;
            vpc[1][rr] = uz;
            if (g.hbx) {
              const int pr = (2 * i + rr) & 3;  // v' ring row of zv + rr
              s_vp[pr * W + c] = ux;
              s_vp[(4 + pr) * W + c] = uz;
            }
          }
        }
#pragma unroll
        for (int q = 0; q < 2 * M; ++q) {
          wxz[q] = wxz[q + 2];
          wzz[q] = wzz[q + 2];
        }
        if (g.hbx) tma::bar_sync(2, NV);  // this iteration's v' rows are in s_vp
        // v'' rows zv-1 (rr = 0) and zv (rr = 1); v' rows zv-2 .. zv+1 are in vpp / vpc
        if (do_v) {
#pragma unroll
          for (int rr = 0; rr < 2; ++rr) {
            const int qv = zv - 1 + rr;
            float2 vv[2] = {rr ? vpc[0][0] : vpp[0][1], rr ? vpc[1][0] : vpp[1][1]};
            const int zsd = zside(qv);
            if (zframe(qv) && g.xfr && (zsd != 0 || g.xsd != 0)) {
              // A.v row qv (rows zv-2, zv-1 sit in the previous slot, zv, zv+1 in this one)
              const float2* vo_r = s_v + ((rr ? os : osp) * 4 + (rr ? 0 : 1)) * W;
              if (g.xsd == 0) {
                // z-side edge: neighbour row qv + zsd
                const int zd = zdist(qv);
                const float2* vz_r = s_v + ((zsd > 0 ? os : osp) * 4 + rr) * W + c;
#pragma unroll
                for (int f = 0; f < 2; ++f) {
                  const float2 vn = zsd > 0 ? vpc[f][rr] : vpp[f][rr];
                  vv[f] = ph_edge(s_wt[f * h.wstride + zd], vv[f],
                                  ph_side(k, vn, vo_r[f * 2 * W + c], vz_r[f * 2 * W]));
                }
              } else {
                const float2* vp_r = s_vp + ((2 * i - 1 + rr) & 3) * W;  // v' row qv
                if (zsd == 0) {
                  // x-side edge: neighbour column x + xsd
#pragma unroll
                  for (int f = 0; f < 2; ++f)
                    vv[f] = ph_edge(s_wt[f * h.wstride + g.xds], vv[f],
                                    ph_side(k, vp_r[f * 4 * W + g.cn], vo_r[f * 2 * W + c],
                                            vo_r[f * 2 * W + g.cn]));
                } else {
                  // corner: both sides
                  const int dist = min(g.xds, zdist(qv));
                  const float2* vz_r = s_v + ((zsd > 0 ? os : osp) * 4 + rr) * W + c;
#pragma unroll
                  for (int f = 0; f < 2; ++f) {
                    const float2 fo = vo_r[f * 2 * W + c];
                    const float2 vn = zsd > 0 ? vpc[f][rr] : vpp[f][rr];
                    const float2 hx = ph_side(k, vp_r[f * 4 * W + g.cn], fo, vo_r[f * 2 * W + g.cn]);
                    const float2 hz = ph_side(k, vn, fo, vz_r[f * 2 * W]);
                    vv[f] = ph_corner(s_wt[f * h.wstride + dist], vv[f], hx, hz);
                  }
                }
              }
            }
            const int vr = ring(vw, rr, LVV);  // v'' ring row of qv
            s_vv[vr * W + c] = vv[0];
            s_vv[(LVV + vr) * W + c] = vv[1];
            if (g.o_any && qv >= g.za && qv < g.zb) {
              ovx[rr ? gm.ld : 0] = vv[0];
              ovz[rr ? gm.ld : 0] = vv[1];
            }
          }
        }
        ovx += 2 * gm.ld;
        ovz += 2 * gm.ld;
#pragma unroll
        for (int f = 0; f < 2; ++f) {
          vpp[f][0] = vpc[f][0];
          vpp[f][1] = vpc[f][1];
        }
        mv0 = __ldg(pv);
        mv1 = __ldg(pv + mp.pitch);
        pv += 2 * mp.pitch;
        tma::bar_sync(1, NT);  // v'' rows zv-1, zv are in the ring; slots of i-1 are free
        if (tid == 0 && live && i + 1 + P < g.I) {
          tma::fence_proxy_async();
          issue(i + 1 + P);
        }
        vw = ring(vw, 2, LVV);
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
      tma::bar_sync(1, NT);  // pairs with the velocity role's segment barrier
      float2 wvx[WN], wvz[WN];
#pragma unroll
      for (int q = 0; q < WN; ++q) wvx[q] = wvz[q] = make_float2(0.0f, 0.0f);
      float2* ot0 = o.txx + g.obase + (long long)(g.zv0 - 4 - M) * gm.ld;
      float2* ot1 = o.tzz + g.obase + (long long)(g.zv0 - 4 - M) * gm.ld;
      float2* ot2 = o.txz + g.obase + (long long)(g.zv0 - 4 - M) * gm.ld;
      float2 spp[3][2];  // previous iteration's s' rows [field][row]
#pragma unroll
      for (int f = 0; f < 3; ++f) spp[f][0] = spp[f][1] = make_float2(0.0f, 0.0f);
      const long long prow0 = (long long)(g.zv0 - 3 - M + kPairRowPad) * mp.pitch + pcol + g.XV;
      const float4* pl = mp.l + prow0;
      const float2* pu = mp.mu + prow0;
      float4 ml0 = __ldg(pl), ml1 = __ldg(pl + mp.pitch);
      float2 mu0 = __ldg(pu), mu1 = __ldg(pu + mp.pitch);
      pl += 2 * mp.pitch;
      pu += 2 * mp.pitch;
      int os = gb % NO, osp = (gb + NO - 1) % NO;
      uint32_t ph = (uint32_t)((gb / NO) & 1);
      // v'' ring rows: z-window entries zv-3, zv-2 (written last iteration) and
      // the x-window rows q, q+1 (q = zv-3-M)
      int ve = LVV - 2, vb = LVV - 2 - M;
      for (int i = 0; i < g.I; ++i) {
        const int zv = g.zv0 + 2 * i, q = zv - 3 - M;
        if (live) live = tma::mbar_wait_bounded(&bars[os], ph, err) && live;
        // the v'' window advances by two rows: rows q-M .. q+M-1 move down, and
        // v'' rows q+M, q+M+1 (= zv-3, zv-2) enter at the top
        if (i > 0) {
#pragma unroll
          for (int t = 0; t < 2 * M; ++t) {
            wvx[t] = wvx[t + 2];
            wvz[t] = wvz[t + 2];
          }
#pragma unroll
          for (int rr = 0; rr < 2; ++rr) {
            const int vr = ring(ve, rr, LVV);
            wvx[2 * M + rr] = s_vv[vr * W + c];
            wvz[2 * M + rr] = s_vv[(LVV + vr) * W + c];
          }
        }
        float2 spc[3][2];  // s' rows q, q+1 [field][row]
        if (do_s) {
#pragma unroll
          for (int rr = 0; rr < 2; ++rr) {
            const int vr = ring(vb, rr, LVV);  // v'' ring row of q + rr
            const float2* rvx = s_vv + vr * W + c;
            const float2* rvz = s_vv + (LVV + vr) * W + c;
            float2 dvxdx = make_float2(0.0f, 0.0f), dvzdx = dvxdx, dvxdz = dvxdx, dvzdz = dvxdx;
#pragma unroll
            for (int l = 1; l <= N; ++l) {
              const float2 a = k.a[l - 1];
              dvxdx = p_fma(a, p_sub(m1, rvx[l], rvx[1 - l]), dvxdx);
              dvzdx = p_fma(a, p_sub(m1, rvz[l - 1], rvz[-l]), dvzdx);
              dvxdz = p_fma(a, p_sub(m1, wvx[rr + M + l], wvx[rr + M - l + 1]), dvxdz);
              dvzdz = p_fma(a, p_sub(m1, wvz[rr + M + l - 1], wvz[rr + M - l]), dvzdz);
            }
            float2 sxx = s_o[(os * 6 + 0 + rr) * W + c + TN];
            float2 szz = s_o[(os * 6 + 2 + rr) * W + c + TN];
            float2 sxz = s_o[(os * 6 + 4 + rr) * W + c + TN];
            if (zinner(q + rr) && g.xin) {
              const float4 ml = rr ? ml1 : ml0;  // {lam, lam, l2m, l2m}
              const float2 mu = rr ? mu1 : mu0;
              const float2 ex = p_mul(dvxdx, k.dtx), ez = p_mul(dvzdz, k.dtz);
              sxx = p_add(sxx, p_fma(hi2(ml), ex, p_mul(lo2(ml), ez)));
              szz = p_add(szz, p_fma(lo2(ml), ex, p_mul(hi2(ml), ez)));
              sxz = p_fma(mu, p_fma(dvxdz, k.dtz, p_mul(dvzdx, k.dtx)), sxz);
            }
            spc[0][rr] = sxx;
            spc[1][rr] = szz;
            spc[2][rr] = sxz;
            if (g.hbx) {
              const int sr = (2 * i + rr) & 3;  // s' ring row of q + rr
              s_sp[sr * W + c] = sxx;
              s_sp[(4 + sr) * W + c] = szz;
              s_sp[(8 + sr) * W + c] = sxz;
            }
          }
        }
        if (g.hbx) tma::bar_sync(3, NV);  // this iteration's s' rows are in s_sp
        // s'' rows q-1 (rr = 0) and q (rr = 1); s' rows q-2 .. q+1 are in spp / spc
        if (g.o_any) {
#pragma unroll
          for (int rr = 0; rr < 2; ++rr) {
            const int qs = q - 1 + rr;
            if (qs < g.za || qs >= g.zb) continue;
            float2 v[3];
#pragma unroll
            for (int f = 0; f < 3; ++f) v[f] = rr ? spc[f][0] : spp[f][1];
            const int zsd = zside(qs);
            if (zframe(qs) && g.xfr && (zsd != 0 || g.xsd != 0)) {
              // old stress row qs (rows q-2, q-1 in the previous slot, q, q+1 in this one)
              const float2* so_r = s_o + ((rr ? os : osp) * 6 + (rr ? 0 : 1)) * W + TN;
              if (g.xsd == 0) {
                const float4 wt = s_wt[2 * h.wstride + zdist(qs)];
                const float2* sz_r = s_o + ((zsd > 0 ? os : osp) * 6 + rr) * W + TN + c;
#pragma unroll
                for (int f = 0; f < 3; ++f) {
                  const float2 sn = zsd > 0 ? spc[f][rr] : spp[f][rr];
                  v[f] = ph_edge(wt, v[f], ph_side(k, sn, so_r[f * 2 * W + c], sz_r[f * 2 * W]));
                }
              } else {
                const float2* sp_r = s_sp + ((2 * i - 1 + rr) & 3) * W;  // s' row qs
                if (zsd == 0) {
                  const float4 wt = s_wt[2 * h.wstride + g.xds];
#pragma unroll
                  for (int f = 0; f < 3; ++f)
                    v[f] = ph_edge(wt, v[f],
                                   ph_side(k, sp_r[f * 4 * W + g.cn], so_r[f * 2 * W + c],
                                           so_r[f * 2 * W + g.cn]));
                } else {
                  const float4 wt = s_wt[2 * h.wstride + min(g.xds, zdist(qs))];
                  const float2* sz_r = s_o + ((zsd > 0 ? os : osp) * 6 + rr) * W + TN + c;
#pragma unroll
                  for (int f = 0; f < 3; ++f) {
                    const float2 fo = so_r[f * 2 * W + c];
                    const float2 sn = zsd > 0 ? spc[f][rr] : spp[f][rr];
                    const float2 hx = ph_side(k, sp_r[f * 4 * W + g.cn], fo, so_r[f * 2 * W + g.cn]);
                    const float2 hz = ph_side(k, sn, fo, sz_r[f * 2 * W]);
                    v[f] = ph_corner(wt, v[f], hx, hz);
                  }
                }
              }
            }
            const long long d = rr ? gm.ld : 0;
            ot0[d] = v[0];
            ot1[d] = v[1];
            ot2[d] = v[2];
          }
        }
        ot0 += 2 * gm.ld;
        ot1 += 2 * gm.ld;
        ot2 += 2 * gm.ld;
#pragma unroll
        for (int f = 0; f < 3; ++f) {
          spp[f][0] = spc[f][0];
          spp[f][1] = spc[f][1];
        }
        ml0 = __ldg(pl);
        ml1 = __ldg(pl + mp.pitch);
        mu0 = __ldg(pu);
        mu1 = __ldg(pu + mp.pitch);
        pl += 2 * mp.pitch;
        pu += 2 * mp.pitch;
        tma::bar_sync(1, NT);
        ve = ring(ve, 2, LVV);
        vb = ring(vb, 2, LVV);
        osp = os;
        os = os + 1 == NO ? 0 : os + 1;
        ph ^= os == 0 ? 1u : 0u;
      }
      gb += g.I;
    }
  }
}

namespace {

// Pair variants: (form 0; threads per role; TMA prefetch depth in row pairs;
// CTAs per SM the register budget targets).  Deeper prefetch keeps more HBM
// reads in flight per SM; narrower CTAs keep two or three of them resident.
#define FOMO_PAIR_VARIANTS(X, NN)                                                         \
  X(0, NN, 0, 128, 1, 2) X(1, NN, 0, 96, 2, 2) X(2, NN, 0, 96, 3, 2) X(3, NN, 0, 64, 3, 3) \
  X(4, NN, 0, 128, 3, 1)
constexpr int kPairNV[] = {128, 96, 96, 64, 128};
constexpr int kNumPair = sizeof(kPairNV) / sizeof(kPairNV[0]);
constexpr int kMaxDynSmemPair = 227 * 1024;

template <int N, int F, int NV, int P>
size_t pair_smem_bytes(int wstride) {
  static_assert(F == 0, "one kernel form");
  using S = PairShape<N, NV, P>;
  return (size_t)S::O_WT * 8 + (size_t)3 * wstride * 16 + sizeof(uint64_t) * S::NO;
}

template <int N, int F, int NV, int P, int MINB>
auto pair_kernel() {
  return k_el_pair<N, NV, P, MINB>;
}

template <int N, int F, int NV, int P, int MINB>
cudaError_t launch_p(cudaStream_t st, const SweepPlan& sp, int set, const PairCoef& k,
                     const HabcDev& h, const PairPack& mp, const PairOut& o, int* err) {
  auto kern = pair_kernel<N, F, NV, P, MINB>();
  static std::atomic<int> attr_set{0};
  if (!attr_set.load(std::memory_order_acquire)) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kMaxDynSmemPair);
    if (e != cudaSuccess) return e;
    attr_set.store(1, std::memory_order_release);
  }
  if (sp.smem > (size_t)kMaxDynSmemPair) return cudaErrorInvalidValue;
  kern<<<(unsigned)sp.grid, 2 * NV, sp.smem, st>>>(sp.tm[set][0], sp.tm[set][1], sp.tm[set][2],
                                                    sp.tm[set][3], sp.tm[set][4], sp.gm, k, h, mp,
                                                    o, sp.d_bounds, err);
  return cudaGetLastError();
}

template <int N, int F, int NV, int P, int MINB>
int occ_p(size_t smem) {
  int nb = 0;
  auto kern = pair_kernel<N, F, NV, P, MINB>();
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmemPair);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 2 * NV, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nb;
}

// Copies the five elastic planes into the pair pack (layout in sweep2d.cuh).
__global__ void k_pair_pack(int nx, int nz, int ld, ElMat m, float4* pv, float4* pl, float2* pu,
                            int pitch, long long cells) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < cells;
       q += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(q / pitch) - kPairRowPad;
    const int x = (int)(q % pitch) - kPairColPad;
    const bool in = z >= 0 && z < nz && x >= 0 && x < nx;
    const long long p = in ? (long long)z * ld + x : 0;
    const float bx = in ? m.bx[p] : 0.0f, bz = in ? m.bz[p] : 0.0f;
    const float la = in ? m.lam[p] : 0.0f, l2 = in ? m.l2m[p] : 0.0f, mu = in ? m.mut[p] : 0.0f;
    pv[q] = make_float4(bx, bx, bz, bz);
    pl[q] = make_float4(la, la, l2, l2);
    pu[q] = make_float2(mu, mu);
  }
}

// Injection then recording on the pair layout, one block per shot (the
// semantics of k_inject_record: sources added in source order by one thread,
// then the receivers sampled after the barrier).
__global__ void k_inject_record_pair(int it, int nt, long long plane, int n_src,
                                     const int* __restrict__ src_lin,
                                     const float* __restrict__ wav, float* txx, float* tzz,
                                     int n_rec, const int* __restrict__ rec_lin,
                                     const float* vx, const float* vz, float* __restrict__ s0,
                                     float* __restrict__ s1) {
  const int s = blockIdx.x;
  const long long so = (long long)(s >> 1) * 2 * plane + (s & 1);
  if (threadIdx.x == 0) {
    for (int q = 0; q < n_src; ++q) {
      const long long p = so + 2LL * src_lin[(long long)s * n_src + q];
      const float w = wav[(long long)(it - 1) * n_src + q];
      txx[p] = __fadd_rn(txx[p], w);
      tzz[p] = __fadd_rn(tzz[p], w);
    }
  }
  __syncthreads();
  const long long ob = (long long)n_rec * ((long long)(it - 1) + (long long)nt * s);
  for (int r = threadIdx.x; r < n_rec; r += blockDim.x) {
    const long long p = so + 2LL * rec_lin[r];
    if (s0) s0[ob + r] = vx[p];
    if (s1) s1[ob + r] = vz[p];
  }
}

// Columns [x0, x0 + nx) of rows [z0, z0 + nz) of one shot of a pair-layout
// field, unpitched.
__global__ void k_pair_unpack(const float* __restrict__ f, long long plane, int ld, int x0, int z0,
                              int nx, int nz, int shot, float* __restrict__ out) {
  const long long n = (long long)nx * nz;
  const long long so = (long long)(shot >> 1) * 2 * plane + (shot & 1);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const long long z = q / nx, x = q - z * nx;
    out[q] = f[so + 2 * ((z + z0) * ld + x + x0)];
  }
}

}  // namespace

int pair_num_variants() { return kNumPair; }

int pair_threads(int v) { return v >= 0 && v < kNumPair ? 2 * kPairNV[v] : 0; }

int pair_txmax(int N, int v) {
  if (v < 0 || v >= kNumPair || N < 1 || N > 5) return 0;
  const int NV = kPairNV[v];
  const int HV = (N + 3) & ~1;
  return (NV - HV - N - 2) & ~1;
}

int pair_box_width(int N, int v) {
  if (v < 0 || v >= kNumPair || N < 1 || N > 5) return 0;
  const int HV = (N + 3) & ~1, TN = 2 * N + 2 - HV;
  return (TN + HV + pair_txmax(N, v) + 2 * N + 2 + 7) & ~7;
}

size_t pair_smem(int N, int v, int wstride) {
#define FOMO_SMEM_P(V, NN, FF, NV, PP, MB) \
  case V: return pair_smem_bytes<NN, FF, NV, PP>(wstride);
#define FOMO_SMEM_PN(NN)                             \
  case NN:                                           \
    switch (v) { FOMO_PAIR_VARIANTS(FOMO_SMEM_P, NN) } \
    break;
  switch (N) { FOMO_SMEM_PN(1) FOMO_SMEM_PN(2) FOMO_SMEM_PN(3) FOMO_SMEM_PN(4) FOMO_SMEM_PN(5) }
#undef FOMO_SMEM_PN
#undef FOMO_SMEM_P
  return 0;
}

int pair_blocks_per_sm(int N, int v, size_t smem) {
#define FOMO_OCC_P(V, NN, FF, NV, PP, MB) \
  case V: return occ_p<NN, FF, NV, PP, MB>(smem);
#define FOMO_OCC_PN(NN)                             \
  case NN:                                          \
    switch (v) { FOMO_PAIR_VARIANTS(FOMO_OCC_P, NN) } \
    break;
  switch (N) { FOMO_OCC_PN(1) FOMO_OCC_PN(2) FOMO_OCC_PN(3) FOMO_OCC_PN(4) FOMO_OCC_PN(5) }
#undef FOMO_OCC_PN
#undef FOMO_OCC_P
  return 0;
}

int pair_pack_pitch(int nx) { return (nx + kPairColPad + 2 * 256 + 15) & ~15; }

size_t pair_pack_floats(int nx, int nz) {
  return (size_t)(nz + 2 * kPairRowPad) * pair_pack_pitch(nx) * 10;
}

cudaError_t build_pair_pack(cudaStream_t st, const Geo2& g, const ElMat& m, float* dst,
                            PairPack& out) {
  if (!dst || (reinterpret_cast<uintptr_t>(dst) & 15)) return cudaErrorInvalidValue;
  const int pitch = pair_pack_pitch(g.nx);
  const long long cells = (long long)(g.nz + 2 * kPairRowPad) * pitch;
  float4* pv = reinterpret_cast<float4*>(dst);
  float4* pl = pv + cells;
  float2* pu = reinterpret_cast<float2*>(pl + cells);
  k_pair_pack<<<1184, 256, 0, st>>>(g.nx, g.nz, g.ld, m, pv, pl, pu, pitch, cells);
  out = PairPack{pv, pl, pu, pitch};
  return cudaGetLastError();
}

PairCoef make_pair_coef(const Coef& c, float dtx, float dtz, const HabcDev& h) {
  PairCoef k;
  for (int l = 0; l < 5; ++l) k.a[l] = make_float2(c.a[l], c.a[l]);
  k.dtx = make_float2(dtx, dtx);
  k.dtz = make_float2(dtz, dtz);
  k.nq = make_float2(-h.q, -h.q);
  k.nqt = make_float2(-h.qt, -h.qt);
  k.nqxt = make_float2(-h.qxt, -h.qxt);
  return k;
}

cudaError_t launch_pair_elastic(cudaStream_t st, const SweepPlan& sp, int v, int set,
                                const PairCoef& k, const HabcDev& h, const PairPack& mp,
                                const PairOut& o, int* err) {
  if (!mp.v || mp.pitch < 1 || h.wstride <= sp.gm.nbc) return cudaErrorInvalidValue;
#define FOMO_LAUNCH_P(V, NN, FF, NV, PP, MB) \
  case V: return launch_p<NN, FF, NV, PP, MB>(st, sp, set, k, h, mp, o, err);
#define FOMO_LAUNCH_PN(NN)                              \
  case NN:                                              \
    switch (v) { FOMO_PAIR_VARIANTS(FOMO_LAUNCH_P, NN) } \
    break;
  switch (sp.N) {
    FOMO_LAUNCH_PN(1) FOMO_LAUNCH_PN(2) FOMO_LAUNCH_PN(3) FOMO_LAUNCH_PN(4) FOMO_LAUNCH_PN(5)
  }
#undef FOMO_LAUNCH_PN
#undef FOMO_LAUNCH_P
  return cudaErrorInvalidValue;
}

cudaError_t launch_inject_record_pair(cudaStream_t st, int it, int nt, int ns, long long plane,
                                      int n_src, const int* src_lin, const float* wav, float* txx,
                                      float* tzz, int n_rec, const int* rec_lin, const float* vx,
                                      const float* vz, float* s0, float* s1) {
  k_inject_record_pair<<<ns, 256, 0, st>>>(it, nt, plane, n_src, src_lin, wav, txx, tzz, n_rec,
                                           rec_lin, vx, vz, s0, s1);
  return cudaGetLastError();
}

cudaError_t launch_pair_unpack(cudaStream_t st, const float* f, long long plane, int ld, int x0,
                               int z0, int nx, int nz, int shot, float* out) {
  k_pair_unpack<<<256, 256, 0, st>>>(f, plane, ld, x0, z0, nx, nz, shot, out);
  return cudaGetLastError();
}

}  // namespace fomo
