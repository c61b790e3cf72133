// sweep3d.cu -- fused, TMA-staged z-marching half steps of elastic3d.
//
// One launch per half step replaces the update kernel and both Higdon passes:
//   velocity: v'  = update(A.v, A.tau)   (elastic3d/update_velocity.jl:17-84)
//             v'' = Higdon(v', A.v)      (boundary/habc/kernels_3d.jl:117-193)
//   stress:   s'  = update(A.tau, B.v)   (elastic3d/update_stress.jl:21-94)
//             s'' = Higdon(s', A.tau)
// written to set B.  The Higdon value of a frame cell needs v' (or s') at its
// interior-ward neighbours, which another thread produces: the CTA's 32 x 16
// threads cover a tile of 30 x 14 output columns plus a one-column ring on
// every side, each thread updating its own column, and the march down z runs
// one plane behind the update (plane z is finished while plane z+1 is
// updated).  So the x / y neighbours come from a shared-memory tile of the
// updated plane and the z neighbours from the thread's own registers; no
// scratch, no second pass, and the same two-pass semantics as the reference's
// deterministic 2D kernels (every Higdon input is a pre-correction value).
//
// Data movement: every input plane of a tile comes by TMA (4D tensor maps over
// the two field sets, no multicast) into a ring of shared-memory slots guarded
// by mbarriers with bounded waits; the x / y derivatives read those boxes, the
// z derivatives read per-thread register windows fed from the same slots.
// Arithmetic is the per-cell kernels' canonical sequence, bit for bit.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>
#include <type_traits>
#include <vector>

#include "sweep3d.cuh"
#include "tma.cuh"

namespace fomo {
namespace {

constexpr int kTX = 32, kTY = 16, kNT = kTX * kTY;
constexpr int kOX = kTX - 2, kOY = kTY - 2;  // output columns / rows of a tile
constexpr int kCW = 36;                      // centre box width: 32 + up to 3 alignment columns
constexpr int kMaxGrid3 = 1184;

__host__ __device__ constexpr int al32(int n) { return (n + 31) & ~31; }

template <int N>
struct F3 {
  static constexpr int XW = (2 * N + 38) & ~3;  // x-halo box width (>= 2N + 35, 16-byte rows)
  static constexpr int YH = kTY + 2 * N;        // y-halo box rows
  static constexpr int C = kTY * kCW, X = kTY * XW, Y = YH * kCW, XY = YH * XW;
  // velocity slot (floats)
  static constexpr int V_AV = 0;                  // A.v      [3][TY][CW]
  static constexpr int V_XX = V_AV + al32(3 * C); // txx      [TY][XW]
  static constexpr int V_XZ = V_XX + al32(X);     // txz      [TY][XW]
  static constexpr int V_XY = V_XZ + al32(X);     // txy      [YH][XW]
  static constexpr int V_YY = V_XY + al32(XY);    // tyy      [YH][CW]
  static constexpr int V_YZ = V_YY + al32(Y);     // tyz      [YH][CW]
  static constexpr int V_WN = V_YZ + al32(Y);     // txz, tyz, tzz at z+N [3][TY][CW]
  static constexpr int V_MB = V_WN + al32(3 * C); // bx, by, bz [3][TY][CW]
  static constexpr int V_SLOT = V_MB + al32(3 * C);
  static constexpr unsigned V_BYTES = 4u * (9 * C + 2 * X + XY + 2 * Y);
  // stress slot (floats)
  static constexpr int S_V = 0;                   // B.v vx, vy, vz [3][YH][XW]
  static constexpr int S_WN = S_V + al32(3 * XY); // vx, vy, vz at z+N [3][TY][CW]
  static constexpr int S_AT = S_WN + al32(3 * C); // A.tau [6][TY][CW]
  static constexpr int S_MT = S_AT + al32(6 * C); // lam, l2m, mxy, mxz, myz [5][TY][CW]
  static constexpr int S_SLOT = S_MT + al32(5 * C);
  static constexpr unsigned S_BYTES = 4u * (3 * XY + 14 * C);
  // acoustic velocity slot (floats)
  static constexpr int A_AV = 0;                   // A.v [3][TY][CW]
  static constexpr int A_PX = A_AV + al32(3 * C);  // p x-halo [TY][XW]
  static constexpr int A_PY = A_PX + al32(X);      // p y-halo [YH][CW]
  static constexpr int A_WN = A_PY + al32(Y);      // p at z+N [TY][CW]
  static constexpr int A_MB = A_WN + al32(C);      // bx, by, bz [3][TY][CW]
  static constexpr int A_SLOT = A_MB + al32(3 * C);
  static constexpr unsigned A_BYTES = 4u * (7 * C + X + Y);
  // acoustic pressure slot (floats)
  static constexpr int P_AP = 0;                   // A.p [TY][CW]
  static constexpr int P_VX = P_AP + al32(C);      // B.vx x-halo [TY][XW]
  static constexpr int P_VY = P_VX + al32(X);      // B.vy y-halo [YH][CW]
  static constexpr int P_WN = P_VY + al32(Y);      // B.vz at z+N [TY][CW]
  static constexpr int P_KP = P_WN + al32(C);      // kappa [TY][CW]
  static constexpr int P_SLOT = P_KP + al32(C);
  static constexpr unsigned P_BYTES = 4u * (3 * C + X + Y);
};

struct F3Maps {
  CUtensorMap c1, c3, c6, xh, yh, xyh, xyh3, m1, m3, m5;
};

__device__ __forceinline__ void load_4d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                        int f, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(tma::saddr(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(f), "r"(tma::saddr(bar))
      : "memory");
}

// Staggered sums (the canonical sequence of fomo_internal.cuh's dm / dp):
// over shared memory (f at the cell, element stride S) ...
template <int N, int S>
__device__ __forceinline__ float sdm(const float* f, const Coef& c) {
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l)
    acc = __fmaf_rn(c.a[l - 1], __fsub_rn(f[(l - 1) * S], f[-l * S]), acc);
  return acc;
}
template <int N, int S>
__device__ __forceinline__ float sdp(const float* f, const Coef& c) {
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l)
    acc = __fmaf_rn(c.a[l - 1], __fsub_rn(f[l * S], f[-(l - 1) * S]), acc);
  return acc;
}
// ... and over a register window w[k] = plane z - N + k
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

__device__ __forceinline__ float ld3(const Geo3& g, const float* __restrict__ f, int x, int y,
                                     int z) {
  return (x >= 0 && x < g.nx && y >= 0 && y < g.ny && z >= 0 && z < g.nz)
             ? __ldg(f + x + g.sy * y + g.sz * z)
             : 0.0f;
}

// The Higdon blend of one field (k_habc3_pass1's sequence, sides summed in x,
// y, z order).  The mean over nd sides divides by nd: x / 1 and x / 2 are
// x and x * 0.5 exactly (both round the same quotient), so only corner cells
// (nd = 3) take the IEEE division.
constexpr int kWt = 256;  // weight-table entries per kind staged in shared memory

__device__ __forceinline__ float blend3(const HabcDev& h, const float* s_wt, int kind, int dist,
                                        int nd, float fc, float sum) {
  const float w = dist < kWt ? s_wt[dist] : habc_weight(h, kind, dist);
  const float p = __fmul_rn(__fsub_rn(1.0f, w), sum);
  const float m = nd == 1 ? p : (nd == 2 ? __fmul_rn(p, 0.5f) : __fdiv_rn(p, 3.0f));
  return __fmaf_rn(w, fc, m);
}

}  // namespace

// ---------------------------------------------------------------------------
// The march of one half step (PH below).
// Iteration i of a segment [z0, z1) of a tile updates plane z = z0 - 1 + i
// (i = 0 .. z1 - z0 + 1) and finishes plane z - 1.  TMA slot k (of R) holds the
// boxes of one plane; a slot is refilled two iterations after its plane was
// updated (its centre box of the old field group serves the Higdon terms of
// the next iteration), so R - 2 planes are in flight ahead of the update.  The
// updated values of every thread go to a three-plane tile ring in shared
// memory for the neighbours' Higdon terms.
// ---------------------------------------------------------------------------
// PH: 0 elastic velocity, 1 elastic stress, 2 acoustic velocity, 3 acoustic
// pressure (acoustic3d/update_velocity.jl:16-53, update_pressure.jl:16-50).
// The acoustic phases fit 64 registers a thread: two CTAs per SM where the
// shared memory allows.
template <int N, int R, int PH>
__global__ void __launch_bounds__(kNT, PH >= 2 ? 2 : 1)
    k_el3_fused(const __grid_constant__ F3Maps mp, Geo3 g, Coef c, float dtdh, HabcDev h,
                float* __restrict__ st, int A, int B, const int4* __restrict__ segs, int nseg,
                int* __restrict__ sched, int* __restrict__ err) {
  using S = F3<N>;
  constexpr bool EL = PH < 2;                 // elastic (9 fields a set) or acoustic (4)
  constexpr bool SECOND = PH == 1 || PH == 3;  // stress / pressure: reads B's velocities
  constexpr int NSET = EL ? 9 : 4;
  constexpr int NF = PH == 0 ? 3 : (PH == 1 ? 6 : (PH == 2 ? 3 : 1));  // fields updated
  constexpr int SLOT = PH == 0 ? S::V_SLOT : (PH == 1 ? S::S_SLOT : (PH == 2 ? S::A_SLOT : S::P_SLOT));
  constexpr unsigned BYTES =
      PH == 0 ? S::V_BYTES : (PH == 1 ? S::S_BYTES : (PH == 2 ? S::A_BYTES : S::P_BYTES));
  // centre boxes of the old field group, and the z-window entries (plane z + N)
  constexpr int OLD = PH == 0 ? S::V_AV : (PH == 1 ? S::S_AT : (PH == 2 ? S::A_AV : S::P_AP));
  constexpr int WIN = PH == 0 ? S::V_WN : (PH == 1 ? S::S_WN : (PH == 2 ? S::A_WN : S::P_WN));
  extern __shared__ __align__(128) float sm[];
  float* slots = sm;
  constexpr int NK = SECOND ? 1 : 3;                // Higdon weight ramps used
  float* tring = sm + R * SLOT;  // [3 planes][NF][NT]
  float* s_wt = tring + 3 * NF * kNT;  // [NK][kWt]
  uint64_t* bars = reinterpret_cast<uint64_t*>(s_wt + NK * kWt);
  __shared__ int s_next;
  const int t = threadIdx.x, r = threadIdx.y, tid = r * kTX + t;
  const bool own_out = t >= 1 && t <= kOX && r >= 1 && r <= kOY;
  if (tid == 0) {
    for (int q = 0; q < R; ++q) tma::mbar_init(&bars[q], 1);
    tma::mbar_init_fence();
  }
  for (int k = tid; k < NK * kWt; k += kNT) {
    const int kind = SECOND ? 3 : k / kWt, d = k % kWt;
    s_wt[k] = d < h.wstride ? __ldg(h.wtab + kind * h.wstride + d) : 1.0f;
  }
  // z-window fields: txz, tyz, tzz of A (elastic velocity), vx, vy, vz of B
  // (stress), p of A (acoustic velocity), vz of B (pressure)
  constexpr int NW = EL ? 3 : 1;
  const int wf0 = PH == 0 ? A * 9 + 7 : (PH == 1 ? B * 9 : (PH == 2 ? A * 4 + 3 : B * 4 + 2));
  const float* w0 = st + (long long)wf0 * g.vol;
  const float* w1 = st + (long long)(PH == 0 ? A * 9 + 8 : B * 9 + 1) * g.vol;
  const float* w2 = st + (long long)(PH == 0 ? A * 9 + 5 : B * 9 + 2) * g.vol;
  float* ob = st + (long long)(B * NSET + (PH == 1 ? 3 : (PH == 3 ? 3 : 0))) * g.vol;
  int q = 0;             // slot of the current iteration
  uint32_t ph = 0;       // its mbarrier phase parity
  long long gk = 0;      // iterations so far (all segments)
  long long ok_upto = 0, issued = 0;
  bool live = true;
  // Segments are handed out in list order (a counter in device memory): the
  // tiles in flight are neighbours, and faster CTAs take more of them.
  for (;;) {
    __syncthreads();  // the previous segment's readers are done with every slot and tile
    if (tid == 0) s_next = atomicAdd(&sched[0], 1);
    __syncthreads();
    const int sgi = s_next;
    if (sgi >= nseg) break;
    const int4 sg = segs[sgi];  // {tile x, tile y, z0, z1}
    const int x0 = sg.x * kOX - 1, y0 = sg.y * kOY - 1, z0 = sg.z, z1 = sg.w;
    const int x = x0 + t, y = y0 + r;
    const int bxc = x0 & ~3, shc = x0 - bxc;
    const int bxh = (x0 - N) & ~3, shh = x0 - bxh;
    const int nit = z1 - z0 + 2;
    const bool out_ok = own_out && x < g.nx && y < g.ny;
    // The ring rows (warps 0 and 15) only feed the y-side Higdon terms of the
    // tile's first / last output row: the back band's (neighbour y - 1) and the
    // front band's (neighbour y + 1).  Elsewhere those warps skip the update.
    const bool ring_idle = (r == 0 && !(y0 + 1 >= g.ny - 1 - g.nbc)) ||
                           (r == kTY - 1 && !(y0 + kOY <= g.nbc));
    const bool in_xy = x >= N && x < g.nx - N && y >= N && y < g.ny - N && !ring_idle;
    // x / y part of the frame classification (kernels_3d.jl:117-150)
    const int sx = x <= g.nbc ? 1 : (x >= g.nx - 1 - g.nbc ? -1 : 0);
    const int sy = y <= g.nbc ? 1 : (y >= g.ny - 1 - g.nbc ? -1 : 0);
    const bool fr_xy = x >= 1 && x <= g.nx - 2 && y >= 1 && y <= g.ny - 2;
    const int nd_xy = (sx != 0) + (sy != 0);
    const int dist_xy = min(min(x, g.nx - 1 - x), min(y, g.ny - 1 - y));
    auto issue = [&](int i, int slot) {
      float* s = slots + slot * SLOT;
      uint64_t* bar = &bars[slot];
      const int z = z0 - 1 + i;
      tma::mbar_expect_tx(bar, BYTES);
      if constexpr (PH == 3) {
        load_4d(s + S::P_AP, &mp.c1, bxc, y0, z, A * 4 + 3, bar);
        load_4d(s + S::P_VX, &mp.xh, bxh, y0, z, B * 4 + 0, bar);
        load_4d(s + S::P_VY, &mp.yh, bxc, y0 - N, z, B * 4 + 1, bar);
        load_4d(s + S::P_WN, &mp.c1, bxc, y0, z + N, B * 4 + 2, bar);
        load_4d(s + S::P_KP, &mp.m1, bxc, y0, z, 3, bar);
      } else if constexpr (PH == 2) {
        load_4d(s + S::A_AV, &mp.c3, bxc, y0, z, A * 4, bar);
        load_4d(s + S::A_PX, &mp.xh, bxh, y0, z, A * 4 + 3, bar);
        load_4d(s + S::A_PY, &mp.yh, bxc, y0 - N, z, A * 4 + 3, bar);
        load_4d(s + S::A_WN, &mp.c1, bxc, y0, z + N, A * 4 + 3, bar);
        load_4d(s + S::A_MB, &mp.m3, bxc, y0, z, 0, bar);
      } else if constexpr (PH == 1) {
        load_4d(s + S::S_V, &mp.xyh3, bxh, y0 - N, z, B * 9, bar);
        load_4d(s + S::S_WN, &mp.c3, bxc, y0, z + N, B * 9, bar);
        load_4d(s + S::S_AT, &mp.c6, bxc, y0, z, A * 9 + 3, bar);
        load_4d(s + S::S_MT, &mp.m5, bxc, y0, z, 3, bar);
      } else {
        const int fa = A * 9;
        load_4d(s + S::V_AV, &mp.c3, bxc, y0, z, fa + 0, bar);
        load_4d(s + S::V_XX, &mp.xh, bxh, y0, z, fa + 3, bar);
        load_4d(s + S::V_XZ, &mp.xh, bxh, y0, z, fa + 7, bar);
        load_4d(s + S::V_XY, &mp.xyh, bxh, y0 - N, z, fa + 6, bar);
        load_4d(s + S::V_YY, &mp.yh, bxc, y0 - N, z, fa + 4, bar);
        load_4d(s + S::V_YZ, &mp.yh, bxc, y0 - N, z, fa + 8, bar);
        load_4d(s + S::V_WN, &mp.c1, bxc, y0, z + N, fa + 7, bar);
        load_4d(s + S::V_WN + S::C, &mp.c1, bxc, y0, z + N, fa + 8, bar);
        load_4d(s + S::V_WN + 2 * S::C, &mp.c1, bxc, y0, z + N, fa + 5, bar);
        load_4d(s + S::V_MB, &mp.m3, bxc, y0, z, 0, bar);
      }
    };
    if (tid == 0 && live) {
      tma::fence_proxy_async();
      int sl = q;
      for (int i = 0; i < R && i < nit; ++i) {
        issue(i, sl);
        sl = sl + 1 == R ? 0 : sl + 1;
      }
      issued = gk + min(R, nit);
    }
    // z windows (length 2N + 3): in phase p of the three-iteration cycle, plane
    // z's window is w[p .. p + 2N] and w[p + 2N] arrives from the slot; after
    // phase 2 the window moves down by three entries.  The updated (U) and old
    // (O) values of the last three planes rotate by phase as well, so the
    // cycle's three bodies carry no register moves besides the window's.
    float wa[2 * N + 3], wb[2 * N + 3], wc[2 * N + 3];
#pragma unroll
    for (int k = 0; k < 2 * N; ++k) {
      const int z = z0 - 1 - N + k;
      wa[k] = ld3(g, w0, x, y, z);
      if constexpr (NW == 3) {
        wb[k] = ld3(g, w1, x, y, z);
        wc[k] = ld3(g, w2, x, y, z);
      }
    }
    float U[3][NF], O[3][NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) U[1][f] = U[2][f] = O[1][f] = O[2][f] = 0.0f;
    const int ce = r * kCW + t + shc;  // this thread's cell in a centre box
    int qp = q;                         // slot of the previous iteration (plane z - 1)
    int qp2 = q;                        // slot of plane z - 2 (refilled after this iteration's barrier)
    auto body = [&](auto P, int i) {
      constexpr int p = decltype(P)::value, p1 = (p + 2) % 3, p2 = (p + 1) % 3;
      const int z = z0 - 1 + i;
      const float* s = slots + q * SLOT;
      if (live) {
        live = tma::mbar_wait_bounded(&bars[q], ph, err);
        if (live) ok_upto = gk + i + 1;
      }
      float(&wA)[2 * N + 1] = *reinterpret_cast<float(*)[2 * N + 1]>(&wa[p]);
      [[maybe_unused]] float(&wB)[2 * N + 1] = *reinterpret_cast<float(*)[2 * N + 1]>(&wb[p]);
      [[maybe_unused]] float(&wC)[2 * N + 1] = *reinterpret_cast<float(*)[2 * N + 1]>(&wc[p]);
      wA[2 * N] = s[WIN + ce];
      if constexpr (NW == 3) {
        wB[2 * N] = s[WIN + S::C + ce];
        wC[2 * N] = s[WIN + 2 * S::C + ce];
      }
      float(&o)[NF] = O[p];
      float(&u)[NF] = U[p];
#pragma unroll
      for (int f = 0; f < NF; ++f) u[f] = o[f] = s[OLD + f * S::C + ce];
      if (in_xy && z + g.z0 >= N && z + g.z0 < g.gnz - N) {
        if constexpr (PH == 3) {
          const float dx = sdp<N, 1>(s + S::P_VX + r * S::XW + t + shh, c);
          const float dy = sdp<N, kCW>(s + S::P_VY + (r + N) * kCW + t + shc, c);
          const float dz = wdm<N>(wA, c);
          u[0] = __fmaf_rn(__fmul_rn(s[S::P_KP + ce], dtdh), __fadd_rn(__fadd_rn(dx, dy), dz), o[0]);
        } else if constexpr (PH == 2) {
          const float dx = sdm<N, 1>(s + S::A_PX + r * S::XW + t + shh, c);
          const float dy = sdm<N, kCW>(s + S::A_PY + (r + N) * kCW + t + shc, c);
          const float dz = wdp<N>(wA, c);
          u[0] = __fmaf_rn(__fmul_rn(s[S::A_MB + ce], dtdh), dx, o[0]);
          u[1] = __fmaf_rn(__fmul_rn(s[S::A_MB + S::C + ce], dtdh), dy, o[1]);
          u[2] = __fmaf_rn(__fmul_rn(s[S::A_MB + 2 * S::C + ce], dtdh), dz, o[2]);
        } else if constexpr (PH == 1) {
          const float* pvx = s + S::S_V + (r + N) * S::XW + t + shh;
          const float* pvy = pvx + S::XY;
          const float* pvz = pvx + 2 * S::XY;
          const float dxx = sdp<N, 1>(pvx, c), dyy = sdp<N, S::XW>(pvy, c), dzz = wdm<N>(wC, c);
          const float dxy = sdm<N, S::XW>(pvx, c), dyx = sdm<N, 1>(pvy, c);
          const float dxz = wdp<N>(wA, c), dzx = sdm<N, 1>(pvz, c);
          const float dyz = wdp<N>(wB, c), dzy = sdm<N, S::XW>(pvz, c);
          const float lm = s[S::S_MT + ce], l2 = s[S::S_MT + S::C + ce];
          u[0] = __fmaf_rn(__fmaf_rn(lm, dzz, __fmaf_rn(lm, dyy, __fmul_rn(l2, dxx))), dtdh, o[0]);
          u[1] = __fmaf_rn(__fmaf_rn(lm, dzz, __fmaf_rn(l2, dyy, __fmul_rn(lm, dxx))), dtdh, o[1]);
          u[2] = __fmaf_rn(__fmaf_rn(l2, dzz, __fmaf_rn(lm, dyy, __fmul_rn(lm, dxx))), dtdh, o[2]);
          u[3] = __fmaf_rn(__fmul_rn(s[S::S_MT + 2 * S::C + ce], __fadd_rn(dxy, dyx)), dtdh, o[3]);
          u[4] = __fmaf_rn(__fmul_rn(s[S::S_MT + 3 * S::C + ce], __fadd_rn(dxz, dzx)), dtdh, o[4]);
          u[5] = __fmaf_rn(__fmul_rn(s[S::S_MT + 4 * S::C + ce], __fadd_rn(dyz, dzy)), dtdh, o[5]);
        } else {
          const float* pxx = s + S::V_XX + r * S::XW + t + shh;
          const float* pxz = s + S::V_XZ + r * S::XW + t + shh;
          const float* pxy = s + S::V_XY + (r + N) * S::XW + t + shh;
          const float* pyy = s + S::V_YY + (r + N) * kCW + t + shc;
          const float* pyz = s + S::V_YZ + (r + N) * kCW + t + shc;
          const float a1 = sdm<N, 1>(pxx, c), a2 = sdp<N, S::XW>(pxy, c), a3 = wdm<N>(wA, c);
          const float b1 = sdp<N, 1>(pxy, c), b2 = sdm<N, kCW>(pyy, c), b3 = wdm<N>(wB, c);
          const float c1 = sdp<N, 1>(pxz, c), c2 = sdp<N, kCW>(pyz, c), c3 = wdp<N>(wC, c);
          u[0] = __fmaf_rn(__fmul_rn(s[S::V_MB + ce], dtdh), __fadd_rn(__fadd_rn(a1, a2), a3), o[0]);
          u[1] = __fmaf_rn(__fmul_rn(s[S::V_MB + S::C + ce], dtdh),
                           __fadd_rn(__fadd_rn(b1, b2), b3), o[1]);
          u[2] = __fmaf_rn(__fmul_rn(s[S::V_MB + 2 * S::C + ce], dtdh),
                           __fadd_rn(__fadd_rn(c1, c2), c3), o[2]);
        }
      }
      float* tcur = tring + p * NF * kNT;   // tile ring planes by phase: z, z - 1
      const float* tprev = tring + p1 * NF * kNT;
#pragma unroll
      for (int f = 0; f < NF; ++f) tcur[f * kNT + tid] = u[f];
      __syncthreads();  // plane z's tile is complete; plane z-2's slot is free
      if (tid == 0 && live && i >= 2 && i + R - 2 < nit) {
        tma::fence_proxy_async();
        issue(i + R - 2, qp2);
        issued = gk + i + R - 1;
      }
      // finish plane z - 1: Higdon(updated, old) on frame cells, the update elsewhere
      const int zq = z - 1;
      if (i >= 1 && out_ok && zq >= z0) {
        const int zg = zq + g.z0;  // global plane: frame classification
        const float(&u1)[NF] = U[p1];
        const float(&u2)[NF] = U[p2];
        const float(&o1)[NF] = O[p1];
        const float(&o2)[NF] = O[p2];
        float vv[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) vv[f] = u1[f];
        const int sz = zg <= g.nbc ? 1 : (zg >= g.gnz - 1 - g.nbc ? -1 : 0);
        const int nd = (fr_xy && zg >= 1 && zg <= g.gnz - 2) ? nd_xy + (sz != 0) : 0;
        if (nd > 0) {
          const int dist = min(dist_xy, min(zg, g.gnz - 1 - zg));
          const float* tp = tprev + tid;
          const float* ap = slots + qp * SLOT + OLD + ce;
#pragma unroll
          for (int f = 0; f < NF; ++f) {
            float sum = 0.0f;
            if (sx) sum = __fadd_rn(sum, higdon_side(h, tp[f * kNT + sx], o1[f], ap[f * S::C + sx]));
            if (sy)
              sum = __fadd_rn(sum, higdon_side(h, tp[f * kNT + sy * kTX], o1[f],
                                               ap[f * S::C + sy * kCW]));
            if (sz)
              sum = __fadd_rn(sum, higdon_side(h, sz > 0 ? u[f] : u2[f], o1[f],
                                               sz > 0 ? o[f] : o2[f]));
            vv[f] = blend3(h, s_wt + (SECOND ? 0 : f) * kWt, SECOND ? 3 : f, dist, nd, u1[f], sum);
          }
        }
        const long long oi = x + g.sy * y + g.sz * zq;
#pragma unroll
        for (int f = 0; f < NF; ++f) ob[f * g.vol + oi] = vv[f];
      }
      qp2 = qp;
      qp = q;
      if (++q == R) {
        q = 0;
        ph ^= 1u;
      }
    };
    for (int i = 0; i < nit;) {
      body(std::integral_constant<int, 0>{}, i);
      if (++i >= nit) break;
      body(std::integral_constant<int, 1>{}, i);
      if (++i >= nit) break;
      body(std::integral_constant<int, 2>{}, i);
      ++i;
#pragma unroll
      for (int k = 0; k < 2 * N; ++k) {
        wa[k] = wa[k + 3];
        if constexpr (NW == 3) {
          wb[k] = wb[k + 3];
          wc[k] = wc[k + 3];
        }
      }
    }
    gk += nit;
  }
  // after a timed-out wait, give the copies still in flight a bounded time to land
  if (tid == 0 && !live)
    for (long long k = ok_upto; k < issued; ++k)
      tma::mbar_wait_bounded(&bars[k % R], (uint32_t)((k / R) & 1), err);
  // the last CTA to finish rearms the counter for the next launch
  if (tid == 0) {
    __threadfence();
    if (atomicAdd(&sched[1], 1) == (int)gridDim.x - 1) {
      sched[0] = 0;
      sched[1] = 0;
      __threadfence();
    }
  }
}

// ---- host side --------------------------------------------------------------
namespace {

PFN_cuTensorMapEncodeTiled_v12000 g_enc3 = nullptr;
std::once_flag g_enc3_once;

PFN_cuTensorMapEncodeTiled_v12000 encoder3() {
  std::call_once(g_enc3_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_enc3 = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    else
      cudaGetLastError();
  });
  return g_enc3;
}

constexpr size_t kMaxDynSmem3 = 227 * 1024;
constexpr int kRing = 4;  // TMA slots per CTA (two planes in flight ahead of the update)

template <int N, int PH>
constexpr size_t smem_bytes3() {
  using S = F3<N>;
  const int slot = PH == 0 ? S::V_SLOT : (PH == 1 ? S::S_SLOT : (PH == 2 ? S::A_SLOT : S::P_SLOT));
  const int nf = PH == 0 ? 3 : (PH == 1 ? 6 : (PH == 2 ? 3 : 1));
  const int nk = (PH == 1 || PH == 3) ? 1 : 3;
  return (size_t)kRing * slot * 4 + (size_t)3 * nf * kNT * 4 + (size_t)nk * kWt * 4 +
         (size_t)kRing * 8;
}
static_assert(smem_bytes3<5, 1>() + 1024 <= kMaxDynSmem3, "the widest stress plan fits an SM");

size_t smem_of(int N, int ph) {
#define FOMO_SM3(NN) \
  case NN:           \
    return ph == 0 ? smem_bytes3<NN, 0>() : ph == 1 ? smem_bytes3<NN, 1>() : ph == 2 ? smem_bytes3<NN, 2>() : smem_bytes3<NN, 3>();
  switch (N) { FOMO_SM3(1) FOMO_SM3(2) FOMO_SM3(3) FOMO_SM3(4) default: FOMO_SM3(5) }
#undef FOMO_SM3
}
int xw_of(int N) { return (2 * N + 38) & ~3; }

CUresult encode4(CUtensorMap* m, const void* base, const Geo3& g, int nf, int bw, int bh, int bf) {
  cuuint64_t dims[4] = {(cuuint64_t)g.nx, (cuuint64_t)g.ny, (cuuint64_t)g.nz, (cuuint64_t)nf};
  cuuint64_t strides[3] = {(cuuint64_t)g.ld * 4, (cuuint64_t)g.sz * 4, (cuuint64_t)g.vol * 4};
  cuuint32_t box[4] = {(cuuint32_t)bw, (cuuint32_t)bh, 1, (cuuint32_t)bf};
  cuuint32_t es[4] = {1, 1, 1, 1};
  return encoder3()(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void*>(base), dims, strides,
                    box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

F3Maps maps_of(const Fused3Plan& p) {
  F3Maps m;
  m.c1 = p.c1;
  m.c3 = p.c3;
  m.c6 = p.c6;
  m.xh = p.xh;
  m.yh = p.yh;
  m.xyh = p.xyh;
  m.xyh3 = p.xyh3;
  m.m1 = p.m1;
  m.m3 = p.m3;
  m.m5 = p.m5;
  return m;
}

// Sets the kernel's shared-memory limit once; returns its resident CTAs per SM
// (0 if the query fails).
template <int N, int PH>
int prepare3() {
  auto kern = k_el3_fused<N, kRing, PH>;
  static std::once_flag once;
  static int per_sm = 0;
  std::call_once(once, [&] {
    int nb = 0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_bytes3<N, PH>()) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, kNT, smem_bytes3<N, PH>()) ==
            cudaSuccess)
      per_sm = nb;
    else
      cudaGetLastError();
  });
  return per_sm;
}
int per_sm3(int N, int ph) {
#define FOMO_PS3(NN) \
  case NN:           \
    return ph == 0 ? prepare3<NN, 0>() : ph == 1 ? prepare3<NN, 1>() : ph == 2 ? prepare3<NN, 2>() : prepare3<NN, 3>();
  switch (N) { FOMO_PS3(1) FOMO_PS3(2) FOMO_PS3(3) FOMO_PS3(4) default: FOMO_PS3(5) }
#undef FOMO_PS3
}

template <int N, int PH>
cudaError_t launch3(cudaStream_t st, const Fused3Plan& p, const Geo3& g, float* state, int A,
                    int B, const Coef& c, float dtdh, const HabcDev& h, int* err) {
  auto kern = k_el3_fused<N, kRing, PH>;
  if (prepare3<N, PH>() < 1) return cudaErrorInvalidConfiguration;
  const int grid = (PH == 0 || PH == 2) ? p.grid_v : p.grid_s;
  kern<<<grid, dim3(kTX, kTY), smem_bytes3<N, PH>(), st>>>(maps_of(p), g, c, dtdh, h, state,
                                                                 A, B, p.d_segs, p.nseg, p.d_sched,
                                                                 err);
  return cudaGetLastError();
}

template <int PH>
cudaError_t launch_any(cudaStream_t st, const Fused3Plan& p, const Geo3& g, float* state, int A,
                       int B, const Coef& c, float dtdh, const HabcDev& h, int* err) {
  switch (p.N) {
    case 1: return launch3<1, PH>(st, p, g, state, A, B, c, dtdh, h, err);
    case 2: return launch3<2, PH>(st, p, g, state, A, B, c, dtdh, h, err);
    case 3: return launch3<3, PH>(st, p, g, state, A, B, c, dtdh, h, err);
    case 4: return launch3<4, PH>(st, p, g, state, A, B, c, dtdh, h, err);
    case 5: return launch3<5, PH>(st, p, g, state, A, B, c, dtdh, h, err);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

bool fused3_supported(int N) { return N >= 1 && N <= 5 && encoder3(); }

size_t fused3_table_bytes(const Geo3& g) {
  const long long ntiles = (long long)((g.nx + kOX - 1) / kOX) * ((g.ny + kOY - 1) / kOY);
  return (size_t)(ntiles + 4 * kMaxGrid3) * sizeof(int4) + 512;
}

cudaError_t fused3_make_plan(Fused3Plan& p, const Geo3& g, int N, bool elastic, float* state,
                             const float* mat, void* d_table, cudaStream_t st) {
  if (!fused3_supported(N)) return cudaErrorNotSupported;
  p.N = N;
  p.ntx = (g.nx + kOX - 1) / kOX;
  p.nty = (g.ny + kOY - 1) / kOY;
  p.elastic = elastic;
  p.smem_v = smem_of(N, elastic ? 0 : 2);
  p.smem_s = smem_of(N, elastic ? 1 : 3);
  int dev = 0, nsm = 148;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  // Persistent CTAs: one per SM for the elastic phases (a CTA holds an SM's
  // registers and most of its shared memory), two for the acoustic ones where
  // they fit; at least 16 planes of work each.  The segment list
  // runs through the tiles in order, whole z columns, so the tiles marching
  // side by side are neighbours and read each other's halo rows from L2; the
  // last wave of tiles is cut into four z chunks (chunk-major) so that the
  // CTAs finish together.
  const int ntiles = p.ntx * p.nty;
  const int zlo = g.zlo, zhi = g.zhi, nzo = zhi - zlo;  // planes updated
  if (zlo < 0 || zhi > g.nz || nzo < 1 || g.gnz < g.nz || g.z0 < 0 || g.z0 + g.nz > g.gnz)
    return cudaErrorInvalidValue;
  const long long total = (long long)ntiles * nzo;
  const int ph0 = elastic ? 0 : 2;
  const int pv = per_sm3(N, ph0), ps = per_sm3(N, ph0 + 1);
  if (pv < 1 || ps < 1) return cudaErrorInvalidConfiguration;
  auto grid_of = [&](int per_sm) {
    return (int)std::max(1LL, std::min<long long>({(long long)per_sm * nsm, (long long)kMaxGrid3,
                                                   total / 16}));
  };
  p.grid_v = grid_of(pv);
  p.grid_s = grid_of(ps);
  const int G = std::max(p.grid_v, p.grid_s);
  const int L = std::min(ntiles, G), K = nzo >= 64 ? 4 : 1;
  std::vector<int4> segs;
  segs.reserve((size_t)ntiles + 3 * (size_t)L);
  for (int tile = 0; tile < ntiles - L; ++tile)
    segs.push_back(make_int4(tile % p.ntx, tile / p.ntx, zlo, zhi));
  for (int k = 0; k < K; ++k) {
    const int z0 = zlo + (int)((long long)nzo * k / K), z1 = zlo + (int)((long long)nzo * (k + 1) / K);
    for (int tile = ntiles - L; tile < ntiles; ++tile)
      segs.push_back(make_int4(tile % p.ntx, tile / p.ntx, z0, z1));
  }
  p.nseg = (int)segs.size();
  char* tb = static_cast<char*>(d_table);
  p.d_sched = reinterpret_cast<int*>(tb);
  p.d_segs = reinterpret_cast<int4*>(tb + 256);
  e = cudaMemsetAsync(p.d_sched, 0, 2 * sizeof(int), st);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(p.d_segs, segs.data(), segs.size() * sizeof(int4), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(st);  // segs is a host temporary
  if (e != cudaSuccess) return e;
  const int XW = xw_of(N), YH = kTY + 2 * N;
  CUresult r = CUDA_SUCCESS;
  auto ok = [&](CUresult x) {
    if (x != CUDA_SUCCESS) r = x;
  };
  const int nst = elastic ? 18 : 8, nmat = elastic ? 8 : 4;  // field planes of both sets
  ok(encode4(&p.c1, state, g, nst, kCW, kTY, 1));
  ok(encode4(&p.c3, state, g, nst, kCW, kTY, 3));
  ok(encode4(&p.xh, state, g, nst, XW, kTY, 1));
  ok(encode4(&p.yh, state, g, nst, kCW, YH, 1));
  ok(encode4(&p.m1, mat, g, nmat, kCW, kTY, 1));
  ok(encode4(&p.m3, mat, g, nmat, kCW, kTY, 3));
  if (elastic) {
    ok(encode4(&p.c6, state, g, nst, kCW, kTY, 6));
    ok(encode4(&p.xyh, state, g, nst, XW, YH, 1));
    ok(encode4(&p.xyh3, state, g, nst, XW, YH, 3));
    ok(encode4(&p.m5, mat, g, nmat, kCW, kTY, 5));
  }
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t fused3_velocity(cudaStream_t st, const Fused3Plan& p, const Geo3& g, float* state,
                            int A, int B, const Coef& c, float dtdh, const HabcDev& h, int* err) {
  return p.elastic ? launch_any<0>(st, p, g, state, A, B, c, dtdh, h, err)
                   : launch_any<2>(st, p, g, state, A, B, c, dtdh, h, err);
}

cudaError_t fused3_stress(cudaStream_t st, const Fused3Plan& p, const Geo3& g, float* state,
                          int A, int B, const Coef& c, float dtdh, const HabcDev& h, int* err) {
  return p.elastic ? launch_any<1>(st, p, g, state, A, B, c, dtdh, h, err)
                   : launch_any<3>(st, p, g, state, A, B, c, dtdh, h, err);
}

}  // namespace fomo
