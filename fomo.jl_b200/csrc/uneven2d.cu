// uneven2d.cu -- acoustic2d over many shots whose grids differ in size.
//
// The reference batches shots only on one shared model (acoustic2d/batch.jl);
// shots on different grids run as separate acoustic2d calls.  Here every shot
// keeps its own padded grid, materials and Higdon coefficients, and one time
// step is three kernels over a flat list of (shot, tile) work items covering
// all shots:
//   velocity update + fused HABC   (acoustic2d/fused_kernels.jl:27-63, kernels_det.jl)
//   pressure update + fused HABC   (fused_kernels.jl:86-114)
//   inject into p, record p/vx/vz  (inject_source.jl:4-24, fused_kernels.jl:137-149)
// The whole nt-step run is captured once into a CUDA graph and replayed with a
// single launch.  The tile shape is chosen by timing candidates on the problem
// itself (cached per problem shape).  Each shot equals a single acoustic2d
// run bit for bit (same per-cell arithmetic as the two-phase kernels).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "solver2d_kernels.cuh"
#include "tma.cuh"

namespace fomo {
namespace {

struct UShot {
  long long st;     // state offset: set k field f at st + (3k + f) * plane (vx, vz, p)
  long long mat;    // material offset: bx, bz, kappa at mat + f * plane
  long long plane;  // ld * nz
  long long wav0;   // wavelet offset (n_src, nt)
  long long seis0;  // seismogram offset: p, vx, vz blocks of n_rec * nt
  int nx, nz, ld;   // padded grid, row pitch
  int tiles_x, tile0;
  int n_src, src0, n_rec, rec0;
  float q, qt, qxt;
};

template <int N>
__global__ void __launch_bounds__(256, 8) k_uac_vel(const UShot* __restrict__ shots,
                                                 const int* __restrict__ tile_shot,
                                                 float* __restrict__ state,
                                                 const float* __restrict__ mat, Coef c, float dtx,
                                                 float dtz, const float* __restrict__ wtab,
                                                 int nbc, int wstride, int set) {
  const int tile = blockIdx.x;
  const UShot sh = shots[tile_shot[tile]];
  const int lt = tile - sh.tile0;
  const int tz = lt / sh.tiles_x, tx = lt - tz * sh.tiles_x;
  const int x = tx * blockDim.x + threadIdx.x, z = tz * blockDim.y + threadIdx.y;
  if (x >= sh.nx || z >= sh.nz) return;
  const Geo2 g{sh.nx, sh.nz, sh.ld, N, nbc, sh.plane};
  const HabcDev h{sh.q, sh.qt, sh.qxt, nbc, wstride, wtab};
  const float* A = state + sh.st + (long long)set * 3 * sh.plane;
  float* B = state + sh.st + (long long)(1 - set) * 3 * sh.plane;
  const float* m = mat + sh.mat;
  float ux, uz;
  ac_vel_cell<N>(g, c, dtx, dtz, h, A + 2 * sh.plane, A, A + sh.plane, m, m + sh.plane, x, z, ux,
                 uz);
  const long long p = (long long)z * sh.ld + x;
  B[p] = ux;
  B[sh.plane + p] = uz;
}

template <int N>
__global__ void __launch_bounds__(256) k_uac_prs(const UShot* __restrict__ shots,
                                                 const int* __restrict__ tile_shot,
                                                 float* __restrict__ state,
                                                 const float* __restrict__ mat, Coef c, float dtx,
                                                 float dtz, const float* __restrict__ wtab,
                                                 int nbc, int wstride, int set) {
  const int tile = blockIdx.x;
  const UShot sh = shots[tile_shot[tile]];
  const int lt = tile - sh.tile0;
  const int tz = lt / sh.tiles_x, tx = lt - tz * sh.tiles_x;
  const int x = tx * blockDim.x + threadIdx.x, z = tz * blockDim.y + threadIdx.y;
  if (x >= sh.nx || z >= sh.nz) return;
  const Geo2 g{sh.nx, sh.nz, sh.ld, N, nbc, sh.plane};
  const HabcDev h{sh.q, sh.qt, sh.qxt, nbc, wstride, wtab};
  const float* A = state + sh.st + (long long)set * 3 * sh.plane;
  float* B = state + sh.st + (long long)(1 - set) * 3 * sh.plane;
  const float u = ac_prs_cell<N>(g, c, dtx, dtz, h, A + 2 * sh.plane, B, B + sh.plane,
                                 mat + sh.mat + 2 * sh.plane, x, z);
  B[2 * sh.plane + (long long)z * sh.ld + x] = u;
}

// One block per shot: sources in order into p, then p/vx/vz at the receivers.
__global__ void k_uinject_record(const UShot* __restrict__ shots, float* __restrict__ state,
                                 const int* __restrict__ src_lin, const float* __restrict__ wav,
                                 const int* __restrict__ rec_lin, float* __restrict__ seis, int it,
                                 int nt, int set_out) {
  const UShot& sh = shots[blockIdx.x];
  float* B = state + sh.st + (long long)set_out * 3 * sh.plane;
  float* p = B + 2 * sh.plane;
  if (threadIdx.x == 0)
    for (int q = 0; q < sh.n_src; ++q) {
      const long long k = src_lin[sh.src0 + q];
      p[k] = __fadd_rn(p[k], wav[sh.wav0 + (long long)(it - 1) * sh.n_src + q]);
    }
  __syncthreads();
  const long long blk = (long long)sh.n_rec * nt, o = sh.seis0 + (long long)sh.n_rec * (it - 1);
  for (int r = threadIdx.x; r < sh.n_rec; r += blockDim.x) {
    const long long k = rec_lin[sh.rec0 + r];
    seis[o + r] = p[k];
    seis[o + blk + r] = B[k];
    seis[o + 2 * blk + r] = B[sh.plane + k];
  }
}

// ---------------------------------------------------------------------------
// Fused single-sweep form of the step: one launch per time step covers every
// shot.  A CTA of NTX threads owns a strip of TXO = NTX - 2N - 2 output columns
// of one shot plus N + 1 columns on each side, one column per thread, and
// walks down z doing both half steps in one pass:
//   velocity at row zv: v' = update(A.v, A.p); v'' = Higdon(v', A.v) one row
//     behind (row zv - 1), its x neighbours from a shared-memory tile ring, its
//     z neighbours from the thread's registers;
//   pressure at row zp = zv - N - 1: p' = update(A.p, v''), reading vx'' rows
//     from a shared ring (x derivative) and vz'' from a register window (z
//     derivative); p'' = Higdon(p', A.p) one row behind.
// The edge columns of the strip only feed the neighbours' stencils and Higdon
// terms.  Every input row comes by TMA (per-shot tensor maps, no multicast)
// into a ring of slots guarded by mbarriers with bounded waits; a slot is
// refilled two rows after its use (its old-value boxes serve the next row's
// Higdon terms).  Persistent CTAs take (shot, strip, z range) segments from a
// list in order through a counter in device memory.  The arithmetic is the
// two-phase kernels' per-cell sequence (ac_vel_at / ac_prs_at and the Higdon
// edge and corner blends), so results are equal bit for bit.
// ---------------------------------------------------------------------------
struct AcShot {
  long long st;     // state offset: set k field f at st + (3k + f) * plane (vx, vz, p)
  long long mat;    // material offset: bx, bz, kappa at mat + f * plane
  long long plane;  // ld * nz
  int nx, nz, ld, unused;
  float q, qt, qxt, unused2;
};
constexpr int kAcMaps = 5;  // per shot: state x-halo row, state row, state 2 rows, material row, 2 rows
constexpr int kAcR = 4;     // TMA slots (two rows each)
constexpr int kAcVK = 8;    // vx'' ring rows
constexpr int kAcWt = 256;  // weight-table entries per kind staged in shared memory

__host__ __device__ constexpr int ac_al32(int n) { return (n + 31) & ~31; }

template <int N, int NTX>
struct AcShape {
  static constexpr int TXO = NTX - 2 * N - 2;            // output columns per strip
  static constexpr int XW = (NTX + 2 * N + 3 + 3) & ~3;  // p row with x halos (+3 alignment)
  static constexpr int CW = (NTX + 3 + 3) & ~3;          // row of the strip (+3 alignment)
  // one slot = the boxes of one iteration (two rows each; [plane][row][x])
  static constexpr int S_PX = 0;                          // p, rows zv, zv+1, x halos
  static constexpr int S_PW = S_PX + ac_al32(2 * XW);     // p, rows zv+N, zv+N+1 (z window)
  static constexpr int S_AV = S_PW + ac_al32(2 * CW);     // vx, vz, rows zv, zv+1
  static constexpr int S_MB = S_AV + ac_al32(4 * CW);     // bx, bz, rows zv, zv+1
  static constexpr int S_AP = S_MB + ac_al32(4 * CW);     // p, rows zp, zp+1
  static constexpr int S_KP = S_AP + ac_al32(2 * CW);     // kappa, rows zp, zp+1
  static constexpr int SLOT = S_KP + ac_al32(2 * CW);
  static constexpr unsigned BYTES = 4u * (2 * XW + 14 * CW);
  static_assert(XW <= 256 && CW <= 256, "a TMA box row holds at most 256 elements");
  static constexpr size_t smem() {
    return (size_t)kAcR * SLOT * 4 + (size_t)(12 + 6 + kAcVK) * NTX * 4 + 3 * kAcWt * 4 +
           (size_t)kAcR * 8;
  }
};

__device__ __forceinline__ void ac_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                           uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(tma::saddr(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(tma::saddr(bar))
      : "memory");
}

// staggered sums over shared memory (element stride 1) and register windows
template <int N>
__device__ __forceinline__ float ac_sdm(const float* f, const Coef& c) {
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l) acc = __fmaf_rn(c.a[l - 1], __fsub_rn(f[l - 1], f[-l]), acc);
  return acc;
}
template <int N>
__device__ __forceinline__ float ac_sdp(const float* f, const Coef& c) {
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l) acc = __fmaf_rn(c.a[l - 1], __fsub_rn(f[l], f[1 - l]), acc);
  return acc;
}
template <int N>
__device__ __forceinline__ float ac_wdm(const float (&w)[2 * N + 1], const Coef& c) {
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l) acc = __fmaf_rn(c.a[l - 1], __fsub_rn(w[N + l - 1], w[N - l]), acc);
  return acc;
}
template <int N>
__device__ __forceinline__ float ac_wdp(const float (&w)[2 * N + 1], const Coef& c) {
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l) acc = __fmaf_rn(c.a[l - 1], __fsub_rn(w[N + l], w[N - l + 1]), acc);
  return acc;
}

// the Higdon value of one field (kernels_det.jl:22-57): edge or corner blend of
// the side terms toward the interior-ward neighbours
__device__ __forceinline__ float ac_higdon(const HabcDev& h, float w, int sx, int sz, float fc,
                                           float fo, float fx, float fox, float fz, float foz) {
  if (sx != 0 && sz != 0)
    return higdon_corner(w, fc, higdon_side(h, fx, fo, fox), higdon_side(h, fz, fo, foz));
  if (sx != 0) return higdon_edge(w, fc, higdon_side(h, fx, fo, fox));
  return higdon_edge(w, fc, higdon_side(h, fz, fo, foz));
}

// The steps one launch runs, and the per-step injection and recording
// (inject_source.jl:4-24, fused_kernels.jl:137-149) it does between them.
struct AcRun {
  const UShot* tab;  // per shot: offsets, sources and receivers
  const int* src_lin;
  const float* wav;
  const int* rec_lin;
  float* seis;
  int ns, nsteps, it0, nt, set0;  // shots; steps of this launch; first step (1-based); run length
};

// Grid-wide barrier of a cooperative launch: an arrival counter and a
// generation word in device memory, the wait bounded (about a second) and
// recorded in *err when it gives up; returns false from then on.
__device__ __forceinline__ bool ac_grid_barrier(unsigned* cnt, unsigned* gen, int* err, bool ok,
                                                int* s_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    if (ok) {
      const unsigned g0 = *(volatile unsigned*)gen;
      __threadfence();  // this CTA's writes before its arrival
      if (atomicAdd(cnt, 1u) == gridDim.x - 1) {
        atomicExch(cnt, 0u);
        __threadfence();
        atomicAdd(gen, 1u);
      } else {
        for (int spin = 0; *(volatile unsigned*)gen == g0; ++spin) {
          if (spin > (1 << 24)) {
            atomicOr(err, 4);
            ok = false;
            break;
          }
          __nanosleep(64);
        }
      }
      __threadfence();
      // the next TMA reads (async proxy) see the other CTAs' stores
      asm volatile("fence.proxy.async;" ::: "memory");
    }
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

template <int N, int NTX>
__global__ void __launch_bounds__(NTX, NTX <= 128 ? 4 : 2) k_uac_sweep(const AcShot* __restrict__ shots,
                                                 const CUtensorMap* __restrict__ maps,
                                                 const int4* __restrict__ segs, int nseg,
                                                 int* __restrict__ sched, float* __restrict__ state,
                                                 Coef c, float dtx, float dtz,
                                                 const float* __restrict__ wtab, int nbc,
                                                 int wstride, AcRun run, int* __restrict__ err) {
  using S = AcShape<N, NTX>;
  // Two rows per iteration.  The pressure rows trail the velocity rows by D:
  // their vz'' window (own registers) must be finished one iteration earlier
  // (D >= N + 2) and their vx'' rows, which other threads write after the
  // barrier, two iterations earlier (D >= 5).
  constexpr int R = kAcR, D = (N + 2 > 5 ? N + 2 : 5), VK = kAcVK;
  constexpr int WV = D + N + 1;  // vz'' window: rows zp - N .. zv
  // vx'' ring: rows written after one barrier and rows read before the next
  // never share an entry (D mod VK not in 2..4), and a row read is not yet
  // replaced (VK > D - 2)
  static_assert(VK > D - 2 && D % VK != 2 && D % VK != 3 && D % VK != 4, "vx'' ring depth");
  extern __shared__ __align__(128) float sm[];
  float* slots = sm;
  float* vt = sm + R * S::SLOT;  // v' tile ring [3 iterations][2 rows][vx, vz][NTX]
  float* pt = vt + 12 * NTX;     // p' tile ring [3 iterations][2 rows][NTX]
  float* vr = pt + 6 * NTX;      // vx'' rows [VK][NTX]
  float* s_wt = vr + VK * NTX;   // weight ramps of vx, vz, p [3][kAcWt]
  uint64_t* bars = reinterpret_cast<uint64_t*>(s_wt + 3 * kAcWt);
  __shared__ int s_next;
  const int t = threadIdx.x;
  if (t == 0) {
    for (int k = 0; k < R; ++k) tma::mbar_init(&bars[k], 1);
    tma::mbar_init_fence();
  }
  for (int k = t; k < 3 * kAcWt; k += NTX) {
    const int kind = k / kAcWt, d = k % kAcWt;
    s_wt[k] = d < wstride ? __ldg(wtab + kind * wstride + d) : 1.0f;
  }
  auto weight = [&](int kind, int dist) {
    return dist < kAcWt ? s_wt[kind * kAcWt + dist]
                        : (dist < wstride ? __ldg(wtab + kind * wstride + dist) : 1.0f);
  };
  const bool v_lane = t >= 1 && t <= NTX - 2;           // v'' (x neighbours in the strip)
  const bool p_lane = t >= N && t <= NTX - N - 1;       // p' (vx'' x window in the strip)
  const bool o_lane = t >= N + 1 && t <= NTX - N - 2;   // output columns
  __shared__ int s_ok;
  int q = 0;  // TMA slot of the current iteration
  uint32_t ph = 0;
  long long gk = 0, ok_upto = 0, issued = 0;
  bool live = true, synced = true;
  // sched: [0], [1] segment counters of even / odd steps, [2], [3] grid barrier
  unsigned* bcnt = reinterpret_cast<unsigned*>(sched + 2);
  unsigned* bgen = reinterpret_cast<unsigned*>(sched + 3);
  for (int step = 0; step < run.nsteps; ++step) {
  const int set = (run.set0 + step) & 1;
  int* ctr = sched + (step & 1);
  for (;;) {
    __syncthreads();  // the previous segment's readers are done with every slot and ring
    if (t == 0) s_next = atomicAdd(ctr, 1);
    __syncthreads();
    const int sgi = s_next;
    if (sgi >= nseg) break;
    const int4 sg = segs[sgi];  // {shot, first output column, z0, z1}
    const AcShot sh = shots[sg.x];
    const CUtensorMap* mp = maps + kAcMaps * sg.x;
    const int X0 = sg.y, z0 = sg.z, z1 = sg.w;
    const int nx = sh.nx, nz = sh.nz, ld = sh.ld;
    const int xl = X0 - N - 1;  // column of lane 0
    const int x = xl + t;
    const int bxc = xl & ~3, shc = xl - bxc;
    const int bxh = (xl - N) & ~3, shh = xl - bxh;
    const int zs = z0 - N - 2;  // first velocity row
    // the last iteration finishes pressure row z1 - 1 (zp >= z1 - 1)
    const int nit = (z1 - 1 + D - zs + 1) / 2 + 1;
    const HabcDev h{sh.q, sh.qt, sh.qxt, nbc, wstride, wtab};
    const float* A = state + sh.st + (long long)set * 3 * sh.plane;
    float* B = state + sh.st + (long long)(1 - set) * 3 * sh.plane;
    const int pl = (int)sh.plane;
    const bool x_in = x >= N && x < nx - N;
    // x part of the frame classification (kernels_fused.jl:28-52)
    const bool fx = x >= 1 && x <= nx - 2;
    const int sx = x <= nbc ? 1 : (x >= nx - 1 - nbc ? -1 : 0);
    const int xdist = min(x, nx - 1 - x);
    const bool v_out = o_lane && x < nx;
    const int fa = set * 3;
    auto issue = [&](int i, int slot) {
      float* s = slots + slot * S::SLOT;
      uint64_t* bar = &bars[slot];
      const int zv = zs + 2 * i, zp = zv - D;
      tma::mbar_expect_tx(bar, S::BYTES);
      ac_load_3d(s + S::S_PX, mp + 0, bxh, zv, fa + 2, bar);
      ac_load_3d(s + S::S_PW, mp + 1, bxc, zv + N, fa + 2, bar);
      ac_load_3d(s + S::S_AV, mp + 2, bxc, zv, fa + 0, bar);
      ac_load_3d(s + S::S_MB, mp + 4, bxc, zv, 0, bar);
      ac_load_3d(s + S::S_AP, mp + 1, bxc, zp, fa + 2, bar);
      ac_load_3d(s + S::S_KP, mp + 3, bxc, zp, 2, bar);
    };
    if (t == 0 && live) {
      tma::fence_proxy_async();
      int sl = q;
      for (int i = 0; i < R && i < nit; ++i) {
        issue(i, sl);
        sl = sl + 1 == R ? 0 : sl + 1;
      }
      issued = gk + min(R, nit);
    }
    // z windows: wp[k] = p row zv - N + k (k < 2N + 2), for the velocity's z
    // derivative; wv[k] = vz'' row zp - N + k (k < WV), for the pressure's.
    float wp[2 * N + 2], wv[WV];
    {
      const float* pa = A + 2 * sh.plane;
#pragma unroll
      for (int k = 0; k < 2 * N; ++k) {
        const int z = zs - N + k;
        wp[k] = (x >= 0 && x < nx && z >= 0 && z < nz) ? __ldcg(pa + (long long)z * ld + x) : 0.0f;
      }
#pragma unroll
      for (int k = 0; k < WV; ++k) wv[k] = 0.0f;
    }
    // v', A.v, p', A.p of this iteration's two rows [phase][row]; the other
    // phase holds the previous iteration's
    float VX[2][2], VZ[2][2], AX[2][2], AZ[2][2], PP[2][2], AP[2][2];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) VX[a][b] = VZ[a][b] = AX[a][b] = AZ[a][b] = PP[a][b] = AP[a][b] = 0.0f;
    const int ce = t + shc;
    const float* s = slots + q * S::SLOT;  // boxes of the current iteration
    const float* sp = s;                    // ... and of the previous one
    int qp = q, qp2 = q;
    int ts = 0, tsp = 0;  // tile-ring entries of this and the previous iteration
    int ov = (zs - 1) * ld + x;      // output offset of v'' row zv - 1
    int op = (zs - D - 1) * ld + x;  // ... and of p'' row zp - 1
    auto body = [&](auto P, int i) {
      constexpr int p = decltype(P)::value, o = 1 - p;
      const int zv = zs + 2 * i, zp = zv - D;
      if (live) {
        live = tma::mbar_wait_bounded(&bars[q], ph, err);
        if (live) ok_upto = gk + i + 1;
      }
      wp[2 * N] = s[S::S_PW + ce];
      wp[2 * N + 1] = s[S::S_PW + S::CW + ce];
      float* vrow = vt + ts * 4 * NTX + t;  // [row][vx, vz][NTX]
      float* prow = pt + ts * 2 * NTX + t;
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        // velocity update, row zv + r (acoustic2d/fused_kernels.jl:27-63)
        AX[p][r] = VX[p][r] = s[S::S_AV + r * S::CW + ce];
        AZ[p][r] = VZ[p][r] = s[S::S_AV + (2 + r) * S::CW + ce];
        if (x_in && zv + r >= N && zv + r < nz - N) {
          const float dpdx = ac_sdm<N>(s + S::S_PX + r * S::XW + t + shh, c);
          const float dpdz = ac_wdp<N>(*reinterpret_cast<const float(*)[2 * N + 1]>(&wp[r]), c);
          VX[p][r] = __fmaf_rn(__fmul_rn(s[S::S_MB + r * S::CW + ce], dtx), dpdx, VX[p][r]);
          VZ[p][r] = __fmaf_rn(__fmul_rn(s[S::S_MB + (2 + r) * S::CW + ce], dtz), dpdz, VZ[p][r]);
        }
        // pressure update, row zp + r (fused_kernels.jl:86-114)
        AP[p][r] = PP[p][r] = s[S::S_AP + r * S::CW + ce];
        if (p_lane && x_in && zp + r >= N && zp + r < nz - N) {
          const float dvxdx = ac_sdp<N>(vr + ((zp + r) & (VK - 1)) * NTX + t, c);
          const float dvzdz = ac_wdm<N>(*reinterpret_cast<const float(*)[2 * N + 1]>(&wv[r]), c);
          PP[p][r] = __fmaf_rn(s[S::S_KP + r * S::CW + ce],
                               __fmaf_rn(dvxdx, dtx, __fmul_rn(dvzdz, dtz)), PP[p][r]);
        }
        vrow[r * 2 * NTX] = VX[p][r];
        vrow[r * 2 * NTX + NTX] = VZ[p][r];
        prow[r * NTX] = PP[p][r];
      }
      __syncthreads();  // rows zv, zv+1 (v') and zp, zp+1 (p') are complete
      if (t == 0 && live && i >= 2 && i + R - 2 < nit) {
        tma::fence_proxy_async();
        issue(i + R - 2, qp2);
        issued = gk + i + R - 1;
      }
      if (i >= 1) {
        const float* vprev = vt + tsp * 4 * NTX + t;
        const float* pprev = pt + tsp * 2 * NTX + t;
        // v'' of rows zv - 1 (r = 0) and zv (r = 1) (kernels_det.jl:22-57)
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const int zq = zv - 1 + r;
          // the row, its upper (zq - 1) and lower (zq + 1) neighbours
          const float fcx = r ? VX[p][0] : VX[o][1], fcz = r ? VZ[p][0] : VZ[o][1];
          const float ocx = r ? AX[p][0] : AX[o][1], ocz = r ? AZ[p][0] : AZ[o][1];
          float ux = fcx, uz = fcz;
          if (v_lane && fx && zq >= 1 && zq <= nz - 2) {
            const int sz = zq <= nbc ? 1 : (zq >= nz - 1 - nbc ? -1 : 0);
            if (sx | sz) {
              const int dist = min(xdist, min(zq, nz - 1 - zq));
              const float* vrw = r ? vrow : vprev + 2 * NTX;  // v' of row zq
              const float* arw = r ? s + S::S_AV + ce : sp + S::S_AV + S::CW + ce;  // A.v of row zq
              const float dnx = r ? VX[p][1] : VX[p][0], upx = r ? VX[o][1] : VX[o][0];
              const float dnz = r ? VZ[p][1] : VZ[p][0], upz = r ? VZ[o][1] : VZ[o][0];
              const float adx = r ? AX[p][1] : AX[p][0], aux = r ? AX[o][1] : AX[o][0];
              const float adz = r ? AZ[p][1] : AZ[p][0], auz = r ? AZ[o][1] : AZ[o][0];
              ux = ac_higdon(h, weight(0, dist), sx, sz, ux, ocx, vrw[sx], arw[sx],
                             sz > 0 ? dnx : upx, sz > 0 ? adx : aux);
              uz = ac_higdon(h, weight(1, dist), sx, sz, uz, ocz, vrw[NTX + sx],
                             arw[2 * S::CW + sx], sz > 0 ? dnz : upz, sz > 0 ? adz : auz);
            }
          }
          vr[(zq & (VK - 1)) * NTX + t] = ux;
          wv[D + N - 1 + r] = uz;
          if (v_out && zq >= z0 && zq < z1) {
            B[ov + r * ld] = ux;
            B[pl + ov + r * ld] = uz;
          }
        }
        // p'' of rows zp - 1 (r = 0) and zp (r = 1)
        if (o_lane) {
#pragma unroll
          for (int r = 0; r < 2; ++r) {
            const int zq = zp - 1 + r;
            float u = r ? PP[p][0] : PP[o][1];
            if (fx && zq >= 1 && zq <= nz - 2) {
              const int sz = zq <= nbc ? 1 : (zq >= nz - 1 - nbc ? -1 : 0);
              if (sx | sz) {
                const int dist = min(xdist, min(zq, nz - 1 - zq));
                const float* prw = r ? prow : pprev + NTX;
                const float* arw = r ? s + S::S_AP + ce : sp + S::S_AP + S::CW + ce;
                const float dn = r ? PP[p][1] : PP[p][0], up = r ? PP[o][1] : PP[o][0];
                const float ad = r ? AP[p][1] : AP[p][0], au = r ? AP[o][1] : AP[o][0];
                u = ac_higdon(h, weight(2, dist), sx, sz, u, r ? AP[p][0] : AP[o][1], prw[sx],
                              arw[sx], sz > 0 ? dn : up, sz > 0 ? ad : au);
              }
            }
            if (x < nx && zq >= z0 && zq < z1) B[2 * pl + op + r * ld] = u;
          }
        }
      }
      // advance: windows, tile ring, offsets, slots
#pragma unroll
      for (int k = 0; k < 2 * N; ++k) wp[k] = wp[k + 2];
#pragma unroll
      for (int k = 0; k + 2 < WV; ++k) wv[k] = wv[k + 2];
      tsp = ts;
      ts = ts == 2 ? 0 : ts + 1;
      ov += 2 * ld;
      op += 2 * ld;
      sp = s;
      qp2 = qp;
      qp = q;
      if (++q == R) {
        q = 0;
        ph ^= 1u;
        s = slots;
      } else {
        s += S::SLOT;
      }
    };
    for (int i = 0; i < nit;) {
      body(std::integral_constant<int, 0>{}, i);
      if (++i >= nit) break;
      body(std::integral_constant<int, 1>{}, i);
      ++i;
    }
    gk += nit;
  }
  // every strip of every shot has finished this step: inject into p, then
  // record p, vx, vz (sources in order, CTA b takes shots b, b + grid, ...)
  synced = ac_grid_barrier(bcnt, bgen, err, synced, &s_ok);
  const int it = run.it0 + step;
  for (int sh = blockIdx.x; sh < run.ns; sh += gridDim.x) {
    const UShot u = run.tab[sh];
    float* Bo = state + u.st + (long long)(1 - set) * 3 * u.plane;
    float* p = Bo + 2 * u.plane;
    if (t == 0)
      for (int k = 0; k < u.n_src; ++k) {
        const long long cell = run.src_lin[u.src0 + k];
        p[cell] = __fadd_rn(__ldcg(p + cell), run.wav[u.wav0 + (long long)(it - 1) * u.n_src + k]);
      }
    __syncthreads();
    const long long blk = (long long)u.n_rec * run.nt, o = u.seis0 + (long long)u.n_rec * (it - 1);
    for (int r = t; r < u.n_rec; r += NTX) {
      const long long cell = run.rec_lin[u.rec0 + r];
      run.seis[o + r] = __ldcg(p + cell);
      run.seis[o + blk + r] = __ldcg(Bo + cell);
      run.seis[o + 2 * blk + r] = __ldcg(Bo + u.plane + cell);
    }
  }
  if (blockIdx.x == 0 && t == 0) sched[(step + 1) & 1] = 0;  // rearm the next step's counter
  synced = ac_grid_barrier(bcnt, bgen, err, synced, &s_ok);
  }
  if (t == 0 && !live)
    for (long long k = ok_upto; k < issued; ++k)
      tma::mbar_wait_bounded(&bars[k % R], (uint32_t)((k / R) & 1), err);
}

// ---- fused sweep: host side ----
PFN_cuTensorMapEncodeTiled_v12000 g_acenc = nullptr;
std::once_flag g_acenc_once;
PFN_cuTensorMapEncodeTiled_v12000 ac_encoder() {
  std::call_once(g_acenc_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_acenc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    else
      cudaGetLastError();
  });
  return g_acenc;
}

constexpr int kAcNTX[] = {128, 224};  // strip widths the autotuner tries (threads per CTA; a
                                      // row box of the widest holds 224 + 2N + 3 <= 256 columns)
constexpr int kAcNumNTX = 2;

template <int N, int NTX>
cudaError_t ac_launch_t(cudaStream_t st, int grid, const AcShot* shots, const CUtensorMap* maps,
                        const int4* segs, int nseg, int* sched, float* state, const Coef& c,
                        float dtdh, const float* wtab, int nbc, int wstride, const AcRun& run,
                        int* err) {
  auto kern = k_uac_sweep<N, NTX>;
  static std::once_flag once;
  static cudaError_t attr = cudaSuccess;
  std::call_once(once, [&] {
    attr = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)AcShape<N, NTX>::smem());
  });
  if (attr != cudaSuccess) return attr;
  // the counters and the barrier start from zero; the CTAs wait on one another
  // between steps, so the launch is cooperative (all of them resident)
  cudaError_t e = cudaMemsetAsync(sched, 0, 4 * sizeof(int), st);
  if (e != cudaSuccess) return e;
  float dtx = dtdh, dtz = dtdh;
  Coef cc = c;
  AcRun rr = run;
  void* args[] = {(void*)&shots, (void*)&maps,   (void*)&segs, (void*)&nseg, (void*)&sched,
                  (void*)&state, (void*)&cc,     (void*)&dtx,  (void*)&dtz,  (void*)&wtab,
                  (void*)&nbc,   (void*)&wstride, (void*)&rr,  (void*)&err};
  return cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(NTX), args,
                                     AcShape<N, NTX>::smem(), st);
}

template <int N, int NTX>
int ac_resident() {
  int nb = 0, dev = 0, nsm = 148;
  if (cudaFuncSetAttribute(k_uac_sweep<N, NTX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)AcShape<N, NTX>::smem()) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_uac_sweep<N, NTX>, NTX,
                                                    AcShape<N, NTX>::smem()) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return nb * nsm;
}

// Dispatch over (N, strip width): the launch, the resident CTA count, the strip's
// output columns and the box widths of its tensor maps.
struct AcForm {
  int resident = 0, txo = 0, xw = 0, cw = 0;
};
template <int N, int NTX>
AcForm ac_form_t() {
  using S = AcShape<N, NTX>;
  return AcForm{ac_resident<N, NTX>(), S::TXO, S::XW, S::CW};
}
AcForm ac_form(int N, int k) {
#define FOMO_ACF(NN)                                                       \
  case NN:                                                                 \
    return k == 0 ? ac_form_t<NN, 128>() : ac_form_t<NN, 224>();
  switch (N) { FOMO_ACF(2) FOMO_ACF(3) FOMO_ACF(4) FOMO_ACF(5) }
#undef FOMO_ACF
  return AcForm{};
}
cudaError_t ac_launch(int N, int k, cudaStream_t st, int grid, const AcShot* shots,
                      const CUtensorMap* maps, const int4* segs, int nseg, int* sched,
                      float* state, const Coef& c, float dtdh, const float* wtab, int nbc,
                      int wstride, const AcRun& run, int* err) {
#define FOMO_ACL(NN)                                                                          \
  case NN:                                                                                    \
    return k == 0 ? ac_launch_t<NN, 128>(st, grid, shots, maps, segs, nseg, sched, state, c, \
                                         dtdh, wtab, nbc, wstride, run, err)                  \
                  : ac_launch_t<NN, 224>(st, grid, shots, maps, segs, nseg, sched, state, c, \
                                         dtdh, wtab, nbc, wstride, run, err);
  switch (N) { FOMO_ACL(2) FOMO_ACL(3) FOMO_ACL(4) FOMO_ACL(5) }
#undef FOMO_ACL
  return cudaErrorInvalidValue;
}

CUresult ac_encode(CUtensorMap* m, const float* base, int nx, int nz, int ld, long long plane,
                   int nplanes, int bw, int bp) {
  cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)nz, (cuuint64_t)nplanes};
  cuuint64_t strides[2] = {(cuuint64_t)ld * 4, (cuuint64_t)plane * 4};
  cuuint32_t box[3] = {(cuuint32_t)bw, 2, (cuuint32_t)bp};  // two rows per iteration
  cuuint32_t es[3] = {1, 1, 1};
  return ac_encoder()(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims,
                      strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

struct Tile {
  int bx, by;
};
constexpr Tile kTiles[] = {{32, 8}, {64, 4}, {128, 2}, {16, 16}, {32, 4}};
constexpr int kNumTiles = sizeof(kTiles) / sizeof(kTiles[0]);

struct UKey {
  int N, ns;
  long long cells;
  bool operator<(const UKey& o) const { return std::tie(N, ns, cells) < std::tie(o.N, o.ns, o.cells); }
};
std::mutex g_umu;
std::map<UKey, int> g_utune;

template <int N>
void launch_step(cudaStream_t st, int nblk, Tile t, const UShot* shots, const int* tile_shot,
                 float* state, const float* mat, const Coef& c, float dtdh, const float* wtab,
                 int nbc, int wstride, int set) {
  const dim3 b(t.bx, t.by);
  k_uac_vel<N><<<nblk, b, 0, st>>>(shots, tile_shot, state, mat, c, dtdh, dtdh, wtab, nbc, wstride,
                                   set);
  k_uac_prs<N><<<nblk, b, 0, st>>>(shots, tile_shot, state, mat, c, dtdh, dtdh, wtab, nbc, wstride,
                                   set);
}

void launch_step_n(int N, cudaStream_t st, int nblk, Tile t, const UShot* shots,
                   const int* tile_shot, float* state, const float* mat, const Coef& c, float dtdh,
                   const float* wtab, int nbc, int wstride, int set) {
  switch (N) {
    case 1: launch_step<1>(st, nblk, t, shots, tile_shot, state, mat, c, dtdh, wtab, nbc, wstride, set); break;
    case 2: launch_step<2>(st, nblk, t, shots, tile_shot, state, mat, c, dtdh, wtab, nbc, wstride, set); break;
    case 3: launch_step<3>(st, nblk, t, shots, tile_shot, state, mat, c, dtdh, wtab, nbc, wstride, set); break;
    case 4: launch_step<4>(st, nblk, t, shots, tile_shot, state, mat, c, dtdh, wtab, nbc, wstride, set); break;
    case 5: launch_step<5>(st, nblk, t, shots, tile_shot, state, mat, c, dtdh, wtab, nbc, wstride, set); break;
  }
}

int run_uneven(fomo_ctx* ctx, float dh, float dt, int nt, int nbc, int fd_order, int ns,
               const fomo_shot2d* shots, const fomo_opts* opts, fomo_stats* stats) {
  if (!ctx) return FOMO_EARG;
  const int N = order_to_N(fd_order);
  if (N < 0) return fail(ctx, FOMO_EARG, "Unsupported FD order: " + std::to_string(fd_order));
  if (ns < 1 || !shots) return fail(ctx, FOMO_EARG, "no shots");
  if (nt < 1 || nbc < 0 || !(dh > 0.0f) || !(dt > 0.0f))
    return fail(ctx, FOMO_EARG, "invalid dh, dt, nt or nbc");
  if (opts && (opts->flags & FOMO_F_DEVICE_PTRS))
    return fail(ctx, FOMO_EUNSUPPORTED, "the uneven batch takes host arrays");
  if (opts && opts->precision != FOMO_FP32)
    return fail(ctx, FOMO_EUNSUPPORTED, "the uneven batch stores FP32 only");
  const int pad = nbc + N;
  if (pad < 2) return fail(ctx, FOMO_EARG, "nbc + fd_order/2 must be >= 2");
  FOMO_CU(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;

  // ---- per-shot validation, geometry and offsets ----
  std::vector<UShot> tab(ns);
  std::vector<int32_t> src_lin, rec_lin;
  long long off_state = 0, off_mat = 0, off_wav = 0, off_seis = 0, off_model = 0;
  long long cells = 0;
  std::vector<float> wt_ref;
  int wstride = 0, zone = 0;
  for (int s = 0; s < ns; ++s) {
    const fomo_shot2d& in = shots[s];
    const std::string tag = "shot " + std::to_string(s + 1) + ": ";
    if (in.nx < 1 || in.nz < 1 || !in.vp || !in.rho)
      return fail(ctx, FOMO_EARG, tag + "model arrays and a positive grid are required");
    if (in.n_src < 0 || in.n_rec < 0 || (in.n_src && (!in.sx || !in.sz || !in.wavelet)) ||
        (in.n_rec && (!in.rx || !in.rz)))
      return fail(ctx, FOMO_EARG, tag + "invalid acquisition");
    UShot& u = tab[s];
    u.nx = in.nx + 2 * pad;
    u.nz = in.nz + 2 * pad;
    u.ld = (u.nx + 31) & ~31;
    u.plane = (long long)u.ld * u.nz;
    if (u.plane > (1LL << 31)) return fail(ctx, FOMO_EARG, tag + "padded grid exceeds 2^31 cells");
    u.st = off_state;
    off_state += 6 * u.plane;
    u.mat = off_mat;
    off_mat += 3 * u.plane;
    u.wav0 = off_wav;
    off_wav += (long long)in.n_src * nt;
    u.seis0 = off_seis;
    off_seis += 3LL * in.n_rec * nt;
    u.n_src = in.n_src;
    u.src0 = (int)src_lin.size();
    u.n_rec = in.n_rec;
    u.rec0 = (int)rec_lin.size();
    for (int k = 0; k < in.n_src; ++k) {
      if (in.sx[k] < 1 || in.sx[k] > in.nx || in.sz[k] < 1 || in.sz[k] > in.nz)
        return fail(ctx, FOMO_EARG, tag + "source index out of range");
      src_lin.push_back((in.sx[k] - 1 + pad) + u.ld * (in.sz[k] - 1 + pad));
    }
    for (int k = 0; k < in.n_rec; ++k) {
      if (in.rx[k] < 1 || in.rx[k] > in.nx || in.rz[k] < 1 || in.rz[k] > in.nz)
        return fail(ctx, FOMO_EARG, tag + "receiver index out of range");
      rec_lin.push_back((in.rx[k] - 1 + pad) + u.ld * (in.rz[k] - 1 + pad));
    }
    float v_ref = in.v_ref;
    const long long nint = (long long)in.nx * in.nz;
    if (!(v_ref > 0.0f)) {  // minimum(vp[vp .> 0]) (acoustic2d.jl:55)
      v_ref = INFINITY;
      for (long long k = 0; k < nint; ++k)
        if (in.vp[k] > 0.0f && in.vp[k] < v_ref) v_ref = in.vp[k];
      if (!std::isfinite(v_ref)) return fail(ctx, FOMO_EARG, tag + "vp has no positive value");
    }
    const HabcHost hh = make_habc(pad, v_ref, dt, dh);
    u.q = hh.q;
    u.qt = hh.qt;
    u.qxt = hh.qxt;
    if (s == 0) {
      wt_ref = hh.wtab;  // the ramps depend on pad only, shared by every shot
      wstride = hh.wstride;
      zone = hh.nbc;
    }
    off_model = std::max(off_model, 2 * nint);
    cells += (long long)u.nx * u.nz;
  }

  // ---- tile shape: FOMO_UNEVEN_TILE="bx,by" pins it, else timed once per shape ----
  int tsel = -1;
  if (const char* env = std::getenv("FOMO_UNEVEN_TILE")) {
    int bx = 0, by = 0;
    if (std::sscanf(env, "%d,%d", &bx, &by) == 2)
      for (int k = 0; k < kNumTiles; ++k)
        if (kTiles[k].bx == bx && kTiles[k].by == by) tsel = k;
    if (tsel < 0) return fail(ctx, FOMO_EARG, "bad FOMO_UNEVEN_TILE (one of 32,8 64,4 128,2 16,16 32,4)");
  }
  const UKey key{N, ns, cells};
  if (tsel < 0) {
    std::lock_guard<std::mutex> lk(g_umu);
    auto it = g_utune.find(key);
    if (it != g_utune.end()) tsel = it->second;
  }
  auto tiles_for = [&](Tile t, std::vector<int>& tile_shot) {
    tile_shot.clear();
    for (int s = 0; s < ns; ++s) {
      UShot& u = tab[s];
      u.tiles_x = (u.nx + t.bx - 1) / t.bx;
      u.tile0 = (int)tile_shot.size();
      const long long n = (long long)u.tiles_x * ((u.nz + t.by - 1) / t.by);
      tile_shot.insert(tile_shot.end(), (size_t)n, s);
    }
  };
  long long max_tiles = 0;
  for (int k = 0; k < kNumTiles; ++k) {
    std::vector<int> ts;
    tiles_for(kTiles[k], ts);
    max_tiles = std::max(max_tiles, (long long)ts.size());
  }

  // ---- workspace ----
  Arena ar;
  const size_t o_state = ar.take<float>(off_state);
  const size_t o_mat = ar.take<float>(off_mat);
  const size_t o_model = ar.take<float>(off_model);
  const size_t o_wav = ar.take<float>(std::max(off_wav, 1LL));
  const size_t o_seis = ar.take<float>(std::max(off_seis, 1LL));
  const size_t o_src = ar.take<int32_t>(std::max<size_t>(src_lin.size(), 1));
  const size_t o_rec = ar.take<int32_t>(std::max<size_t>(rec_lin.size(), 1));
  const size_t o_tab = ar.take<UShot>(ns);
  const size_t o_tiles = ar.take<int>(max_tiles);
  const size_t o_w = ar.take<float>(wt_ref.size());
  // fused sweep: shot table, five tensor maps per shot, segment list, counter
  long long max_seg = 3LL * 4096;
  for (int s = 0; s < ns; ++s) max_seg += (tab[s].nx + 63) / 64;
  const size_t o_ashot = ar.take<AcShot>(ns);
  const size_t o_maps = ar.take<CUtensorMap>((size_t)kAcMaps * ns);
  const size_t o_segs = ar.take<int4>(max_seg);
  const size_t o_sched = ar.take<int>(4);
  int rc;
  if ((rc = ensure_workspace(ctx, ar.off))) return rc;
  float* d_state = ws_ptr<float>(ctx, o_state);
  float* d_mat = ws_ptr<float>(ctx, o_mat);
  float* d_model = ws_ptr<float>(ctx, o_model);
  float* d_wav = ws_ptr<float>(ctx, o_wav);
  float* d_seis = ws_ptr<float>(ctx, o_seis);
  int32_t* d_src = ws_ptr<int32_t>(ctx, o_src);
  int32_t* d_rec = ws_ptr<int32_t>(ctx, o_rec);
  UShot* d_tab = ws_ptr<UShot>(ctx, o_tab);
  int* d_tiles = ws_ptr<int>(ctx, o_tiles);
  float* d_w = ws_ptr<float>(ctx, o_w);

  // ---- materials per shot (device preparation, one model staging buffer) ----
  const float dtdh = dt / dh;
  for (int s = 0; s < ns; ++s) {
    const fomo_shot2d& in = shots[s];
    const long long nint = (long long)in.nx * in.nz;
    FOMO_CU(ctx, cudaMemcpyAsync(d_model, in.vp, 4 * nint, cudaMemcpyHostToDevice, st));
    FOMO_CU(ctx, cudaMemcpyAsync(d_model + nint, in.rho, 4 * nint, cudaMemcpyHostToDevice, st));
    float* m = d_mat + tab[s].mat;
    FOMO_CU(ctx, launch_medium2d(st, 1, in.nx, in.nz, pad, tab[s].ld, dtdh, d_model, nullptr,
                                 d_model + nint, m, m + tab[s].plane, m + 2 * tab[s].plane, nullptr,
                                 nullptr));
    if (in.n_src)
      FOMO_CU(ctx, cudaMemcpyAsync(d_wav + tab[s].wav0, in.wavelet, 4LL * in.n_src * nt,
                                   cudaMemcpyHostToDevice, st));
    // the staging buffer is reused by the next shot: wait for this one's reads
    FOMO_CU(ctx, cudaStreamSynchronize(st));
  }
  if (!src_lin.empty())
    FOMO_CU(ctx, cudaMemcpyAsync(d_src, src_lin.data(), 4 * src_lin.size(), cudaMemcpyHostToDevice, st));
  if (!rec_lin.empty())
    FOMO_CU(ctx, cudaMemcpyAsync(d_rec, rec_lin.data(), 4 * rec_lin.size(), cudaMemcpyHostToDevice, st));
  FOMO_CU(ctx, cudaMemcpyAsync(d_w, wt_ref.data(), 4 * wt_ref.size(), cudaMemcpyHostToDevice, st));

  Coef c;
  for (int l = 0; l < 5; ++l) c.a[l] = kFD[N][l];

  // ---- fused single sweep (the default from order 4): strip width autotuned ----
  const char* env_sweep = std::getenv("FOMO_UNEVEN_SWEEP");
  const bool fused = N >= 2 && ac_encoder() && !std::getenv("FOMO_UNEVEN_TILE") &&
                     !(opts && opts->kernel == FOMO_KERNEL_TWO_PHASE);
  AcShot* d_ashot = ws_ptr<AcShot>(ctx, o_ashot);
  CUtensorMap* d_maps = ws_ptr<CUtensorMap>(ctx, o_maps);
  int4* d_segs = ws_ptr<int4>(ctx, o_segs);
  int* d_sched = ws_ptr<int>(ctx, o_sched);
  int a_grid = 0, a_nseg = 0, a_k = -1;
  // Builds the tables of strip width kAcNTX[k]; returns FOMO_OK or a negative
  // code, and a_grid = 0 when that width does not fit an SM.
  auto ac_build = [&](int k) -> int {
    const AcForm f = ac_form(N, k);
    a_grid = 0;
    if (f.resident < 1) return FOMO_OK;
    std::vector<AcShot> at(ns);
    std::vector<CUtensorMap> mh((size_t)kAcMaps * ns);
    std::vector<int4> sg;
    for (int s = 0; s < ns; ++s) {
      const UShot& u = tab[s];
      at[s] = AcShot{u.st, u.mat, u.plane, u.nx, u.nz, u.ld, 0, u.q, u.qt, u.qxt, 0.0f};
      const float* bs = d_state + u.st;
      const float* bm = d_mat + u.mat;
      CUresult r = ac_encode(&mh[kAcMaps * s + 0], bs, u.nx, u.nz, u.ld, u.plane, 6, f.xw, 1);
      if (r == CUDA_SUCCESS) r = ac_encode(&mh[kAcMaps * s + 1], bs, u.nx, u.nz, u.ld, u.plane, 6, f.cw, 1);
      if (r == CUDA_SUCCESS) r = ac_encode(&mh[kAcMaps * s + 2], bs, u.nx, u.nz, u.ld, u.plane, 6, f.cw, 2);
      if (r == CUDA_SUCCESS) r = ac_encode(&mh[kAcMaps * s + 3], bm, u.nx, u.nz, u.ld, u.plane, 3, f.cw, 1);
      if (r == CUDA_SUCCESS) r = ac_encode(&mh[kAcMaps * s + 4], bm, u.nx, u.nz, u.ld, u.plane, 3, f.cw, 2);
      if (r != CUDA_SUCCESS) return fail(ctx, FOMO_ECUDA, "uneven sweep: tensor map encoding failed");
    }
    // Strips in order of decreasing height (the longest segments first, a
    // shot's strips side by side so that neighbours share halo rows in L2); the
    // last wave of strips is cut into four z chunks (chunk-major) so that the
    // persistent CTAs finish together.
    std::vector<int> order(ns);
    for (int s = 0; s < ns; ++s) order[s] = s;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return tab[a].nz > tab[b].nz; });
    for (int s : order)
      for (int x0 = 0; x0 < tab[s].nx; x0 += f.txo) sg.push_back(make_int4(s, x0, 0, tab[s].nz));
    a_grid = std::min<int>(f.resident, (int)sg.size());
    const int L = std::min<int>(a_grid, (int)sg.size());
    std::vector<int4> tail(sg.end() - L, sg.end());
    sg.resize(sg.size() - L);
    for (int k2 = 0; k2 < 4; ++k2)
      for (const int4& e : tail) {
        const int za = (int)((long long)e.w * k2 / 4), zb = (int)((long long)e.w * (k2 + 1) / 4);
        if (zb > za) sg.push_back(make_int4(e.x, e.y, za, zb));
      }
    if ((long long)sg.size() > max_seg) return fail(ctx, FOMO_ECUDA, "uneven sweep: segment table");
    a_nseg = (int)sg.size();
    FOMO_CU(ctx, cudaMemcpyAsync(d_ashot, at.data(), sizeof(AcShot) * ns, cudaMemcpyHostToDevice, st));
    FOMO_CU(ctx, cudaMemcpyAsync(d_maps, mh.data(), sizeof(CUtensorMap) * mh.size(),
                                 cudaMemcpyHostToDevice, st));
    FOMO_CU(ctx, cudaMemcpyAsync(d_segs, sg.data(), sizeof(int4) * sg.size(), cudaMemcpyHostToDevice, st));
    FOMO_CU(ctx, cudaStreamSynchronize(st));  // host tables change before the next build
    return FOMO_OK;
  };
  // one cooperative launch runs steps it0 .. it0 + nsteps - 1, injecting and
  // recording after each
  auto ac_run = [&](cudaStream_t s2, int it0, int nsteps) {
    const AcRun run{d_tab, d_src, d_wav, d_rec, d_seis, ns, nsteps, it0, nt, (it0 - 1) & 1};
    return ac_launch(N, a_k, s2, a_grid, d_ashot, d_maps, d_segs, a_nseg, d_sched, d_state, c,
                     dtdh, d_w, zone, wstride, run, ctx->d_flag);
  };
  if (fused) {
    FOMO_CU(ctx, cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), st));
    // the in-kernel injection and recording read the shot table
    FOMO_CU(ctx, cudaMemcpyAsync(d_tab, tab.data(), sizeof(UShot) * ns, cudaMemcpyHostToDevice, st));
    int pin = -1;
    if (env_sweep)
      for (int k = 0; k < kAcNumNTX; ++k)
        if (std::atoi(env_sweep) == kAcNTX[k]) pin = k;
    const UKey key{-N, ns, cells};  // negative order: the fused form's cache entries
    if (pin < 0) {
      std::lock_guard<std::mutex> lk(g_umu);
      auto it = g_utune.find(key);
      if (it != g_utune.end()) pin = it->second;
    }
    if (pin < 0) {  // time each strip width on three steps of the zero state
      FOMO_CU(ctx, cudaMemsetAsync(d_state, 0, 4 * off_state, st));
      float best = 1e30f;
      for (int k = 0; k < kAcNumNTX; ++k) {
        if ((rc = ac_build(k))) return rc;
        if (a_grid < 1) continue;
        a_k = k;
        FOMO_CU(ctx, ac_run(st, 1, 1));
        FOMO_CU(ctx, cudaEventRecord(ctx->ev0, st));
        FOMO_CU(ctx, ac_run(st, 1, 3));
        FOMO_CU(ctx, cudaEventRecord(ctx->ev1, st));
        FOMO_CU(ctx, cudaEventSynchronize(ctx->ev1));
        float ms = 0.0f;
        FOMO_CU(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        if (ms < best) {
          best = ms;
          pin = k;
        }
      }
      if (pin < 0) return fail(ctx, FOMO_ECUDA, "uneven sweep: no strip width fits an SM");
      std::lock_guard<std::mutex> lk(g_umu);
      g_utune[key] = pin;
    }
    if ((rc = ac_build(pin))) return rc;
    if (a_grid < 1) return fail(ctx, FOMO_ECUDA, "uneven sweep: the strip width does not fit an SM");
    a_k = pin;
  }
  std::vector<int> tile_shot;
  auto upload_tiles = [&](int k) -> int {
    tiles_for(kTiles[k], tile_shot);
    FOMO_CU(ctx, cudaMemcpyAsync(d_tab, tab.data(), sizeof(UShot) * ns, cudaMemcpyHostToDevice, st));
    FOMO_CU(ctx, cudaMemcpyAsync(d_tiles, tile_shot.data(), 4 * tile_shot.size(),
                                 cudaMemcpyHostToDevice, st));
    FOMO_CU(ctx, cudaStreamSynchronize(st));  // host vectors change before the next upload
    return FOMO_OK;
  };

  if (!fused && tsel < 0) {  // time each tile shape on three steps of the zero state
    FOMO_CU(ctx, cudaMemsetAsync(d_state, 0, 4 * off_state, st));
    float best = 1e30f;
    for (int k = 0; k < kNumTiles; ++k) {
      if ((rc = upload_tiles(k))) return rc;
      const int nblk = (int)tile_shot.size();
      launch_step_n(N, st, nblk, kTiles[k], d_tab, d_tiles, d_state, d_mat, c, dtdh, d_w, zone,
                    wstride, 0);
      FOMO_CU(ctx, cudaEventRecord(ctx->ev0, st));
      for (int r = 0; r < 3; ++r)
        launch_step_n(N, st, nblk, kTiles[k], d_tab, d_tiles, d_state, d_mat, c, dtdh, d_w, zone,
                      wstride, r & 1);
      FOMO_CU(ctx, cudaEventRecord(ctx->ev1, st));
      FOMO_CU(ctx, cudaEventSynchronize(ctx->ev1));
      float ms = 0.0f;
      FOMO_CU(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
      if (ms < best) {
        best = ms;
        tsel = k;
      }
    }
    std::lock_guard<std::mutex> lk(g_umu);
    g_utune[key] = tsel;
  }
  if (!fused && (rc = upload_tiles(tsel))) return rc;
  const int nblk = (int)tile_shot.size();
  const Tile t = fused ? Tile{0, 0} : kTiles[tsel];

  // ---- zero state, capture the whole run, replay it once ----
  FOMO_CU(ctx, cudaMemsetAsync(d_state, 0, 4 * off_state, st));
  FOMO_CU(ctx, cudaMemsetAsync(d_seis, 0, 4 * std::max(off_seis, 1LL), st));
  FOMO_CU(ctx, cudaStreamSynchronize(st));
  float ms = 0.0f;
  if (fused) {  // the whole run is one persistent launch
    FOMO_CU(ctx, cudaEventRecord(ctx->ev0, st));
    FOMO_CU(ctx, ac_run(st, 1, nt));
    FOMO_CU(ctx, cudaEventRecord(ctx->ev1, st));
    FOMO_CU(ctx, cudaStreamSynchronize(st));
    FOMO_CU(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    int hflag = 0;
    FOMO_CU(ctx, cudaMemcpy(&hflag, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (hflag)
      return fail(ctx, FOMO_ECUDA, "uneven sweep: a bounded TMA wait or grid barrier timed out");
  }
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // Capture on the context's own stream: the caller's stream may be the
  // legacy default stream, which cannot be captured.  Replay on the caller's.
  const cudaStream_t cs = ctx->own_stream;
  if (!fused) {  // velocity / pressure kernels: the run captured into one graph
    FOMO_CU(ctx, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    for (int it = 1; it <= nt; ++it) {
      const int A = (it - 1) & 1;
      launch_step_n(N, cs, nblk, t, d_tab, d_tiles, d_state, d_mat, c, dtdh, d_w, zone, wstride, A);
      k_uinject_record<<<ns, 256, 0, cs>>>(d_tab, d_state, d_src, d_wav, d_rec, d_seis, it, nt,
                                           1 - A);
    }
    cudaError_t ce = cudaStreamEndCapture(cs, &graph);
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, "capture of the uneven-batch run");
    ce = cudaGraphInstantiate(&exec, graph, 0);
    if (ce != cudaSuccess) {
      cudaGraphDestroy(graph);
      return cuda_fail(ctx, ce, "cudaGraphInstantiate");
    }
    FOMO_CU(ctx, cudaEventRecord(ctx->ev0, st));
    ce = cudaGraphLaunch(exec, st);
    if (ce == cudaSuccess) ce = cudaEventRecord(ctx->ev1, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, "uneven-batch graph launch");
    FOMO_CU(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  }

  // ---- seismograms back to each shot's buffers ----
  for (int s = 0; s < ns; ++s) {
    const fomo_shot2d& in = shots[s];
    const long long blk = (long long)in.n_rec * nt;
    float* outs[3] = {in.seis_p, in.seis_vx, in.seis_vz};
    for (int k = 0; k < 3; ++k)
      if (outs[k] && blk)
        FOMO_CU(ctx, cudaMemcpyAsync(outs[k], d_seis + tab[s].seis0 + k * blk, 4 * blk,
                                     cudaMemcpyDeviceToHost, st));
  }
  FOMO_CU(ctx, cudaStreamSynchronize(st));
  if (stats) {
    std::memset(stats, 0, sizeof *stats);
    stats->kernel_time_s = ms * 1e-3;
    stats->cell_updates = (double)cells * nt;
    // acoustic: vx, vz, p read and written + bx, bz, kappa read = 9 words per cell
    stats->alg_bytes = 36.0 * (double)cells * nt;
    stats->n_shots = ns;
    stats->gpu_launches = fused ? 1 : 3 * nt;
    stats->kernel = fused ? FOMO_KERNEL_SINGLE_SWEEP : FOMO_KERNEL_TWO_PHASE;
    stats->sweep_config = fused ? kAcNTX[a_k] * 1000 : t.bx * 1000 + t.by;
  }
  return FOMO_OK;
}

}  // namespace
}  // namespace fomo

extern "C" int fomo_acoustic2d_uneven(fomo_ctx* ctx, float dh, float dt, int32_t nt, int32_t nbc,
                                      int32_t fd_order, int32_t n_shots, const fomo_shot2d* shots,
                                      const fomo_opts* opts, fomo_stats* stats) {
  return fomo::run_uneven(ctx, dh, dt, nt, nbc, fd_order, n_shots, shots, opts, stats);
}
