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
#include <vector>

#include "solver2d_kernels.cuh"

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
  std::vector<int> tile_shot;
  auto upload_tiles = [&](int k) -> int {
    tiles_for(kTiles[k], tile_shot);
    FOMO_CU(ctx, cudaMemcpyAsync(d_tab, tab.data(), sizeof(UShot) * ns, cudaMemcpyHostToDevice, st));
    FOMO_CU(ctx, cudaMemcpyAsync(d_tiles, tile_shot.data(), 4 * tile_shot.size(),
                                 cudaMemcpyHostToDevice, st));
    FOMO_CU(ctx, cudaStreamSynchronize(st));  // host vectors change before the next upload
    return FOMO_OK;
  };

  if (tsel < 0) {  // time each tile shape on three steps of the zero state
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
  if ((rc = upload_tiles(tsel))) return rc;
  const int nblk = (int)tile_shot.size();
  const Tile t = kTiles[tsel];

  // ---- zero state, capture the whole run, replay it once ----
  FOMO_CU(ctx, cudaMemsetAsync(d_state, 0, 4 * off_state, st));
  FOMO_CU(ctx, cudaMemsetAsync(d_seis, 0, 4 * std::max(off_seis, 1LL), st));
  FOMO_CU(ctx, cudaStreamSynchronize(st));
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // Capture on the context's own stream: the caller's stream may be the
  // legacy default stream, which cannot be captured.  Replay on the caller's.
  const cudaStream_t cs = ctx->own_stream;
  FOMO_CU(ctx, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  for (int it = 1; it <= nt; ++it) {
    const int A = (it - 1) & 1;
    launch_step_n(N, cs, nblk, t, d_tab, d_tiles, d_state, d_mat, c, dtdh, d_w, zone, wstride, A);
    k_uinject_record<<<ns, 256, 0, cs>>>(d_tab, d_state, d_src, d_wav, d_rec, d_seis, it, nt, 1 - A);
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
  float ms = 0.0f;
  FOMO_CU(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));

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
    stats->gpu_launches = 3 * nt;
    stats->kernel = FOMO_KERNEL_TWO_PHASE;
    stats->sweep_config = t.bx * 1000 + t.by;
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
