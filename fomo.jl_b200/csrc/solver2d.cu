// solver2d.cu -- host drivers of the 2D solvers (acoustic2d, elastic2d,
// scalar2d and the _batch variants): validation, workspace layout, device
// medium preparation, the time loop and the result download.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>

#include "solver2d_kernels.cuh"
#include "mixed2d.cuh"
#include "replica2d.cuh"
#include "sweep2d.cuh"

namespace fomo {
// learned corrector (corrector.cu)
cudaError_t corr_forward_device(cudaStream_t st, int h, int w, const float* u, const float* up,
                                const float* c2, long long ld, int n_src, const int* src,
                                const float* inj_next, const float* inj_prev,
                                const float* params, void* scratch, float* y, bool pack);
size_t corr_scratch_bytes(long long npix);
namespace {

enum Phys { kAcoustic = 0, kElastic = 1, kScalar = 2 };

struct Plan2 {
  Phys phys;
  int nx, nz, nt, nbc, fd_order, N, M, pad, nxp, nzp;
  int ld;  // row pitch: nxp rounded up to 32 floats (128-byte rows, TMA-legal strides)
  long long plane;
  float dh, dt, v_ref;
  int ns, n_src, n_rec;
  bool dev;
  int snap_interval, nsnap;
  int kernel;
  bool fp16 = false;  // elastic: binary16 wavefield storage (mixed2d.cuh)
  bool sponge = false;  // boundary = :sponge (FOMO_F_SPONGE) instead of HABC
  float sponge_factor = 0.015f;
};

int check_indices(fomo_ctx* ctx, const char* what, const int32_t* ix, const int32_t* iz,
                  long long n, int nx, int nz) {
  for (long long k = 0; k < n; ++k)
    if (ix[k] < 1 || ix[k] > nx || iz[k] < 1 || iz[k] > nz)
      return fail(ctx, FOMO_EARG,
                  std::string(what) + " index out of range: need 1 <= x <= " + std::to_string(nx) +
                      ", 1 <= z <= " + std::to_string(nz) + " (got " + std::to_string(ix[k]) + ", " +
                      std::to_string(iz[k]) + ")");
  return FOMO_OK;
}

// Copies a small index/value array to the host when the caller passed device
// pointers (validation and linear-index construction happen on the host).
template <class T>
int host_copy(fomo_ctx* ctx, const T* src, long long n, bool dev, std::vector<T>& out) {
  out.resize((size_t)std::max<long long>(n, 0));
  if (n <= 0) return FOMO_OK;
  if (dev) {
    FOMO_CU(ctx, cudaMemcpy(out.data(), src, sizeof(T) * n, cudaMemcpyDeviceToHost));
  } else {
    std::memcpy(out.data(), src, sizeof(T) * n);
  }
  return FOMO_OK;
}

int make_plan(fomo_ctx* ctx, Phys phys, const fomo_grid2d* g, const fomo_acq* acq,
              int snap_interval, const fomo_opts* opts, bool batch, Plan2& P) {
  if (!ctx) return FOMO_EARG;
  if (!g || !acq) return fail(ctx, FOMO_EARG, "grid and acquisition descriptors are required");
  P.phys = phys;
  P.nx = g->nx;
  P.nz = g->nz;
  P.nt = g->nt;
  P.nbc = g->nbc;
  P.fd_order = g->fd_order;
  P.dh = g->dh;
  P.dt = g->dt;
  P.v_ref = g->v_ref;
  P.N = order_to_N(g->fd_order);
  if (P.N < 0) return fail(ctx, FOMO_EARG, "Unsupported FD order: " + std::to_string(g->fd_order));
  if (P.nx < 1 || P.nz < 1) return fail(ctx, FOMO_EARG, "grid must be at least 1x1");
  if (P.nt < 1) return fail(ctx, FOMO_EARG, "nt must be >= 1");
  if (!(P.dh > 0.0f) || !(P.dt > 0.0f)) return fail(ctx, FOMO_EARG, "dh and dt must be > 0");
  if (P.nbc < 0) return fail(ctx, FOMO_EARG, "nbc must be >= 0");
  P.M = P.N;
  P.pad = P.nbc + P.M;
  if (P.pad < 2) return fail(ctx, FOMO_EARG, "nbc + fd_order/2 must be >= 2");
  P.nxp = P.nx + 2 * P.pad;
  P.nzp = P.nz + 2 * P.pad;
  P.ld = (P.nxp + 31) & ~31;
  P.plane = (long long)P.ld * P.nzp;
  P.ns = acq->n_shots;
  P.n_src = acq->n_src;
  P.n_rec = acq->n_rec;
  if (P.ns < 1) return fail(ctx, FOMO_EARG, "at least 1 shot is required");
  if (!batch && P.ns != 1) return fail(ctx, FOMO_EARG, "single-shot solver takes n_shots == 1");
  if (P.n_src < 0 || P.n_rec < 0) return fail(ctx, FOMO_EARG, "negative source/receiver count");
  if (P.n_src > 0 && (!acq->sx || !acq->sz || !acq->wavelet))
    return fail(ctx, FOMO_EARG, "sources need sx, sz and a wavelet matrix");
  if (P.n_rec > 0 && (!acq->rx || !acq->rz)) return fail(ctx, FOMO_EARG, "receivers need rx, rz");
  if (snap_interval < 0) return fail(ctx, FOMO_EARG, "snap_interval must be >= 0");
  P.snap_interval = snap_interval;
  P.nsnap = snap_interval > 0 ? P.nt / snap_interval : 0;
  P.dev = opts && (opts->flags & FOMO_F_DEVICE_PTRS);
  P.kernel = opts ? opts->kernel : FOMO_KERNEL_AUTO;
  if (opts && opts->precision == FOMO_FP16 && phys == kElastic) {
    P.fp16 = true;  // two-phase kernels with binary16 storage
  } else if (opts && opts->precision != FOMO_FP32) {
    return fail(ctx, FOMO_EUNSUPPORTED,
                phys == kElastic ? "elastic2d stores FP32 or FP16 (BF16 is not accurate enough)"
                                 : "this solver stores FP32 only");
  }
  if (opts && (opts->flags & FOMO_F_SPONGE)) {  // acoustic2d.jl:65-87, elastic2d.jl:63-87
    if (phys == kScalar)
      return fail(ctx, FOMO_EUNSUPPORTED, "scalar2d has no sponge boundary (HABC only)");
    if (P.fp16) return fail(ctx, FOMO_EUNSUPPORTED, "the sponge boundary stores FP32 only");
    if (P.kernel == FOMO_KERNEL_SINGLE_SWEEP)
      return fail(ctx, FOMO_EUNSUPPORTED, "the sponge boundary runs the two-phase kernels");
    if (!(opts->sponge_factor >= 0.0f) || !std::isfinite(opts->sponge_factor))
      return fail(ctx, FOMO_EARG, "sponge_factor must be finite and >= 0");
    P.sponge = true;
    P.sponge_factor = opts->sponge_factor;
  }
  if ((long long)P.nxp * P.nzp > (1LL << 31))
    return fail(ctx, FOMO_EARG, "padded grid exceeds 2^31 cells");
  return FOMO_OK;
}

float min_positive(const std::vector<float>& v) {
  float m = INFINITY;
  for (float x : v)
    if (x > 0.0f && x < m) m = x;
  return m;
}

// Autotuner of the single-sweep kernel: times each (variant, strip width,
// z-segments) candidate on the problem itself and keeps the fastest; the
// choice is cached per (N, padded grid, shots) for the process.
struct TuneKey {
  int N, nx, nz, ns, h16;
  bool operator<(const TuneKey& o) const {
    return std::tie(N, nx, nz, ns, h16) < std::tie(o.N, o.nx, o.nz, o.ns, o.h16);
  }
};
struct TuneVal {
  int variant, TX, per_sm;
  float frame_weight;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune;

// sets16 / o16: the binary16 arrays (set-major, sweep field order) and the
// binary16 outputs of set 1 for the binary16 storage form; null for FP32.
template <class FieldFn>
int tune_sweep(fomo_ctx* ctx, cudaStream_t st, SweepPlan& sp, int N, const Geo2& g, int ns,
               float* const sets[2][5], const Coef& c, float dtx, float dtz, const HabcDev& h,
               const ElMat& m, FieldFn field, long long* d_bounds, __half* const* sets16 = nullptr,
               const ElOut16* o16 = nullptr) {
  const bool h16 = sets16 != nullptr;
  const TuneKey key{N, g.nx, g.nz, ns, h16 ? 1 : 0};
  // FOMO_SWEEP_CONFIG="variant,TX,ctas_per_sm" pins the configuration (tests, sweeps)
  if (const char* env = std::getenv("FOMO_SWEEP_CONFIG")) {
    int v = 0, tx = 0, per_sm = 0;
    float fw = kFrameWeight;
    const int nr = std::sscanf(env, "%d,%d,%d,%f", &v, &tx, &per_sm, &fw);
    if (nr >= 3 && v >= 0 && v < sweep_num_variants() && per_sm >= 1) {
      if (sweep_variant_h16(v) != h16)
        return fail(ctx, FOMO_EARG, "FOMO_SWEEP_CONFIG names a variant of the other storage form");
      FOMO_CU(ctx, make_sweep_plan(sp, N, v, tx, per_sm, g, ns, sets, fw, d_bounds, st, sets16));
      return FOMO_OK;
    }
    return fail(ctx, FOMO_EARG, "bad FOMO_SWEEP_CONFIG (want variant,TX,ctas_per_sm[,frame_weight])");
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      FOMO_CU(ctx, make_sweep_plan(sp, N, it->second.variant, it->second.TX, it->second.per_sm, g,
                                   ns, sets, it->second.frame_weight, d_bounds, st, sets16));
      return FOMO_OK;
    }
  }
  ElFields a{field(0, 0), field(0, 1), field(0, 2), field(0, 3), field(0, 4)};
  ElOut o{field(1, 0), field(1, 1), field(1, 2), field(1, 3), field(1, 4)};
  cudaEvent_t e0, e1;
  FOMO_CU(ctx, cudaEventCreate(&e0));
  FOMO_CU(ctx, cudaEventCreate(&e1));
  float best = 1e30f;
  TuneVal bv{-1, 0, 0, kFrameWeight};
  auto time_plan = [&](const SweepPlan& cand, float& ms) -> int {
    FOMO_CU(ctx, launch_sweep_elastic(st, cand, 0, c, dtx, dtz, h, a, m, o, ctx->d_flag, o16));
    FOMO_CU(ctx, cudaEventRecord(e0, st));
    for (int r = 0; r < 3; ++r)
      FOMO_CU(ctx, launch_sweep_elastic(st, cand, 0, c, dtx, dtz, h, a, m, o, ctx->d_flag, o16));
    FOMO_CU(ctx, cudaEventRecord(e1, st));
    FOMO_CU(ctx, cudaEventSynchronize(e1));
    FOMO_CU(ctx, cudaEventElapsedTime(&ms, e0, e1));
    return FOMO_OK;
  };
  // Candidates: the warp-specialized sweeps and, for FP32 batches with the
  // pair pack built, the shot-pair sweeps (the older families measured slower
  // on every problem; FOMO_SWEEP_CONFIG still selects them).
  const bool pairs_ok = !h16 && m.ppack != nullptr && ns >= 2;
  for (int v = 0; v < sweep_num_variants(); ++v) {
    if (sweep_variant_h16(v) != h16) continue;
    if (sweep_variant_pair(v) ? !pairs_ok : !sweep_variant_ws(v)) continue;
    int txs[4];
    int ntx = sweep_tx_candidates(v, N, g.nx, txs, 4);
    for (int k = 0; k < ntx; ++k) {
      SweepPlan cand;
      if (make_sweep_plan(cand, N, v, txs[k], 64, g, ns, sets, kFrameWeight, d_bounds, st,
                          sets16) != cudaSuccess)
        continue;
      const int full = cand.per_sm;  // all resident CTAs; also try one fewer
      for (int per_sm = full; per_sm >= 1 && per_sm >= full - 1; --per_sm) {
        if (make_sweep_plan(cand, N, v, txs[k], per_sm, g, ns, sets, kFrameWeight, d_bounds,
                            st, sets16) != cudaSuccess)
          continue;
        float ms = 0.0f;
        if (int rc = time_plan(cand, ms)) return rc;
        if (ms < best) {
          best = ms;
          bv = TuneVal{v, txs[k], per_sm, kFrameWeight};
        }
      }
    }
  }
  // then the cost weight of frame cells for the row-range split
  if (bv.variant >= 0)
    for (float fw : {0.0f, 0.07f, 0.3f, 0.6f, 1.2f}) {
      SweepPlan cand;
      if (make_sweep_plan(cand, N, bv.variant, bv.TX, bv.per_sm, g, ns, sets, fw, d_bounds, st,
                          sets16) != cudaSuccess)
        continue;
      float ms = 0.0f;
      if (int rc = time_plan(cand, ms)) return rc;
      if (ms < best) {
        best = ms;
        bv.frame_weight = fw;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (bv.variant < 0) return fail(ctx, FOMO_ECUDA, "no single-sweep configuration fits");
  FOMO_CU(ctx, make_sweep_plan(sp, N, bv.variant, bv.TX, bv.per_sm, g, ns, sets, bv.frame_weight,
                               d_bounds, st, sets16));
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = bv;
  return FOMO_OK;
}

struct Outs {
  float* seis[3];
  int nseis;
  float* snaps;
};

// Per-step extension of the scalar loop (learned correction, wavefield
// snapshots).  correct() runs after the step and the injection of step it and
// before the recording; u2 = u^{n+1}, u1 = u^n, u0 = u^{n-1} (padded, pitched).
struct ScalarHook {
  virtual ~ScalarHook() = default;
  // wav: the run's device wavelet matrix (n_src, nt)
  virtual int begin(fomo_ctx*, cudaStream_t, const Plan2&, const float*) { return FOMO_OK; }
  virtual int correct(fomo_ctx*, cudaStream_t, int, float*, const float*, const float*,
                      const float*, const Plan2&) {
    return FOMO_OK;
  }
  virtual int after_step(fomo_ctx*, cudaStream_t, int, const float*, const Plan2&) { return FOMO_OK; }
  virtual bool corrects() const { return false; }
  virtual int launches_per_step() const { return 0; }
};

// Common run: model (vp, vs, rho per phys), acquisition, outputs.
int run2d(fomo_ctx* ctx, Plan2& P, const float* vp, const float* vs, const float* rho,
          const fomo_acq* acq, Outs outs, const fomo_opts* opts, fomo_stats* stats,
          ScalarHook* hook = nullptr) {
  FOMO_CU(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const long long nint = (long long)P.nx * P.nz;
  if (!vp || (P.phys != kScalar && !rho) || (P.phys == kElastic && !vs))
    return fail(ctx, FOMO_EARG, "model arrays are required");

  // ---- indices: validate (utils/checks.jl:8-13) and pad (source.jl:18-28) ----
  std::vector<int32_t> hsx, hsz, hrx, hrz;
  long long nsrc_all = (long long)P.n_src * P.ns;
  int rc;
  if ((rc = host_copy(ctx, acq->sx, nsrc_all, P.dev, hsx)) ||
      (rc = host_copy(ctx, acq->sz, nsrc_all, P.dev, hsz)) ||
      (rc = host_copy(ctx, acq->rx, (long long)P.n_rec, P.dev, hrx)) ||
      (rc = host_copy(ctx, acq->rz, (long long)P.n_rec, P.dev, hrz)))
    return rc;
  if ((rc = check_indices(ctx, "source", hsx.data(), hsz.data(), nsrc_all, P.nx, P.nz)) ||
      (rc = check_indices(ctx, "receiver", hrx.data(), hrz.data(), P.n_rec, P.nx, P.nz)))
    return rc;
  std::vector<int32_t> src_lin(nsrc_all), rec_lin(P.n_rec);
  for (long long k = 0; k < nsrc_all; ++k)
    src_lin[k] = (hsx[k] - 1 + P.pad) + P.ld * (hsz[k] - 1 + P.pad);
  for (int r = 0; r < P.n_rec; ++r) rec_lin[r] = (hrx[r] - 1 + P.pad) + P.ld * (hrz[r] - 1 + P.pad);

  // ---- v_ref default: minimum(vp > 0) (acoustic2d.jl:55) ----
  if (P.sponge && !(P.v_ref > 0.0f)) P.v_ref = 1.0f;  // v_ref is ignored with the sponge
  if (!(P.v_ref > 0.0f)) {
    std::vector<float> hvp;
    if ((rc = host_copy(ctx, vp, nint, P.dev, hvp))) return rc;
    P.v_ref = min_positive(hvp);
    if (!std::isfinite(P.v_ref)) return fail(ctx, FOMO_EARG, "vp has no positive value for v_ref");
  }
  HabcHost hh = make_habc(P.pad, P.v_ref, P.dt, P.dh);

  int kernel = P.kernel;
  // the replica of the reference's CUDA.jl step exists for elastic HABC FP32 runs
  const bool replica = kernel == FOMO_KERNEL_REPLICA;
  if (replica && (P.phys != kElastic || P.fp16 || P.sponge || hook))
    return fail(ctx, FOMO_EARG,
                "FOMO_KERNEL_REPLICA replicates the elastic2d HABC FP32 step only");
  if (P.sponge) kernel = FOMO_KERNEL_TWO_PHASE;
  if (kernel == FOMO_KERNEL_AUTO) kernel = pick_kernel_2d((int)P.phys, P.N, P.nxp, P.nzp, P.ns);
  if (kernel == FOMO_KERNEL_SINGLE_SWEEP && !sweep2d_supported((int)P.phys, P.N))
    kernel = FOMO_KERNEL_TWO_PHASE;

  // ---- workspace layout ----
  const int nmat = P.phys == kElastic ? 5 : (P.phys == kAcoustic ? 3 : 1);
  const int nfield = P.phys == kElastic ? 5 : (P.phys == kAcoustic ? 3 : 1);
  const int nsets = P.phys == kScalar ? 3 : 2;
  const long long seis_n = (long long)P.n_rec * P.nt * P.ns;
  // Shots allocated per field: single-sweep FP32 elastic runs may take the
  // shot-pair sweep, whose pair-interleaved fields hold an even number of shots
  // (an odd batch carries one all-zero shot).
  const bool sweep = kernel == FOMO_KERNEL_SINGLE_SWEEP;
  const bool pair_ok = sweep && !P.fp16 && P.phys == kElastic;
  const int nsa = pair_ok ? P.ns + (P.ns & 1) : P.ns;
  Arena ar;
  size_t o_model = P.dev ? 0 : ar.take<float>(3 * nint);
  size_t o_mat = ar.take<float>(nmat * P.plane);
  size_t o_state = ar.take<float>((long long)nsets * nfield * nsa * P.plane);
  size_t o_state16 = P.fp16 ? ar.take<__half>((long long)nsets * nfield * P.ns * P.plane) : 0;
  size_t o_unpack = ((P.fp16 || pair_ok) && opts && opts->final_state)
                        ? ar.take<float>(P.nxp * (long long)P.nzp)
                        : 0;
  const std::vector<float> damp = P.sponge ? sponge_table(P.nbc, P.sponge_factor) : std::vector<float>();
  if (P.sponge) hh.wtab = damp.empty() ? std::vector<float>(1, 1.0f) : damp;
  size_t o_w = ar.take<float>(hh.wtab.size());
  size_t o_src = ar.take<int32_t>(std::max<long long>(nsrc_all, 1));
  size_t o_rec = ar.take<int32_t>(std::max(P.n_rec, 1));
  size_t o_wav = P.dev ? 0 : ar.take<float>(std::max<long long>((long long)P.n_src * P.nt, 1));
  size_t o_seis = P.dev ? 0 : ar.take<float>(std::max<long long>(outs.nseis * seis_n, 1));
  size_t o_snap = (!P.dev && outs.snaps && P.nsnap) ? ar.take<float>(P.nsnap * nint) : 0;
  size_t o_bounds = ar.take<long long>(kMaxGrid + 1);
  size_t o_it = ar.take<int>(1);  // device step index of replayed chunks
  // Two-phase runs of up to 2 M shot-cells, which are bound by launch latency,
  // inject and record inside the step's last update kernel on tagged cells
  // (CellTags) instead of a separate launch.  Larger grids keep the
  // separate kernel: a step costs tens of microseconds there, and the tag code
  // raises the acoustic pressure kernel from 40 to 54 registers (6 -> 4 blocks
  // per SM).
  const bool tagged = !P.fp16 && !hook && (long long)P.nxp * P.nzp * P.ns <= 2000000LL &&
                      (P.phys == kScalar || kernel == FOMO_KERNEL_TWO_PHASE);
  CellTagHost tags;
  if (tagged) tags = make_cell_tags(src_lin.data(), (int)nsrc_all, rec_lin.data(), P.n_rec);
  const int n_ent = (int)tags.lin.size();
  size_t o_tag = tagged ? ar.take<int32_t>(P.plane) : 0;
  size_t o_ent = tagged ? ar.take<int4>(std::max(n_ent, 1)) : 0;
  size_t o_elin = tagged ? ar.take<int32_t>(std::max(n_ent, 1)) : 0;
  size_t o_list = tagged ? ar.take<int32_t>(std::max<size_t>(tags.list.size(), 1)) : 0;
  size_t o_pack = sweep ? ar.take<float>(sweep_pack_floats(P.nxp, P.nzp)) : 0;
  size_t o_ppack = pair_ok ? ar.take<float>(pair_pack_floats(P.nxp, P.nzp)) : 0;
  // replica: strip backups of the five fields, three weight planes, frame scratch
  const long long rep_total = replica ? replica_frame_total(P.nxp, P.nzp, hh.nbc) : 0;
  size_t o_rep = replica ? ar.take<float>((long long)5 * P.ns * P.plane) : 0;
  size_t o_repw = replica ? ar.take<float>(3 * P.plane) : 0;
  size_t o_repscr = replica ? ar.take<float>(std::max(1LL, 3 * rep_total * P.ns)) : 0;
  if ((rc = ensure_workspace(ctx, ar.off))) return rc;

  const float* d_vp = vp;
  const float* d_vs = vs;
  const float* d_rho = rho;
  const float* d_wav = acq->wavelet;
  if (!P.dev) {
    float* m = ws_ptr<float>(ctx, o_model);
    FOMO_CU(ctx, cudaMemcpyAsync(m, vp, sizeof(float) * nint, cudaMemcpyHostToDevice, st));
    d_vp = m;
    if (vs) {
      FOMO_CU(ctx, cudaMemcpyAsync(m + nint, vs, sizeof(float) * nint, cudaMemcpyHostToDevice, st));
      d_vs = m + nint;
    }
    if (rho) {
      FOMO_CU(ctx,
              cudaMemcpyAsync(m + 2 * nint, rho, sizeof(float) * nint, cudaMemcpyHostToDevice, st));
      d_rho = m + 2 * nint;
    }
    if (P.n_src > 0) {
      float* w = ws_ptr<float>(ctx, o_wav);
      FOMO_CU(ctx, cudaMemcpyAsync(w, acq->wavelet, sizeof(float) * P.n_src * P.nt,
                                   cudaMemcpyHostToDevice, st));
      d_wav = w;
    }
  }
  float* d_mat = ws_ptr<float>(ctx, o_mat);
  float* d_state = ws_ptr<float>(ctx, o_state);
  __half* d_state16 = P.fp16 ? ws_ptr<__half>(ctx, o_state16) : nullptr;
  float* d_w = ws_ptr<float>(ctx, o_w);
  int32_t* d_src = ws_ptr<int32_t>(ctx, o_src);
  int32_t* d_rec = ws_ptr<int32_t>(ctx, o_rec);
  FOMO_CU(ctx, cudaMemcpyAsync(d_w, hh.wtab.data(), sizeof(float) * hh.wtab.size(),
                               cudaMemcpyHostToDevice, st));
  if (nsrc_all)
    FOMO_CU(ctx, cudaMemcpyAsync(d_src, src_lin.data(), sizeof(int32_t) * nsrc_all,
                                 cudaMemcpyHostToDevice, st));
  if (P.n_rec)
    FOMO_CU(ctx, cudaMemcpyAsync(d_rec, rec_lin.data(), sizeof(int32_t) * P.n_rec,
                                 cudaMemcpyHostToDevice, st));
  float* d_seis[3] = {nullptr, nullptr, nullptr};
  for (int k = 0; k < outs.nseis; ++k)
    d_seis[k] = P.dev ? outs.seis[k] : (outs.seis[k] ? ws_ptr<float>(ctx, o_seis) + k * seis_n : nullptr);
  float* d_snap = P.dev ? outs.snaps : (o_snap ? ws_ptr<float>(ctx, o_snap) : nullptr);
  if (!outs.snaps) d_snap = nullptr;

  // ---- medium (device) ----
  float dtdh = P.dt / P.dh;  // Float32(dt / dh)
  FOMO_CU(ctx, launch_medium2d(st, P.phys == kElastic ? 0 : (P.phys == kAcoustic ? 1 : 2), P.nx,
                               P.nz, P.pad, P.ld, dtdh, d_vp, d_vs, d_rho, d_mat, d_mat + P.plane,
                               d_mat + 2 * P.plane, d_mat + 3 * P.plane, d_mat + 4 * P.plane));
  // ---- zero state (reset!, batch.jl:30-35) ----
  FOMO_CU(ctx, cudaMemsetAsync(d_state, 0, sizeof(float) * nsets * nfield * nsa * P.plane, st));
  if (P.fp16) {
    FOMO_CU(ctx, cudaMemsetAsync(d_state16, 0, sizeof(__half) * nsets * nfield * P.ns * P.plane, st));
    // fold the storage scales into the materials (powers of two: exact)
    k_scale<<<256, 256, 0, st>>>(d_mat, 2 * P.plane, kFp16Sv / kFp16St);
    k_scale<<<256, 256, 0, st>>>(d_mat + 2 * P.plane, 3 * P.plane, kFp16St / kFp16Sv);
  }
  if (!P.dev)
    for (int k = 0; k < outs.nseis; ++k)
      if (d_seis[k]) FOMO_CU(ctx, cudaMemsetAsync(d_seis[k], 0, sizeof(float) * seis_n, st));

  int* d_it = ws_ptr<int>(ctx, o_it);
  FOMO_CU(ctx, cudaMemsetAsync(d_it, 0, sizeof(int), st));
  CellTags tg;
  if (tagged) {
    int32_t* d_tag = ws_ptr<int32_t>(ctx, o_tag);
    FOMO_CU(ctx, cudaMemsetAsync(d_tag, 0xFF, sizeof(int32_t) * P.plane, st));  // -1
    if (n_ent) {
      FOMO_CU(ctx, cudaMemcpyAsync(ws_ptr<int4>(ctx, o_ent), tags.ent.data(), sizeof(int4) * n_ent,
                                   cudaMemcpyHostToDevice, st));
      FOMO_CU(ctx, cudaMemcpyAsync(ws_ptr<int32_t>(ctx, o_elin), tags.lin.data(),
                                   sizeof(int32_t) * n_ent, cudaMemcpyHostToDevice, st));
      FOMO_CU(ctx, cudaMemcpyAsync(ws_ptr<int32_t>(ctx, o_list), tags.list.data(),
                                   sizeof(int32_t) * tags.list.size(), cudaMemcpyHostToDevice, st));
      k_set_tags<<<cdiv(n_ent, 256), 256, 0, st>>>(d_tag, ws_ptr<int32_t>(ctx, o_elin), n_ent);
    }
    tg.tag = d_tag;
    tg.ent = ws_ptr<int4>(ctx, o_ent);
    tg.list = ws_ptr<int32_t>(ctx, o_list);
    tg.wav = d_wav;
    tg.n_src = P.n_src;
    tg.n_rec = P.n_rec;
    tg.nt = P.nt;
    tg.s0 = d_seis[0];
    tg.s1 = d_seis[1];
    tg.s2 = d_seis[2];
    tg.it0 = d_it;
  }

  Geo2 g{P.nxp, P.nzp, P.ld, P.M, hh.nbc, P.plane};
  Coef c;
  for (int l = 0; l < 5; ++l) c.a[l] = kFD[P.N][l];
  HabcDev h{hh.q, hh.qt, hh.qxt, P.sponge ? P.nbc : hh.nbc, hh.wstride, d_w};
  const float dtx = dtdh, dtz = dtdh;
  auto field = [&](int set, int f) { return d_state + ((long long)set * nfield + f) * nsa * P.plane; };
  auto hfield = [&](int set, int f) {
    return HField{field(set, f), d_state16 + ((long long)set * nfield + f) * P.ns * P.plane};
  };

  ElMat emat{d_mat, d_mat + P.plane, d_mat + 2 * P.plane, d_mat + 3 * P.plane, d_mat + 4 * P.plane};
  SweepPlan sp;
  if (sweep) {
    FOMO_CU(ctx, build_sweep_pack(st, g, emat, ws_ptr<float>(ctx, o_pack)));
    if (pair_ok) {
      PairPack pp;
      FOMO_CU(ctx, build_pair_pack(st, g, emat, ws_ptr<float>(ctx, o_ppack), pp));
      emat.ppack = ws_ptr<float>(ctx, o_ppack);
      emat.ppack_pitch = pp.pitch;
    }
    float* sets[2][5] = {{field(0, 2), field(0, 3), field(0, 4), field(0, 0), field(0, 1)},
                         {field(1, 2), field(1, 3), field(1, 4), field(1, 0), field(1, 1)}};
    __half* sets16[10];
    ElOut16 o16{};
    if (P.fp16) {
      const int order[5] = {2, 3, 4, 0, 1};  // txx, tzz, txz, vx, vz
      for (int s2 = 0; s2 < 2; ++s2)
        for (int f = 0; f < 5; ++f) sets16[s2 * 5 + f] = hfield(s2, order[f]).f16;
      o16 = ElOut16{hfield(1, 0).f16, hfield(1, 1).f16, hfield(1, 2).f16, hfield(1, 3).f16,
                    hfield(1, 4).f16};
    }
    rc = tune_sweep(ctx, st, sp, P.N, g, P.ns, sets, c, dtx, dtz, h, emat,
                    [&](int set, int f) { return field(set, f); },
                    ws_ptr<long long>(ctx, o_bounds), P.fp16 ? sets16 : nullptr,
                    P.fp16 ? &o16 : nullptr);
    if (rc) return rc;
    // the tuning launches ran on the zero state; restore it
    FOMO_CU(ctx, cudaMemsetAsync(d_state, 0, sizeof(float) * nsets * nfield * nsa * P.plane, st));
    if (P.fp16)
      FOMO_CU(ctx, cudaMemsetAsync(d_state16, 0, sizeof(__half) * nsets * nfield * P.ns * P.plane,
                                   st));
  }
  FOMO_CU(ctx, cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), st));
  // the shot-pair sweep's fields are pair-interleaved (sweep2d.cuh)
  const bool pairs = sweep && sp.family == 5;
  // the replica updates set 0 in place, with backups and scratch of its own
  RepFields rw{};
  float *rep_wv = nullptr, *rep_wz = nullptr, *rep_wt = nullptr, *rep_scr = nullptr;
  if (replica) {
    float* ro = ws_ptr<float>(ctx, o_rep);
    const long long fs = (long long)P.ns * P.plane;
    rw = RepFields{field(0, 0), field(0, 1), field(0, 2), field(0, 3), field(0, 4),
                   ro,          ro + fs,     ro + 2 * fs, ro + 3 * fs, ro + 4 * fs};
    FOMO_CU(ctx, cudaMemsetAsync(ro, 0, sizeof(float) * 5 * fs, st));
    rep_wv = ws_ptr<float>(ctx, o_repw);
    rep_wz = rep_wv + P.plane;
    rep_wt = rep_wz + P.plane;
    rep_scr = ws_ptr<float>(ctx, o_repscr);
    FOMO_CU(ctx, replica_setup(st, g, h, rep_wv, rep_wz, rep_wt));
  }

  dim3 blk(32, 8), grd(cdiv(P.nxp, 32), cdiv(P.nzp, 8), P.ns);
  int launches = 0;
  // FOMO_F_PROFILE: event pairs around the sweep kernel(s) of a window of steps
  const bool prof = opts && (opts->flags & FOMO_F_PROFILE) && P.nt >= 2;
  const int w0 = P.nt / 2, nw = prof ? std::min(16, P.nt - w0) : 0;
  std::vector<cudaEvent_t> pev(2 * nw, nullptr);
  for (auto& e : pev) FOMO_CU(ctx, cudaEventCreate(&e));
  auto prof_mark = [&](int it, int which) -> cudaError_t {
    int k = it - 1 - w0;
    if (k < 0 || k >= nw) return cudaSuccess;
    return cudaEventRecord(pev[2 * k + which], st);
  };
  int sweeps_per_step = 0;
  if (hook)
    if (int hr = hook->begin(ctx, st, P, d_wav)) return hr;
  FOMO_CU(ctx, cudaEventRecord(ctx->ev0, st));
  int A = 0, B = 1, C2 = 2;  // scalar: A = u^{n-1}, B = u^n, C2 = u^{n+1}
  // One two-phase step, set a -> set b, on stream s (j: the step's index in its
  // chunk, for the tagged kernels), with the sponge and tag variants chosen here.
  auto el_two_phase = [&](cudaStream_t s, int a, int b, int j) {
    const ElFields fa{field(a, 0), field(a, 1), field(a, 2), field(a, 3), field(a, 4)};
    auto go = [&](auto spc, auto tgc) {
      constexpr bool SPV = decltype(spc)::value, TGV = decltype(tgc)::value;
      switch (P.N) {
#define FOMO_EL2_CASE(NN)                                                                        \
  case NN:                                                                                       \
    k_el_vel<NN, SPV><<<grd, blk, 0, s>>>(g, c, dtx, dtz, h, fa, emat, field(b, 0), field(b, 1)); \
    k_el_str<NN, SPV, TGV><<<grd, blk, 0, s>>>(g, c, dtx, dtz, h, fa, field(b, 0), field(b, 1),   \
                                               emat, field(b, 2), field(b, 3), field(b, 4), tg,  \
                                               j);                                               \
    break;
        FOMO_EL2_CASE(1) FOMO_EL2_CASE(2) FOMO_EL2_CASE(3) FOMO_EL2_CASE(4) FOMO_EL2_CASE(5)
#undef FOMO_EL2_CASE
      }
    };
    if (P.sponge) {
      if (tagged) go(std::true_type{}, std::true_type{});
      else go(std::true_type{}, std::false_type{});
    } else {
      if (tagged) go(std::false_type{}, std::true_type{});
      else go(std::false_type{}, std::false_type{});
    }
  };
  // One scalar leapfrog step u^{n+1} (set n) from u^n (set b) and u^{n-1} (set a).
  auto sc_step = [&](cudaStream_t s, int a, int b, int n, int j, const D2Coef& dc) {
    auto go = [&](auto tgc) {
      constexpr bool TGV = decltype(tgc)::value;
      switch (P.N) {
#define FOMO_SC2_CASE(NN)                                                                     \
  case NN:                                                                                    \
    k_sc_step<NN, TGV><<<grd, blk, 0, s>>>(g, dc, h, field(b, 0), field(a, 0), d_mat,          \
                                           field(n, 0), tg, j);                               \
    break;
        FOMO_SC2_CASE(1) FOMO_SC2_CASE(2) FOMO_SC2_CASE(3) FOMO_SC2_CASE(4) FOMO_SC2_CASE(5)
#undef FOMO_SC2_CASE
      }
    };
    if (tagged) go(std::true_type{});
    else go(std::false_type{});
  };
  auto ac_two_phase = [&](cudaStream_t s, int a, int b, int j) {
    const float* bx = d_mat;
    const float* bz = d_mat + P.plane;
    const float* kap = d_mat + 2 * P.plane;
    auto go = [&](auto spc, auto tgc) {
      constexpr bool SPV = decltype(spc)::value, TGV = decltype(tgc)::value;
      switch (P.N) {
#define FOMO_AC2_CASE(NN)                                                                        \
  case NN:                                                                                       \
    if constexpr (TGV) {                                                                         \
      k_ac_vel<NN, SPV><<<grd, blk, 0, s>>>(g, c, dtx, dtz, h, field(a, 2), field(a, 0),         \
                                            field(a, 1), bx, bz, field(b, 0), field(b, 1));      \
      k_ac_prs<NN, SPV, true><<<grd, blk, 0, s>>>(g, c, dtx, dtz, h, field(a, 2), field(b, 0),   \
                                                  field(b, 1), kap, field(b, 2), tg, j);         \
    } else {                                                                                     \
      k_ac_vel8<NN, SPV><<<grd, blk, 0, s>>>(g, c, dtx, dtz, h, field(a, 2), field(a, 0),        \
                                             field(a, 1), bx, bz, field(b, 0), field(b, 1));     \
      k_ac_prs8<NN, SPV><<<grd, blk, 0, s>>>(g, c, dtx, dtz, h, field(a, 2), field(b, 0),        \
                                             field(b, 1), kap, field(b, 2), tg, j);              \
    }                                                                                            \
    break;
        FOMO_AC2_CASE(1) FOMO_AC2_CASE(2) FOMO_AC2_CASE(3) FOMO_AC2_CASE(4) FOMO_AC2_CASE(5)
#undef FOMO_AC2_CASE
      }
    };
    if (P.sponge) {
      if (tagged) go(std::true_type{}, std::true_type{});
      else go(std::true_type{}, std::false_type{});
    } else {
      if (tagged) go(std::false_type{}, std::true_type{});
      else go(std::false_type{}, std::false_type{});
    }
  };
  // Acoustic, scalar and two-phase elastic runs on small grids are bound by
  // launch latency.  A chunk of K steps (the updates, inject/record; the interior snapshot where
  // the step is a multiple of snap_interval; the advance of a device step
  // index) is captured once and replayed; the remaining steps launch one by
  // one.  K is a multiple of the buffer rotation (2 acoustic, 3 scalar: a chunk
  // returns the buffers to their start) and of snap_interval, so every replay
  // runs the same node sequence.  Results are identical to step-by-step
  // launches (FOMO_F_STEP_LAUNCH).
  int it_first = 1;
  cudaGraphExec_t chunk_exec = nullptr;
  struct ExecGuard {  // the chunk's replays finish before it is destroyed, on every return path
    cudaGraphExec_t& e;
    cudaStream_t s;
    ~ExecGuard() {
      if (e) {
        cudaStreamSynchronize(s);
        cudaGraphExecDestroy(e);
      }
    }
  } exec_guard{chunk_exec, st};
  // Snapshot streaming: with host outputs, the frames of replayed chunk k are
  // copied to the caller's buffer on the copy stream once chunk k has run (an
  // event per chunk), while later chunks compute.  Only the frames of the
  // step-by-step remainder are copied after the time loop.
  struct ChunkEvents {
    std::vector<cudaEvent_t> ev;
    ~ChunkEvents() {
      for (auto e : ev) cudaEventDestroy(e);
    }
  } chunk_ev;
  int streamed_chunks = 0, frames_per_chunk = 0;
  auto replay = [&](int nchunk) -> cudaError_t {
    cudaError_t e = cudaSuccess;
    for (int k = 0; e == cudaSuccess && k < nchunk; ++k) {
      e = cudaGraphLaunch(chunk_exec, st);
      if (e == cudaSuccess && k < (int)chunk_ev.ev.size()) e = cudaEventRecord(chunk_ev.ev[k], st);
    }
    return e;
  };
  {
    const bool scalar = P.phys == kScalar;
    const bool elastic = P.phys == kElastic;
    const bool chunks_ok = (!elastic || kernel == FOMO_KERNEL_TWO_PHASE) && !P.fp16 && !hook &&
                           !prof && !(opts && (opts->flags & FOMO_F_STEP_LAUNCH));
    const int si = (!scalar && d_snap && P.snap_interval > 0) ? P.snap_interval : 0;
    const int period = scalar ? 3 : 2;  // buffer rotation: scalar u^{n-1}, u^n, u^{n+1}
    int K = 0;
    if (chunks_ok && (scalar ? !d_snap : true)) {
      if (si == 0) {
        K = 64 / period * period;
      } else if (si <= 256) {
        K = si * std::max(1, (64 + si / 2) / si);
        if (K % period) K *= period;
      }
    }
    const int nchunk = K > 0 ? P.nt / K : 0;
    if (nchunk >= 2) {
      if (si && !P.dev && outs.snaps) {
        chunk_ev.ev.assign(nchunk, nullptr);
        for (auto& e : chunk_ev.ev) FOMO_CU(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        frames_per_chunk = K / si;
      }
      const cudaStream_t cs = ctx->own_stream;  // the caller's may be uncapturable
      const float* bx = d_mat;
      const float* bz = d_mat + P.plane;
      const float* kap = d_mat + 2 * P.plane;
      cudaGraph_t graph = nullptr;
      cudaError_t ce = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
      if (ce == cudaSuccess && scalar) {
        D2Coef dc;
        dc.two_c0 = 2.0f * kD2C0[P.N];
        for (int l = 0; l < 5; ++l) dc.d[l] = kD2[P.N][l];
        int a = A, b = B, n = C2, nodes = 0;
        for (int j = 0; j < K; ++j) {
          sc_step(cs, a, b, n, j, dc);
          ++nodes;
          if (!tagged) {
            k_inject_record_at<<<1, 256, 0, cs>>>(d_it, j, P.nt, P.plane, P.n_src, d_src, d_wav,
                                                  field(n, 0), nullptr, P.n_rec, d_rec,
                                                  field(n, 0), nullptr, nullptr, d_seis[0],
                                                  nullptr, nullptr);
            ++nodes;
          }
          const int t = a;
          a = b;
          b = n;
          n = t;
        }
        k_step_add<<<1, 1, 0, cs>>>(d_it, K);
        ++nodes;
        ce = cudaStreamEndCapture(cs, &graph);
        if (ce == cudaSuccess) ce = cudaGraphInstantiate(&chunk_exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (ce == cudaSuccess) ce = replay(nchunk);
        if (ce == cudaSuccess) {
          launches += nchunk * nodes;
          it_first = nchunk * K + 1;
          if (frames_per_chunk) streamed_chunks = nchunk;
        }
      } else if (ce == cudaSuccess && elastic) {
        int a = A, b = B, nodes = 0;
        for (int j = 0; j < K; ++j) {
          el_two_phase(cs, a, b, j);
          nodes += 2;
          if (!tagged) {
            k_inject_record_at<<<P.ns, 256, 0, cs>>>(d_it, j, P.nt, P.plane, P.n_src, d_src, d_wav,
                                                     field(b, 2), field(b, 3), P.n_rec, d_rec,
                                                     field(b, 0), field(b, 1), nullptr, d_seis[0],
                                                     d_seis[1], nullptr);
            ++nodes;
          }
          if (si && (j + 1) % si == 0) {
            k_snap_at<<<dim3(cdiv(P.nx, 128), P.nz), 128, 0, cs>>>(
                d_it, j, si, field(b, 1) + P.pad + (long long)P.pad * P.ld, P.ld, P.nx, P.nz,
                d_snap);
            ++nodes;
          }
          std::swap(a, b);
        }
        k_step_add<<<1, 1, 0, cs>>>(d_it, K);
        ++nodes;
        ce = cudaStreamEndCapture(cs, &graph);
        if (ce == cudaSuccess) ce = cudaGraphInstantiate(&chunk_exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (ce == cudaSuccess) ce = replay(nchunk);
        if (ce == cudaSuccess) {
          launches += nchunk * nodes;
          it_first = nchunk * K + 1;
          if (frames_per_chunk) streamed_chunks = nchunk;
        }
      } else if (ce == cudaSuccess) {
        int a = A, b = B, nodes = 0;
        for (int j = 0; j < K; ++j) {
          ac_two_phase(cs, a, b, j);
          nodes += 2;
          if (!tagged) {
            k_inject_record_at<<<P.ns, 256, 0, cs>>>(d_it, j, P.nt, P.plane, P.n_src, d_src, d_wav,
                                                     field(b, 2), nullptr, P.n_rec, d_rec,
                                                     field(b, 2), field(b, 0), field(b, 1),
                                                     d_seis[0], d_seis[1], d_seis[2]);
            ++nodes;
          }
          if (si && (j + 1) % si == 0) {
            k_snap_at<<<dim3(cdiv(P.nx, 128), P.nz), 128, 0, cs>>>(
                d_it, j, si, field(b, 2) + P.pad + (long long)P.pad * P.ld, P.ld, P.nx, P.nz,
                d_snap);
            ++nodes;
          }
          std::swap(a, b);
        }
        k_step_add<<<1, 1, 0, cs>>>(d_it, K);
        ++nodes;
        ce = cudaStreamEndCapture(cs, &graph);
        if (ce == cudaSuccess) ce = cudaGraphInstantiate(&chunk_exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (ce == cudaSuccess) ce = replay(nchunk);
        if (ce == cudaSuccess) {
          launches += nchunk * nodes;
          it_first = nchunk * K + 1;
          if (frames_per_chunk) streamed_chunks = nchunk;
        }
      }
      if (ce != cudaSuccess)
        return fail(ctx, FOMO_ECUDA, std::string("replayed step chunk: ") + cudaGetErrorString(ce));
    }
  }
  // Step-by-step runs with host snapshots copy frame k-1 once frame k is written:
  // the host waits on that pageable copy while the GPU still holds snap_interval
  // queued steps.  (Replayed chunks stream their frames after the loop instead.)
  const bool lag_stream = !P.dev && d_snap && outs.snaps && P.snap_interval > 0 &&
                          streamed_chunks == 0;
  ChunkEvents frame_ev;
  if (lag_stream) {
    frame_ev.ev.assign(2, nullptr);
    for (auto& e : frame_ev.ev) FOMO_CU(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  long long lag_done = 0;  // frames [0, lag_done) copied during the loop
  // Seismograms of step-by-step runs (the large-batch single sweep) are copied
  // the same way, in blocks of kSeisBlock steps, one block behind: each block is
  // one strided copy per component ((n_rec, steps) per shot, pitch n_rec * nt).
  constexpr int kSeisBlock = 128;
  const bool seis_stream = !P.dev && seis_n > 0 && it_first == 1 && P.nt >= 2 * kSeisBlock;
  ChunkEvents seis_ev;
  if (seis_stream) {
    seis_ev.ev.assign(2, nullptr);
    for (auto& e : seis_ev.ev) FOMO_CU(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  long long seis_done = 0;  // time steps [0, seis_done) of every seismogram copied
  auto copy_seis = [&](long long t0, long long t1, cudaStream_t s) -> cudaError_t {
    const size_t pitch = sizeof(float) * (size_t)P.n_rec * P.nt;
    for (int k = 0; k < outs.nseis; ++k) {
      if (!outs.seis[k]) continue;
      cudaError_t e = cudaMemcpy2DAsync(outs.seis[k] + (long long)P.n_rec * t0, pitch,
                                        d_seis[k] + (long long)P.n_rec * t0, pitch,
                                        sizeof(float) * (size_t)P.n_rec * (t1 - t0), P.ns,
                                        cudaMemcpyDeviceToHost, s);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  };
  for (int it = it_first; it <= P.nt; ++it) {
    FOMO_CU(ctx, prof_mark(it, 0));
    if (P.phys == kElastic && replica) {
      FOMO_CU(ctx, replica_step(st, P.N, g, c, dtx, dtz, h, rw, emat, rep_wv, rep_wz, rep_wt,
                                rep_scr, P.ns, it, P.nt, P.n_src, d_src, d_wav, P.n_rec, d_rec,
                                d_seis[0], d_seis[1]));
      const int rl = 2 + (rep_total > 0 ? 4 : 0) + (P.n_src > 0) + (P.n_rec > 0);
      launches += rl;
      sweeps_per_step = rl;
      FOMO_CU(ctx, prof_mark(it, 1));
    } else if (P.phys == kElastic) {
      ElFields a{field(A, 0), field(A, 1), field(A, 2), field(A, 3), field(A, 4)};
      const ElMat& m = emat;
      if (P.fp16 && kernel == FOMO_KERNEL_SINGLE_SWEEP) {
        ElOut o{field(B, 0), field(B, 1), field(B, 2), field(B, 3), field(B, 4)};
        const ElOut16 o16{hfield(B, 0).f16, hfield(B, 1).f16, hfield(B, 2).f16, hfield(B, 3).f16,
                          hfield(B, 4).f16};
        FOMO_CU(ctx, launch_sweep_elastic(st, sp, A, c, dtx, dtz, h, a, m, o, ctx->d_flag, &o16));
        launches += 1;
        sweeps_per_step = 1;
      } else if (P.fp16) {
        HSet ha{{hfield(A, 0), hfield(A, 1), hfield(A, 2), hfield(A, 3), hfield(A, 4)}};
#define FOMO_ELH_CASE(NN)                                                                       \
  case NN:                                                                                      \
    k_elh_vel<NN><<<grd, blk, 0, st>>>(g, c, dtx, dtz, h, ha, m, hfield(B, 0), hfield(B, 1));   \
    k_elh_str<NN><<<grd, blk, 0, st>>>(g, c, dtx, dtz, h, ha, hfield(B, 0), hfield(B, 1), m,    \
                                       hfield(B, 2), hfield(B, 3), hfield(B, 4));               \
    break;
        switch (P.N) { FOMO_ELH_CASE(1) FOMO_ELH_CASE(2) FOMO_ELH_CASE(3) FOMO_ELH_CASE(4) FOMO_ELH_CASE(5) }
#undef FOMO_ELH_CASE
        launches += 2;
        sweeps_per_step = 2;
      } else if (kernel == FOMO_KERNEL_SINGLE_SWEEP) {
        ElOut o{field(B, 0), field(B, 1), field(B, 2), field(B, 3), field(B, 4)};
        FOMO_CU(ctx, launch_sweep_elastic(st, sp, A, c, dtx, dtz, h, a, m, o, ctx->d_flag));
        launches += 1;
        sweeps_per_step = 1;
      } else {
        el_two_phase(st, A, B, it - it_first);  // *d_it = it_first - 1 after the chunks
        launches += 2;
        sweeps_per_step = 2;
      }
      FOMO_CU(ctx, prof_mark(it, 1));
      if (P.fp16)
        k_elh_inject_record<<<P.ns, 256, 0, st>>>(it, P.nt, g, P.n_src, d_src, d_wav, hfield(B, 2),
                                                  hfield(B, 3), P.n_rec, d_rec, hfield(B, 0),
                                                  hfield(B, 1), d_seis[0], d_seis[1]);
      else if (pairs)
        FOMO_CU(ctx, launch_inject_record_pair(st, it, P.nt, P.ns, P.plane, P.n_src, d_src, d_wav,
                                               field(B, 2), field(B, 3), P.n_rec, d_rec,
                                               field(B, 0), field(B, 1), d_seis[0], d_seis[1]));
      else if (!tagged)
        k_inject_record<<<P.ns, 256, 0, st>>>(it, P.nt, P.plane, P.n_src, d_src, d_wav, field(B, 2),
                                              field(B, 3), P.n_rec, d_rec, field(B, 0), field(B, 1),
                                              nullptr, d_seis[0], d_seis[1], nullptr);
      if (!tagged) launches += 1;
    } else if (P.phys == kAcoustic) {
      ac_two_phase(st, A, B, it - it_first);  // *d_it = it_first - 1 after the chunks
      sweeps_per_step = 2;
      FOMO_CU(ctx, prof_mark(it, 1));
      launches += 2;
      if (!tagged) {
        k_inject_record<<<P.ns, 256, 0, st>>>(it, P.nt, P.plane, P.n_src, d_src, d_wav, field(B, 2),
                                              nullptr, P.n_rec, d_rec, field(B, 2), field(B, 0),
                                              field(B, 1), d_seis[0], d_seis[1], d_seis[2]);
        launches += 1;
      }
    } else {
      D2Coef dc;
      dc.two_c0 = 2.0f * kD2C0[P.N];
      for (int l = 0; l < 5; ++l) dc.d[l] = kD2[P.N][l];
      sc_step(st, A, B, C2, it - it_first, dc);  // *d_it = it_first - 1 after the chunks
      sweeps_per_step = 1;
      FOMO_CU(ctx, prof_mark(it, 1));
      if (hook && hook->corrects()) {
        // inject, correct u^{n+1}, then record the corrected field
        k_inject_record<<<1, 256, 0, st>>>(it, P.nt, P.plane, P.n_src, d_src, d_wav, field(C2, 0),
                                           nullptr, 0, d_rec, nullptr, nullptr, nullptr, nullptr,
                                           nullptr, nullptr);
        if (int hr = hook->correct(ctx, st, it, field(C2, 0), field(B, 0), field(A, 0), d_mat, P))
          return hr;
        k_inject_record<<<1, 256, 0, st>>>(it, P.nt, P.plane, 0, d_src, d_wav, nullptr, nullptr,
                                           P.n_rec, d_rec, field(C2, 0), nullptr, nullptr,
                                           d_seis[0], nullptr, nullptr);
        launches += 3 + hook->launches_per_step();
      } else if (!tagged) {
        k_inject_record<<<1, 256, 0, st>>>(it, P.nt, P.plane, P.n_src, d_src, d_wav, field(C2, 0),
                                           nullptr, P.n_rec, d_rec, field(C2, 0), nullptr, nullptr,
                                           d_seis[0], nullptr, nullptr);
        launches += 2;
      } else {
        launches += 1;
      }
      if (hook)
        if (int hr = hook->after_step(ctx, st, it, field(C2, 0), P)) return hr;
    }
    FOMO_CU(ctx, cudaGetLastError());
    // snapshot of the interior (fused_kernels.jl:192-195): p (acoustic), vz (elastic)
    if (P.fp16 && d_snap && P.snap_interval > 0 && it % P.snap_interval == 0) {
      const int k = it / P.snap_interval - 1;
      k_elh_unpack<<<dim3(cdiv(P.nx, 128), P.nz), 128, 0, st>>>(
          g, hfield(B, 1), 0, P.pad, P.pad, P.nx, P.nz, kFp16Sv, d_snap + (long long)k * nint);
    } else if (pairs && d_snap && P.snap_interval > 0 && it % P.snap_interval == 0) {
      const int k = it / P.snap_interval - 1;  // vz of shot 0, interior
      FOMO_CU(ctx, launch_pair_unpack(st, field(B, 1), P.plane, P.ld, P.pad, P.pad, P.nx, P.nz, 0,
                                      d_snap + (long long)k * nint));
    } else if (d_snap && P.snap_interval > 0 && it % P.snap_interval == 0) {
      int k = it / P.snap_interval - 1;
      const float* src = (P.phys == kAcoustic ? field(B, 2) : field(replica ? A : B, 1)) + P.pad +
                         (long long)P.pad * P.ld;
      FOMO_CU(ctx, cudaMemcpy2DAsync(d_snap + (long long)k * nint, sizeof(float) * P.nx, src,
                                     sizeof(float) * P.ld, sizeof(float) * P.nx, P.nz,
                                     cudaMemcpyDeviceToDevice, st));
    }
    if (seis_stream && it % kSeisBlock == 0) {
      const int b = it / kSeisBlock - 1;  // steps [b, b + 1) * kSeisBlock are enqueued
      FOMO_CU(ctx, cudaEventRecord(seis_ev.ev[b & 1], st));
      if (b >= 1) {
        FOMO_CU(ctx, cudaStreamWaitEvent(ctx->copy_stream, seis_ev.ev[(b - 1) & 1], 0));
        FOMO_CU(ctx, copy_seis((long long)(b - 1) * kSeisBlock, (long long)b * kSeisBlock,
                               ctx->copy_stream));
        seis_done = (long long)b * kSeisBlock;
      }
    }
    if (lag_stream && it % P.snap_interval == 0) {
      const int k = it / P.snap_interval - 1;
      FOMO_CU(ctx, cudaEventRecord(frame_ev.ev[k & 1], st));
      if (k >= 1) {
        FOMO_CU(ctx, cudaStreamWaitEvent(ctx->copy_stream, frame_ev.ev[(k - 1) & 1], 0));
        FOMO_CU(ctx, cudaMemcpyAsync(outs.snaps + (long long)(k - 1) * nint,
                                     d_snap + (long long)(k - 1) * nint, sizeof(float) * nint,
                                     cudaMemcpyDeviceToHost, ctx->copy_stream));
        lag_done = k;
      }
    }
    if (P.phys == kScalar) {
      int t = A;
      A = B;
      B = C2;
      C2 = t;
    } else {
      if (!replica) std::swap(A, B);  // the replica updates in place
    }
  }
  FOMO_CU(ctx, cudaEventRecord(ctx->ev1, st));

  // ---- results ----
  if (!P.dev) {
    // frames of the replayed chunks first: each waits only for its own chunk (a
    // copy into pageable memory returns when done, so these overlap the chunks
    // that follow; a copy on st would wait for the whole loop)
    const long long streamed =
        streamed_chunks ? (long long)streamed_chunks * frames_per_chunk : lag_done;
    for (int k = 0; k < streamed_chunks; ++k) {
      FOMO_CU(ctx, cudaStreamWaitEvent(ctx->copy_stream, chunk_ev.ev[k], 0));
      const long long f0 = (long long)k * frames_per_chunk;
      FOMO_CU(ctx, cudaMemcpyAsync(outs.snaps + f0 * nint, d_snap + f0 * nint,
                                   sizeof(float) * frames_per_chunk * nint,
                                   cudaMemcpyDeviceToHost, ctx->copy_stream));
    }
    if (seis_n && seis_done == 0) {
      for (int k = 0; k < outs.nseis; ++k)
        if (outs.seis[k])
          FOMO_CU(ctx, cudaMemcpyAsync(outs.seis[k], d_seis[k], sizeof(float) * seis_n,
                                       cudaMemcpyDeviceToHost, st));
    } else if (seis_n) {
      FOMO_CU(ctx, copy_seis(seis_done, P.nt, st));
    }
    if (d_snap && P.nsnap > streamed)
      FOMO_CU(ctx, cudaMemcpyAsync(outs.snaps + streamed * nint, d_snap + streamed * nint,
                                   sizeof(float) * (P.nsnap - streamed) * nint,
                                   cudaMemcpyDeviceToHost, st));
  }
  if (opts && opts->final_state) {
    // (nxp, nzp, nfield, ns) unpitched host layout; scalar returns (u^n, u^{n-1})
    const long long hp = (long long)P.nxp * P.nzp;
    for (int s = 0; s < P.ns; ++s)
      for (int f = 0; f < (P.phys == kScalar ? 2 : nfield); ++f) {
        if (P.fp16) {  // unscaled FP32 copy of the stored field
          float* tmp = ws_ptr<float>(ctx, o_unpack);
          k_elh_unpack<<<dim3(cdiv(P.nxp, 128), P.nzp), 128, 0, st>>>(
              g, hfield(A, f), (long long)s * P.plane, 0, 0, P.nxp, P.nzp,
              f < 2 ? kFp16Sv : kFp16St, tmp);
          FOMO_CU(ctx, cudaMemcpyAsync(opts->final_state + ((long long)s * nfield + f) * hp, tmp,
                                       sizeof(float) * hp, cudaMemcpyDeviceToHost, st));
          FOMO_CU(ctx, cudaStreamSynchronize(st));  // tmp is reused by the next field
          continue;
        }
        if (pairs) {
          float* tmp = ws_ptr<float>(ctx, o_unpack);
          FOMO_CU(ctx, launch_pair_unpack(st, field(A, f), P.plane, P.ld, 0, 0, P.nxp, P.nzp, s,
                                          tmp));
          FOMO_CU(ctx, cudaMemcpyAsync(opts->final_state + ((long long)s * nfield + f) * hp, tmp,
                                       sizeof(float) * hp, cudaMemcpyDeviceToHost, st));
          FOMO_CU(ctx, cudaStreamSynchronize(st));  // tmp is reused by the next field
          continue;
        }
        const float* src = P.phys == kScalar ? field(f == 0 ? B : A, 0)
                                             : field(A, f) + (long long)s * P.plane;
        FOMO_CU(ctx, cudaMemcpy2DAsync(opts->final_state + ((long long)s * nfield + f) * hp,
                                       sizeof(float) * P.nxp, src, sizeof(float) * P.ld,
                                       sizeof(float) * P.nxp, P.nzp, cudaMemcpyDeviceToHost, st));
      }
  }
  FOMO_CU(ctx, cudaStreamSynchronize(st));
  if (streamed_chunks || lag_done || seis_done)
    FOMO_CU(ctx, cudaStreamSynchronize(ctx->copy_stream));
  if (kernel == FOMO_KERNEL_SINGLE_SWEEP) {
    int hflag = 0;
    FOMO_CU(ctx, cudaMemcpy(&hflag, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (hflag) return fail(ctx, FOMO_ECUDA, "single-sweep kernel: a bounded TMA wait timed out");
  }
  float ms = 0.0f;
  FOMO_CU(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  double sweep_ms = 0.0;
  for (int k = 0; k < nw; ++k) {
    float t = 0.0f;
    FOMO_CU(ctx, cudaEventElapsedTime(&t, pev[2 * k], pev[2 * k + 1]));
    sweep_ms += t;
  }
  for (auto& e : pev) cudaEventDestroy(e);
  if (nw) sweep_ms /= nw;
  if (stats) {
    stats->kernel_time_s = ms * 1e-3;
    const double cells = (double)P.nxp * P.nzp;
    stats->cell_updates = cells * P.nt * P.ns;
    // wavefield words read + written per shot-cell, material words per cell
    double wpc = P.phys == kElastic ? 10.0 : (P.phys == kAcoustic ? 6.0 : 3.0);
    double wm = P.phys == kElastic ? 5.0 : (P.phys == kAcoustic ? 3.0 : 1.0);
    double wbytes = 4.0;  // bytes of a stored wavefield word
    if (P.fp16) {         // binary16 outside the FP32 band
      const double inner = (double)std::max(0, P.nxp - 2 * kFp16Band) * std::max(0, P.nzp - 2 * kFp16Band);
      wbytes = (4.0 * (cells - inner) + 2.0 * inner) / cells;
    }
    stats->alg_bytes = (double)P.nt * cells * (wbytes * wpc * P.ns + 4.0 * wm);
    stats->n_shots = P.ns;
    stats->gpu_launches = launches;
    stats->kernel = kernel;
    stats->status = FOMO_OK;
    stats->sweep_ms = sweep_ms;
    stats->sweep_launches = sweeps_per_step;
    stats->sweep_config = kernel == FOMO_KERNEL_SINGLE_SWEEP
                              ? sp.variant * 1000000 + sp.gm.TX * 1000 + sp.per_sm
                              : 0;
  }
  return FOMO_OK;
}

// ---- scalar2d extensions: strided snapshots and the learned correction ----
__global__ void k_snap_stride(const float* __restrict__ u, long long ld, int pad, int nx, int nz,
                              int stride, int mx, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= mx || i * stride >= nx || j * stride >= nz) return;
  out[i + (long long)mx * j] = u[(long long)(pad + j * stride) * ld + pad + i * stride];
}

// u (interior origin, pitch ld) += y (window with a margin of `mg` cells on
// every side, row length nx + 2 mg), except within src_r cells of a source.
__global__ void k_add_interior(float* __restrict__ u, long long ld, int nx, int nz, int mg,
                               const float* __restrict__ y, const int* __restrict__ src, int n_src,
                               int src_r) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y;
  if (x >= nx || z >= nz) return;
  for (int q = 0; q < n_src; ++q)
    if (abs(x - src[2 * q]) <= src_r && abs(z - src[2 * q + 1]) <= src_r) return;
  float* p = u + (long long)z * ld + x;
  *p = __fadd_rn(*p, y[(long long)(z + mg) * (nx + 2 * mg) + x + mg]);
}

struct SnapHook : ScalarHook {
  int from = 1, every = 1, stride = 1, mx = 0, mz = 0, count = 0;
  float* out = nullptr;  // device (mx, mz, count)
  int after_step(fomo_ctx* ctx, cudaStream_t st, int it, const float* u2, const Plan2& P) override {
    if (it < from || (it - from) % every != 0) return FOMO_OK;
    const int k = (it - from) / every;
    if (k >= count) return FOMO_OK;
    k_snap_stride<<<dim3(cdiv(mx, 128), mz), 128, 0, st>>>(u2, P.ld, P.pad, P.nx, P.nz, stride, mx,
                                                        out + (long long)k * mx * mz);
    FOMO_CU(ctx, cudaGetLastError());
    return FOMO_OK;
  }
};

// The corrector sees a window reaching kCorrMargin cells into the absorbing
// zone (its receptive field), so interior cells get real neighbours, and the
// values injected at the sources in this and the previous step.  The
// correction is added to interior cells except within kCorrSrcR cells of a
// source, the cells its training targets leave out.
constexpr int kCorrMargin = 3;
constexpr int kCorrSrcR = 3;

struct CorrHook : ScalarHook {
  const float* params = nullptr;  // host or device (kNParam floats)
  bool dev = false;
  std::vector<int> src_xz;        // 0-based interior source cells
  const float* wav = nullptr;     // device wavelet matrix (n_src, nt) of the run
  float* d_params = nullptr;
  float* d_y = nullptr;
  int* d_src = nullptr;      // window coordinates
  int* d_src_int = nullptr;  // interior coordinates
  void* scratch = nullptr;
  int mg = 0;
  ~CorrHook() override {
    if (d_params) cudaFree(d_params);
    if (d_y) cudaFree(d_y);
    if (d_src) cudaFree(d_src);
    if (d_src_int) cudaFree(d_src_int);
    if (scratch) cudaFree(scratch);
  }
  bool corrects() const override { return true; }
  int launches_per_step() const override { return 5; }
  int begin(fomo_ctx* ctx, cudaStream_t st, const Plan2& P, const float* d_wav) override {
    wav = d_wav;
    mg = std::min(kCorrMargin, P.pad);
    const long long npix = (long long)(P.nx + 2 * mg) * (P.nz + 2 * mg);
    const int np = fomo_corr_param_count();
    FOMO_CU(ctx, cudaMalloc(&d_params, sizeof(float) * np));
    FOMO_CU(ctx, cudaMalloc(&d_y, sizeof(float) * npix));
    FOMO_CU(ctx, cudaMalloc(&d_src, sizeof(int) * std::max<size_t>(src_xz.size(), 2)));
    FOMO_CU(ctx, cudaMalloc(&d_src_int, sizeof(int) * std::max<size_t>(src_xz.size(), 2)));
    if (!src_xz.empty())
      FOMO_CU(ctx, cudaMemcpyAsync(d_src_int, src_xz.data(), sizeof(int) * src_xz.size(),
                                   cudaMemcpyHostToDevice, st));
    FOMO_CU(ctx, cudaMalloc(&scratch, corr_scratch_bytes(npix)));
    FOMO_CU(ctx, cudaMemcpyAsync(d_params, params, sizeof(float) * np,
                                 dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    // source cells in window coordinates (the window starts mg cells outside)
    std::vector<int> win(src_xz);
    for (int& v : win) v += mg;
    if (!win.empty())
      FOMO_CU(ctx, cudaMemcpyAsync(d_src, win.data(), sizeof(int) * win.size(),
                                   cudaMemcpyHostToDevice, st));
    FOMO_CU(ctx, cudaStreamSynchronize(st));  // src_xz is host memory owned by this hook
    return FOMO_OK;
  }
  int correct(fomo_ctx* ctx, cudaStream_t st, int it, float* u2, const float* u1, const float* u0,
              const float* c2, const Plan2& P) override {
    const long long off = (long long)P.pad * P.ld + P.pad;             // interior origin
    const long long wof = (long long)(P.pad - mg) * P.ld + (P.pad - mg);  // window origin
    const int ns = (int)src_xz.size() / 2;
    const float* inj_next = wav ? wav + (long long)(it - 1) * ns : nullptr;
    const float* inj_prev = (wav && it > 1) ? wav + (long long)(it - 2) * ns : nullptr;
    FOMO_CU(ctx, corr_forward_device(st, P.nz + 2 * mg, P.nx + 2 * mg, u1 + wof, u0 + wof,
                                     c2 + wof, P.ld, ns, d_src, inj_next, inj_prev, d_params,
                                     scratch, d_y, it == 1));
    k_add_interior<<<dim3(cdiv(P.nx, 128), P.nz), 128, 0, st>>>(
        u2 + off, P.ld, P.nx, P.nz, mg, d_y, d_src_int, ns, kCorrSrcR);
    FOMO_CU(ctx, cudaGetLastError());
    return FOMO_OK;
  }
};

}  // namespace
}  // namespace fomo

using namespace fomo;

extern "C" {

int fomo_acoustic2d(fomo_ctx* ctx, const fomo_grid2d* g, const float* vp, const float* rho,
                    const fomo_acq* acq, int32_t snap_interval, float* seis_p, float* seis_vx,
                    float* seis_vz, float* snaps, const fomo_opts* opts, fomo_stats* stats) {
  Plan2 P;
  int rc = make_plan(ctx, kAcoustic, g, acq, snap_interval, opts, false, P);
  if (rc) return rc;
  Outs o{{seis_p, seis_vx, seis_vz}, 3, snaps};
  return run2d(ctx, P, vp, nullptr, rho, acq, o, opts, stats);
}

int fomo_acoustic2d_batch(fomo_ctx* ctx, const fomo_grid2d* g, const float* vp, const float* rho,
                          const fomo_acq* acq, float* seis_p, float* seis_vx, float* seis_vz,
                          const fomo_opts* opts, fomo_stats* stats) {
  Plan2 P;
  int rc = make_plan(ctx, kAcoustic, g, acq, 0, opts, true, P);
  if (rc) return rc;
  Outs o{{seis_p, seis_vx, seis_vz}, 3, nullptr};
  return run2d(ctx, P, vp, nullptr, rho, acq, o, opts, stats);
}

int fomo_elastic2d(fomo_ctx* ctx, const fomo_grid2d* g, const float* vp, const float* vs,
                   const float* rho, const fomo_acq* acq, int32_t snap_interval, float* seis_vx,
                   float* seis_vz, float* snaps, const fomo_opts* opts, fomo_stats* stats) {
  Plan2 P;
  int rc = make_plan(ctx, kElastic, g, acq, snap_interval, opts, false, P);
  if (rc) return rc;
  Outs o{{seis_vx, seis_vz, nullptr}, 2, snaps};
  return run2d(ctx, P, vp, vs, rho, acq, o, opts, stats);
}

int fomo_elastic2d_batch(fomo_ctx* ctx, const fomo_grid2d* g, const float* vp, const float* vs,
                         const float* rho, const fomo_acq* acq, float* seis_vx, float* seis_vz,
                         const fomo_opts* opts, fomo_stats* stats) {
  Plan2 P;
  int rc = make_plan(ctx, kElastic, g, acq, 0, opts, true, P);
  if (rc) return rc;
  Outs o{{seis_vx, seis_vz, nullptr}, 2, nullptr};
  return run2d(ctx, P, vp, vs, rho, acq, o, opts, stats);
}

int fomo_scalar2d(fomo_ctx* ctx, const fomo_grid2d* g, const float* vp, const fomo_acq* acq,
                  float* seis_u, const fomo_opts* opts, fomo_stats* stats) {
  Plan2 P;
  int rc = make_plan(ctx, kScalar, g, acq, 0, opts, false, P);
  if (rc) return rc;
  Outs o{{seis_u, nullptr, nullptr}, 1, nullptr};
  return run2d(ctx, P, vp, nullptr, nullptr, acq, o, opts, stats);
}

int fomo_scalar2d_snapshots(fomo_ctx* ctx, const fomo_grid2d* g, const float* vp,
                            const fomo_acq* acq, int32_t snap_from, int32_t snap_every,
                            int32_t stride, float* snaps, float* seis_u, const fomo_opts* opts,
                            fomo_stats* stats) {
  if (!opts || !(opts->flags & FOMO_F_DEVICE_PTRS))
    return fail(ctx, FOMO_EUNSUPPORTED, "scalar2d snapshots need FOMO_F_DEVICE_PTRS");
  if (!g || snap_from < 1 || snap_every < 1 || stride < 1 || !snaps)
    return fail(ctx, FOMO_EARG, "bad snapshot arguments");
  Plan2 P;
  int rc = make_plan(ctx, kScalar, g, acq, 0, opts, false, P);
  if (rc) return rc;
  SnapHook hk;
  hk.from = snap_from;
  hk.every = snap_every;
  hk.stride = stride;
  hk.mx = (g->nx + stride - 1) / stride;
  hk.mz = (g->nz + stride - 1) / stride;
  hk.count = g->nt >= snap_from ? (g->nt - snap_from) / snap_every + 1 : 0;
  hk.out = snaps;
  Outs o{{seis_u, nullptr, nullptr}, 1, nullptr};
  return run2d(ctx, P, vp, nullptr, nullptr, acq, o, opts, stats, &hk);
}

int fomo_scalar2d_corrected(fomo_ctx* ctx, const fomo_grid2d* g, const float* vp,
                            const fomo_acq* acq, const float* params, float* seis_u,
                            const fomo_opts* opts, fomo_stats* stats) {
  if (!params) return fail(ctx, FOMO_EARG, "corrector parameters are required");
  Plan2 P;
  int rc = make_plan(ctx, kScalar, g, acq, 0, opts, false, P);
  if (rc) return rc;
  CorrHook hk;
  hk.params = params;
  hk.dev = opts && (opts->flags & FOMO_F_DEVICE_PTRS);
  std::vector<int32_t> hx, hz;
  if ((rc = host_copy(ctx, acq->sx, P.n_src, P.dev, hx)) ||
      (rc = host_copy(ctx, acq->sz, P.n_src, P.dev, hz)))
    return rc;
  for (int q = 0; q < P.n_src; ++q) {
    hk.src_xz.push_back(hx[q] - 1);
    hk.src_xz.push_back(hz[q] - 1);
  }
  Outs o{{seis_u, nullptr, nullptr}, 1, nullptr};
  return run2d(ctx, P, vp, nullptr, nullptr, acq, o, opts, stats, &hk);
}

int fomo_debug_medium2d(fomo_ctx* ctx, int32_t kind, int32_t nx, int32_t nz, int32_t pad,
                        float dt, float dh, const float* vp, const float* vs, const float* rho,
                        float* out) {
  if (!ctx || !vp || !out || nx < 1 || nz < 1 || pad < 1 || kind < 0 || kind > 2)
    return fail(ctx, FOMO_EARG, "bad debug_medium2d arguments");
  if ((kind == 0 && (!vs || !rho)) || (kind == 1 && !rho))
    return fail(ctx, FOMO_EARG, "model arrays missing");
  FOMO_CU(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  long long nint = (long long)nx * nz, plane = (long long)(nx + 2 * pad) * (nz + 2 * pad);
  int nf = kind == 0 ? 5 : (kind == 1 ? 3 : 1);
  Arena ar;
  size_t om = ar.take<float>(3 * nint), oo = ar.take<float>(nf * plane);
  int rc = ensure_workspace(ctx, ar.off);
  if (rc) return rc;
  float* m = ws_ptr<float>(ctx, om);
  float* o = ws_ptr<float>(ctx, oo);
  FOMO_CU(ctx, cudaMemcpyAsync(m, vp, sizeof(float) * nint, cudaMemcpyHostToDevice, st));
  if (vs) FOMO_CU(ctx, cudaMemcpyAsync(m + nint, vs, sizeof(float) * nint, cudaMemcpyHostToDevice, st));
  if (rho)
    FOMO_CU(ctx, cudaMemcpyAsync(m + 2 * nint, rho, sizeof(float) * nint, cudaMemcpyHostToDevice, st));
  FOMO_CU(ctx, launch_medium2d(st, kind, nx, nz, pad, nx + 2 * pad, dt / dh, m, vs ? m + nint : nullptr,
                               rho ? m + 2 * nint : nullptr, o, o + plane, o + 2 * plane,
                               o + 3 * plane, o + 4 * plane));
  FOMO_CU(ctx, cudaMemcpyAsync(out, o, sizeof(float) * nf * plane, cudaMemcpyDeviceToHost, st));
  FOMO_CU(ctx, cudaStreamSynchronize(st));
  return FOMO_OK;
}

}  // extern "C"
