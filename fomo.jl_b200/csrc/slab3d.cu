// slab3d.cu -- z-slab domain decomposition of one 3D model (fomo_slab3d_*).
//
// The fields are stored x fastest, then y, then z, so a z-slab of a field is
// one contiguous block and so is every halo: the exchange between slabs is a
// plain copy of whole planes (NCCL send/recv between GPUs, a device copy
// between slabs of one device), with no packing kernel.
//
// Each slab holds its owned planes plus `halo` = N planes on each side and
// advances them with the fused half steps of sweep3d.cu, which classify the
// Higdon frame by GLOBAL z and address the slab's local volume.  The update of
// an owned plane reads the z windows of three fields (elastic velocity: txz,
// tyz, tzz; stress: vx, vy, vz; acoustic: p, then vz) N planes beyond it and
// everything else in-plane, so those fields are the halo.  The Higdon z terms
// of a band plane read the half-step value of the plane next to it on the
// interior side; cuts are therefore kept clear of the z bands of the frame and
// of those planes.  Under those two rules every owned plane equals the single-device
// run's, bit for bit.  The planes just outside a slab's owned range are
// updated as well (the march recomputes the plane before and after each
// segment) from partly stale halo data; those values only feed Higdon z terms,
// which the cut rule excludes, and are never stored.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "fomo_internal.cuh"
#include "sweep3d.cuh"

struct fomo_slab3d {
  fomo_ctx* ctx = nullptr;
  bool elastic = true;
  int N = 0, nt = 0, n_src = 0, n_rec = 0;
  fomo::Geo3 g;
  float* state = nullptr;   // caller memory: 2 sets x nfield volumes
  void* mem = nullptr;      // one allocation for everything below
  float* mat = nullptr;     // materials of the held planes
  float* wt = nullptr;      // Higdon weight ramps
  int* src = nullptr;       // linear index per source (-1: another slab's)
  int* rec = nullptr;       // linear index per receiver (-1: another slab's)
  float* wav = nullptr;     // (n_src, nt)
  float* seis = nullptr;    // 3 x (n_rec, nt)
  int* err = nullptr;       // bounded-wait timeouts
  std::vector<uint8_t> owned;
  fomo::Fused3Plan fp;
  fomo::Coef c;
  fomo::HabcDev h;
  float dtdh = 0.0f;
};

namespace fomo {
namespace {

// Layout of slab [z_lo, z_hi) of the padded grid; "" or why the cut is refused.
std::string slab_layout(int elastic, const fomo_grid3d* gp, int z_lo, int z_hi,
                        fomo_slab3d_layout* L) {
  if (!gp) return "grid is required";
  const int N = order_to_N(gp->fd_order);
  if (N < 0) return "Unsupported FD order: " + std::to_string(gp->fd_order);
  if (gp->nx < 1 || gp->ny < 1 || gp->nz < 1 || gp->nt < 1 || gp->nbc < 0 || !(gp->dh > 0.0f) ||
      !(gp->dt > 0.0f))
    return "invalid 3D grid";
  const int pad = gp->nbc + N;
  if (pad < 2) return "nbc + fd_order/2 must be >= 2";
  std::memset(L, 0, sizeof *L);
  L->nxp = gp->nx + 2 * pad;
  L->nyp = gp->ny + 2 * pad;
  L->nzp = gp->nz + 2 * pad;
  L->ld = (L->nxp + 31) & ~31;
  L->plane = (int64_t)L->ld * L->nyp;
  L->halo = N;
  L->nfield = elastic ? 9 : 4;
  // The Higdon z bands are planes 1..fr and nzp-1-fr..nzp-2 (fr = pad - 1);
  // a band plane's z term reads the half-step value of its interior-side
  // neighbour (fr + 1, or nzp - 2 - fr), so each band and that plane stay in
  // one slab.
  const int fr = pad - 1;
  L->cut_min = fr + 2;
  L->cut_max = L->nzp - 2 - fr;
  L->z_lo = z_lo;
  L->z_hi = z_hi;
  if (z_lo < 0 || z_hi > L->nzp || z_lo >= z_hi)
    return "slab planes [" + std::to_string(z_lo) + ", " + std::to_string(z_hi) +
           ") are not inside the padded grid of " + std::to_string(L->nzp) + " planes";
  auto cut_ok = [&](int c) { return c >= L->cut_min && c <= L->cut_max; };
  if ((z_lo > 0 && !cut_ok(z_lo)) || (z_hi < L->nzp && !cut_ok(z_hi)))
    return "slab cuts must lie in [" + std::to_string(L->cut_min) + ", " +
           std::to_string(L->cut_max) + "] (outside the Higdon z bands)";
  if ((z_lo > 0 || z_hi < L->nzp) && z_hi - z_lo < N)
    return "a slab with a neighbour must own at least fd_order/2 planes";
  L->z_base = std::max(z_lo - N, 0);
  L->nz_local = std::min(z_hi + N, L->nzp) - L->z_base;
  if (L->plane * L->nz_local > (1LL << 31) - 1) return "slab volume exceeds 2^31 cells";
  L->state_floats = 2LL * L->nfield * L->plane * L->nz_local;
  return "";
}

}  // namespace
}  // namespace fomo

using namespace fomo;

extern "C" {

int fomo_slab3d_layout_of(fomo_ctx* ctx, int32_t elastic, const fomo_grid3d* g, int32_t z_lo,
                          int32_t z_hi, fomo_slab3d_layout* out) {
  if (!out) return fail(ctx, FOMO_EARG, "layout output is required");
  const std::string why = slab_layout(elastic, g, z_lo, z_hi, out);
  return why.empty() ? FOMO_OK : fail(ctx, FOMO_EARG, why);
}

int fomo_slab3d_create(fomo_ctx* ctx, int32_t elastic, const fomo_grid3d* gp, const float* vp,
                       const float* vs, const float* rho, const fomo_acq3d* acq, int32_t z_lo,
                       int32_t z_hi, float* state, fomo_slab3d** out) {
  if (!ctx) return FOMO_EARG;
  if (!out) return fail(ctx, FOMO_EARG, "slab output is required");
  *out = nullptr;
  fomo_slab3d_layout L;
  const std::string why = slab_layout(elastic, gp, z_lo, z_hi, &L);
  if (!why.empty()) return fail(ctx, FOMO_EARG, why);
  if (!acq || !vp || !rho || (elastic && !vs))
    return fail(ctx, FOMO_EARG, "acquisition and model arrays are required");
  if (!state || ((uintptr_t)state & 15))
    return fail(ctx, FOMO_EARG, "state must be 16-byte aligned device memory");
  if (acq->n_src < 0 || acq->n_rec < 0 ||
      (acq->n_src > 0 && (!acq->sx || !acq->sy || !acq->sz || !acq->wavelet)) ||
      (acq->n_rec > 0 && (!acq->rx || !acq->ry || !acq->rz)))
    return fail(ctx, FOMO_EARG, "invalid 3D acquisition");
  const int N = L.halo, pad = gp->nbc + N, nt = gp->nt;
  if (!fused3_supported(N))
    return fail(ctx, FOMO_EUNSUPPORTED, "z-slabs need the fused 3D half steps (TMA encoder)");
  const int nx = gp->nx, ny = gp->ny, nz = gp->nz;
  for (int k = 0; k < acq->n_src; ++k)
    if (acq->sx[k] < 1 || acq->sx[k] > nx || acq->sy[k] < 1 || acq->sy[k] > ny ||
        acq->sz[k] < 1 || acq->sz[k] > nz)
      return fail(ctx, FOMO_EARG, "source index out of range");
  for (int k = 0; k < acq->n_rec; ++k)
    if (acq->rx[k] < 1 || acq->rx[k] > nx || acq->ry[k] < 1 || acq->ry[k] > ny ||
        acq->rz[k] < 1 || acq->rz[k] > nz)
      return fail(ctx, FOMO_EARG, "receiver index out of range");
  const long long nint = (long long)nx * ny * nz;
  float v_ref = gp->v_ref;
  if (!(v_ref > 0.0f)) {
    v_ref = INFINITY;
    for (long long k = 0; k < nint; ++k)
      if (vp[k] > 0.0f && vp[k] < v_ref) v_ref = vp[k];
    if (!std::isfinite(v_ref)) return fail(ctx, FOMO_EARG, "vp has no positive value for v_ref");
  }

  auto* s = new fomo_slab3d;
  auto bail = [&](int rc) {
    if (s->mem) cudaFree(s->mem);
    delete s;
    return rc;
  };
  s->ctx = ctx;
  s->elastic = elastic != 0;
  s->N = N;
  s->nt = nt;
  s->n_src = acq->n_src;
  s->n_rec = acq->n_rec;
  s->state = state;
  Geo3& g = s->g;
  g.nx = L.nxp;
  g.ny = L.nyp;
  g.nz = L.nz_local;
  g.ld = L.ld;
  g.sy = L.ld;
  g.sz = L.plane;
  g.vol = L.plane * L.nz_local;
  g.M = N;
  g.nbc = pad - 1;
  g.z0 = L.z_base;
  g.gnz = L.nzp;
  g.zlo = z_lo - L.z_base;
  g.zhi = z_hi - L.z_base;

  // points of the owned planes, as linear indices of the held volume
  std::vector<int32_t> src_lin(std::max(acq->n_src, 1), -1), rec_lin(std::max(acq->n_rec, 1), -1);
  auto lin = [&](int a, int b, int c) -> int32_t {
    const int zg = c - 1 + pad;
    if (zg < z_lo || zg >= z_hi) return -1;
    return (int32_t)((a - 1 + pad) + g.sy * (b - 1 + pad) + g.sz * (zg - L.z_base));
  };
  for (int k = 0; k < acq->n_src; ++k) src_lin[k] = lin(acq->sx[k], acq->sy[k], acq->sz[k]);
  s->owned.assign(std::max(acq->n_rec, 0), 0);
  for (int k = 0; k < acq->n_rec; ++k) {
    rec_lin[k] = lin(acq->rx[k], acq->ry[k], acq->rz[k]);
    s->owned[k] = rec_lin[k] >= 0;
  }
  HabcHost hh = make_habc(pad, v_ref, gp->dt, gp->dh);
  const std::vector<float> wt3 = habc3_ramps(pad, hh.wstride);
  const int nmat = elastic ? 8 : 4;
  const long long seis_n = (long long)acq->n_rec * nt;
  Arena ar;
  const size_t o_mat = ar.take<float>(nmat * g.vol);
  const size_t o_tab = ar.take<char>(fused3_table_bytes(g));
  const size_t o_wt = ar.take<float>(wt3.size());
  const size_t o_src = ar.take<int32_t>(src_lin.size());
  const size_t o_rec = ar.take<int32_t>(rec_lin.size());
  const size_t o_wav = ar.take<float>(std::max(1LL, (long long)acq->n_src * nt));
  const size_t o_seis = ar.take<float>(std::max(1LL, 3 * seis_n));
  const size_t o_err = ar.take<int>(1);
  // raw model planes the held volume reads (edge-replicated padding, and the
  // staggered averages one plane below)
  const int kz0 = std::min(std::max(L.z_base - pad, 0), nz - 1);
  const int kz1 = std::min(std::max(L.z_base + L.nz_local - pad, 0), nz - 1);
  const long long nraw = (long long)nx * ny * (kz1 - kz0 + 1);
  FOMO_CU(ctx, cudaSetDevice(ctx->device));
  float* raw = nullptr;  // freed once the materials are built
  if (cudaMalloc(&s->mem, ar.off) != cudaSuccess) {
    cudaGetLastError();
    s->mem = nullptr;
    return bail(fail(ctx, FOMO_ENOMEM, "z-slab: device allocation failed"));
  }
  if (cudaMalloc(&raw, sizeof(float) * 3 * nraw) != cudaSuccess) {
    cudaGetLastError();
    return bail(fail(ctx, FOMO_ENOMEM, "z-slab: device allocation failed"));
  }
  char* base = static_cast<char*>(s->mem);
  s->mat = reinterpret_cast<float*>(base + o_mat);
  s->wt = reinterpret_cast<float*>(base + o_wt);
  s->src = reinterpret_cast<int*>(base + o_src);
  s->rec = reinterpret_cast<int*>(base + o_rec);
  s->wav = reinterpret_cast<float*>(base + o_wav);
  s->seis = reinterpret_cast<float*>(base + o_seis);
  s->err = reinterpret_cast<int*>(base + o_err);
  cudaStream_t st = ctx->stream;
  const long long off = (long long)nx * ny * kz0;
  int rc = FOMO_OK;
  auto cu = [&](cudaError_t e, const char* where) {
    if (e != cudaSuccess && rc == FOMO_OK) rc = cuda_fail(ctx, e, where);
  };
  cu(cudaMemcpyAsync(raw, vp + off, 4 * nraw, cudaMemcpyHostToDevice, st), "slab vp");
  cu(cudaMemcpyAsync(raw + 2 * nraw, rho + off, 4 * nraw, cudaMemcpyHostToDevice, st), "slab rho");
  if (elastic)
    cu(cudaMemcpyAsync(raw + nraw, vs + off, 4 * nraw, cudaMemcpyHostToDevice, st), "slab vs");
  cu(cudaMemcpyAsync(s->wt, wt3.data(), 4 * wt3.size(), cudaMemcpyHostToDevice, st), "slab ramps");
  cu(cudaMemcpyAsync(s->src, src_lin.data(), 4 * src_lin.size(), cudaMemcpyHostToDevice, st),
     "slab sources");
  cu(cudaMemcpyAsync(s->rec, rec_lin.data(), 4 * rec_lin.size(), cudaMemcpyHostToDevice, st),
     "slab receivers");
  if (acq->n_src)
    cu(cudaMemcpyAsync(s->wav, acq->wavelet, 4LL * acq->n_src * nt, cudaMemcpyHostToDevice, st),
       "slab wavelet");
  cu(cudaMemsetAsync(s->seis, 0, 4 * std::max(1LL, 3 * seis_n), st), "slab seismograms");
  cu(cudaMemsetAsync(s->err, 0, sizeof(int), st), "slab status");
  cu(cudaMemsetAsync(state, 0, 4 * L.state_floats, st), "slab state");
  if (rc == FOMO_OK)
    cu(medium3d(st, elastic, g, raw, elastic ? raw + nraw : raw, raw + 2 * nraw, nx, ny, nz, pad,
                kz0, s->mat),
       "k_medium3d");
  if (rc == FOMO_OK)
    cu(fused3_make_plan(s->fp, g, N, elastic, state, s->mat, base + o_tab, st),
       "fused3_make_plan");  // synchronizes the stream: the host arrays above are free
  if (rc != FOMO_OK) cudaStreamSynchronize(st);
  cudaFree(raw);
  if (rc != FOMO_OK) return bail(rc);
  for (int l = 0; l < 5; ++l) s->c.a[l] = kFD[N][l];
  s->h = HabcDev{hh.q, hh.qt, hh.qxt, hh.nbc, hh.wstride, s->wt};
  s->dtdh = gp->dt / gp->dh;
  *out = s;
  return FOMO_OK;
}

int fomo_slab3d_step(fomo_slab3d* s, int32_t it, int32_t half) {
  if (!s) return FOMO_EARG;
  fomo_ctx* ctx = s->ctx;
  if (it < 1 || it > s->nt || (half != 0 && half != 1))
    return fail(ctx, FOMO_EARG, "slab step: it must be in 1..nt and half 0 or 1");
  const int A = (it + 1) & 1, B = it & 1;
  FOMO_CU(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  if (half == 0) {
    FOMO_CU(ctx, fused3_velocity(st, s->fp, s->g, s->state, A, B, s->c, s->dtdh, s->h, s->err));
  } else {
    FOMO_CU(ctx, fused3_stress(st, s->fp, s->g, s->state, A, B, s->c, s->dtdh, s->h, s->err));
    const long long n = (long long)s->n_rec * s->nt;
    FOMO_CU(ctx, inject_record3(st, s->elastic, s->g, s->state, B, it, s->nt, s->n_src, s->src,
                                s->wav, s->n_rec, s->rec, s->seis, s->seis + n, s->seis + 2 * n));
  }
  return FOMO_OK;
}

int fomo_slab3d_seismograms(fomo_slab3d* s, float* svx, float* svy, float* svz, uint8_t* owned) {
  if (!s) return FOMO_EARG;
  fomo_ctx* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  FOMO_CU(ctx, cudaSetDevice(ctx->device));
  FOMO_CU(ctx, cudaStreamSynchronize(st));
  int flag = 0;
  FOMO_CU(ctx, cudaMemcpy(&flag, s->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) return fail(ctx, FOMO_ECUDA, "z-slab half step: a bounded TMA wait timed out");
  const long long n = (long long)s->n_rec * s->nt;
  float* outs[3] = {svx, svy, svz};
  for (int k = 0; k < 3; ++k)
    if (outs[k] && n)
      FOMO_CU(ctx, cudaMemcpy(outs[k], s->seis + k * n, 4 * n, cudaMemcpyDeviceToHost));
  if (owned && s->n_rec) std::memcpy(owned, s->owned.data(), s->owned.size());
  return FOMO_OK;
}

void fomo_slab3d_destroy(fomo_slab3d* s) {
  if (!s) return;
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->ctx->stream);
  if (s->mem) cudaFree(s->mem);
  delete s;
}

}  // extern "C"
