// noalloc.cu -- fomo_scalar2d_noalloc: the scalar2d solver for callers that
// cannot allocate device memory.
//
// Some callers may not call cudaMalloc: a plugin running inside a framework
// whose caching allocator owns every device byte, a service with a fixed device
// budget, or code that must not trigger an allocation (and the implicit device
// synchronisation cudaFree brings) in the middle of its own schedule.  For them
// this entry point keeps every working buffer (the three leapfrog wavefields,
// c^2, the HABC weight table, the padded source/receiver indices and an error
// word) in one file-scope __device__ array of fixed size.  The caller passes the
// inputs and outputs as device pointers; nothing here calls cudaMalloc,
// cudaFree or any allocating library routine.
//
// Properties a user must know:
//  * The array (kNoallocBytes = 32 MiB) is held by every GPU that loads this
//    library until the process exits.
//  * Problems whose working set exceeds it are rejected with FOMO_EARG.
//  * All calls share the one array: two calls whose work overlaps on the GPU
//    (other streams, other host threads) race and corrupt each other.
//  * The array keeps the previous call's contents; each call clears the
//    wavefields and the error word before it starts.
//  * Every call looks up the array's device address (cudaGetSymbolAddress,
//    which allocates nothing) on the current device and context, so a device
//    reset or a different current context never leaves it a stale address.
//  * The call is synchronous: it returns once the run has finished on its
//    stream and the results are in the caller's buffers.
//  * Like the other C entry points it makes none of the reference's argument
//    checks on the time step (the centered CFL bound of utils/checks.jl:61-70)
//    or on dispersion: an unstable dt runs and its result grows without bound.
//    The caller (or a binding such as the Python mirror) makes those checks.
#include <algorithm>
#include <cstdio>

#include "solver2d_kernels.cuh"

namespace fomo {
namespace {

constexpr size_t kNoallocBytes = size_t(32) << 20;

// Working memory of fomo_scalar2d_noalloc (see the file comment).  In host
// code this name is only a handle for cudaGetSymbolAddress, never an address.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

void set_err(char* err, int len, const char* msg) {
  if (err && len > 0) std::snprintf(err, (size_t)len, "%s", msg);
}

// The array's device address in the current device's current context.  Looked
// up on every call (no cache), so it always belongs to the context the call
// launches in.
int scratch_address(unsigned char** out, char* err, int len) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    char b[256];
    std::snprintf(b, sizeof b, "cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
    set_err(err, len, b);
    return FOMO_ECUDA;
  }
  *out = static_cast<unsigned char*>(p);
  return FOMO_OK;
}

inline size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

// Padded linear source/receiver indices with the range check of
// utils/checks.jl:8-13 (a bad index sets *flag and is never used), and the
// HABC weight table of boundary/habc/habc.jl:17-44 by distance-to-edge.
__global__ void k_noalloc_prep(int nx, int nz, int pad, int nxp, int n_src,
                               const int32_t* __restrict__ sx, const int32_t* __restrict__ sz,
                               int n_rec, const int32_t* __restrict__ rx,
                               const int32_t* __restrict__ rz, int32_t* src_lin, int32_t* rec_lin,
                               int wstride, float* wtab, int* flag) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n_src) {
    int x = sx[t], z = sz[t];
    if (x < 1 || x > nx || z < 1 || z > nz) {
      atomicOr(flag, 1);
      src_lin[t] = 0;
    } else {
      src_lin[t] = (x - 1 + pad) + nxp * (z - 1 + pad);
    }
  }
  if (t < n_rec) {
    int x = rx[t], z = rz[t];
    if (x < 1 || x > nx || z < 1 || z > nz) {
      atomicOr(flag, 2);
      rec_lin[t] = 0;
    } else {
      rec_lin[t] = (x - 1 + pad) + nxp * (z - 1 + pad);
    }
  }
  if (t < 3 * wstride) {
    const double offs[3] = {0.0, 0.5, 0.75};
    int k = t / wstride, d = t % wstride;
    double w = ((double)d - offs[k]) / (double)(pad - 1);
    w = fmin(fmax(w, 0.0), 1.0);
    wtab[t] = (float)w;
  }
}

template <int N>
void launch_step(cudaStream_t st, dim3 grd, dim3 blk, const Geo2& g, const D2Coef& dc,
                 const HabcDev& h, const float* u1, const float* u0, const float* c2, float* u2) {
  k_sc_step<N><<<grd, blk, 0, st>>>(g, dc, h, u1, u0, c2, u2);
}

}  // namespace
}  // namespace fomo

using namespace fomo;

extern "C" int fomo_scalar2d_noalloc(const fomo_grid2d* g, const float* vp, const fomo_acq* acq,
                                     float* seis_u, void* stream, char* err, int32_t err_len) {
  if (!g || !acq || !vp) {
    set_err(err, err_len, "grid, acquisition and vp are required");
    return FOMO_EARG;
  }
  const int N = order_to_N(g->fd_order);
  if (N < 0) {
    set_err(err, err_len, "Unsupported FD order");
    return FOMO_EARG;
  }
  if (g->nx < 1 || g->nz < 1 || g->nt < 1 || g->nbc < 0 || !(g->dh > 0.0f) || !(g->dt > 0.0f)) {
    set_err(err, err_len, "invalid grid (need nx, nz, nt >= 1, nbc >= 0, dh, dt > 0)");
    return FOMO_EARG;
  }
  if (!(g->v_ref > 0.0f)) {
    set_err(err, err_len, "v_ref must be given (> 0); the no-alloc entry does not scan vp");
    return FOMO_EARG;
  }
  if (acq->n_shots != 1 || acq->n_src < 0 || acq->n_rec < 0 ||
      (acq->n_src > 0 && (!acq->sx || !acq->sz || !acq->wavelet)) ||
      (acq->n_rec > 0 && (!acq->rx || !acq->rz || !seis_u))) {
    set_err(err, err_len, "invalid acquisition (one shot; sources need sx, sz, wavelet)");
    return FOMO_EARG;
  }
  const int pad = g->nbc + N;
  if (pad < 2) {
    set_err(err, err_len, "nbc + fd_order/2 must be >= 2");
    return FOMO_EARG;
  }
  const int nxp = g->nx + 2 * pad, nzp = g->nz + 2 * pad;
  const long long plane = (long long)nxp * nzp;
  const int wstride = pad + 2;
  // carve: 3 wavefields | c2 | weights | src idx | rec idx | error word
  const size_t o_u = 0;
  const size_t o_c2 = o_u + up256(3 * sizeof(float) * (size_t)plane);
  const size_t o_w = o_c2 + up256(sizeof(float) * (size_t)plane);
  const size_t o_src = o_w + up256(sizeof(float) * 3 * (size_t)wstride);
  const size_t o_rec = o_src + up256(sizeof(int32_t) * (size_t)acq->n_src);
  const size_t o_flag = o_rec + up256(sizeof(int32_t) * (size_t)acq->n_rec);
  const size_t need = o_flag + 256;
  if (need > kNoallocBytes) {
    char b[256];
    std::snprintf(b, sizeof b,
                  "problem needs %zu bytes of working memory; the no-alloc limit is %zu bytes "
                  "(about %lld padded cells)",
                  need, kNoallocBytes, (long long)(kNoallocBytes / 16));
    set_err(err, err_len, b);
    return FOMO_EARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    set_err(err, err_len, "no current CUDA device");
    return FOMO_ECUDA;
  }
  unsigned char* base = nullptr;
  int rc = scratch_address(&base, err, err_len);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  float* u = reinterpret_cast<float*>(base + o_u);
  float* c2 = reinterpret_cast<float*>(base + o_c2);
  float* wtab = reinterpret_cast<float*>(base + o_w);
  int32_t* src_lin = reinterpret_cast<int32_t*>(base + o_src);
  int32_t* rec_lin = reinterpret_cast<int32_t*>(base + o_rec);
  int* flag = reinterpret_cast<int*>(base + o_flag);

  // HABC coefficients (boundary/habc/habc.jl:17-44), float32 as the reference computes them
  const float r = (g->v_ref * g->dt) / g->dh;
  const float b = 0.45f, beta = 1.0f, br = beta + r, den = br * (1.0f - b);
  HabcDev h{(b * br - r) / den, (b * br - beta) / den, b / (b - 1.0f), pad - 1, wstride, wtab};
  Geo2 geo{nxp, nzp, nxp, N, pad - 1, plane};
  D2Coef dc;
  dc.two_c0 = 2.0f * kD2C0[N];
  for (int l = 0; l < 5; ++l) dc.d[l] = kD2[N][l];

  cudaError_t e = cudaMemsetAsync(u, 0, 3 * sizeof(float) * (size_t)plane, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(flag, 0, sizeof(int), st);
  if (e == cudaSuccess) {
    int nthr = std::max(std::max(acq->n_src, acq->n_rec), 3 * wstride);
    k_noalloc_prep<<<cdiv(nthr, 256), 256, 0, st>>>(g->nx, g->nz, pad, nxp, acq->n_src, acq->sx,
                                                    acq->sz, acq->n_rec, acq->rx, acq->rz, src_lin,
                                                    rec_lin, wstride, wtab, flag);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = launch_medium2d(st, 2, g->nx, g->nz, pad, nxp, g->dt / g->dh, vp, nullptr, nullptr, c2, nullptr,
                        nullptr, nullptr, nullptr);
  int hflag = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    char b2[256];
    std::snprintf(b2, sizeof b2, "CUDA error during set-up: %s", cudaGetErrorString(e));
    set_err(err, err_len, b2);
    return FOMO_ECUDA;
  }
  if (hflag) {
    set_err(err, err_len, (hflag & 1) ? "source index out of range" : "receiver index out of range");
    return FOMO_EARG;
  }

  dim3 blk(32, 8), grd(cdiv(nxp, 32), cdiv(nzp, 8), 1);
  float* buf[3] = {u, u + plane, u + 2 * plane};
  int A = 0, B = 1, C = 2;  // u^{n-1}, u^n, u^{n+1}
  for (int it = 1; it <= g->nt && e == cudaSuccess; ++it) {
    switch (N) {
      case 1: launch_step<1>(st, grd, blk, geo, dc, h, buf[B], buf[A], c2, buf[C]); break;
      case 2: launch_step<2>(st, grd, blk, geo, dc, h, buf[B], buf[A], c2, buf[C]); break;
      case 3: launch_step<3>(st, grd, blk, geo, dc, h, buf[B], buf[A], c2, buf[C]); break;
      case 4: launch_step<4>(st, grd, blk, geo, dc, h, buf[B], buf[A], c2, buf[C]); break;
      default: launch_step<5>(st, grd, blk, geo, dc, h, buf[B], buf[A], c2, buf[C]); break;
    }
    k_inject_record<<<1, 256, 0, st>>>(it, g->nt, plane, acq->n_src, src_lin, acq->wavelet,
                                       buf[C], nullptr, acq->n_rec, rec_lin, buf[C], nullptr,
                                       nullptr, seis_u, nullptr, nullptr);
    e = cudaGetLastError();
    int t = A;
    A = B;
    B = C;
    C = t;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    char b3[256];
    std::snprintf(b3, sizeof b3, "CUDA error in the time loop: %s", cudaGetErrorString(e));
    set_err(err, err_len, b3);
    return FOMO_ECUDA;
  }
  set_err(err, err_len, "");
  return FOMO_OK;
}
