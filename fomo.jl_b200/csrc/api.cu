// api.cu -- context, errors, workspace and host-side helpers of libfomo_b200.
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "fomo_internal.cuh"

namespace fomo {

// utils/FD_utils.jl:5-11 (Float64 literals rounded to Float32, as Julia does)
const float kFD[6][5] = {
    {0, 0, 0, 0, 0},
    {(float)1.0, 0, 0, 0, 0},
    {(float)1.125, (float)-0.041666667, 0, 0, 0},
    {(float)1.171875, (float)-0.065104167, (float)0.0046875, 0, 0},
    {(float)1.1962890625, (float)-0.079752604167, (float)0.0095703125, (float)-0.000697544643, 0},
    {(float)1.2115478515625, (float)-0.089721679687, (float)0.0138427734375,
     (float)-0.00176565987723, (float)0.0001186795166},
};
// utils/FD_centered.jl:27-41
const float kD2C0[6] = {0, (float)-2.0, (float)(-5.0 / 2.0), (float)(-49.0 / 18.0),
                        (float)(-205.0 / 72.0), (float)(-5269.0 / 1800.0)};
const float kD2[6][5] = {
    {0, 0, 0, 0, 0},
    {(float)1.0, 0, 0, 0, 0},
    {(float)(4.0 / 3.0), (float)(-1.0 / 12.0), 0, 0, 0},
    {(float)(3.0 / 2.0), (float)(-3.0 / 20.0), (float)(1.0 / 90.0), 0, 0},
    {(float)(8.0 / 5.0), (float)(-1.0 / 5.0), (float)(8.0 / 315.0), (float)(-1.0 / 560.0), 0},
    {(float)(5.0 / 3.0), (float)(-5.0 / 21.0), (float)(5.0 / 126.0), (float)(-5.0 / 1008.0),
     (float)(1.0 / 3150.0)},
};

int fail(fomo_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

int cuda_fail(fomo_ctx* ctx, cudaError_t e, const char* where) {
  char buf[512];
  std::snprintf(buf, sizeof buf, "CUDA error %d (%s) at %s", (int)e, cudaGetErrorString(e), where);
  return fail(ctx, e == cudaErrorMemoryAllocation ? FOMO_ENOMEM : FOMO_ECUDA, buf);
}

int ensure_workspace(fomo_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->ws_bytes) return FOMO_OK;
  if (ctx->ws) {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->ws);
    ctx->ws = nullptr;
    ctx->ws_bytes = 0;
  }
  size_t want = bytes + (bytes >> 4);  // headroom so nearby sizes reuse it
  cudaError_t e = cudaMalloc(&ctx->ws, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    e = cudaMalloc(&ctx->ws, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      ctx->ws = nullptr;
      return cuda_fail(ctx, e, "workspace cudaMalloc");
    }
    want = bytes;
  }
  ctx->ws_bytes = want;
  return FOMO_OK;
}

// boundary/habc/habc.jl:17-44.  q, qt, qxt in float32 (Float32 arithmetic in
// the reference), weights clamp((dist - off)/(pad - 1), 0, 1) in Float64 then
// rounded to float32, tabulated by distance-to-edge.
HabcHost make_habc(int pad, float v_ref, float dt, float dh) {
  HabcHost h;
  h.nbc = pad - 1;
  const float r = (v_ref * dt) / dh;  // Float32(v_ref * dt / dh), left to right
  const float b = 0.45f, beta = 1.0f;
  float br = beta + r;
  float den = br * (1.0f - b);
  h.q = (b * br - r) / den;
  h.qt = (b * br - beta) / den;
  h.qxt = b / (b - 1.0f);
  h.wstride = pad + 2;
  h.wtab.resize(3 * h.wstride);
  const double offs[3] = {0.0, 0.5, 0.75};
  for (int k = 0; k < 3; ++k)
    for (int d = 0; d < h.wstride; ++d) {
      double w = ((double)d - offs[k]) / (double)(pad - 1);
      w = std::min(std::max(w, 0.0), 1.0);
      h.wtab[k * h.wstride + d] = (float)w;
    }
  return h;
}

std::vector<float> sponge_table(int nbc, float factor) {
  std::vector<float> t((size_t)std::max(nbc, 0));
  for (int d = 0; d < nbc; ++d) {
    const float r = factor * (float)(nbc - d);
    const float rr = r * r;
    t[(size_t)d] = (float)std::exp(-(double)rr);
  }
  return t;
}

}  // namespace fomo

using namespace fomo;

extern "C" {

int fomo_version(void) { return FOMO_ABI_VERSION; }

int fomo_create(fomo_ctx** out, int device) {
  if (!out) return FOMO_EARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return FOMO_ECUDA;
  }
  if (device < 0 || device >= n) return FOMO_EARG;
  fomo_ctx* c = new fomo_ctx();
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      cudaMalloc(&c->d_flag, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return FOMO_ECUDA;
  }
  c->stream = c->own_stream;
  *out = c;
  return FOMO_OK;
}

void fomo_destroy(fomo_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  if (ctx->ws) cudaFree(ctx->ws);
  if (ctx->d_flag) cudaFree(ctx->d_flag);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  delete ctx;
}

const char* fomo_last_error(const fomo_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int fomo_set_stream(fomo_ctx* ctx, void* stream) {
  if (!ctx) return FOMO_EARG;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return FOMO_OK;
}

int fomo_trim(fomo_ctx* ctx) {
  if (!ctx) return FOMO_EARG;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->ws) cudaFree(ctx->ws);
  ctx->ws = nullptr;
  ctx->ws_bytes = 0;
  return FOMO_OK;
}

// utils/checks.jl:39-48 (staggered) and :61-70 (centered).
int fomo_check_numerics(float vmax, float dh, float dt, int32_t fd_order, int32_t centered,
                        float* dt_max) {
  int N = order_to_N(fd_order);
  if (N < 0 || !(vmax > 0.0f) || !(dh > 0.0f)) return FOMO_EARG;
  float dmax;
  if (!centered) {
    float s = 0.0f;
    for (int l = 0; l < N; ++l) s += std::fabs(kFD[N][l]);
    dmax = dh / (vmax * std::sqrt(2.0f) * s);
  } else {
    float s = 0.0f;
    for (int l = 0; l < N; ++l) s += std::fabs(kD2[N][l]);
    float lam_max = std::fabs(kD2C0[N]) + 2.0f * s;
    dmax = 2.0f * dh / (vmax * std::sqrt(2.0f * lam_max));
  }
  if (dt_max) *dt_max = dmax;
  return dt <= dmax ? FOMO_OK : FOMO_EARG;
}

}  // extern "C"
