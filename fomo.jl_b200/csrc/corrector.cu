// corrector.cu -- learned per-step dispersion corrector for coarse-grid runs
// (no reference counterpart).
//
// Network: three 3x3 convolutions, bias-free, ReLU between them:
//   features (6 channels) -> 16 -> 16 -> 1, the features being
//   u^n, u^{n-1}, c2 u^n, c2^2 u^n, and at the source cells the values
//   injected in this step and in the previous one (0 elsewhere).
// Every input channel is linear in the wave's amplitude and the network has
// no bias, so the correction is positively homogeneous: it scales with the
// amplitude and needs no normalisation.  The correction is added to u^{n+1}
// after the coarse scalar step and the source injection.
//
// Tensor-core path: activations are BF16 in NHWC with 16 channels (32 bytes a
// pixel), weights BF16, accumulation FP32, via mma.sync m16n8k16 implicit
// GEMMs: a warp takes 16 consecutive pixels of a row (M), one conv tap's 16
// input channels per k-step (K = 16, 9 taps), 8 output channels per n-tile.
//   forward            Y[p, co]   = sum_tap sum_ci X[p + tap, ci] W[tap, ci, co]
//   backward (data)    dX[p, ci]  = sum_tap sum_co dY[p - tap, co] W[tap, ci, co]
//                                 = the forward kernel on flipped, transposed weights
//   backward (weights) dW[tap, ci, co] = sum_p X[p + tap, ci] dY[p, co]
//                        (M = ci, N = co, K = pixels; per-block partials reduced
//                         in block order, so gradients are deterministic)
// Parameters are FP32 masters: W1[9][6][16], W2[9][16][16], W3[9][16] (co = 1).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "fomo_internal.cuh"

namespace fomo {
namespace {

constexpr int kC = 16;                       // channel stride of every activation
constexpr int kCin = 6;                      // feature channels
constexpr int kNW1 = 9 * kCin * 16;          // 864
constexpr int kNW2 = 9 * 16 * 16;            // 2304
constexpr int kNW3 = 9 * 16;                 // 144
constexpr int kNParam = kNW1 + kNW2 + kNW3;  // 3312
// packed B fragments, [tap][ntile][lane][2] uint32 each
constexpr int kF16 = 9 * 2 * 64;  // 16 output channels (2 n-tiles)
constexpr int kF8 = 9 * 1 * 64;   // 1 output channel (1 n-tile, 7 zero columns)
constexpr int kOffF1 = 0, kOffF2 = kOffF1 + kF16, kOffF3 = kOffF2 + kF16;
constexpr int kOffT3 = kOffF3 + kF8, kOffT2 = kOffT3 + kF16;
constexpr int kNFrag = kOffT2 + kF16;

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(lo)) |
         ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(hi)) << 16);
}
__device__ __forceinline__ float bf(uint16_t u) { return __bfloat162float(__ushort_as_bfloat16(u)); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// W[tap][ci][co] of a layer with ci_n x co_n channels (zero outside)
__device__ __forceinline__ float wat(const float* W, int ci_n, int co_n, int tap, int ci, int co) {
  return (ci < ci_n && co < co_n) ? W[(tap * ci_n + ci) * co_n + co] : 0.0f;
}

// B fragment of m16n8k16 (k x n): reg0 = (k = 2t, 2t+1; n = g), reg1 = (k = 2t+8, 2t+9; n = g)
// with t = lane & 3, g = lane >> 2.  Forward: B[k = ci][n = co] of tap.
// Transposed (backward data): tap' = 8 - tap, B[k = co][n = ci].
__global__ void k_pack(const float* __restrict__ P, uint32_t* __restrict__ F) {
  const float* W1 = P;
  const float* W2 = P + kNW1;
  const float* W3 = P + kNW1 + kNW2;
  for (int i = threadIdx.x; i < kNFrag / 2; i += blockDim.x) {
    int part, base;
    if (i < kOffF2 / 2) { part = 0; base = kOffF1 / 2; }
    else if (i < kOffF3 / 2) { part = 1; base = kOffF2 / 2; }
    else if (i < kOffT3 / 2) { part = 2; base = kOffF3 / 2; }
    else if (i < kOffT2 / 2) { part = 3; base = kOffT3 / 2; }
    else { part = 4; base = kOffT2 / 2; }
    const int nt_n = part == 2 ? 1 : 2;
    int r = i - base;
    const int lane = r & 31;
    r >>= 5;
    const int nt = r % nt_n, tap = r / nt_n;
    const int t = lane & 3, g = lane >> 2, n = nt * 8 + g;
    float v[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int k = 2 * t + (e & 1) + (e >> 1) * 8;
      switch (part) {
        case 0: v[e] = wat(W1, kCin, 16, tap, k, n); break;
        case 1: v[e] = wat(W2, 16, 16, tap, k, n); break;
        case 2: v[e] = wat(W3, 16, 1, tap, k, n); break;
        case 3: v[e] = wat(W3, 16, 1, 8 - tap, n, k); break;   // dY3 (1 ch) -> dH2 (16 ch)
        default: v[e] = wat(W2, 16, 16, 8 - tap, n, k); break;  // dPre2 -> dH1
      }
    }
    F[2 * i] = pack2(v[0], v[1]);
    F[2 * i + 1] = pack2(v[2], v[3]);
  }
}

// 3x3 "same" convolution, zero padding.  A block = 4 warps x 16 pixels of one
// row.  MODE 0: ReLU -> bf16 (16 ch); 1: linear, channel 0 -> fp32;
// 2: multiply by (act > 0) (ReLU derivative of the layer input) -> bf16.
template <int NT, int MODE>
__global__ void __launch_bounds__(128) k_conv(int H, int W, const uint16_t* __restrict__ x,
                                              const uint32_t* __restrict__ frag,
                                              const uint16_t* __restrict__ act, void* out) {
  __shared__ uint32_t sf[9 * NT * 64];
  for (int i = threadIdx.x; i < 9 * NT * 64; i += 128) sf[i] = frag[i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int x0 = (blockIdx.x * 4 + warp) * 16;
  const int y = blockIdx.y;
  const long long img = (long long)blockIdx.z * H * W;
  if (x0 >= W) return;
  float acc[NT][4];
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0f;
#pragma unroll
  for (int tap = 0; tap < 9; ++tap) {
    const int yy = y + tap / 3 - 1, dx = tap % 3 - 1;
    const bool rok = yy >= 0 && yy < H;
    const int xa = x0 + g + dx, xb = xa + 8;
    const uint16_t* row = x + (img + (long long)yy * W) * kC;
    auto ld = [&](int xx, int ch) -> uint32_t {
      return (rok && xx >= 0 && xx < W) ? __ldg(reinterpret_cast<const uint32_t*>(row + xx * kC + ch))
                                        : 0u;
    };
    const uint32_t a0 = ld(xa, 2 * t), a1 = ld(xb, 2 * t), a2 = ld(xa, 2 * t + 8),
                   a3 = ld(xb, 2 * t + 8);
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const uint32_t* b = sf + ((tap * NT + nt) * 32 + lane) * 2;
      mma_bf16(acc[nt], a0, a1, a2, a3, b[0], b[1]);
    }
  }
  const int pa = x0 + g, pb = pa + 8;
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    const int px = half ? pb : pa;
    if (px >= W) continue;
    const long long pix = img + (long long)y * W + px;
    if (MODE == 1) {
      if (t == 0) reinterpret_cast<float*>(out)[pix] = acc[0][2 * half];
      continue;
    }
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const int co = nt * 8 + 2 * t;
      float v0 = acc[nt][2 * half], v1 = acc[nt][2 * half + 1];
      if (MODE == 0) {
        v0 = fmaxf(v0, 0.0f);
        v1 = fmaxf(v1, 0.0f);
      } else {
        const uint32_t a = *reinterpret_cast<const uint32_t*>(act + pix * kC + co);
        if (!(bf((uint16_t)(a & 0xffffu)) > 0.0f)) v0 = 0.0f;
        if (!(bf((uint16_t)(a >> 16)) > 0.0f)) v1 = 0.0f;
      }
      reinterpret_cast<uint32_t*>(out)[(pix * kC + co) / 2] = pack2(v0, v1);
    }
  }
}

// Weight gradient partials: block b sums k-steps [b*ks_per, (b+1)*ks_per) of 16
// pixels (W % 16 == 0, so a k-step is 16 pixels of one row).
// D[m = ci][n = co] += A[ci][p] B[p][co],  A[ci][p] = X[p + tap, ci],  B = dY.
template <int NT>
__global__ void __launch_bounds__(128) k_wgrad(int H, int W, long long nks, int ks_per,
                                               const uint16_t* __restrict__ x,
                                               const uint16_t* __restrict__ dy,
                                               float* __restrict__ partial) {
  constexpr int NO = 8 * NT;
  __shared__ float red[4][9 * 16 * NO];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float acc[9][NT][4];
#pragma unroll
  for (int k = 0; k < 9; ++k)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) acc[k][nt][0] = acc[k][nt][1] = acc[k][nt][2] = acc[k][nt][3] = 0.0f;
  const int wpr = W / 16;  // k-steps per row
  const long long ks0 = (long long)blockIdx.x * ks_per;
  const long long ks1 = min(nks, ks0 + ks_per);
  for (long long ks = ks0 + warp; ks < ks1; ks += 4) {
    const long long rowid = ks / wpr;  // n*H + y
    const int x0 = (int)(ks - rowid * wpr) * 16;
    const int y = (int)(rowid % H);
    const long long img = (rowid / H) * (long long)H * W;
    const uint16_t* dyr = dy + (img + (long long)y * W + x0) * kC;
    uint32_t b[NT][2];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const int co = nt * 8 + g;
      const int k0 = 2 * t;
      b[nt][0] = (uint32_t)dyr[k0 * kC + co] | ((uint32_t)dyr[(k0 + 1) * kC + co] << 16);
      b[nt][1] = (uint32_t)dyr[(k0 + 8) * kC + co] | ((uint32_t)dyr[(k0 + 9) * kC + co] << 16);
    }
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int yy = y + tap / 3 - 1, dx = tap % 3 - 1;
      const bool rok = yy >= 0 && yy < H;
      const uint16_t* xr = x + (img + (long long)yy * W) * kC;
      auto xv = [&](int j, int ci) -> uint32_t {  // X at pixel x0+j shifted by the tap
        const int xx = x0 + j + dx;
        return (rok && xx >= 0 && xx < W) ? (uint32_t)xr[xx * kC + ci] : 0u;
      };
      const int j0 = 2 * t;
      const uint32_t a0 = xv(j0, g) | (xv(j0 + 1, g) << 16);
      const uint32_t a1 = xv(j0, g + 8) | (xv(j0 + 1, g + 8) << 16);
      const uint32_t a2 = xv(j0 + 8, g) | (xv(j0 + 9, g) << 16);
      const uint32_t a3 = xv(j0 + 8, g + 8) | (xv(j0 + 9, g + 8) << 16);
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) mma_bf16(acc[tap][nt], a0, a1, a2, a3, b[nt][0], b[nt][1]);
    }
  }
  // D fragment: (row g / g+8 = ci, cols 2t, 2t+1 = co within the n-tile)
#pragma unroll
  for (int tap = 0; tap < 9; ++tap)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int ci = g + (e >> 1) * 8, co = nt * 8 + 2 * t + (e & 1);
        red[warp][(tap * 16 + ci) * NO + co] = acc[tap][nt][e];
      }
  __syncthreads();
  for (int i = threadIdx.x; i < 9 * 16 * NO; i += 128)
    partial[(long long)blockIdx.x * 9 * 16 * NO + i] =
        ((red[0][i] + red[1][i]) + red[2][i]) + red[3][i];
}

// Sum the partials in block order into the logical gradient layout.
__global__ void k_wgrad_reduce(int nblk, int NO, const float* __restrict__ partial, int ci_n,
                               int co_n, float* __restrict__ grad) {
  const int n = 9 * ci_n * co_n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int co = i % co_n, ci = (i / co_n) % ci_n, tap = i / (co_n * ci_n);
    const int j = (tap * 16 + ci) * NO + co;
    float s = 0.0f;
    for (int b = 0; b < nblk; ++b) s += partial[(long long)b * 9 * 16 * NO + j];
    grad[i] = s;
  }
}

// Masked mean-square loss: r = m (y - t); dY = 2 r / count (bf16, channel 0);
// per-block partial sums of r^2 (fixed-order, deterministic).
__global__ void k_loss(long long npix, const float* __restrict__ y, const float* __restrict__ tgt,
                       const float* __restrict__ mask, float inv_count, uint16_t* __restrict__ dy,
                       float* __restrict__ part) {
  __shared__ float s[256];
  float acc = 0.0f;
  for (long long p = blockIdx.x * 256LL + threadIdx.x; p < npix; p += gridDim.x * 256LL) {
    const float r = (mask ? mask[p] : 1.0f) * (y[p] - tgt[p]);
    acc += r * r;
    uint32_t* d = reinterpret_cast<uint32_t*>(dy + p * kC);
    d[0] = pack2(2.0f * r * inv_count, 0.0f);
#pragma unroll
    for (int k = 1; k < kC / 2; ++k) d[k] = 0u;
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

__global__ void k_sum(int n, const float* __restrict__ a, float scale, float* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    float s = 0.0f;
    for (int i = 0; i < n; ++i) s += a[i];
    *out = s * scale;
  }
}

__global__ void k_adam(int n, float* __restrict__ p, const float* __restrict__ g,
                       float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// Window origin of image k: off[k] when an offset table is given, else k*stride.
__device__ __forceinline__ long long img_base(const long long* off, long long stride, int k) {
  return off ? off[k] : (long long)k * stride;
}

// features of the (h, w) windows of fields with row pitch ld, times scale[k]:
// (u, u_prev, c2 u, c2^2 u, s_next, s_prev) where s_* is the value injected at
// a source cell of the window in this / the previous step (n_src sources per
// window at src[2(k n_src + q)], values inj_next / inj_prev[k n_src + q]).
__global__ void k_features(int H, int W, const float* __restrict__ u, const float* __restrict__ up,
                           const float* __restrict__ c2, long long ld, const long long* u_off,
                           long long u_stride, const long long* c_off, long long c_stride,
                           const float* __restrict__ scale, int n_src, const int* __restrict__ src,
                           const float* __restrict__ inj_next, const float* __restrict__ inj_prev,
                           uint16_t* __restrict__ feat) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, k = blockIdx.z;
  if (x >= W) return;
  const long long q = img_base(u_off, u_stride, k) + (long long)y * ld + x;
  const float s = scale ? scale[k] : 1.0f;
  const float a = __fmul_rn(u[q], s), b = __fmul_rn(up[q], s);
  const float c = c2[img_base(c_off, c_stride, k) + (long long)y * ld + x];
  const float ca = __fmul_rn(c, a);
  float sn = 0.0f, sp = 0.0f;
  for (int j = 0; j < n_src; ++j) {
    const int i = k * n_src + j;
    if (src[2 * i] == x && src[2 * i + 1] == y) {
      if (inj_next) sn = __fadd_rn(sn, __fmul_rn(inj_next[i], s));
      if (inj_prev) sp = __fadd_rn(sp, __fmul_rn(inj_prev[i], s));
    }
  }
  uint32_t* f = reinterpret_cast<uint32_t*>(feat + (((long long)k * H + y) * W + x) * kC);
  f[0] = pack2(a, b);
  f[1] = pack2(ca, __fmul_rn(c, ca));
  f[2] = pack2(sn, sp);
#pragma unroll
  for (int j = 3; j < kC / 2; ++j) f[j] = 0u;
}

// Training target: the part of u^{n+1} the coarse step misses,
//   target = s * (u_next - (scalar step(u, u_prev) + injection)),
// with the scalar step's exact arithmetic (scalar2d.jl:29-53, as the solver
// kernel); mask = 1 where the stencil and the network's 7x7 receptive field
// fit the window and outside a square of half-width src_r around the source,
// else 0 (and target 0).
struct D2C {
  float two_c0;
  float d[5];
};
template <int N>
__global__ void k_target(int H, int W, D2C cf, const float* __restrict__ u,
                         const float* __restrict__ up, const float* __restrict__ un,
                         const float* __restrict__ c2, long long ld, const long long* u_off,
                         long long u_stride, const long long* c_off, long long c_stride,
                         const float* __restrict__ scale, const int* __restrict__ src,
                         const float* __restrict__ inj, int src_r, float* __restrict__ tgt,
                         float* __restrict__ mask) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, k = blockIdx.z;
  if (x >= W) return;
  const long long o = ((long long)k * H + y) * W + x;
  const int sx = src ? src[2 * k] : -1000000, sz = src ? src[2 * k + 1] : -1000000;
  const bool near_src = abs(x - sx) <= src_r && abs(y - sz) <= src_r;
  constexpr int E = N > 3 ? N : 3;  // the stencil and the network's receptive field fit
  if (x < E || x >= W - E || y < E || y >= H - E || near_src) {
    tgt[o] = 0.0f;
    if (mask) mask[o] = 0.0f;
    return;
  }
  const long long q = img_base(u_off, u_stride, k) + (long long)y * ld + x;
  const float uc = u[q];
  float lap = __fmul_rn(cf.two_c0, uc);
#pragma unroll
  for (int l = 1; l <= N; ++l) {
    const float nb = __fadd_rn(__fadd_rn(__fadd_rn(u[q + l], u[q - l]), u[q + l * ld]), u[q - l * ld]);
    lap = __fmaf_rn(cf.d[l - 1], nb, lap);
  }
  const float c = c2[img_base(c_off, c_stride, k) + (long long)y * ld + x];
  float nxt = __fmaf_rn(c, lap, __fsub_rn(__fmul_rn(2.0f, uc), up[q]));
  if (x == sx && y == sz && inj) nxt = __fadd_rn(nxt, inj[k]);
  const float s = scale ? scale[k] : 1.0f;
  tgt[o] = __fmul_rn(__fsub_rn(un[q], nxt), s);
  if (mask) mask[o] = 1.0f;
}

struct Bufs {
  uint32_t* frag;
  uint16_t *h1, *h2, *d3, *dh2, *dh1;
  float *y, *part, *lpart;
};

int plan_bufs(fomo_ctx* ctx, long long npix, int nblk, int nlb, Bufs& b) {
  Arena ar;
  const size_t o_f = ar.take<uint32_t>(kNFrag);
  const size_t o_h1 = ar.take<uint16_t>(npix * kC), o_h2 = ar.take<uint16_t>(npix * kC);
  const size_t o_d3 = ar.take<uint16_t>(npix * kC), o_dh2 = ar.take<uint16_t>(npix * kC);
  const size_t o_dh1 = ar.take<uint16_t>(npix * kC);
  const size_t o_y = ar.take<float>(npix);
  const size_t o_p = ar.take<float>((size_t)std::max(nblk, 1) * 9 * 16 * 16);
  const size_t o_l = ar.take<float>(std::max(nlb, 1));
  if (int rc = ensure_workspace(ctx, ar.off)) return rc;
  b.frag = ws_ptr<uint32_t>(ctx, o_f);
  b.h1 = ws_ptr<uint16_t>(ctx, o_h1);
  b.h2 = ws_ptr<uint16_t>(ctx, o_h2);
  b.d3 = ws_ptr<uint16_t>(ctx, o_d3);
  b.dh2 = ws_ptr<uint16_t>(ctx, o_dh2);
  b.dh1 = ws_ptr<uint16_t>(ctx, o_dh1);
  b.y = ws_ptr<float>(ctx, o_y);
  b.part = ws_ptr<float>(ctx, o_p);
  b.lpart = ws_ptr<float>(ctx, o_l);
  return FOMO_OK;
}

cudaError_t forward(cudaStream_t st, int n, int h, int w, const uint16_t* feat, const float* params,
                    const Bufs& b, float* y, bool pack = true) {
  if (pack) k_pack<<<1, 256, 0, st>>>(params, b.frag);
  const dim3 grid((w + 63) / 64, h, n);
  k_conv<2, 0><<<grid, 128, 0, st>>>(h, w, feat, b.frag + kOffF1, nullptr, b.h1);
  k_conv<2, 0><<<grid, 128, 0, st>>>(h, w, b.h1, b.frag + kOffF2, nullptr, b.h2);
  k_conv<1, 1><<<grid, 128, 0, st>>>(h, w, b.h2, b.frag + kOffF3, nullptr, y);
  return cudaGetLastError();
}

int check_dims(fomo_ctx* ctx, int n, int h, int w, bool grad) {
  if (n < 1 || h < 1 || w < 1) return fail(ctx, FOMO_EARG, "corrector: empty batch");
  if (grad && (w % 16)) return fail(ctx, FOMO_EARG, "corrector gradients need width % 16 == 0");
  if ((long long)n * h * w > (1LL << 31)) return fail(ctx, FOMO_EARG, "corrector batch too large");
  return FOMO_OK;
}

}  // namespace

// Device-side helpers used by the corrected coarse solver.
cudaError_t corr_forward_device(cudaStream_t st, int h, int w, const float* u, const float* up,
                                const float* c2, long long ld, int n_src, const int* src,
                                const float* inj_next, const float* inj_prev,
                                const float* params, void* scratch, float* y, bool pack);
size_t corr_scratch_bytes(long long npix);

size_t corr_scratch_bytes(long long npix) {
  return 4 * (size_t)kNFrag + 3 * (size_t)npix * kC * 2 + 64 * 4;
}

cudaError_t corr_forward_device(cudaStream_t st, int h, int w, const float* u, const float* up,
                                const float* c2, long long ld, int n_src, const int* src,
                                const float* inj_next, const float* inj_prev,
                                const float* params, void* scratch, float* y, bool pack) {
  const long long npix = (long long)h * w;
  Bufs b{};
  char* s = static_cast<char*>(scratch);
  b.frag = reinterpret_cast<uint32_t*>(s);
  uint16_t* feat = reinterpret_cast<uint16_t*>(s + 4 * (size_t)kNFrag);
  b.h1 = feat + npix * kC;
  b.h2 = b.h1 + npix * kC;
  k_features<<<dim3((w + 127) / 128, h, 1), 128, 0, st>>>(
      h, w, u, up, c2, ld, nullptr, 0, nullptr, 0, nullptr, n_src, src, inj_next, inj_prev, feat);
  return forward(st, 1, h, w, feat, params, b, y, pack);
}

}  // namespace fomo

using namespace fomo;

extern "C" {

int fomo_corr_param_count(void) { return kNParam; }

int fomo_corr_features(fomo_ctx* ctx, int32_t n, int32_t h, int32_t w, const float* u,
                       const float* u_prev, const float* c2, int64_t ld, const int64_t* u_off,
                       int64_t u_stride, const int64_t* c2_off, int64_t c2_stride,
                       const float* scale, int32_t n_src, const int32_t* src,
                       const float* inj_next, const float* inj_prev, uint16_t* feat) {
  if (!ctx) return FOMO_EARG;
  if (int rc = check_dims(ctx, n, h, w, false)) return rc;
  if (!u || !u_prev || !c2 || !feat || ld < w || n_src < 0 || (n_src > 0 && !src))
    return fail(ctx, FOMO_EARG, "corrector features: bad arguments");
  k_features<<<dim3((w + 127) / 128, h, n), 128, 0, ctx->stream>>>(
      h, w, u, u_prev, c2, ld, reinterpret_cast<const long long*>(u_off), u_stride,
      reinterpret_cast<const long long*>(c2_off), c2_stride, scale, n_src, src, inj_next,
      inj_prev, feat);
  FOMO_CU(ctx, cudaGetLastError());
  return FOMO_OK;
}

int fomo_corr_target(fomo_ctx* ctx, int32_t n, int32_t h, int32_t w, int32_t fd_order,
                     const float* u, const float* u_prev, const float* u_next, const float* c2,
                     int64_t ld, const int64_t* u_off, int64_t u_stride, const int64_t* c2_off,
                     int64_t c2_stride, const float* scale, const int32_t* src, const float* inj,
                     int32_t src_r, float* target, float* mask) {
  if (!ctx) return FOMO_EARG;
  if (int rc = check_dims(ctx, n, h, w, false)) return rc;
  const int N = order_to_N(fd_order);
  if (N < 0) return fail(ctx, FOMO_EARG, "Unsupported FD order: " + std::to_string(fd_order));
  if (!u || !u_prev || !u_next || !c2 || !target || ld < w)
    return fail(ctx, FOMO_EARG, "corrector target: bad arguments");
  D2C cf;
  cf.two_c0 = 2.0f * kD2C0[N];
  for (int l = 0; l < 5; ++l) cf.d[l] = kD2[N][l];
  const dim3 grid((w + 127) / 128, h, n);
  const long long* uo = reinterpret_cast<const long long*>(u_off);
  const long long* co = reinterpret_cast<const long long*>(c2_off);
#define FOMO_TGT(NN)                                                                          \
  case NN:                                                                                    \
    k_target<NN><<<grid, 128, 0, ctx->stream>>>(h, w, cf, u, u_prev, u_next, c2, ld, uo,       \
                                                u_stride, co, c2_stride, scale, src, inj, src_r, \
                                                target, mask);                                 \
    break;
  switch (N) { FOMO_TGT(1) FOMO_TGT(2) FOMO_TGT(3) FOMO_TGT(4) FOMO_TGT(5) }
#undef FOMO_TGT
  FOMO_CU(ctx, cudaGetLastError());
  return FOMO_OK;
}

int fomo_corr_forward(fomo_ctx* ctx, int32_t n, int32_t h, int32_t w, const uint16_t* feat,
                      const float* params, float* y) {
  if (!ctx) return FOMO_EARG;
  if (int rc = check_dims(ctx, n, h, w, false)) return rc;
  if (!feat || !params || !y) return fail(ctx, FOMO_EARG, "corrector forward: null pointer");
  Bufs b{};
  if (int rc = plan_bufs(ctx, (long long)n * h * w, 1, 1, b)) return rc;
  FOMO_CU(ctx, forward(ctx->stream, n, h, w, feat, params, b, y));
  return FOMO_OK;
}

int fomo_corr_gradients(fomo_ctx* ctx, int32_t n, int32_t h, int32_t w, const uint16_t* feat,
                        const float* target, const float* mask, const float* params, float* grad,
                        float* loss, float* y_out) {
  if (!ctx) return FOMO_EARG;
  if (int rc = check_dims(ctx, n, h, w, true)) return rc;
  if (!feat || !target || !params || !grad || !loss)
    return fail(ctx, FOMO_EARG, "corrector gradients: null pointer");
  cudaStream_t st = ctx->stream;
  const long long npix = (long long)n * h * w, nks = npix / 16;
  const int ks_per = 64;
  const int nblk = (int)((nks + ks_per - 1) / ks_per);
  const int nlb = (int)std::min<long long>(1024, (npix + 255) / 256);
  Bufs b{};
  if (int rc = plan_bufs(ctx, npix, nblk, nlb, b)) return rc;
  float* y = y_out ? y_out : b.y;
  FOMO_CU(ctx, forward(st, n, h, w, feat, params, b, y));
  // loss and dY3
  const float count = (float)npix;  // the loss is a mean over every pixel (mask zeros included)
  const dim3 grid((w + 63) / 64, h, n);
  k_loss<<<nlb, 256, 0, st>>>(npix, y, target, mask, 1.0f / count, b.d3, b.lpart);
  k_sum<<<1, 32, 0, st>>>(nlb, b.lpart, 1.0f / count, loss);
  // layer 3: dW3 = sum h2[p+tap] dY3[p];  dH2 = conv_t(dY3, W3) * (h2 > 0)
  k_wgrad<1><<<nblk, 128, 0, st>>>(h, w, nks, ks_per, b.h2, b.d3, b.part);
  k_wgrad_reduce<<<2, 128, 0, st>>>(nblk, 8, b.part, 16, 1, grad + kNW1 + kNW2);
  k_conv<2, 2><<<grid, 128, 0, st>>>(h, w, b.d3, b.frag + kOffT3, b.h2, b.dh2);
  // layer 2: dW2 = sum h1[p+tap] dPre2[p];  dH1 = conv_t(dPre2, W2) * (h1 > 0)
  k_wgrad<2><<<nblk, 128, 0, st>>>(h, w, nks, ks_per, b.h1, b.dh2, b.part);
  k_wgrad_reduce<<<18, 128, 0, st>>>(nblk, 16, b.part, 16, 16, grad + kNW1);
  k_conv<2, 2><<<grid, 128, 0, st>>>(h, w, b.dh2, b.frag + kOffT2, b.h1, b.dh1);
  // layer 1: dW1 = sum feat[p+tap] dPre1[p]
  k_wgrad<2><<<nblk, 128, 0, st>>>(h, w, nks, ks_per, feat, b.dh1, b.part);
  k_wgrad_reduce<<<5, 128, 0, st>>>(nblk, 16, b.part, kCin, 16, grad);
  FOMO_CU(ctx, cudaGetLastError());
  return FOMO_OK;
}

int fomo_corr_adam(fomo_ctx* ctx, int32_t count, float* params, const float* grad, float* m,
                   float* v, float lr, float beta1, float beta2, float eps, int32_t step) {
  if (!ctx) return FOMO_EARG;
  if (count < 1 || !params || !grad || !m || !v || step < 1)
    return fail(ctx, FOMO_EARG, "corrector adam: bad arguments");
  const float c1 = 1.0f - std::pow(beta1, (float)step), c2 = 1.0f - std::pow(beta2, (float)step);
  k_adam<<<(count + 255) / 256, 256, 0, ctx->stream>>>(count, params, grad, m, v, lr, beta1, beta2,
                                                      eps, c1, c2);
  FOMO_CU(ctx, cudaGetLastError());
  return FOMO_OK;
}

}  // extern "C"
