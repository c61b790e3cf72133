// fomo_internal.cuh -- shared internals of libfomo_b200 (sm_100a).
//
// Built with --fmad=false: the only fused multiply-adds are the explicit
// __fmaf_rn calls below, so every kernel rounds in exactly the sequence the
// CPU oracle restates (canonical arithmetic, see stencil helpers).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/fomo_b200.h"

struct fomo_ctx {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // snapshot copies that overlap the time loop
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  void* ws = nullptr;  // device workspace, grown on demand and reused
  size_t ws_bytes = 0;
  int* d_flag = nullptr;  // device status word (non-finite sentinel)
  std::string err;
};

namespace fomo {

// Record an error message on the context and return the code.
int fail(fomo_ctx* ctx, int code, const std::string& msg);
int cuda_fail(fomo_ctx* ctx, cudaError_t e, const char* where);

#define FOMO_CU(ctx, call)                                   \
  do {                                                       \
    cudaError_t _e = (call);                                 \
    if (_e != cudaSuccess) return fomo::cuda_fail(ctx, _e, #call); \
  } while (0)

// Bump allocator over the context workspace (256-byte aligned regions).
struct Arena {
  size_t off = 0;
  template <class T>
  size_t take(size_t count) {
    size_t o = off;
    off += (count * sizeof(T) + 255) & ~size_t(255);
    return o;
  }
};
int ensure_workspace(fomo_ctx* ctx, size_t bytes);
template <class T>
inline T* ws_ptr(fomo_ctx* ctx, size_t off) {
  return reinterpret_cast<T*>(static_cast<char*>(ctx->ws) + off);
}

// utils/FD_utils.jl:5-11 and utils/FD_centered.jl:27-41, as float32 values of
// the reference's Float64 literals.
extern const float kFD[6][5];
extern const float kD2C0[6];
extern const float kD2[6][5];

struct Coef {
  float a[5];
};

// Higdon parameters: q, qt, qxt (habc.jl:17-44, float32) and the weight ramp
// tables w(dist) for offsets 0 / 0.5 / 0.75 (vx / vz / tau,p,u).
struct HabcHost {
  int nbc;  // zone = pad - 1
  float q, qt, qxt;
  std::vector<float> wtab;  // 3 * (pad + 2)
  int wstride;
};
HabcHost make_habc(int pad, float v_ref, float dt, float dh);
// Cerjan sponge damping by distance to the padded edge, d = 0 .. nbc-1
// (boundary/sponge.jl:31-48): exp(-r^2), r = factor * (nbc - d) in float32, the
// exponential in double rounded once to float32.
std::vector<float> sponge_table(int nbc, float factor);

// In sponge mode nbc is the user's layer count and wtab the sponge_table.
struct HabcDev {
  float q, qt, qxt;
  int nbc;
  int wstride;
  const float* wtab;
};

// FP16 wavefield storage (elastic2d, mixed2d.cuh and the sweep's binary16
// form): cells within kFp16Band of the padded grid's edge stay FP32; stored
// velocities are scaled by kFp16Sv, stresses by kFp16St (powers of two).
constexpr int kFp16Band = 32;
constexpr float kFp16Sv = 4194304.0f;  // 2^22
constexpr float kFp16St = 1.0f;

// Padded 2D geometry (0-based x in [0,nx), z in [0,nz)).
struct Geo2 {
  int nx, nz;      // padded
  int ld;          // row pitch in elements (>= nx)
  int M;           // fd_order / 2
  int nbc;         // HABC zone = pad - 1
  long long plane; // ld * nz
};

__device__ __forceinline__ bool interior2(const Geo2& g, int x, int z) {
  return x >= g.M && x < g.nx - g.M && z >= g.M && z < g.nz - g.M;
}

// kernels_fused.jl:28-52: frame = 1<=x<=nx-2, 1<=z<=nz-2 within nbc of an edge.
// side: +1 -> neighbour at +1 (left/top band), -1 -> at -1 (right/bottom), 0 none.
__device__ __forceinline__ bool frame2(const Geo2& g, int x, int z, int& sx, int& sz,
                                       int& dist) {
  if (x < 1 || x > g.nx - 2 || z < 1 || z > g.nz - 2) return false;
  sx = x <= g.nbc ? 1 : (x >= g.nx - 1 - g.nbc ? -1 : 0);
  sz = z <= g.nbc ? 1 : (z >= g.nz - 1 - g.nbc ? -1 : 0);
  if (sx == 0 && sz == 0) return false;
  dist = min(min(x, g.nx - 1 - x), min(z, g.nz - 1 - z));
  return true;
}

__device__ __forceinline__ float habc_weight(const HabcDev& h, int kind, int dist) {
  return dist < h.wstride ? __ldg(h.wtab + kind * h.wstride + dist) : 1.0f;
}

// kernels_det.jl:22-57 side term:  -q*f[nb] - qt*fo[p] - qxt*fo[nb]
__device__ __forceinline__ float higdon_side(const HabcDev& h, float f_nb, float fo_p,
                                             float fo_nb) {
  float s = __fmul_rn(-h.q, f_nb);
  s = __fmaf_rn(-h.qt, fo_p, s);
  return __fmaf_rn(-h.qxt, fo_nb, s);
}
__device__ __forceinline__ float higdon_edge(float w, float fc, float s) {
  return __fmaf_rn(w, fc, __fmul_rn(__fsub_rn(1.0f, w), s));
}
__device__ __forceinline__ float higdon_corner(float w, float fc, float sx, float sz) {
  return __fmaf_rn(w, fc, __fmul_rn(__fmul_rn(__fsub_rn(1.0f, w), 0.5f), __fadd_rn(sx, sz)));
}

// Staggered derivative sums, accumulated l = 1..N with one fma per term.
//   dm: sum a_l (f[p+(l-1)s] - f[p-l s])    (backward-staggered)
//   dp: sum a_l (f[p+l s]   - f[p-(l-1)s])  (forward-staggered)
template <int N>
__device__ __forceinline__ float dm(const float* __restrict__ f, long long p, long long s,
                                    const Coef& c) {
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l)
    acc = __fmaf_rn(c.a[l - 1], __fsub_rn(__ldg(f + p + (l - 1) * s), __ldg(f + p - l * s)), acc);
  return acc;
}
template <int N>
__device__ __forceinline__ float dp(const float* __restrict__ f, long long p, long long s,
                                    const Coef& c) {
  float acc = 0.0f;
#pragma unroll
  for (int l = 1; l <= N; ++l)
    acc = __fmaf_rn(c.a[l - 1], __fsub_rn(__ldg(f + p + l * s), __ldg(f + p - (l - 1) * s)), acc);
  return acc;
}

// Host side of the cell tags (CellTags, solver2d_kernels.cuh): one entry per
// distinct source or receiver cell (linear pitched index within a shot's
// plane), listing the source indices s * n_src + q (ascending) then the
// receiver indices at that cell.  src_lin holds all shots' sources.
struct CellTagHost {
  std::vector<int32_t> lin;  // entry -> cell
  std::vector<int4> ent;     // sources list[x, y), receivers list[z, w)
  std::vector<int32_t> list;
};
inline CellTagHost make_cell_tags(const int32_t* src_lin, int n_src, const int32_t* rec_lin,
                                  int n_rec) {
  CellTagHost t;
  std::map<int32_t, int> at;
  std::vector<std::vector<int32_t>> srcs, recs;
  auto entry = [&](int32_t lin) {
    auto it = at.find(lin);
    if (it != at.end()) return it->second;
    const int e = (int)t.lin.size();
    at[lin] = e;
    t.lin.push_back(lin);
    srcs.emplace_back();
    recs.emplace_back();
    return e;
  };
  for (int k = 0; k < n_src; ++k) srcs[entry(src_lin[k])].push_back(k);
  for (int k = 0; k < n_rec; ++k) recs[entry(rec_lin[k])].push_back(k);
  t.ent.resize(t.lin.size());
  for (size_t e = 0; e < t.lin.size(); ++e) {
    t.ent[e].x = (int)t.list.size();
    t.list.insert(t.list.end(), srcs[e].begin(), srcs[e].end());
    t.ent[e].y = t.ent[e].z = (int)t.list.size();
    t.list.insert(t.list.end(), recs[e].begin(), recs[e].end());
    t.ent[e].w = (int)t.list.size();
  }
  return t;
}

// Host helpers
inline int order_to_N(int fd_order) {
  if (fd_order < 2 || fd_order > 10 || (fd_order & 1)) return -1;
  return fd_order / 2;
}
inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

// Device medium preparation (medium.cu).
cudaError_t launch_medium2d(cudaStream_t st, int kind, int nx, int nz, int pad, int ld, float dtdh,
                            const float* vp, const float* vs, const float* rho, float* out0,
                            float* out1, float* out2, float* out3, float* out4);

}  // namespace fomo
