// medium.cu -- device-side model preparation (one pass, no padded temporaries).
//
// The padded value at (x, z) is the raw model at the clamped interior index,
// which is what utils/pad_array.jl:8-22 produces (x strips, then full rows).
// Everything is IEEE float32 without contraction, matching the Julia host
// arithmetic bit for bit.
#include "fomo_internal.cuh"

namespace fomo {
namespace {

struct Raw2 {
  const float* a;
  int nx, nz, pad;
  __device__ __forceinline__ float at(int x, int z) const {
    int ii = min(max(x - pad, 0), nx - 1);
    int jj = min(max(z - pad, 0), nz - 1);
    return __ldg(a + (long long)jj * nx + ii);
  }
};

// utils/pad_array.jl:30-67 vacuum rules
__device__ __forceinline__ float harm2(float r1, float r2) {
  if (r1 == 0.0f && r2 == 0.0f) return 0.0f;
  if (r1 == 0.0f) return __fdiv_rn(2.0f, r2);
  if (r2 == 0.0f) return __fdiv_rn(2.0f, r1);
  return __fdiv_rn(2.0f, __fadd_rn(r1, r2));
}

// elastic2d/medium.jl:59-69
__device__ __forceinline__ float harm4(float m1, float m2, float m3, float m4) {
  if (m1 == 0.0f || m2 == 0.0f || m3 == 0.0f || m4 == 0.0f) return 0.0f;
  float s = __fadd_rn(__fadd_rn(__fadd_rn(__frcp_rn(m1), __frcp_rn(m2)), __frcp_rn(m3)),
                      __frcp_rn(m4));
  return __fdiv_rn(4.0f, s);
}

__device__ __forceinline__ float mu_at(const Raw2& rho, const Raw2& vs, int x, int z) {
  float v = vs.at(x, z);
  return __fmul_rn(rho.at(x, z), __fmul_rn(v, v));
}

// kind 0 elastic: out0..4 = bx, bz, lam, lam2mu, mu_txz
// kind 1 acoustic: out0..2 = bx, bz, kappa
// kind 2 scalar: out0 = c2 = (vp * dt/dh)^2
__global__ void k_medium2d(int kind, int nx, int nz, int pad, int ld, float dtdh, Raw2 vp, Raw2 vs,
                           Raw2 rho, float* __restrict__ o0, float* __restrict__ o1,
                           float* __restrict__ o2, float* __restrict__ o3,
                           float* __restrict__ o4) {
  int nxp = nx + 2 * pad, nzp = nz + 2 * pad;
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int z = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= nxp || z >= nzp) return;
  long long p = (long long)z * ld + x;
  if (kind == 2) {
    float t = __fmul_rn(vp.at(x, z), dtdh);
    o0[p] = __fmul_rn(t, t);
    return;
  }
  // buoyancy: bx row 0 copies row 1; bz last column copies the one before
  int xb = max(x, 1);
  o0[p] = harm2(rho.at(xb - 1, z), rho.at(xb, z));
  int zb = min(z, nzp - 2);
  o1[p] = harm2(rho.at(x, zb), rho.at(x, zb + 1));
  float r = rho.at(x, z), v = vp.at(x, z);
  float rv2 = __fmul_rn(r, __fmul_rn(v, v));
  if (kind == 1) {
    o2[p] = rv2;  // kappa = rho * vp^2 (acoustic2d/medium.jl:44)
    return;
  }
  float mu = mu_at(rho, vs, x, z);
  float two_mu = __fmul_rn(2.0f, mu);
  float lam = __fsub_rn(rv2, two_mu);
  o2[p] = lam;
  o3[p] = __fadd_rn(lam, two_mu);
  // mu_txz: row 0 copies row 1, then the last column copies the one before
  int xm = max(x, 1), zm = min(z, nzp - 2);
  o4[p] = harm4(mu_at(rho, vs, xm - 1, zm), mu_at(rho, vs, xm, zm), mu_at(rho, vs, xm - 1, zm + 1),
                mu_at(rho, vs, xm, zm + 1));
}

}  // namespace

cudaError_t launch_medium2d(cudaStream_t st, int kind, int nx, int nz, int pad, int ld, float dtdh,
                            const float* vp, const float* vs, const float* rho, float* out0,
                            float* out1, float* out2, float* out3, float* out4) {
  int nxp = nx + 2 * pad, nzp = nz + 2 * pad;
  dim3 b(32, 8), gr(cdiv(nxp, 32), cdiv(nzp, 8));
  Raw2 a{vp, nx, nz, pad}, s{vs ? vs : vp, nx, nz, pad}, r{rho ? rho : vp, nx, nz, pad};
  k_medium2d<<<gr, b, 0, st>>>(kind, nx, nz, pad, ld, dtdh, a, s, r, out0, out1, out2, out3, out4);
  return cudaGetLastError();
}

}  // namespace fomo
