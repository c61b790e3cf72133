// fomo_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of Fomo.jl's staggered-grid time stepping (the checker for
// libfomo_b200, never shipped, never on the product path).  Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
//
// Templated on the arithmetic type: T=float is the FP32 oracle (same rounding
// sequence as the CUDA kernels, so GPU==oracle is expected bit-exact), T=double
// is the FP64 oracle of the same scheme used for error reporting.
//
// Parity pinning: the reference ships no golden vectors and Julia is absent
// here, so absolute seismogram values are pinned by the reference's own test
// properties (tests/test_oracle_pins.py): the HABC absorption calibration of
// test/verify_patch.jl:9-11 (1.245e-2 for zone=pad-1, 1.336e-2 for zone=nbc),
// exact mirror symmetry under causal shielding (verify_patch.jl:59-73),
// multi-source linearity (:97-104), and the scalar same-scheme CPU transcription
// (verify_scalar.jl:33-86) and det-HABC CPU reference (verify_det_graph.jl:59-94),
// which this file restates.
//
// Canonical arithmetic (shared with fomo.jl_b200/csrc/stencil.cuh).  The
// reference writes `acc += c*(a-b)` and `v += b*(dtx*X + dtz*Z)`; CUDA.jl's
// NVPTX backend contracts these into FMAs.  This restatement fixes one
// contraction explicitly:
//   acc = fma(c, a-b, acc)
//   vx  = fma(bx, fma(dtx, X, dtz*Z), vx)                (elastic velocity)
//   v   = fma(b*dtx, D, v)                               (acoustic velocity)
//   p   = fma(kappa, fma(X, dtx, Z*dtz), p)              (acoustic pressure)
//   ex = X*dtx; ez = Z*dtz; txx = txx + fma(l2m, ex, lam*ez)
//                           tzz = tzz + fma(lam, ex, l2m*ez)
//   txz = fma(mu_txz, fma(Xz, dtz, Zx*dtx), txz)
//   Higdon side term  s = fma(-qxt, fo[n], fma(-qt, fo[p], (-q)*f[n]))
//   edge   f' = fma(w, f, (1-w)*s);  corner f' = fma(w, f, ((1-w)*0.5)*(sx+sz))
// Host preparation (padding, buoyancy, Lame, HABC weights) is IEEE without
// contraction, exactly as the Julia host code computes it (this file must be
// compiled with -ffp-contract=off).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// utils/FD_utils.jl:5-11 (staggered coefficients, orders 2..10)
const float kFD[6][5] = {
    {0, 0, 0, 0, 0},
    {(float)1.0, 0, 0, 0, 0},
    {(float)1.125, (float)-0.041666667, 0, 0, 0},
    {(float)1.171875, (float)-0.065104167, (float)0.0046875, 0, 0},
    {(float)1.1962890625, (float)-0.079752604167, (float)0.0095703125, (float)-0.000697544643, 0},
    {(float)1.2115478515625, (float)-0.089721679687, (float)0.0138427734375,
     (float)-0.00176565987723, (float)0.0001186795166},
};
// utils/FD_centered.jl:27-41 (centered second derivative)
const float kD2C0[6] = {0, (float)-2.0, (float)(-5.0 / 2.0), (float)(-49.0 / 18.0), (float)(-205.0 / 72.0),
                        (float)(-5269.0 / 1800.0)};
const float kD2[6][5] = {
    {0, 0, 0, 0, 0},
    {(float)1.0, 0, 0, 0, 0},
    {(float)(4.0 / 3.0), (float)(-1.0 / 12.0), 0, 0, 0},
    {(float)(3.0 / 2.0), (float)(-3.0 / 20.0), (float)(1.0 / 90.0), 0, 0},
    {(float)(8.0 / 5.0), (float)(-1.0 / 5.0), (float)(8.0 / 315.0), (float)(-1.0 / 560.0), 0},
    {(float)(5.0 / 3.0), (float)(-5.0 / 21.0), (float)(5.0 / 126.0), (float)(-5.0 / 1008.0),
     (float)(1.0 / 3150.0)},
};

inline int order_to_N(int fd_order) {
  if (fd_order < 2 || fd_order > 10 || (fd_order & 1)) return -1;
  return fd_order / 2;
}

inline float fmaT(float a, float b, float c) { return std::fmaf(a, b, c); }
inline double fmaT(double a, double b, double c) { return std::fma(a, b, c); }

// ---------------------------------------------------------------------------
// Reduced-precision wavefield storage (no reference counterpart).  A stored
// value is the FP32 result rounded to nearest-even into IEEE binary16 (with
// subnormals, overflow to inf) or bfloat16; these restate those formats'
// published rounding rules bit by bit so the oracle does not depend on a
// compiler's half-precision support.
// ---------------------------------------------------------------------------
enum StoreKind { kStoreF32 = 0, kStoreF16 = 1, kStoreBF16 = 2 };

inline float bits_f(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
inline uint32_t f_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}

inline float round_fp16(float x) {
  const uint32_t u = f_bits(x), sign = u & 0x80000000u, a = u & 0x7fffffffu;
  if (a >= 0x7f800000u) return x;                              // inf, nan
  if (a >= 0x477ff000u) return bits_f(sign | 0x7f800000u);     // >= 65520 -> inf
  if (a >= 0x38800000u) {                                      // |x| >= 2^-14: 10-bit mantissa
    uint32_t r = (a + 0x0fffu + ((a >> 13) & 1u)) & ~0x1fffu;
    return bits_f(sign | r);
  }
  // subnormal binary16: multiples of 2^-24 (x * 2^24 is exact)
  const float k = std::nearbyint(std::fabs(x) * 16777216.0f);
  return bits_f(sign | f_bits(k * (1.0f / 16777216.0f)));
}

inline float round_bf16(float x) {
  uint32_t u = f_bits(x);
  if ((u & 0x7fffffffu) > 0x7f800000u) return x;  // nan
  u = (u + 0x7fffu + ((u >> 16) & 1u)) & 0xffff0000u;
  return bits_f(u);
}

inline float round_store(float x, int kind) {
  return kind == kStoreF16 ? round_fp16(x) : (kind == kStoreBF16 ? round_bf16(x) : x);
}
inline double round_store(double x, int) { return x; }

// Storage format and power-of-two scales of the stored velocity (sv) and
// stress (st) fields: stored v = sv * v, stored tau = st * tau.  The scales are
// folded into the coefficients (b * sv/st, lambda * st/sv, ...), so the FP32
// arithmetic on scaled values equals the unscaled arithmetic times a power of
// two; the scales only place the values inside the storage format's range.
// Cells closer than fp32_band to a grid edge keep FP32 storage (0: none).
struct StoreSpec {
  int kind = kStoreF32;
  float sv = 1.0f, st = 1.0f;
  int fp32_band = 0;
};

// 1-based (i,j) -> linear index of a column-major (x fastest) padded grid.
struct G2 {
  int nx, nz;
  inline size_t at(int i, int j) const { return (size_t)(i - 1) + (size_t)nx * (size_t)(j - 1); }
  size_t n() const { return (size_t)nx * (size_t)nz; }
};

// utils/pad_array.jl:8-22 -- edge replication (x strips first, then z strips
// over full rows, which equals clamped indexing).
template <class T>
std::vector<T> pad_array(const float* d, int nx, int nz, int pad) {
  G2 g{nx + 2 * pad, nz + 2 * pad};
  std::vector<T> r(g.n());
  for (int j = 1; j <= g.nz; ++j) {
    int jj = std::min(std::max(j - pad, 1), nz);
    for (int i = 1; i <= g.nx; ++i) {
      int ii = std::min(std::max(i - pad, 1), nx);
      r[g.at(i, j)] = (T)d[(size_t)(ii - 1) + (size_t)nx * (jj - 1)];
    }
  }
  return r;
}

// utils/pad_array.jl:30-67 -- harmonic buoyancy with vacuum rules.
template <class T>
inline T harm2(T r1, T r2) {
  if (r1 == T(0) && r2 == T(0)) return T(0);
  if (r1 == T(0)) return T(2) / r2;
  if (r2 == T(0)) return T(2) / r1;
  return T(2) / (r1 + r2);
}

template <class T>
void staggered_buoyancy(const G2& g, const std::vector<T>& rho, std::vector<T>& bx,
                        std::vector<T>& bz) {
  bx.assign(g.n(), T(0));
  bz.assign(g.n(), T(0));
  for (int j = 1; j <= g.nz; ++j)
    for (int i = 2; i <= g.nx; ++i) bx[g.at(i, j)] = harm2(rho[g.at(i - 1, j)], rho[g.at(i, j)]);
  for (int j = 1; j <= g.nz; ++j) bx[g.at(1, j)] = bx[g.at(2, j)];
  for (int j = 1; j <= g.nz - 1; ++j)
    for (int i = 1; i <= g.nx; ++i) bz[g.at(i, j)] = harm2(rho[g.at(i, j)], rho[g.at(i, j + 1)]);
  for (int i = 1; i <= g.nx; ++i) bz[g.at(i, g.nz)] = bz[g.at(i, g.nz - 1)];
}

// elastic2d/medium.jl:52-74 -- Lame parameters and 4-point harmonic mu at txz.
template <class T>
inline T harm4(T m1, T m2, T m3, T m4) {
  if (m1 == T(0) || m2 == T(0) || m3 == T(0) || m4 == T(0)) return T(0);
  return T(4) / (T(1) / m1 + T(1) / m2 + T(1) / m3 + T(1) / m4);
}

template <class T>
void elastic_params(const G2& g, const std::vector<T>& vp, const std::vector<T>& vs,
                    const std::vector<T>& rho, std::vector<T>& lam, std::vector<T>& lam2mu,
                    std::vector<T>& mu_txz) {
  size_t n = g.n();
  std::vector<T> mu(n);
  lam.resize(n);
  lam2mu.resize(n);
  for (size_t k = 0; k < n; ++k) {
    mu[k] = rho[k] * (vs[k] * vs[k]);
    lam[k] = rho[k] * (vp[k] * vp[k]) - T(2) * mu[k];
    lam2mu[k] = lam[k] + T(2) * mu[k];
  }
  mu_txz.assign(n, T(0));
  for (int j = 1; j <= g.nz - 1; ++j)
    for (int i = 2; i <= g.nx; ++i)
      mu_txz[g.at(i, j)] = harm4(mu[g.at(i - 1, j)], mu[g.at(i, j)], mu[g.at(i - 1, j + 1)],
                                 mu[g.at(i, j + 1)]);
  for (int j = 1; j <= g.nz; ++j) mu_txz[g.at(1, j)] = mu_txz[g.at(2, j)];
  for (int i = 1; i <= g.nx; ++i) mu_txz[g.at(i, g.nz)] = mu_txz[g.at(i, g.nz - 1)];
}

// boundary/habc/habc.jl:17-44 -- Higdon coefficients (in T) and weight ramps.
template <class T>
struct Habc {
  int nbc;  // = pad - 1, the zone width every loop uses
  T q, qt, qxt;
  // weight tables by distance-to-edge for offsets 0 (vx), 0.5 (vz), 0.75 (tau/p)
  std::vector<T> wtab[3];
};

template <class T>
Habc<T> init_habc(int pad, float v_ref, float dt, float dh) {
  Habc<T> h;
  h.nbc = pad - 1;
  T r = (T)v_ref * (T)dt / (T)dh;
  T b = (T)0.45f, beta = T(1);
  h.q = (b * (beta + r) - r) / ((beta + r) * (T(1) - b));
  h.qt = (b * (beta + r) - beta) / ((beta + r) * (T(1) - b));
  h.qxt = b / (b - T(1));
  const double offs[3] = {0.0, 0.5, 0.75};
  for (int k = 0; k < 3; ++k) {
    h.wtab[k].resize(pad + 2);
    for (int d = 0; d < pad + 2; ++d) {
      double w = ((double)d - offs[k]) / (double)(pad - 1);
      w = std::min(std::max(w, 0.0), 1.0);
      h.wtab[k][d] = (T)w;
    }
  }
  return h;
}

template <class T>
inline T habc_w(const Habc<T>& h, int kind, int dist) {
  const std::vector<T>& t = h.wtab[kind];
  return dist < (int)t.size() ? t[dist] : T(1);
}

// kernels_fused.jl:28-52 -- the frame: 2<=i<=nx-1, 2<=j<=nz-1 and within nbc+1
// of an edge.  Stored as a list (sides encoded) for the two-pass update.
struct FramePt {
  size_t idx;
  int i, j;
  int8_t sx, sz;  // -1 left/top neighbour is i+1/j+1 ... encoded: +1 => use +1 neighbour, -1 => -1 neighbour, 0 => none
  int dist;
};

std::vector<FramePt> frame_points(const G2& g, int nbc) {
  std::vector<FramePt> f;
  for (int j = 2; j <= g.nz - 1; ++j)
    for (int i = 2; i <= g.nx - 1; ++i) {
      bool L = i <= nbc + 1, R = i >= g.nx - nbc, T_ = j <= nbc + 1, B = j >= g.nz - nbc;
      if (!(L || R || T_ || B)) continue;
      FramePt p;
      p.idx = g.at(i, j);
      p.i = i;
      p.j = j;
      p.sx = L ? 1 : (R ? -1 : 0);
      p.sz = T_ ? 1 : (B ? -1 : 0);
      p.dist = std::min(std::min(i - 1, g.nx - i), std::min(j - 1, g.nz - j));
      f.push_back(p);
    }
  return f;
}

// kernels_det.jl:22-57 -- Higdon value from read-only pre-correction fields.
template <class T>
inline T higdon_side(T q, T qt, T qxt, T f_nb, T fo_p, T fo_nb) {
  T s = (-q) * f_nb;
  s = fmaT(-qt, fo_p, s);
  s = fmaT(-qxt, fo_nb, s);
  return s;
}

template <class T>
inline T habc_value(const G2& g, const Habc<T>& h, const FramePt& p, const T* f, const T* fo,
                    T w) {
  T fc = f[p.idx];
  T one_m_w = T(1) - w;
  if (p.sx != 0 && p.sz != 0) {
    size_t nbx = p.sx > 0 ? p.idx + 1 : p.idx - 1;
    size_t nbz = p.sz > 0 ? p.idx + g.nx : p.idx - g.nx;
    T sx = higdon_side(h.q, h.qt, h.qxt, f[nbx], fo[p.idx], fo[nbx]);
    T sz = higdon_side(h.q, h.qt, h.qxt, f[nbz], fo[p.idx], fo[nbz]);
    return fmaT(w, fc, (one_m_w * T(0.5)) * (sx + sz));
  } else if (p.sx != 0) {
    size_t nb = p.sx > 0 ? p.idx + 1 : p.idx - 1;
    T s = higdon_side(h.q, h.qt, h.qxt, f[nb], fo[p.idx], fo[nb]);
    return fmaT(w, fc, one_m_w * s);
  } else {
    size_t nb = p.sz > 0 ? p.idx + g.nx : p.idx - g.nx;
    T s = higdon_side(h.q, h.qt, h.qxt, f[nb], fo[p.idx], fo[nb]);
    return fmaT(w, fc, one_m_w * s);
  }
}

// kernels_det.jl:60-132 -- pass 1 into scratch, pass 2 write-back.
template <class T>
void habc_det(const G2& g, const Habc<T>& h, const std::vector<FramePt>& fr, int kind, T* f,
              const T* fo, std::vector<T>& scr) {
  scr.resize(fr.size());
  const long n = (long)fr.size();
#pragma omp parallel for schedule(static)
  for (long k = 0; k < n; ++k) scr[k] = habc_value(g, h, fr[k], f, fo, habc_w(h, kind, fr[k].dist));
#pragma omp parallel for schedule(static)
  for (long k = 0; k < n; ++k) f[fr[k].idx] = scr[k];
}

template <class T>
struct Coef {
  int N;
  T a[5];
};

template <class T>
Coef<T> coef(int fd_order) {
  Coef<T> c;
  c.N = order_to_N(fd_order);
  for (int l = 0; l < 5; ++l) c.a[l] = (T)kFD[c.N][l];
  return c;
}

// ---------------------------------------------------------------------------
// elastic2d: elastic2d/fused_kernels.jl:21-124 + loop order :200-240
// (batch: elastic2d/batch.jl:38-183, bit-identical per shot by construction)
// ---------------------------------------------------------------------------
template <class T>
struct ElasticState {
  std::vector<T> vx, vz, txx, tzz, txz, o1, o2, o3;
};

template <class T>
void elastic_vel(const G2& g, int M, const Coef<T>& c, T dtx, T dtz, const T* bx, const T* bz,
                 ElasticState<T>& s) {
  const size_t nx = g.nx;
#pragma omp parallel for schedule(static)
  for (int j = M + 1; j <= g.nz - M; ++j) {
    for (int i = M + 1; i <= g.nx - M; ++i) {
      size_t p = g.at(i, j);
      T dxx = 0, dxzz = 0, dxzx = 0, dzz = 0;
      for (int l = 1; l <= c.N; ++l) {
        T a = c.a[l - 1];
        dxx = fmaT(a, s.txx[p + (l - 1)] - s.txx[p - l], dxx);
        dxzz = fmaT(a, s.txz[p + (size_t)(l - 1) * nx] - s.txz[p - (size_t)l * nx], dxzz);
        dxzx = fmaT(a, s.txz[p + l] - s.txz[p - (l - 1)], dxzx);
        dzz = fmaT(a, s.tzz[p + (size_t)l * nx] - s.tzz[p - (size_t)(l - 1) * nx], dzz);
      }
      s.vx[p] = fmaT(bx[p], fmaT(dtx, dxx, dtz * dxzz), s.vx[p]);
      s.vz[p] = fmaT(bz[p], fmaT(dtx, dxzx, dtz * dzz), s.vz[p]);
    }
  }
}

template <class T>
void elastic_str(const G2& g, int M, const Coef<T>& c, T dtx, T dtz, const T* lam,
                 const T* lam2mu, const T* mutxz, ElasticState<T>& s) {
  const size_t nx = g.nx;
#pragma omp parallel for schedule(static)
  for (int j = M + 1; j <= g.nz - M; ++j) {
    for (int i = M + 1; i <= g.nx - M; ++i) {
      size_t p = g.at(i, j);
      T dvxdx = 0, dvzdz = 0, dvxdz = 0, dvzdx = 0;
      for (int l = 1; l <= c.N; ++l) {
        T a = c.a[l - 1];
        dvxdx = fmaT(a, s.vx[p + l] - s.vx[p - (l - 1)], dvxdx);
        dvzdz = fmaT(a, s.vz[p + (size_t)(l - 1) * nx] - s.vz[p - (size_t)l * nx], dvzdz);
        dvxdz = fmaT(a, s.vx[p + (size_t)l * nx] - s.vx[p - (size_t)(l - 1) * nx], dvxdz);
        dvzdx = fmaT(a, s.vz[p + (l - 1)] - s.vz[p - l], dvzdx);
      }
      T ex = dvxdx * dtx, ez = dvzdz * dtz;
      s.txx[p] = s.txx[p] + fmaT(lam2mu[p], ex, lam[p] * ez);
      s.tzz[p] = s.tzz[p] + fmaT(lam[p], ex, lam2mu[p] * ez);
      s.txz[p] = fmaT(mutxz[p], fmaT(dvxdz, dtz, dvzdx * dtx), s.txz[p]);
    }
  }
}

// ---------------------------------------------------------------------------
// acoustic2d: acoustic2d/fused_kernels.jl:27-114 + loop :166-197
// ---------------------------------------------------------------------------
template <class T>
struct AcousticState {
  std::vector<T> vx, vz, p, o1, o2, o3;
};

template <class T>
void acoustic_vel(const G2& g, int M, const Coef<T>& c, T dtx, T dtz, const T* bx, const T* bz,
                  AcousticState<T>& s) {
  const size_t nx = g.nx;
#pragma omp parallel for schedule(static)
  for (int j = M + 1; j <= g.nz - M; ++j) {
    for (int i = M + 1; i <= g.nx - M; ++i) {
      size_t p = g.at(i, j);
      T dpdx = 0, dpdz = 0;
      for (int l = 1; l <= c.N; ++l) {
        T a = c.a[l - 1];
        dpdx = fmaT(a, s.p[p + (l - 1)] - s.p[p - l], dpdx);
        dpdz = fmaT(a, s.p[p + (size_t)l * nx] - s.p[p - (size_t)(l - 1) * nx], dpdz);
      }
      s.vx[p] = fmaT(bx[p] * dtx, dpdx, s.vx[p]);
      s.vz[p] = fmaT(bz[p] * dtz, dpdz, s.vz[p]);
    }
  }
}

template <class T>
void acoustic_prs(const G2& g, int M, const Coef<T>& c, T dtx, T dtz, const T* kappa,
                  AcousticState<T>& s) {
  const size_t nx = g.nx;
#pragma omp parallel for schedule(static)
  for (int j = M + 1; j <= g.nz - M; ++j) {
    for (int i = M + 1; i <= g.nx - M; ++i) {
      size_t p = g.at(i, j);
      T dvxdx = 0, dvzdz = 0;
      for (int l = 1; l <= c.N; ++l) {
        T a = c.a[l - 1];
        dvxdx = fmaT(a, s.vx[p + l] - s.vx[p - (l - 1)], dvxdx);
        dvzdz = fmaT(a, s.vz[p + (size_t)(l - 1) * nx] - s.vz[p - (size_t)l * nx], dvzdz);
      }
      s.p[p] = fmaT(kappa[p], fmaT(dvxdx, dtx, dvzdz * dtz), s.p[p]);
    }
  }
}

// Cerjan sponge (boundary/sponge.jl:31-48): with d the distance in cells from a
// padded-grid cell to the nearest edge, damp(d) = exp(-r^2), r = factor * (nbc - d),
// for d < nbc (the user's nbc, not pad); damp = 1 elsewhere.  r and r^2 round to
// FP32 as in the reference; exp is taken in double and rounded once to FP32.
// The FP64 oracle uses the same FP32 table (the reference stores it as Float32).
std::vector<float> sponge_table(int nbc, float factor) {
  std::vector<float> t((size_t)std::max(nbc, 0));
  for (int d = 0; d < nbc; ++d) {
    const float r = factor * (float)(nbc - d);
    const float rr = r * r;
    t[(size_t)d] = (float)std::exp(-(double)rr);
  }
  return t;
}

// apply_sponge! (boundary/sponge.jl:55-78): field *= damp over the whole padded grid.
template <class T>
void apply_sponge(const G2& g, const std::vector<float>& damp, T* f) {
  const int nbc = (int)damp.size();
#pragma omp parallel for schedule(static)
  for (int j = 0; j < g.nz; ++j) {
    const int dz = std::min(j, g.nz - 1 - j);
    for (int i = 0; i < g.nx; ++i) {
      const int d = std::min(std::min(i, g.nx - 1 - i), dz);
      if (d < nbc) {
        const size_t q = (size_t)i + (size_t)g.nx * (size_t)j;
        f[q] = f[q] * (T)damp[(size_t)d];
      }
    }
  }
}

// Snapshot of the interior (unpadded) part of a padded field.
template <class T, class O>
void snap_interior(const G2& g, int pad, const T* f, O* out) {
  int nxi = g.nx - 2 * pad, nzi = g.nz - 2 * pad;
  for (int j = 1; j <= nzi; ++j)
    for (int i = 1; i <= nxi; ++i) out[(size_t)(i - 1) + (size_t)nxi * (j - 1)] = (O)f[g.at(i + pad, j + pad)];
}

template <class T>
int run_elastic2d(int nx, int nz, int ns, const float* vp, const float* vs, const float* rho,
                  float dh, float dt, int nt, int nbc, int fd_order, float v_ref, int n_src,
                  const int32_t* sx, const int32_t* sz, const float* wavelet, int n_rec,
                  const int32_t* rx, const int32_t* rz, T* seis_vx, T* seis_vz, int snap_interval,
                  T* snaps, T* final_fields, StoreSpec ss = StoreSpec(),
                  float sponge_factor = -1.0f) {
  int N = order_to_N(fd_order);
  if (N < 0) return -2;
  int M = N, pad = nbc + M;
  if (pad < 2) return -2;
  G2 g{nx + 2 * pad, nz + 2 * pad};
  std::vector<T> vpp = pad_array<T>(vp, nx, nz, pad), vsp = pad_array<T>(vs, nx, nz, pad),
                 rhop = pad_array<T>(rho, nx, nz, pad);
  std::vector<T> bx, bz, lam, lam2mu, mutxz;
  staggered_buoyancy(g, rhop, bx, bz);
  elastic_params(g, vpp, vsp, rhop, lam, lam2mu, mutxz);
  const int sk = ss.kind;
  const T sv = (T)ss.sv, st_ = (T)ss.st;
  if (ss.sv != 1.0f || ss.st != 1.0f) {
    const T rv = sv / st_, rs = st_ / sv;  // exact: powers of two
    for (auto& a : bx) a *= rv;
    for (auto& a : bz) a *= rv;
    for (auto& a : lam) a *= rs;
    for (auto& a : lam2mu) a *= rs;
    for (auto& a : mutxz) a *= rs;
  }
  const int sfmt = sk, zb = ss.fp32_band, zone_f32 = zb > 0;
  auto in_zone = [&](size_t q) {
    const int i = (int)(q % (size_t)g.nx), j = (int)(q / (size_t)g.nx);
    return std::min(std::min(i, g.nx - 1 - i), std::min(j, g.nz - 1 - j)) < zb;
  };
  auto round_all = [&](std::vector<T>& f) {
    if (sfmt == kStoreF32) return;
#pragma omp parallel for schedule(static)
    for (long q = 0; q < (long)f.size(); ++q)
      if (!zone_f32 || !in_zone((size_t)q)) f[q] = round_store(f[q], sfmt);
  };
  const bool sponge = sponge_factor >= 0.0f;  // boundary = :sponge (elastic2d.jl:83-87)
  if (sponge && sk != kStoreF32) return -2;
  const std::vector<float> damp = sponge ? sponge_table(nbc, sponge_factor) : std::vector<float>();
  Habc<T> h = init_habc<T>(pad, v_ref, dt, dh);
  std::vector<FramePt> fr = frame_points(g, h.nbc);
  Coef<T> c = coef<T>(fd_order);
  T dtx = (T)dt / (T)dh, dtz = dtx;
  int nsnap = snap_interval > 0 ? nt / snap_interval : 0;
  size_t ncell = g.n();
  size_t nint = (size_t)nx * nz;
  std::vector<T> scr;
  for (int s = 0; s < ns; ++s) {
    ElasticState<T> st;
    for (auto* v : {&st.vx, &st.vz, &st.txx, &st.tzz, &st.txz, &st.o1, &st.o2, &st.o3})
      v->assign(ncell, T(0));
    for (int it = 1; it <= nt; ++it) {
      if (sponge) {  // legacy loop, elastic2d.jl:180-195
        elastic_vel(g, M, c, dtx, dtz, bx.data(), bz.data(), st);
        apply_sponge(g, damp, st.vx.data());
        apply_sponge(g, damp, st.vz.data());
        elastic_str(g, M, c, dtx, dtz, lam.data(), lam2mu.data(), mutxz.data(), st);
        apply_sponge(g, damp, st.txx.data());
        apply_sponge(g, damp, st.tzz.data());
        apply_sponge(g, damp, st.txz.data());
      } else {
        st.o1 = st.vx;
        st.o2 = st.vz;
        elastic_vel(g, M, c, dtx, dtz, bx.data(), bz.data(), st);
        habc_det(g, h, fr, 0, st.vx.data(), st.o1.data(), scr);
        habc_det(g, h, fr, 1, st.vz.data(), st.o2.data(), scr);
        round_all(st.vx);  // stored v'' (the stress update reads the stored values)
        round_all(st.vz);
        st.o1 = st.txx;
        st.o2 = st.tzz;
        st.o3 = st.txz;
        elastic_str(g, M, c, dtx, dtz, lam.data(), lam2mu.data(), mutxz.data(), st);
        habc_det(g, h, fr, 2, st.txx.data(), st.o1.data(), scr);
        habc_det(g, h, fr, 2, st.tzz.data(), st.o2.data(), scr);
        habc_det(g, h, fr, 2, st.txz.data(), st.o3.data(), scr);
        round_all(st.txx);
        round_all(st.tzz);
        round_all(st.txz);
      }
      for (int q = 0; q < n_src; ++q) {  // batch_acq.jl:58-71, sequential in source order
        size_t p = g.at(sx[(size_t)s * n_src + q] + pad, sz[(size_t)s * n_src + q] + pad);
        T w = (T)wavelet[(size_t)q + (size_t)n_src * (it - 1)] * st_;
        const int k = (zone_f32 && in_zone(p)) ? kStoreF32 : sfmt;
        st.txx[p] = round_store(st.txx[p] + w, k);
        st.tzz[p] = round_store(st.tzz[p] + w, k);
      }
      for (int r = 0; r < n_rec; ++r) {  // batch_acq.jl:108-121
        size_t p = g.at(rx[r] + pad, rz[r] + pad);
        size_t o = (size_t)r + (size_t)n_rec * ((it - 1) + (size_t)nt * s);
        seis_vx[o] = st.vx[p] / sv;
        seis_vz[o] = st.vz[p] / sv;
      }
      if (snaps && snap_interval > 0 && it % snap_interval == 0) {
        int k = it / snap_interval - 1;
        snap_interior(g, pad, st.vz.data(), snaps + nint * ((size_t)k + (size_t)nsnap * s));
        if (sv != T(1))
          for (size_t q = 0; q < nint; ++q) snaps[nint * ((size_t)k + (size_t)nsnap * s) + q] /= sv;
      }
    }
    if (final_fields) {  // unscaled values of the stored fields
      T* o = final_fields + (size_t)s * 5 * ncell;
      const T sc[5] = {sv, sv, st_, st_, st_};
      const std::vector<T>* F[5] = {&st.vx, &st.vz, &st.txx, &st.tzz, &st.txz};
      for (int f = 0; f < 5; ++f)
        for (size_t q = 0; q < ncell; ++q) o[f * ncell + q] = (*F[f])[q] / sc[f];
    }
  }
  return 0;
}

template <class T>
int run_acoustic2d(int nx, int nz, int ns, const float* vp, const float* rho, float dh, float dt,
                   int nt, int nbc, int fd_order, float v_ref, int n_src, const int32_t* sx,
                   const int32_t* sz, const float* wavelet, int n_rec, const int32_t* rx,
                   const int32_t* rz, T* seis_p, T* seis_vx, T* seis_vz, int snap_interval,
                   T* snaps, T* final_fields, int zone_nbc_override,
                   float sponge_factor = -1.0f) {
  int N = order_to_N(fd_order);
  if (N < 0) return -2;
  int M = N, pad = nbc + M;
  if (pad < 2) return -2;
  G2 g{nx + 2 * pad, nz + 2 * pad};
  std::vector<T> vpp = pad_array<T>(vp, nx, nz, pad), rhop = pad_array<T>(rho, nx, nz, pad);
  std::vector<T> bx, bz, kappa(g.n());
  staggered_buoyancy(g, rhop, bx, bz);
  for (size_t k = 0; k < g.n(); ++k) kappa[k] = rhop[k] * (vpp[k] * vpp[k]);  // acoustic2d/medium.jl:44
  Habc<T> h = init_habc<T>(pad, v_ref, dt, dh);
  // zone_nbc_override > 0 restates the pre-v0.2 zone (= nbc) used by the
  // calibration in test/verify_patch.jl:9-11; 0 keeps the production zone pad-1.
  if (zone_nbc_override > 0) h.nbc = zone_nbc_override;
  const bool sponge = sponge_factor >= 0.0f;  // boundary = :sponge (acoustic2d.jl:84-87)
  const std::vector<float> damp = sponge ? sponge_table(nbc, sponge_factor) : std::vector<float>();
  std::vector<FramePt> fr = frame_points(g, h.nbc);
  Coef<T> c = coef<T>(fd_order);
  T dtx = (T)dt / (T)dh, dtz = dtx;
  int nsnap = snap_interval > 0 ? nt / snap_interval : 0;
  size_t ncell = g.n(), nint = (size_t)nx * nz;
  std::vector<T> scr;
  for (int s = 0; s < ns; ++s) {
    AcousticState<T> st;
    for (auto* v : {&st.vx, &st.vz, &st.p, &st.o1, &st.o2, &st.o3}) v->assign(ncell, T(0));
    for (int it = 1; it <= nt; ++it) {
      if (sponge) {  // legacy loop, acoustic2d.jl:213-227
        acoustic_vel(g, M, c, dtx, dtz, bx.data(), bz.data(), st);
        apply_sponge(g, damp, st.vx.data());
        apply_sponge(g, damp, st.vz.data());
        acoustic_prs(g, M, c, dtx, dtz, kappa.data(), st);
        apply_sponge(g, damp, st.p.data());
      } else {
        st.o1 = st.vx;
        st.o2 = st.vz;
        acoustic_vel(g, M, c, dtx, dtz, bx.data(), bz.data(), st);
        habc_det(g, h, fr, 0, st.vx.data(), st.o1.data(), scr);
        habc_det(g, h, fr, 1, st.vz.data(), st.o2.data(), scr);
        st.o3 = st.p;
        acoustic_prs(g, M, c, dtx, dtz, kappa.data(), st);
        habc_det(g, h, fr, 2, st.p.data(), st.o3.data(), scr);
      }
      for (int q = 0; q < n_src; ++q) {  // inject_source.jl:4-24
        size_t p = g.at(sx[(size_t)s * n_src + q] + pad, sz[(size_t)s * n_src + q] + pad);
        st.p[p] += (T)wavelet[(size_t)q + (size_t)n_src * (it - 1)];
      }
      for (int r = 0; r < n_rec; ++r) {  // acoustic2d/fused_kernels.jl:137-149
        size_t p = g.at(rx[r] + pad, rz[r] + pad);
        size_t o = (size_t)r + (size_t)n_rec * ((it - 1) + (size_t)nt * s);
        if (seis_p) seis_p[o] = st.p[p];
        if (seis_vx) seis_vx[o] = st.vx[p];
        if (seis_vz) seis_vz[o] = st.vz[p];
      }
      if (snaps && snap_interval > 0 && it % snap_interval == 0) {
        int k = it / snap_interval - 1;
        snap_interior(g, pad, st.p.data(), snaps + nint * ((size_t)k + (size_t)nsnap * s));
      }
    }
    if (final_fields) {
      T* o = final_fields + (size_t)s * 3 * ncell;
      std::copy(st.vx.begin(), st.vx.end(), o);
      std::copy(st.vz.begin(), st.vz.end(), o + ncell);
      std::copy(st.p.begin(), st.p.end(), o + 2 * ncell);
    }
  }
  return 0;
}

// ---------------------------------------------------------------------------
// scalar2d: scalar2d/scalar2d.jl:29-84 (leapfrog, carried pad ring, HABC with
// f_old = u^n); restates verify_scalar.jl:33-86 (cpu_scalar_step!).
// ---------------------------------------------------------------------------
template <class T>
int run_scalar2d(int nx, int nz, const float* vp, float dh, float dt, int nt, int nbc,
                 int fd_order, float v_ref, int n_src, const int32_t* sx, const int32_t* sz,
                 const float* wavelet, int n_rec, const int32_t* rx, const int32_t* rz, T* seis_u,
                 T* final_fields) {
  int N = order_to_N(fd_order);
  if (N < 0) return -2;
  int M = N, pad = nbc + M;
  if (pad < 2) return -2;
  G2 g{nx + 2 * pad, nz + 2 * pad};
  std::vector<T> c2 = pad_array<T>(vp, nx, nz, pad);
  T r = (T)dt / (T)dh;  // Float32(dt / dh)
  for (auto& v : c2) {
    T t = v * r;
    v = t * t;
  }
  Habc<T> h = init_habc<T>(pad, v_ref, dt, dh);
  std::vector<FramePt> fr = frame_points(g, h.nbc);
  T c0 = (T)kD2C0[N];
  T d2[5];
  for (int l = 0; l < 5; ++l) d2[l] = (T)kD2[N][l];
  T two_c0 = T(2) * c0;
  size_t ncell = g.n();
  const size_t snx = g.nx;
  std::vector<T> u_old(ncell, T(0)), u_cur(ncell, T(0)), u_nxt(ncell, T(0)), scr;
  for (int it = 1; it <= nt; ++it) {
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= g.nz; ++j) {
      for (int i = 1; i <= g.nx; ++i) {
        size_t p = g.at(i, j);
        T uc = u_cur[p], un = uc;
        if (i > M && i <= g.nx - M && j > M && j <= g.nz - M) {
          T lap = two_c0 * uc;
          for (int l = 1; l <= N; ++l) {
            T nb = ((u_cur[p + l] + u_cur[p - l]) + u_cur[p + (size_t)l * snx]) + u_cur[p - (size_t)l * snx];
            lap = fmaT(d2[l - 1], nb, lap);
          }
          un = fmaT(c2[p], lap, T(2) * uc - u_old[p]);
        }
        u_nxt[p] = un;
      }
    }
    habc_det(g, h, fr, 2, u_nxt.data(), u_cur.data(), scr);
    for (int q = 0; q < n_src; ++q) {
      size_t p = g.at(sx[q] + pad, sz[q] + pad);
      u_nxt[p] += (T)wavelet[(size_t)q + (size_t)n_src * (it - 1)];
    }
    for (int rr = 0; rr < n_rec; ++rr) {
      size_t p = g.at(rx[rr] + pad, rz[rr] + pad);
      seis_u[(size_t)rr + (size_t)n_rec * (it - 1)] = u_nxt[p];
    }
    std::swap(u_old, u_cur);  // u_old <- u^n
    std::swap(u_cur, u_nxt);  // u_cur <- u^{n+1}
  }
  if (final_fields) {
    std::copy(u_cur.begin(), u_cur.end(), final_fields);
    std::copy(u_old.begin(), u_old.end(), final_fields + ncell);
  }
  return 0;
}


// ===========================================================================
// 3D: pad_array_3d.jl:8-89, elastic3d/medium.jl:31-123, acoustic3d/medium.jl:33-63,
// habc_3d.jl:23-55, kernels_3d.jl:117-193 (Higdon averaged over the active
// directions, evaluated two-pass from read-only inputs), update kernels of
// elastic3d/update_*.jl and acoustic3d/update_*.jl, loops elastic3d.jl:122-162
// and acoustic3d.jl:134-185.
// ===========================================================================
struct G3 {
  int nx, ny, nz;
  inline size_t at(int i, int j, int k) const {
    return (size_t)(i - 1) + (size_t)nx * ((size_t)(j - 1) + (size_t)ny * (size_t)(k - 1));
  }
  size_t n() const { return (size_t)nx * ny * nz; }
};

template <class T>
std::vector<T> pad_array3(const float* d, int nx, int ny, int nz, int pad) {
  G3 g{nx + 2 * pad, ny + 2 * pad, nz + 2 * pad};
  std::vector<T> r(g.n());
  for (int k = 1; k <= g.nz; ++k) {
    int kk = std::min(std::max(k - pad, 1), nz);
    for (int j = 1; j <= g.ny; ++j) {
      int jj = std::min(std::max(j - pad, 1), ny);
      for (int i = 1; i <= g.nx; ++i) {
        int ii = std::min(std::max(i - pad, 1), nx);
        r[g.at(i, j, k)] = (T)d[(size_t)(ii - 1) + (size_t)nx * ((jj - 1) + (size_t)ny * (kk - 1))];
      }
    }
  }
  return r;
}

// pad_array_3d.jl:37-89: bx (i-1,i; row 1 copies 2), by (j-1,j; copies 2), bz (k,k+1; last copies)
template <class T>
void buoyancy3(const G3& g, const std::vector<T>& rho, std::vector<T>& bx, std::vector<T>& by,
               std::vector<T>& bz) {
  bx.assign(g.n(), T(0));
  by.assign(g.n(), T(0));
  bz.assign(g.n(), T(0));
  for (int k = 1; k <= g.nz; ++k)
    for (int j = 1; j <= g.ny; ++j) {
      for (int i = 2; i <= g.nx; ++i) bx[g.at(i, j, k)] = harm2(rho[g.at(i - 1, j, k)], rho[g.at(i, j, k)]);
      bx[g.at(1, j, k)] = bx[g.at(2, j, k)];
    }
  for (int k = 1; k <= g.nz; ++k) {
    for (int j = 2; j <= g.ny; ++j)
      for (int i = 1; i <= g.nx; ++i) by[g.at(i, j, k)] = harm2(rho[g.at(i, j - 1, k)], rho[g.at(i, j, k)]);
    for (int i = 1; i <= g.nx; ++i) by[g.at(i, 1, k)] = by[g.at(i, 2, k)];
  }
  for (int k = 1; k <= g.nz - 1; ++k)
    for (int j = 1; j <= g.ny; ++j)
      for (int i = 1; i <= g.nx; ++i) bz[g.at(i, j, k)] = harm2(rho[g.at(i, j, k)], rho[g.at(i, j, k + 1)]);
  for (int j = 1; j <= g.ny; ++j)
    for (int i = 1; i <= g.nx; ++i) bz[g.at(i, j, g.nz)] = bz[g.at(i, j, g.nz - 1)];
}

// elastic3d/medium.jl:73-123
template <class T>
void elastic_params3(const G3& g, const std::vector<T>& vp, const std::vector<T>& vs,
                     const std::vector<T>& rho, std::vector<T>& lam, std::vector<T>& l2m,
                     std::vector<T>& mxy, std::vector<T>& mxz, std::vector<T>& myz) {
  size_t n = g.n();
  std::vector<T> mu(n);
  lam.resize(n);
  l2m.resize(n);
  for (size_t q = 0; q < n; ++q) {
    mu[q] = rho[q] * (vs[q] * vs[q]);
    lam[q] = rho[q] * (vp[q] * vp[q]) - T(2) * mu[q];
    l2m[q] = lam[q] + T(2) * mu[q];
  }
  mxy.assign(n, T(0));
  mxz.assign(n, T(0));
  myz.assign(n, T(0));
  for (int k = 1; k <= g.nz; ++k)
    for (int j = 2; j <= g.ny; ++j)
      for (int i = 2; i <= g.nx; ++i)
        mxy[g.at(i, j, k)] = harm4(mu[g.at(i - 1, j - 1, k)], mu[g.at(i, j - 1, k)], mu[g.at(i - 1, j, k)],
                                   mu[g.at(i, j, k)]);
  for (int k = 1; k <= g.nz; ++k)
    for (int j = 1; j <= g.ny; ++j) mxy[g.at(1, j, k)] = mxy[g.at(2, j, k)];
  for (int k = 1; k <= g.nz; ++k)
    for (int i = 1; i <= g.nx; ++i) mxy[g.at(i, 1, k)] = mxy[g.at(i, 2, k)];
  for (int k = 1; k <= g.nz - 1; ++k)
    for (int j = 1; j <= g.ny; ++j)
      for (int i = 2; i <= g.nx; ++i)
        mxz[g.at(i, j, k)] = harm4(mu[g.at(i - 1, j, k)], mu[g.at(i, j, k)], mu[g.at(i - 1, j, k + 1)],
                                   mu[g.at(i, j, k + 1)]);
  for (int k = 1; k <= g.nz; ++k)
    for (int j = 1; j <= g.ny; ++j) mxz[g.at(1, j, k)] = mxz[g.at(2, j, k)];
  for (int j = 1; j <= g.ny; ++j)
    for (int i = 1; i <= g.nx; ++i) mxz[g.at(i, j, g.nz)] = mxz[g.at(i, j, g.nz - 1)];
  for (int k = 1; k <= g.nz - 1; ++k)
    for (int j = 2; j <= g.ny; ++j)
      for (int i = 1; i <= g.nx; ++i)
        myz[g.at(i, j, k)] = harm4(mu[g.at(i, j - 1, k)], mu[g.at(i, j, k)], mu[g.at(i, j - 1, k + 1)],
                                   mu[g.at(i, j, k + 1)]);
  for (int k = 1; k <= g.nz; ++k)
    for (int i = 1; i <= g.nx; ++i) myz[g.at(i, 1, k)] = myz[g.at(i, 2, k)];
  for (int j = 1; j <= g.ny; ++j)
    for (int i = 1; i <= g.nx; ++i) myz[g.at(i, j, g.nz)] = myz[g.at(i, j, g.nz - 1)];
}

// habc_3d.jl:23-55: same q, qt, qxt as 2D; four ramps (offsets 0, .25, .5, .75)
template <class T>
struct Habc3 {
  int nbc;
  T q, qt, qxt;
  std::vector<T> wtab[4];
};

template <class T>
Habc3<T> init_habc3(int pad, float v_ref, float dt, float dh) {
  Habc<T> h2 = init_habc<T>(pad, v_ref, dt, dh);
  Habc3<T> h;
  h.nbc = h2.nbc;
  h.q = h2.q;
  h.qt = h2.qt;
  h.qxt = h2.qxt;
  const double offs[4] = {0.0, 0.25, 0.5, 0.75};
  for (int k = 0; k < 4; ++k) {
    h.wtab[k].resize(pad + 2);
    for (int d = 0; d < pad + 2; ++d) {
      double w = ((double)d - offs[k]) / (double)(pad - 1);
      h.wtab[k][d] = (T)std::min(std::max(w, 0.0), 1.0);
    }
  }
  return h;
}

struct FramePt3 {
  size_t idx;
  int8_t sx, sy, sz;
  int dist;
};

std::vector<FramePt3> frame_points3(const G3& g, int nbc) {
  std::vector<FramePt3> f;
  for (int k = 2; k <= g.nz - 1; ++k)
    for (int j = 2; j <= g.ny - 1; ++j)
      for (int i = 2; i <= g.nx - 1; ++i) {
        int8_t sx = i <= nbc + 1 ? 1 : (i >= g.nx - nbc ? -1 : 0);
        int8_t sy = j <= nbc + 1 ? 1 : (j >= g.ny - nbc ? -1 : 0);
        int8_t sz = k <= nbc + 1 ? 1 : (k >= g.nz - nbc ? -1 : 0);
        if (!sx && !sy && !sz) continue;
        int d = std::min(std::min(std::min(i - 1, g.nx - i), std::min(j - 1, g.ny - j)),
                         std::min(k - 1, g.nz - k));
        f.push_back(FramePt3{g.at(i, j, k), sx, sy, sz, d});
      }
  return f;
}

template <class T>
void habc3_det(const G3& g, const Habc3<T>& h, const std::vector<FramePt3>& fr, int kind, T* f,
               const T* fo, std::vector<T>& scr) {
  scr.resize(fr.size());
  const long n = (long)fr.size();
  const size_t sxs = 1, sys = (size_t)g.nx, szs = (size_t)g.nx * g.ny;
#pragma omp parallel for schedule(static)
  for (long q = 0; q < n; ++q) {
    const FramePt3& p = fr[q];
    T sum = 0;
    int nd = 0;
    if (p.sx) {
      size_t nb = p.sx > 0 ? p.idx + sxs : p.idx - sxs;
      sum = sum + higdon_side(h.q, h.qt, h.qxt, f[nb], fo[p.idx], fo[nb]);
      ++nd;
    }
    if (p.sy) {
      size_t nb = p.sy > 0 ? p.idx + sys : p.idx - sys;
      sum = sum + higdon_side(h.q, h.qt, h.qxt, f[nb], fo[p.idx], fo[nb]);
      ++nd;
    }
    if (p.sz) {
      size_t nb = p.sz > 0 ? p.idx + szs : p.idx - szs;
      sum = sum + higdon_side(h.q, h.qt, h.qxt, f[nb], fo[p.idx], fo[nb]);
      ++nd;
    }
    const std::vector<T>& t = h.wtab[kind];
    T w = p.dist < (int)t.size() ? t[p.dist] : T(1);
    scr[q] = fmaT(w, f[p.idx], ((T(1) - w) * sum) / (T)nd);
  }
#pragma omp parallel for schedule(static)
  for (long q = 0; q < n; ++q) f[fr[q].idx] = scr[q];
}

template <class T>
int run_acoustic3d(int nx, int ny, int nz, const float* vp, const float* rho, float dh, float dt,
                   int nt, int nbc, int fd_order, float v_ref, int n_src, const int32_t* sx,
                   const int32_t* sy, const int32_t* sz, const float* wavelet, int n_rec,
                   const int32_t* rx, const int32_t* ry, const int32_t* rz, T* svx, T* svy, T* svz,
                   int snap_interval, int snap_plane, int snap_index, T* snaps, T* final_fields) {
  int N = order_to_N(fd_order);
  if (N < 0) return -2;
  int M = N, pad = nbc + M;
  if (pad < 2) return -2;
  G3 g{nx + 2 * pad, ny + 2 * pad, nz + 2 * pad};
  std::vector<T> vpp = pad_array3<T>(vp, nx, ny, nz, pad), rhop = pad_array3<T>(rho, nx, ny, nz, pad);
  std::vector<T> bx, by, bz, kap(g.n());
  buoyancy3(g, rhop, bx, by, bz);
  for (size_t q = 0; q < g.n(); ++q) kap[q] = rhop[q] * (vpp[q] * vpp[q]);
  Habc3<T> h = init_habc3<T>(pad, v_ref, dt, dh);
  std::vector<FramePt3> fr = frame_points3(g, h.nbc);
  Coef<T> c = coef<T>(fd_order);
  const T dtdh = (T)dt / (T)dh;
  const size_t n = g.n(), sy_ = (size_t)g.nx, sz_ = (size_t)g.nx * g.ny;
  std::vector<T> vx(n, T(0)), vy(n, T(0)), vz(n, T(0)), p(n, T(0)), o1, o2, o3, scr;
  for (int it = 1; it <= nt; ++it) {
    o1 = vx;
    o2 = vy;
    o3 = vz;
#pragma omp parallel for schedule(static)
    for (int k = M + 1; k <= g.nz - M; ++k)
      for (int j = M + 1; j <= g.ny - M; ++j)
        for (int i = M + 1; i <= g.nx - M; ++i) {
          size_t q = g.at(i, j, k);
          T dx = 0, dy = 0, dz = 0;
          for (int l = 1; l <= N; ++l) {
            T a = c.a[l - 1];
            dx = fmaT(a, p[q + (l - 1)] - p[q - l], dx);
            dy = fmaT(a, p[q + (l - 1) * sy_] - p[q - l * sy_], dy);
            dz = fmaT(a, p[q + l * sz_] - p[q - (l - 1) * sz_], dz);
          }
          vx[q] = fmaT(bx[q] * dtdh, dx, vx[q]);
          vy[q] = fmaT(by[q] * dtdh, dy, vy[q]);
          vz[q] = fmaT(bz[q] * dtdh, dz, vz[q]);
        }
    habc3_det(g, h, fr, 0, vx.data(), o1.data(), scr);
    habc3_det(g, h, fr, 1, vy.data(), o2.data(), scr);
    habc3_det(g, h, fr, 2, vz.data(), o3.data(), scr);
    o1 = p;
#pragma omp parallel for schedule(static)
    for (int k = M + 1; k <= g.nz - M; ++k)
      for (int j = M + 1; j <= g.ny - M; ++j)
        for (int i = M + 1; i <= g.nx - M; ++i) {
          size_t q = g.at(i, j, k);
          T dx = 0, dy = 0, dz = 0;
          for (int l = 1; l <= N; ++l) {
            T a = c.a[l - 1];
            dx = fmaT(a, vx[q + l] - vx[q - (l - 1)], dx);
            dy = fmaT(a, vy[q + l * sy_] - vy[q - (l - 1) * sy_], dy);
            dz = fmaT(a, vz[q + (l - 1) * sz_] - vz[q - l * sz_], dz);
          }
          p[q] = fmaT(kap[q] * dtdh, (dx + dy) + dz, p[q]);
        }
    habc3_det(g, h, fr, 3, p.data(), o1.data(), scr);
    for (int s = 0; s < n_src; ++s)
      p[g.at(sx[s] + pad, sy[s] + pad, sz[s] + pad)] += (T)wavelet[(size_t)s + (size_t)n_src * (it - 1)];
    for (int r = 0; r < n_rec; ++r) {
      size_t q = g.at(rx[r] + pad, ry[r] + pad, rz[r] + pad), o = (size_t)r + (size_t)n_rec * (it - 1);
      svx[o] = vx[q];
      svy[o] = vy[q];
      svz[o] = vz[q];
    }
    if (snaps && snap_interval > 0 && it % snap_interval == 0) {
      T* out = snaps + (size_t)(it / snap_interval - 1) * (snap_plane == 1 ? (size_t)nx * ny
                                                          : snap_plane == 2 ? (size_t)ny * nz
                                                                            : (size_t)nx * nz);
      int si = snap_index + pad;
      if (snap_plane == 0)
        for (int k = 1; k <= nz; ++k)
          for (int i = 1; i <= nx; ++i) out[(i - 1) + (size_t)nx * (k - 1)] = p[g.at(i + pad, si, k + pad)];
      else if (snap_plane == 1)
        for (int j = 1; j <= ny; ++j)
          for (int i = 1; i <= nx; ++i) out[(i - 1) + (size_t)nx * (j - 1)] = p[g.at(i + pad, j + pad, si)];
      else
        for (int k = 1; k <= nz; ++k)
          for (int j = 1; j <= ny; ++j) out[(j - 1) + (size_t)ny * (k - 1)] = p[g.at(si, j + pad, k + pad)];
    }
  }
  if (final_fields) {
    std::copy(vx.begin(), vx.end(), final_fields);
    std::copy(vy.begin(), vy.end(), final_fields + n);
    std::copy(vz.begin(), vz.end(), final_fields + 2 * n);
    std::copy(p.begin(), p.end(), final_fields + 3 * n);
  }
  return 0;
}

template <class T>
int run_elastic3d(int nx, int ny, int nz, const float* vp, const float* vs, const float* rho,
                  float dh, float dt, int nt, int nbc, int fd_order, float v_ref, int n_src,
                  const int32_t* sx, const int32_t* sy, const int32_t* sz, const float* wavelet,
                  int n_rec, const int32_t* rx, const int32_t* ry, const int32_t* rz, T* svx,
                  T* svy, T* svz, int snap_interval, int snap_plane, int snap_index, T* snaps,
                  T* final_fields) {
  int N = order_to_N(fd_order);
  if (N < 0) return -2;
  int M = N, pad = nbc + M;
  if (pad < 2) return -2;
  G3 g{nx + 2 * pad, ny + 2 * pad, nz + 2 * pad};
  std::vector<T> vpp = pad_array3<T>(vp, nx, ny, nz, pad), vsp = pad_array3<T>(vs, nx, ny, nz, pad),
                 rhop = pad_array3<T>(rho, nx, ny, nz, pad);
  std::vector<T> bx, by, bz, lam, l2m, mxy, mxz, myz;
  buoyancy3(g, rhop, bx, by, bz);
  elastic_params3(g, vpp, vsp, rhop, lam, l2m, mxy, mxz, myz);
  Habc3<T> h = init_habc3<T>(pad, v_ref, dt, dh);
  std::vector<FramePt3> fr = frame_points3(g, h.nbc);
  Coef<T> c = coef<T>(fd_order);
  const T dtdh = (T)dt / (T)dh;
  const size_t n = g.n(), Y = (size_t)g.nx, Z = (size_t)g.nx * g.ny;
  std::vector<T> F[9], O[9], scr;  // vx vy vz txx tyy tzz txy txz tyz
  for (auto& v : F) v.assign(n, T(0));
  for (int it = 1; it <= nt; ++it) {
    for (int f = 0; f < 3; ++f) O[f] = F[f];
    T *vx = F[0].data(), *vy = F[1].data(), *vz = F[2].data();
    const T *txx = F[3].data(), *tyy = F[4].data(), *tzz = F[5].data(), *txy = F[6].data(),
            *txz = F[7].data(), *tyz = F[8].data();
#pragma omp parallel for schedule(static)
    for (int k = M + 1; k <= g.nz - M; ++k)
      for (int j = M + 1; j <= g.ny - M; ++j)
        for (int i = M + 1; i <= g.nx - M; ++i) {
          size_t q = g.at(i, j, k);
          T a1 = 0, a2 = 0, a3 = 0, b1 = 0, b2 = 0, b3 = 0, c1 = 0, c2 = 0, c3 = 0;
          for (int l = 1; l <= N; ++l) {  // elastic3d/update_velocity.jl:49-75
            T a = c.a[l - 1];
            a1 = fmaT(a, txx[q + (l - 1)] - txx[q - l], a1);          // dtxxdx
            a2 = fmaT(a, txy[q + l * Y] - txy[q - (l - 1) * Y], a2);  // dtxydy
            a3 = fmaT(a, txz[q + (l - 1) * Z] - txz[q - l * Z], a3);  // dtxzdz
            b1 = fmaT(a, txy[q + l] - txy[q - (l - 1)], b1);          // dtxydx
            b2 = fmaT(a, tyy[q + (l - 1) * Y] - tyy[q - l * Y], b2);  // dtyydy
            b3 = fmaT(a, tyz[q + (l - 1) * Z] - tyz[q - l * Z], b3);  // dtyzdz
            c1 = fmaT(a, txz[q + l] - txz[q - (l - 1)], c1);          // dtxzdx
            c2 = fmaT(a, tyz[q + l * Y] - tyz[q - (l - 1) * Y], c2);  // dtyzdy
            c3 = fmaT(a, tzz[q + l * Z] - tzz[q - (l - 1) * Z], c3);  // dtzzdz
          }
          vx[q] = fmaT(bx[q] * dtdh, (a1 + a2) + a3, vx[q]);
          vy[q] = fmaT(by[q] * dtdh, (b1 + b2) + b3, vy[q]);
          vz[q] = fmaT(bz[q] * dtdh, (c1 + c2) + c3, vz[q]);
        }
    habc3_det(g, h, fr, 0, vx, O[0].data(), scr);
    habc3_det(g, h, fr, 1, vy, O[1].data(), scr);
    habc3_det(g, h, fr, 2, vz, O[2].data(), scr);
    for (int f = 3; f < 9; ++f) O[f] = F[f];
    T *sxx = F[3].data(), *syy = F[4].data(), *szz = F[5].data(), *sxy = F[6].data(),
      *sxz = F[7].data(), *syz = F[8].data();
#pragma omp parallel for schedule(static)
    for (int k = M + 1; k <= g.nz - M; ++k)
      for (int j = M + 1; j <= g.ny - M; ++j)
        for (int i = M + 1; i <= g.nx - M; ++i) {
          size_t q = g.at(i, j, k);
          T dxx = 0, dyy = 0, dzz = 0, dxy = 0, dyx = 0, dxz = 0, dzx = 0, dyz = 0, dzy = 0;
          for (int l = 1; l <= N; ++l) {  // elastic3d/update_stress.jl:51-80
            T a = c.a[l - 1];
            dxx = fmaT(a, vx[q + l] - vx[q - (l - 1)], dxx);
            dyy = fmaT(a, vy[q + l * Y] - vy[q - (l - 1) * Y], dyy);
            dzz = fmaT(a, vz[q + (l - 1) * Z] - vz[q - l * Z], dzz);
            dxy = fmaT(a, vx[q + (l - 1) * Y] - vx[q - l * Y], dxy);
            dyx = fmaT(a, vy[q + (l - 1)] - vy[q - l], dyx);
            dxz = fmaT(a, vx[q + l * Z] - vx[q - (l - 1) * Z], dxz);
            dzx = fmaT(a, vz[q + (l - 1)] - vz[q - l], dzx);
            dyz = fmaT(a, vy[q + l * Z] - vy[q - (l - 1) * Z], dyz);
            dzy = fmaT(a, vz[q + (l - 1) * Y] - vz[q - l * Y], dzy);
          }
          const T lm = lam[q], l2 = l2m[q];
          sxx[q] = fmaT(fmaT(lm, dzz, fmaT(lm, dyy, l2 * dxx)), dtdh, sxx[q]);
          syy[q] = fmaT(fmaT(lm, dzz, fmaT(l2, dyy, lm * dxx)), dtdh, syy[q]);
          szz[q] = fmaT(fmaT(l2, dzz, fmaT(lm, dyy, lm * dxx)), dtdh, szz[q]);
          sxy[q] = fmaT(mxy[q] * (dxy + dyx), dtdh, sxy[q]);
          sxz[q] = fmaT(mxz[q] * (dxz + dzx), dtdh, sxz[q]);
          syz[q] = fmaT(myz[q] * (dyz + dzy), dtdh, syz[q]);
        }
    for (int f = 3; f < 9; ++f) habc3_det(g, h, fr, 3, F[f].data(), O[f].data(), scr);
    for (int s = 0; s < n_src; ++s) {
      size_t q = g.at(sx[s] + pad, sy[s] + pad, sz[s] + pad);
      T w = (T)wavelet[(size_t)s + (size_t)n_src * (it - 1)];
      sxx[q] += w;
      syy[q] += w;
      szz[q] += w;
    }
    for (int r = 0; r < n_rec; ++r) {
      size_t q = g.at(rx[r] + pad, ry[r] + pad, rz[r] + pad), o = (size_t)r + (size_t)n_rec * (it - 1);
      svx[o] = vx[q];
      svy[o] = vy[q];
      svz[o] = vz[q];
    }
    if (snaps && snap_interval > 0 && it % snap_interval == 0) {
      T* out = snaps + (size_t)(it / snap_interval - 1) * (snap_plane == 1 ? (size_t)nx * ny
                                                          : snap_plane == 2 ? (size_t)ny * nz
                                                                            : (size_t)nx * nz);
      int si = snap_index + pad;
      if (snap_plane == 0)
        for (int k = 1; k <= nz; ++k)
          for (int i = 1; i <= nx; ++i) out[(i - 1) + (size_t)nx * (k - 1)] = vz[g.at(i + pad, si, k + pad)];
      else if (snap_plane == 1)
        for (int j = 1; j <= ny; ++j)
          for (int i = 1; i <= nx; ++i) out[(i - 1) + (size_t)nx * (j - 1)] = vz[g.at(i + pad, j + pad, si)];
      else
        for (int k = 1; k <= nz; ++k)
          for (int j = 1; j <= ny; ++j) out[(j - 1) + (size_t)ny * (k - 1)] = vz[g.at(si, j + pad, k + pad)];
    }
  }
  if (final_fields)
    for (int f = 0; f < 9; ++f) std::copy(F[f].begin(), F[f].end(), final_fields + f * n);
  return 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// coupled2d: coupled P-S potentials (equations/coupled2d/*, constant density).
// ---------------------------------------------------------------------------
// utils/FD_centered.jl:15-21 -- centered first-derivative coefficients.
const float kD1[6][5] = {
    {0, 0, 0, 0, 0},
    {(float)0.5, 0, 0, 0, 0},
    {(float)(2.0 / 3.0), (float)(-1.0 / 12.0), 0, 0, 0},
    {(float)(3.0 / 4.0), (float)(-3.0 / 20.0), (float)(1.0 / 60.0), 0, 0},
    {(float)(4.0 / 5.0), (float)(-1.0 / 5.0), (float)(4.0 / 105.0), (float)(-1.0 / 280.0), 0},
    {(float)(5.0 / 6.0), (float)(-5.0 / 21.0), (float)(5.0 / 84.0), (float)(-5.0 / 504.0),
     (float)(1.0 / 1260.0)},
};

// coupled2d/medium.jl:121-126 -- taps exp(-0.5 (k/sigma)^2), k = -r..r, r = ceil(3 sigma),
// rounded to T and divided by their sum (summed in T from k = -r).
template <class T>
std::vector<T> gaussian_taps(double sigma) {
  const int r = (int)std::ceil(3.0 * sigma);
  std::vector<T> k((size_t)(2 * r + 1));
  for (int q = -r; q <= r; ++q) {
    const double x = (double)q / sigma;
    k[(size_t)(q + r)] = (T)std::exp(-0.5 * (x * x));
  }
  T s = T(0);
  for (T v : k) s = s + v;
  for (T& v : k) v = v / s;
  return k;
}

// coupled2d/medium.jl:118-151 -- separable smoothing, x pass then z pass, clamped
// indices; each tap is one multiply and one add (the reference's CPU loop).
template <class T>
std::vector<T> gaussian_smooth(const G2& g, const std::vector<T>& f, const std::vector<T>& taps) {
  const int r = (int)(taps.size() - 1) / 2;
  std::vector<T> tmp(g.n()), out(g.n());
#pragma omp parallel for schedule(static)
  for (int j = 1; j <= g.nz; ++j)
    for (int i = 1; i <= g.nx; ++i) {
      T v = T(0);
      for (int q = -r; q <= r; ++q) {
        const int ii = std::min(std::max(i + q, 1), g.nx);
        v = v + taps[(size_t)(q + r)] * f[g.at(ii, j)];
      }
      tmp[g.at(i, j)] = v;
    }
#pragma omp parallel for schedule(static)
  for (int j = 1; j <= g.nz; ++j)
    for (int i = 1; i <= g.nx; ++i) {
      T v = T(0);
      for (int q = -r; q <= r; ++q) {
        const int jj = std::min(std::max(j + q, 1), g.nz);
        v = v + taps[(size_t)(q + r)] * tmp[g.at(i, jj)];
      }
      out[g.at(i, j)] = v;
    }
  return out;
}

// coupled2d/medium.jl:157-193 -- gradients (x: M < i <= nx-M, every j; z: the
// transpose) and the Laplacian (both ranges) of the smoothed field; 0 elsewhere.
template <class T>
void coupled_derivs(const G2& g, int N, T h, const std::vector<T>& f, T* dx, T* dz, T* lap) {
  const int M = N;
  const T ih2 = T(1) / (h * h);
  const T c0 = (T)kD2C0[N];
  for (size_t q = 0; q < g.n(); ++q) dx[q] = dz[q] = lap[q] = T(0);
#pragma omp parallel for schedule(static)
  for (int j = 1; j <= g.nz; ++j)
    for (int i = 1; i <= g.nx; ++i) {
      const size_t p = g.at(i, j);
      if (i > M && i <= g.nx - M) {
        T v = T(0);
        for (int l = 1; l <= N; ++l) v = v + (T)kD1[N][l - 1] * (f[p + l] - f[p - l]);
        dx[p] = v / h;
      }
      if (j > M && j <= g.nz - M) {
        T v = T(0);
        for (int l = 1; l <= N; ++l)
          v = v + (T)kD1[N][l - 1] * (f[p + (size_t)l * g.nx] - f[p - (size_t)l * g.nx]);
        dz[p] = v / h;
      }
      if (i > M && i <= g.nx - M && j > M && j <= g.nz - M) {
        T a = c0 * f[p], b = c0 * f[p];
        for (int l = 1; l <= N; ++l) {
          a = a + (T)kD2[N][l - 1] * (f[p + l] + f[p - l]);
          b = b + (T)kD2[N][l - 1] * (f[p + (size_t)l * g.nx] + f[p - (size_t)l * g.nx]);
        }
        lap[p] = (a + b) * ih2;
      }
    }
}

// The eight planes of CoupledMedium (medium.jl:46-107): alpha, beta (unsmoothed
// vp^2, vs^2), then d alpha/dx, d alpha/dz, d beta/dx, d beta/dz, lap alpha,
// lap beta of the smoothed fields (smooth_sigma <= 0: no smoothing).
template <class T>
std::vector<T> coupled_medium(const G2& g, int N, const float* vp, const float* vs, int nx,
                              int nz, int pad, float dh, double sigma) {
  const size_t n = g.n();
  std::vector<T> m(8 * n);
  std::vector<T> vpp = pad_array<T>(vp, nx, nz, pad), vsp = pad_array<T>(vs, nx, nz, pad);
  std::vector<T> a(n), b(n);
  for (size_t q = 0; q < n; ++q) {
    a[q] = vpp[q] * vpp[q];
    b[q] = vsp[q] * vsp[q];
  }
  std::vector<T> as = a, bs = b;
  if (sigma > 0) {
    const std::vector<T> taps = gaussian_taps<T>(sigma);
    as = gaussian_smooth(g, a, taps);
    bs = gaussian_smooth(g, b, taps);
  }
  std::copy(a.begin(), a.end(), m.begin());
  std::copy(b.begin(), b.end(), m.begin() + n);
  const T h = (T)dh;
  coupled_derivs(g, N, h, as, m.data() + 2 * n, m.data() + 3 * n, m.data() + 6 * n);
  coupled_derivs(g, N, h, bs, m.data() + 4 * n, m.data() + 5 * n, m.data() + 7 * n);
  return m;
}

template <class T>
struct CoupledState {
  std::vector<T> P, S, dP, dS, o1, o2;
};

// update_fields.jl:27-108, "velocity" half step on M < i, j <= n - M.  The
// operation order (one fma per stencil term, the right-hand sides as written
// below) is this implementation's canonical FP32 sequence; the GPU kernel
// repeats it.
template <class T>
void coupled_vel(const G2& g, int N, const T* m, T dt, T ih, T ih2, CoupledState<T>& s) {
  const int M = N;
  const size_t n = g.n(), nx = g.nx;
  const T c0 = (T)kD2C0[N];
#pragma omp parallel for schedule(static)
  for (int j = M + 1; j <= g.nz - M; ++j)
    for (int i = M + 1; i <= g.nx - M; ++i) {
      const size_t p = g.at(i, j);
      const T* P = s.P.data();
      const T* S = s.S.data();
      T dPx = 0, dPz = 0, dSx = 0, dSz = 0;
      T lPx = c0 * P[p], lPz = c0 * P[p], lSx = c0 * S[p], lSz = c0 * S[p];
      for (int l = 1; l <= N; ++l) {
        const T c1 = (T)kD1[N][l - 1], c2 = (T)kD2[N][l - 1];
        const size_t lz = (size_t)l * nx;
        dPx = fmaT(c1, P[p + l] - P[p - l], dPx);
        dPz = fmaT(c1, P[p + lz] - P[p - lz], dPz);
        lPx = fmaT(c2, P[p + l] + P[p - l], lPx);
        lPz = fmaT(c2, P[p + lz] + P[p - lz], lPz);
        dSx = fmaT(c1, S[p + l] - S[p - l], dSx);
        dSz = fmaT(c1, S[p + lz] - S[p - lz], dSz);
        lSx = fmaT(c2, S[p + l] + S[p - l], lSx);
        lSz = fmaT(c2, S[p + lz] + S[p - lz], lSz);
      }
      dPx = dPx * ih;
      dPz = dPz * ih;
      dSx = dSx * ih;
      dSz = dSz * ih;
      const T lapP = (lPx + lPz) * ih2, lapS = (lSx + lSz) * ih2;
      const T a = m[p], b = m[n + p], ax = m[2 * n + p], az = m[3 * n + p], bx = m[4 * n + p],
              bz = m[5 * n + p], la = m[6 * n + p], lb = m[7 * n + p];
      const T Pc = P[p];
      T rP = Pc * la;
      rP = fmaT(T(2), fmaT(ax, dPx, az * dPz), rP);
      rP = fmaT(T(-2) * Pc, lb, rP);
      rP = fmaT(T(2), fmaT(bx, dSz, -(bz * dSx)), rP);
      rP = fmaT(a, lapP, rP);
      T rS = T(2) * fmaT(bx, dSx, bz * dSz);
      rS = fmaT(T(2), fmaT(bz, dPx, -(bx * dPz)), rS);
      rS = fmaT(b, lapS, rS);
      s.dP[p] = fmaT(dt, rP, s.dP[p]);
      s.dS[p] = fmaT(dt, rS, s.dS[p]);
    }
}

// update_fields.jl:120-141, "position" half step.
template <class T>
void coupled_pos(const G2& g, int M, T dt, CoupledState<T>& s) {
#pragma omp parallel for schedule(static)
  for (int j = M + 1; j <= g.nz - M; ++j)
    for (int i = M + 1; i <= g.nx - M; ++i) {
      const size_t p = g.at(i, j);
      s.P[p] = fmaT(dt, s.dP[p], s.P[p]);
      s.S[p] = fmaT(dt, s.dS[p], s.S[p]);
    }
}

// coupled2d.jl:53-171 and the loop :192-260.  The loop's racy full-grid HABC
// (boundary/habc/kernels.jl:122-190) is applied in the deterministic two-pass
// form (pre-correction neighbours), with weights w_vx for dP/dt, dS/dt and
// w_tau for P, S, and the Higdon coefficients of v_ref_p (P fields) and
// v_ref_s (S fields).
template <class T>
int run_coupled2d(int nx, int nz, const float* vp, const float* vs, float dh, float dt, int nt,
                  int nbc, int fd_order, float v_ref_p, float v_ref_s, double sigma, int n_src,
                  const int32_t* sx, const int32_t* sz, const float* wavelet, int n_rec,
                  const int32_t* rx, const int32_t* rz, T* seis_P, T* seis_S, int snap_interval,
                  T* snaps_P, T* snaps_S, T* medium_out) {
  const int N = order_to_N(fd_order);
  if (N < 0) return -2;
  const int M = N, pad = nbc + M;
  if (pad < 2) return -2;
  G2 g{nx + 2 * pad, nz + 2 * pad};
  const std::vector<T> med = coupled_medium<T>(g, N, vp, vs, nx, nz, pad, dh, sigma);
  if (medium_out) std::copy(med.begin(), med.end(), medium_out);
  Habc<T> hp = init_habc<T>(pad, v_ref_p, dt, dh), hs = init_habc<T>(pad, v_ref_s, dt, dh);
  std::vector<FramePt> fr = frame_points(g, hp.nbc);
  const T tdt = (T)dt, ih = T(1) / (T)dh, ih2 = ih * ih;
  const size_t ncell = g.n(), nint = (size_t)nx * nz;
  CoupledState<T> st;
  for (auto* v : {&st.P, &st.S, &st.dP, &st.dS, &st.o1, &st.o2}) v->assign(ncell, T(0));
  std::vector<T> scr;
  for (int it = 1; it <= nt; ++it) {
    st.o1 = st.dP;
    st.o2 = st.dS;
    coupled_vel(g, N, med.data(), tdt, ih, ih2, st);
    habc_det(g, hp, fr, 0, st.dP.data(), st.o1.data(), scr);
    habc_det(g, hs, fr, 0, st.dS.data(), st.o2.data(), scr);
    st.o1 = st.P;
    st.o2 = st.S;
    coupled_pos(g, M, tdt, st);
    habc_det(g, hp, fr, 2, st.P.data(), st.o1.data(), scr);
    habc_det(g, hs, fr, 2, st.S.data(), st.o2.data(), scr);
    for (int q = 0; q < n_src; ++q) {  // inject_source!(P): coupled2d.jl:239-243
      size_t p = g.at(sx[q] + pad, sz[q] + pad);
      st.P[p] += (T)wavelet[(size_t)q + (size_t)n_src * (it - 1)];
    }
    for (int r = 0; r < n_rec; ++r) {  // coupled2d.jl:245-250
      size_t p = g.at(rx[r] + pad, rz[r] + pad);
      size_t o = (size_t)r + (size_t)n_rec * (it - 1);
      if (seis_P) seis_P[o] = st.P[p];
      if (seis_S) seis_S[o] = st.S[p];
    }
    if (snap_interval > 0 && it % snap_interval == 0) {  // coupled2d.jl:252-258
      const int k = it / snap_interval - 1;
      if (snaps_P) snap_interior(g, pad, st.P.data(), snaps_P + nint * (size_t)k);
      if (snaps_S) snap_interior(g, pad, st.S.data(), snaps_S + nint * (size_t)k);
    }
  }
  return 0;
}

extern "C" {

int oracle_version(void) { return 1; }

void oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// Host preparation exported for the tests (padded column-major arrays).
// kind: 0 = elastic (out: bx,bz,lam,lam2mu,mu_txz), 1 = acoustic (out: bx,bz,kappa).
int oracle_medium2d_f32(int kind, int nx, int nz, const float* vp, const float* vs,
                        const float* rho, int pad, float* out) {
  G2 g{nx + 2 * pad, nz + 2 * pad};
  size_t n = g.n();
  std::vector<float> vpp = pad_array<float>(vp, nx, nz, pad), rhop = pad_array<float>(rho, nx, nz, pad);
  std::vector<float> bx, bz;
  staggered_buoyancy(g, rhop, bx, bz);
  std::copy(bx.begin(), bx.end(), out);
  std::copy(bz.begin(), bz.end(), out + n);
  if (kind == 0) {
    std::vector<float> vsp = pad_array<float>(vs, nx, nz, pad), lam, l2m, mut;
    elastic_params(g, vpp, vsp, rhop, lam, l2m, mut);
    std::copy(lam.begin(), lam.end(), out + 2 * n);
    std::copy(l2m.begin(), l2m.end(), out + 3 * n);
    std::copy(mut.begin(), mut.end(), out + 4 * n);
  } else {
    for (size_t k = 0; k < n; ++k) out[2 * n + k] = rhop[k] * (vpp[k] * vpp[k]);
  }
  return 0;
}

// Higdon coefficients (q, qt, qxt) and the three weight tables (pad+2 each).
int oracle_habc_f32(int pad, float v_ref, float dt, float dh, float* qs, float* wtab) {
  Habc<float> h = init_habc<float>(pad, v_ref, dt, dh);
  qs[0] = h.q;
  qs[1] = h.qt;
  qs[2] = h.qxt;
  for (int k = 0; k < 3; ++k) std::copy(h.wtab[k].begin(), h.wtab[k].end(), wtab + k * (pad + 2));
  return h.nbc;
}

// One two-pass HABC application on a padded field (restates habc_cpu_ref,
// verify_det_graph.jl:59-94).  kind: 0 vx, 1 vz, 2 tau/p.
int oracle_habc_apply_f32(int nxp, int nzp, int pad, float v_ref, float dt, float dh, int kind,
                          float* f, const float* f_old) {
  G2 g{nxp, nzp};
  Habc<float> h = init_habc<float>(pad, v_ref, dt, dh);
  std::vector<FramePt> fr = frame_points(g, h.nbc);
  std::vector<float> scr;
  habc_det(g, h, fr, kind, f, f_old, scr);
  return (int)fr.size();
}

#define ORACLE_PREC_DISPATCH(prec, call32, call64) \
  ((prec) == 64 ? (call64) : ((prec) == 32 ? (call32) : -3))

int oracle_elastic2d(int prec, int nx, int nz, int ns, const float* vp, const float* vs,
                     const float* rho, float dh, float dt, int nt, int nbc, int fd_order,
                     float v_ref, int n_src, const int32_t* sx, const int32_t* sz,
                     const float* wavelet, int n_rec, const int32_t* rx, const int32_t* rz,
                     void* seis_vx, void* seis_vz, int snap_interval, void* snaps,
                     void* final_fields) {
  return ORACLE_PREC_DISPATCH(
      prec,
      run_elastic2d<float>(nx, nz, ns, vp, vs, rho, dh, dt, nt, nbc, fd_order, v_ref, n_src, sx,
                           sz, wavelet, n_rec, rx, rz, (float*)seis_vx, (float*)seis_vz,
                           snap_interval, (float*)snaps, (float*)final_fields),
      run_elastic2d<double>(nx, nz, ns, vp, vs, rho, dh, dt, nt, nbc, fd_order, v_ref, n_src, sx,
                            sz, wavelet, n_rec, rx, rz, (double*)seis_vx, (double*)seis_vz,
                            snap_interval, (double*)snaps, (double*)final_fields));
}

// FP32 arithmetic with wavefields stored as store_kind (0 fp32, 1 fp16,
// 2 bf16) under power-of-two scales sv (velocities) and st (stresses).
int oracle_elastic2d_store(int store_kind, float sv, float st, int fp32_band, int nx, int nz, int ns,
                           const float* vp, const float* vs, const float* rho, float dh, float dt,
                           int nt, int nbc, int fd_order, float v_ref, int n_src, const int32_t* sx,
                           const int32_t* sz, const float* wavelet, int n_rec, const int32_t* rx,
                           const int32_t* rz, float* seis_vx, float* seis_vz, int snap_interval,
                           float* snaps, float* final_fields) {
  StoreSpec ss;
  ss.kind = store_kind;
  ss.sv = sv;
  ss.st = st;
  ss.fp32_band = fp32_band;
  return run_elastic2d<float>(nx, nz, ns, vp, vs, rho, dh, dt, nt, nbc, fd_order, v_ref, n_src,
                              sx, sz, wavelet, n_rec, rx, rz, seis_vx, seis_vz, snap_interval,
                              snaps, final_fields, ss);
}

// Element-wise storage rounding (checked against numpy's float16 in the tests).
void oracle_round_store(int store_kind, const float* x, float* y, long long n) {
  for (long long q = 0; q < n; ++q) y[q] = round_store(x[q], store_kind);
}

int oracle_acoustic2d(int prec, int nx, int nz, int ns, const float* vp, const float* rho,
                      float dh, float dt, int nt, int nbc, int fd_order, float v_ref, int n_src,
                      const int32_t* sx, const int32_t* sz, const float* wavelet, int n_rec,
                      const int32_t* rx, const int32_t* rz, void* seis_p, void* seis_vx,
                      void* seis_vz, int snap_interval, void* snaps, void* final_fields,
                      int zone_nbc_override) {
  return ORACLE_PREC_DISPATCH(
      prec,
      run_acoustic2d<float>(nx, nz, ns, vp, rho, dh, dt, nt, nbc, fd_order, v_ref, n_src, sx, sz,
                            wavelet, n_rec, rx, rz, (float*)seis_p, (float*)seis_vx,
                            (float*)seis_vz, snap_interval, (float*)snaps, (float*)final_fields,
                            zone_nbc_override),
      run_acoustic2d<double>(nx, nz, ns, vp, rho, dh, dt, nt, nbc, fd_order, v_ref, n_src, sx, sz,
                             wavelet, n_rec, rx, rz, (double*)seis_p, (double*)seis_vx,
                             (double*)seis_vz, snap_interval, (double*)snaps,
                             (double*)final_fields, zone_nbc_override));
}

// boundary = :sponge with Cerjan factor sponge_factor (>= 0): the legacy loops
// acoustic2d.jl:213-227 and elastic2d.jl:180-195.
int oracle_acoustic2d_sponge(int prec, float sponge_factor, int nx, int nz, int ns,
                             const float* vp, const float* rho, float dh, float dt, int nt,
                             int nbc, int fd_order, int n_src, const int32_t* sx,
                             const int32_t* sz, const float* wavelet, int n_rec, const int32_t* rx,
                             const int32_t* rz, void* seis_p, void* seis_vx, void* seis_vz,
                             int snap_interval, void* snaps, void* final_fields) {
  if (!(sponge_factor >= 0.0f)) return -2;
  return ORACLE_PREC_DISPATCH(
      prec,
      run_acoustic2d<float>(nx, nz, ns, vp, rho, dh, dt, nt, nbc, fd_order, 1.0f, n_src, sx, sz,
                            wavelet, n_rec, rx, rz, (float*)seis_p, (float*)seis_vx,
                            (float*)seis_vz, snap_interval, (float*)snaps, (float*)final_fields,
                            0, sponge_factor),
      run_acoustic2d<double>(nx, nz, ns, vp, rho, dh, dt, nt, nbc, fd_order, 1.0f, n_src, sx, sz,
                             wavelet, n_rec, rx, rz, (double*)seis_p, (double*)seis_vx,
                             (double*)seis_vz, snap_interval, (double*)snaps,
                             (double*)final_fields, 0, sponge_factor));
}

int oracle_elastic2d_sponge(int prec, float sponge_factor, int nx, int nz, int ns,
                            const float* vp, const float* vs, const float* rho, float dh, float dt,
                            int nt, int nbc, int fd_order, int n_src, const int32_t* sx,
                            const int32_t* sz, const float* wavelet, int n_rec, const int32_t* rx,
                            const int32_t* rz, void* seis_vx, void* seis_vz, int snap_interval,
                            void* snaps, void* final_fields) {
  if (!(sponge_factor >= 0.0f)) return -2;
  return ORACLE_PREC_DISPATCH(
      prec,
      run_elastic2d<float>(nx, nz, ns, vp, vs, rho, dh, dt, nt, nbc, fd_order, 1.0f, n_src, sx,
                           sz, wavelet, n_rec, rx, rz, (float*)seis_vx, (float*)seis_vz,
                           snap_interval, (float*)snaps, (float*)final_fields, StoreSpec(),
                           sponge_factor),
      run_elastic2d<double>(nx, nz, ns, vp, vs, rho, dh, dt, nt, nbc, fd_order, 1.0f, n_src, sx,
                            sz, wavelet, n_rec, rx, rz, (double*)seis_vx, (double*)seis_vz,
                            snap_interval, (double*)snaps, (double*)final_fields, StoreSpec(),
                            sponge_factor));
}

int oracle_coupled2d(int prec, int nx, int nz, const float* vp, const float* vs, float dh,
                     float dt, int nt, int nbc, int fd_order, float v_ref_p, float v_ref_s,
                     double smooth_sigma, int n_src, const int32_t* sx, const int32_t* sz,
                     const float* wavelet, int n_rec, const int32_t* rx, const int32_t* rz,
                     void* seis_P, void* seis_S, int snap_interval, void* snaps_P, void* snaps_S,
                     void* medium_out) {
  return ORACLE_PREC_DISPATCH(
      prec,
      run_coupled2d<float>(nx, nz, vp, vs, dh, dt, nt, nbc, fd_order, v_ref_p, v_ref_s,
                           smooth_sigma, n_src, sx, sz, wavelet, n_rec, rx, rz, (float*)seis_P,
                           (float*)seis_S, snap_interval, (float*)snaps_P, (float*)snaps_S,
                           (float*)medium_out),
      run_coupled2d<double>(nx, nz, vp, vs, dh, dt, nt, nbc, fd_order, v_ref_p, v_ref_s,
                            smooth_sigma, n_src, sx, sz, wavelet, n_rec, rx, rz, (double*)seis_P,
                            (double*)seis_S, snap_interval, (double*)snaps_P, (double*)snaps_S,
                            (double*)medium_out));
}

// sponge_table for the tests (boundary/sponge.jl:31-48).
int oracle_sponge_table(int nbc, float factor, float* out) {
  std::vector<float> t = sponge_table(nbc, factor);
  std::copy(t.begin(), t.end(), out);
  return 0;
}

int oracle_scalar2d(int prec, int nx, int nz, const float* vp, float dh, float dt, int nt,
                    int nbc, int fd_order, float v_ref, int n_src, const int32_t* sx,
                    const int32_t* sz, const float* wavelet, int n_rec, const int32_t* rx,
                    const int32_t* rz, void* seis_u, void* final_fields) {
  return ORACLE_PREC_DISPATCH(
      prec,
      run_scalar2d<float>(nx, nz, vp, dh, dt, nt, nbc, fd_order, v_ref, n_src, sx, sz, wavelet,
                          n_rec, rx, rz, (float*)seis_u, (float*)final_fields),
      run_scalar2d<double>(nx, nz, vp, dh, dt, nt, nbc, fd_order, v_ref, n_src, sx, sz, wavelet,
                           n_rec, rx, rz, (double*)seis_u, (double*)final_fields));
}


int oracle_acoustic3d(int prec, int nx, int ny, int nz, const float* vp, const float* rho, float dh,
                      float dt, int nt, int nbc, int fd_order, float v_ref, int n_src,
                      const int32_t* sx, const int32_t* sy, const int32_t* sz, const float* wavelet,
                      int n_rec, const int32_t* rx, const int32_t* ry, const int32_t* rz, void* svx,
                      void* svy, void* svz, int snap_interval, int snap_plane, int snap_index,
                      void* snaps, void* final_fields) {
  return ORACLE_PREC_DISPATCH(
      prec,
      run_acoustic3d<float>(nx, ny, nz, vp, rho, dh, dt, nt, nbc, fd_order, v_ref, n_src, sx, sy,
                            sz, wavelet, n_rec, rx, ry, rz, (float*)svx, (float*)svy, (float*)svz,
                            snap_interval, snap_plane, snap_index, (float*)snaps,
                            (float*)final_fields),
      run_acoustic3d<double>(nx, ny, nz, vp, rho, dh, dt, nt, nbc, fd_order, v_ref, n_src, sx, sy,
                             sz, wavelet, n_rec, rx, ry, rz, (double*)svx, (double*)svy,
                             (double*)svz, snap_interval, snap_plane, snap_index, (double*)snaps,
                             (double*)final_fields));
}

int oracle_elastic3d(int prec, int nx, int ny, int nz, const float* vp, const float* vs,
                     const float* rho, float dh, float dt, int nt, int nbc, int fd_order,
                     float v_ref, int n_src, const int32_t* sx, const int32_t* sy,
                     const int32_t* sz, const float* wavelet, int n_rec, const int32_t* rx,
                     const int32_t* ry, const int32_t* rz, void* svx, void* svy, void* svz,
                     int snap_interval, int snap_plane, int snap_index, void* snaps,
                     void* final_fields) {
  return ORACLE_PREC_DISPATCH(
      prec,
      run_elastic3d<float>(nx, ny, nz, vp, vs, rho, dh, dt, nt, nbc, fd_order, v_ref, n_src, sx,
                           sy, sz, wavelet, n_rec, rx, ry, rz, (float*)svx, (float*)svy,
                           (float*)svz, snap_interval, snap_plane, snap_index, (float*)snaps,
                           (float*)final_fields),
      run_elastic3d<double>(nx, ny, nz, vp, vs, rho, dh, dt, nt, nbc, fd_order, v_ref, n_src, sx,
                            sy, sz, wavelet, n_rec, rx, ry, rz, (double*)svx, (double*)svy,
                            (double*)svz, snap_interval, snap_plane, snap_index, (double*)snaps,
                            (double*)final_fields));
}

}  // extern "C"
