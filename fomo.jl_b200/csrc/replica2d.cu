// replica2d.cu -- a CUDA C++ replica of Fomo.jl's CUDA.jl time step for
// elastic2d_batch, kept as a same-hardware measurement baseline
// (fomo_opts.kernel = FOMO_KERNEL_REPLICA; AUTO never picks it).
//
// Julia and CUDA.jl cannot run on this machine, so the reference's GPU path is
// restated here with its own decomposition, launch shapes and memory traffic:
// one step is the eight launches of _elastic2d_loop_batch!
// (equations/elastic2d/batch.jl:157-183), on in-place fields of
// (nx, nz, n_shots) with strip backups, full-grid HABC weight planes and a
// frame scratch buffer:
//   1. _bfused_vel_elastic_cuda!  (batch.jl:38-77): (32, 8) threads per block,
//      grid (nx/32, nz/8, ns); back up vx, vz in the strip, update them;
//   2-3. apply_bhabc_det_2! (boundary/habc/kernels_det_batch.jl:90-133): pass 1
//      evaluates the Higdon value of every frame cell into the scratch, pass 2
//      writes it back (256 threads, grid (frame/256, ns));
//   4. _bfused_str_elastic_cuda!  (batch.jl:95-138): back up and update the
//      stresses from the corrected velocities;
//   5-6. apply_bhabc_det_3! (kernels_det_batch.jl:136-182);
//   7. _binject_pair_kernel! (acquisition/batch_acq.jl:58-80): one thread per
//      source adds the wavelet to txx and tzz;
//   8. _brecord2_kernel! (batch_acq.jl:108-130): one thread per receiver.
// No shared memory, no graph, every operand from global memory, as the CUDA.jl
// kernels do.  The arithmetic is the library's canonical sequence (one fma per
// stencil term, the Higdon helpers), so the replica's results equal the
// oracle's bit for bit; only the decomposition is the reference's.
#include "replica2d.cuh"

namespace fomo {
namespace {

// _habc_frame_ij (boundary/habc/kernels_fused.jl:28-45), 0-based: top band,
// bottom band, then the left and right columns row by row.
__device__ __forceinline__ void frame_xz(int idx, int nx, int nz, int nbc, int& x, int& z) {
  const int wd = nx - 2, nh = wd * nbc;
  if (idx < nh) {
    z = 1 + idx / wd;
    x = 1 + idx % wd;
  } else if (idx < 2 * nh) {
    const int t = idx - nh;
    z = nz - 1 - nbc + t / wd;
    x = 1 + t % wd;
  } else {
    const int t = idx - 2 * nh;
    const int q = t / (2 * nbc), r = t % (2 * nbc);
    z = nbc + 1 + q;
    x = r < nbc ? 1 + r : nx - 1 - nbc + (r - nbc);
  }
}

// _habc_det_value_b (kernels_det_batch.jl:13-48) at frame cell (x, z).
__device__ __forceinline__ float det_value(const float* __restrict__ f,
                                           const float* __restrict__ fo,
                                           const float* __restrict__ w, const HabcDev& h, int x,
                                           int z, int nx, int nz, int ld, int nbc) {
  const bool left = x <= nbc, right = x >= nx - 1 - nbc;
  const bool top = z <= nbc, bottom = z >= nz - 1 - nbc;
  const long long p = (long long)z * ld + x;
  const float wt = w[p], fc = f[p];
  const long long px = left ? p + 1 : p - 1;
  const long long pz = top ? p + ld : p - ld;
  if ((left || right) && (top || bottom))
    return higdon_corner(wt, fc, higdon_side(h, f[px], fo[p], fo[px]),
                         higdon_side(h, f[pz], fo[p], fo[pz]));
  if (left || right) return higdon_edge(wt, fc, higdon_side(h, f[px], fo[p], fo[px]));
  return higdon_edge(wt, fc, higdon_side(h, f[pz], fo[p], fo[pz]));
}

__device__ __forceinline__ bool strip(const Geo2& g, int x, int z) {
  return x <= g.nbc + 1 || x >= g.nx - g.nbc - 2 || z <= g.nbc + 1 || z >= g.nz - g.nbc - 2;
}

template <int N>
__global__ void k_rep_vel(Geo2 g, Coef c, float dtx, float dtz, RepFields w, ElMat m) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= g.nx || z >= g.nz) return;
  const long long so = (long long)blockIdx.z * g.plane;
  const long long p = (long long)z * g.ld + x;
  float* vx = w.vx + so;
  float* vz = w.vz + so;
  if (strip(g, x, z)) {
    w.vx_o[so + p] = vx[p];
    w.vz_o[so + p] = vz[p];
  }
  if (interior2(g, x, z)) {
    const float dxx = dm<N>(w.txx + so, p, 1, c);
    const float dxzz = dm<N>(w.txz + so, p, g.ld, c);
    const float dxzx = dp<N>(w.txz + so, p, 1, c);
    const float dzz = dp<N>(w.tzz + so, p, g.ld, c);
    vx[p] = __fmaf_rn(m.bx[p], __fmaf_rn(dtx, dxx, __fmul_rn(dtz, dxzz)), vx[p]);
    vz[p] = __fmaf_rn(m.bz[p], __fmaf_rn(dtx, dxzx, __fmul_rn(dtz, dzz)), vz[p]);
  }
}

template <int N>
__global__ void k_rep_str(Geo2 g, Coef c, float dtx, float dtz, RepFields w, ElMat m) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= g.nx || z >= g.nz) return;
  const long long so = (long long)blockIdx.z * g.plane;
  const long long p = (long long)z * g.ld + x;
  float* txx = w.txx + so;
  float* tzz = w.tzz + so;
  float* txz = w.txz + so;
  if (strip(g, x, z)) {
    w.txx_o[so + p] = txx[p];
    w.tzz_o[so + p] = tzz[p];
    w.txz_o[so + p] = txz[p];
  }
  if (interior2(g, x, z)) {
    const float dvxdx = dp<N>(w.vx + so, p, 1, c);
    const float dvzdz = dm<N>(w.vz + so, p, g.ld, c);
    const float dvxdz = dp<N>(w.vx + so, p, g.ld, c);
    const float dvzdx = dm<N>(w.vz + so, p, 1, c);
    const float lam = m.lam[p], l2m = m.l2m[p];
    const float ex = __fmul_rn(dvxdx, dtx), ez = __fmul_rn(dvzdz, dtz);
    txx[p] = __fadd_rn(txx[p], __fmaf_rn(l2m, ex, __fmul_rn(lam, ez)));
    tzz[p] = __fadd_rn(tzz[p], __fmaf_rn(lam, ex, __fmul_rn(l2m, ez)));
    txz[p] = __fmaf_rn(m.mut[p], __fmaf_rn(dvxdz, dtz, __fmul_rn(dvzdx, dtx)), txz[p]);
  }
}

// pass 1 of the det-HABC for nf fields (fields f[k], backups fo[k], weights w[k])
__global__ void k_rep_habc1(Geo2 g, HabcDev h, RepHabc a, int nf, int total,
                            float* __restrict__ scr) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int s = blockIdx.y;
  int x, z;
  frame_xz(idx, g.nx, g.nz, g.nbc, x, z);
  const long long so = (long long)s * g.plane;
  for (int k = 0; k < nf; ++k)
    scr[((long long)s * nf + k) * total + idx] =
        det_value(a.f[k] + so, a.fo[k] + so, a.w[k], h, x, z, g.nx, g.nz, g.ld, g.nbc);
}

__global__ void k_rep_habc2(Geo2 g, RepHabc a, int nf, int total,
                            const float* __restrict__ scr) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int s = blockIdx.y;
  int x, z;
  frame_xz(idx, g.nx, g.nz, g.nbc, x, z);
  const long long p = (long long)s * g.plane + (long long)z * g.ld + x;
  for (int k = 0; k < nf; ++k) a.f[k][p] = scr[((long long)s * nf + k) * total + idx];
}

__global__ void k_rep_inject(long long plane, int n_src, const int* __restrict__ src_lin,
                             const float* __restrict__ wav, int it, float* txx, float* tzz) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (q >= n_src) return;
  const long long p = (long long)s * plane + src_lin[(long long)s * n_src + q];
  const float v = wav[(long long)(it - 1) * n_src + q];
  txx[p] = __fadd_rn(txx[p], v);
  tzz[p] = __fadd_rn(tzz[p], v);
}

__global__ void k_rep_record(long long plane, int n_rec, const int* __restrict__ rec_lin, int it,
                             int nt, const float* __restrict__ vx, const float* __restrict__ vz,
                             float* __restrict__ s0, float* __restrict__ s1) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (r >= n_rec) return;
  const long long p = (long long)s * plane + rec_lin[r];
  const long long o = (long long)n_rec * ((long long)(it - 1) + (long long)nt * s) + r;
  if (s0) s0[o] = vx[p];
  if (s1) s1[o] = vz[p];
}

// HABC weight planes w(x, z) = table(kind, dist) of init_habc (habc.jl:17-44)
__global__ void k_rep_weights(Geo2 g, HabcDev h, float* __restrict__ wv, float* __restrict__ wz,
                              float* __restrict__ wt) {
  const long long n = (long long)g.nx * g.nz;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(q / g.nx), x = (int)(q % g.nx);
    const int d = min(min(x, g.nx - 1 - x), min(z, g.nz - 1 - z));
    const long long p = (long long)z * g.ld + x;
    wv[p] = habc_weight(h, 0, d);
    wz[p] = habc_weight(h, 1, d);
    wt[p] = habc_weight(h, 2, d);
  }
}

}  // namespace

long long replica_frame_total(int nx, int nz, int nbc) {
  return 2LL * (nx - 2) * nbc + 2LL * nbc * (nz - 2 * nbc - 2);
}

cudaError_t replica_setup(cudaStream_t st, const Geo2& g, const HabcDev& h, float* wv, float* wz,
                          float* wt) {
  k_rep_weights<<<1184, 256, 0, st>>>(g, h, wv, wz, wt);
  return cudaGetLastError();
}

cudaError_t replica_step(cudaStream_t st, int N, const Geo2& g, const Coef& c, float dtx,
                         float dtz, const HabcDev& h, const RepFields& w, const ElMat& m,
                         const float* w_vx, const float* w_vz, const float* w_tau, float* scr,
                         int ns, int it, int nt, int n_src, const int* src_lin, const float* wav,
                         int n_rec, const int* rec_lin, float* s0, float* s1) {
  const dim3 blk(32, 8), grd(cdiv(g.nx, 32), cdiv(g.nz, 8), ns);
  const int total = (int)replica_frame_total(g.nx, g.nz, g.nbc);
  const dim3 fgrd(cdiv(total, 256), ns);
  switch (N) {
#define FOMO_REP_VEL(NN) \
  case NN: k_rep_vel<NN><<<grd, blk, 0, st>>>(g, c, dtx, dtz, w, m); break;
    FOMO_REP_VEL(1) FOMO_REP_VEL(2) FOMO_REP_VEL(3) FOMO_REP_VEL(4) FOMO_REP_VEL(5)
#undef FOMO_REP_VEL
    default: return cudaErrorInvalidValue;
  }
  RepHabc hv{{w.vx, w.vz, nullptr}, {w.vx_o, w.vz_o, nullptr}, {w_vx, w_vz, nullptr}};
  if (total > 0) {
    k_rep_habc1<<<fgrd, 256, 0, st>>>(g, h, hv, 2, total, scr);
    k_rep_habc2<<<fgrd, 256, 0, st>>>(g, hv, 2, total, scr);
  }
  switch (N) {
#define FOMO_REP_STR(NN) \
  case NN: k_rep_str<NN><<<grd, blk, 0, st>>>(g, c, dtx, dtz, w, m); break;
    FOMO_REP_STR(1) FOMO_REP_STR(2) FOMO_REP_STR(3) FOMO_REP_STR(4) FOMO_REP_STR(5)
#undef FOMO_REP_STR
  }
  RepHabc hs{{w.txx, w.tzz, w.txz}, {w.txx_o, w.tzz_o, w.txz_o}, {w_tau, w_tau, w_tau}};
  if (total > 0) {
    k_rep_habc1<<<fgrd, 256, 0, st>>>(g, h, hs, 3, total, scr);
    k_rep_habc2<<<fgrd, 256, 0, st>>>(g, hs, 3, total, scr);
  }
  if (n_src > 0)
    k_rep_inject<<<dim3(cdiv(n_src, 256), ns), 256, 0, st>>>(g.plane, n_src, src_lin, wav, it,
                                                              w.txx, w.tzz);
  if (n_rec > 0)
    k_rep_record<<<dim3(cdiv(n_rec, 256), ns), 256, 0, st>>>(g.plane, n_rec, rec_lin, it, nt,
                                                              w.vx, w.vz, s0, s1);
  return cudaGetLastError();
}

}  // namespace fomo
