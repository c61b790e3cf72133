/*
 * fomo_b200.h -- C ABI of libfomo_b200.so, the B200 (sm_100a) time-stepping
 * engine behind Fomo.jl's public solvers.
 *
 * Each entry point replaces one Fomo.jl public function (and the device loop it
 * drives); the Julia host code keeps the reference's signatures and result
 * NamedTuples and `ccall`s these symbols instead of launching CUDA.jl kernels.
 *
 * Conventions (identical to the reference):
 *  - grids are column-major with x fastest: vp[(i-1) + nx*(j-1)] is vp[i, j];
 *  - source / receiver indices are 1-based and UNPADDED, exactly as the user
 *    passes them to Fomo (the library adds the pad offset,
 *    acquisition/source.jl:18-28, receiver.jl:15-19);
 *  - padded sizes are nx + 2*pad with pad = nbc + fd_order/2
 *    (elastic2d/medium.jl:21-26); the HABC zone is pad-1 (habc.jl:38);
 *  - seismograms are (n_rec, nt[, n_shots]) column-major, snapshots are
 *    (nx, nz, nt/snap_interval) interior slices;
 *  - all arithmetic is FP32 unless fomo_opts.precision selects a 16-bit
 *    storage format (FP32 accumulation always).
 *
 * Errors: every call returns FOMO_OK (0) or a negative FOMO_E* code and never
 * aborts; fomo_last_error() gives the message.  FOMO_EARG corresponds to the
 * reference's ArgumentError (utils/checks.jl:8-71).
 *
 * Threading: a fomo_ctx is used by one host thread at a time; it owns a CUDA
 * stream (or borrows the caller's via fomo_set_stream) and a device
 * workspace that grows on demand and is reused across calls.
 */
#ifndef FOMO_B200_H
#define FOMO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FOMO_ABI_VERSION 2

#if defined(__GNUC__)
#define FOMO_API __attribute__((visibility("default")))
#else
#define FOMO_API
#endif

#define FOMO_OK 0
#define FOMO_EARG (-1)        /* invalid argument (reference: ArgumentError)      */
#define FOMO_ECUDA (-2)       /* CUDA runtime error                                */
#define FOMO_ENOMEM (-3)      /* device allocation failed                          */
#define FOMO_ENONFINITE (-4)  /* NaN/Inf sentinel tripped (fomo_opts.check_every) */
#define FOMO_EUNSUPPORTED (-5)

/* fomo_opts.flags */
#define FOMO_F_DEVICE_PTRS 1u /* every array argument is a device pointer */
#define FOMO_F_PROFILE 2u     /* time the sweep kernels of a window of steps  */
#define FOMO_F_STEP_LAUNCH 4u /* launch every time step from the host (no      */
                              /* replayed CUDA-graph chunks; same results)      */
#define FOMO_F_SPONGE 8u      /* boundary = :sponge: Cerjan layer of the user's  */
                              /* nbc cells (boundary/sponge.jl) instead of HABC;  */
                              /* acoustic2d and elastic2d (+ batch), FP32 only    */

/* fomo_opts.precision: storage format of wavefields and material arrays */
#define FOMO_FP32 0
#define FOMO_FP16 1
#define FOMO_BF16 2

/* fomo_opts.kernel: time-step kernel family (0 lets the autotuner pick) */
#define FOMO_KERNEL_AUTO 0
#define FOMO_KERNEL_TWO_PHASE 1    /* velocity sweep + stress sweep per step      */
#define FOMO_KERNEL_SINGLE_SWEEP 2 /* one fused sweep per step (z-marching tiles); */
                                   /* 3D: two TMA-staged half steps per step, each    */
                                   /* with its Higdon boundary fused (AUTO's pick,    */
                                   /* stats: SINGLE_SWEEP)                            */
#define FOMO_KERNEL_ZMARCH 3       /* elastic3d: z-marching velocity and stress       */
                                   /* updates and two-pass Higdon kernels; TWO_PHASE  */
                                   /* = per-cell updates and two-pass Higdon kernels  */
#define FOMO_KERNEL_REPLICA 4      /* elastic2d(_batch): a CUDA C++ replica of the    */
                                   /* reference's CUDA.jl step (batch.jl:157-183:     */
                                   /* 8 launches, strip backups, frame scratch), a    */
                                   /* measurement baseline; AUTO never picks it       */

typedef struct fomo_ctx fomo_ctx;

/* Grid and run parameters shared by the 2D solvers. */
typedef struct fomo_grid2d {
  int32_t nx, nz;    /* interior (unpadded) grid                                */
  float dh, dt;      /* spacing (m), time step (s)                              */
  int32_t nt;        /* time steps                                              */
  int32_t nbc;       /* absorbing layers (reference keyword nbc, default 50)    */
  int32_t fd_order;  /* 2, 4, 6, 8 or 10                                        */
  float v_ref;       /* HABC reference velocity; <= 0 selects min(vp > 0)       */
} fomo_grid2d;

/* Acquisition: sources per shot and a receiver spread shared by all shots. */
typedef struct fomo_acq {
  int32_t n_shots;      /* 1 for the single-shot solvers                        */
  int32_t n_src;        /* sources per shot                                     */
  const int32_t* sx;    /* (n_src, n_shots), 1-based interior indices           */
  const int32_t* sz;
  const float* wavelet; /* (n_src, nt): injected raw (`f += w[q, it]`)          */
  int32_t n_rec;
  const int32_t* rx;    /* (n_rec), 1-based interior indices                    */
  const int32_t* rz;
} fomo_acq;

typedef struct fomo_opts {
  uint32_t flags;       /* FOMO_F_* */
  int32_t precision;    /* FOMO_FP32 / FOMO_FP16 / FOMO_BF16                    */
  int32_t kernel;       /* FOMO_KERNEL_*                                        */
  int32_t check_every;  /* NaN/Inf sentinel every K steps, 0 = off              */
  float* final_state;   /* optional HOST buffer: padded end-of-run wavefields   */
  float sponge_factor;  /* FOMO_F_SPONGE: Cerjan factor (reference default 0.015) */
} fomo_opts;

typedef struct fomo_stats {
  double kernel_time_s; /* CUDA-event time of the time loop (stats.kernel_time_s) */
  double cell_updates;  /* padded cells x nt x shots                              */
  double alg_bytes;     /* algorithmic HBM bytes of the loop                      */
  int32_t n_shots;
  int32_t gpu_launches; /* kernels launched inside the timed loop                 */
  int32_t kernel;       /* kernel family that ran                                 */
  int32_t status;
  double sweep_ms;      /* FOMO_F_PROFILE: mean device time of one step's sweep    */
                        /* kernel(s) over a window of steps, else 0               */
  int32_t sweep_launches; /* sweep kernels per step                               */
  int32_t sweep_config;   /* single-sweep: variant*1000000 + strip*1000 + z-segments */
} fomo_stats;

/* ---- context ---------------------------------------------------------- */
FOMO_API int fomo_version(void);
FOMO_API int fomo_create(fomo_ctx** out, int device);
FOMO_API void fomo_destroy(fomo_ctx* ctx);
FOMO_API const char* fomo_last_error(const fomo_ctx* ctx);
/* Borrow a caller stream (cudaStream_t); NULL returns to the context's own. */
FOMO_API int fomo_set_stream(fomo_ctx* ctx, void* stream);
/* Release the cached device workspace. */
FOMO_API int fomo_trim(fomo_ctx* ctx);

/* ---- host-side checks shared by the language shims -------------------- */
/* CFL bound (utils/checks.jl:39-48 staggered, :61-70 centered when
 * `centered` != 0): writes dt_max and returns FOMO_EARG when dt > dt_max. */
FOMO_API int fomo_check_numerics(float vmax, float dh, float dt, int32_t fd_order, int32_t centered,
                        float* dt_max);

/* ---- solvers -------------------------------------------------------------
 * Outputs are caller-owned, sized (n_rec, nt, n_shots); `snaps` may be NULL.
 * opts may be NULL (FP32, host pointers, autotuned kernel).
 */

/* acoustic2d (equations/acoustic2d/acoustic2d.jl:47-192; HABC graph/fused loop
 * loop_graph.jl:12-76, fused_kernels.jl:166-197).  acq->n_shots must be 1;
 * acq->n_src sources fire together.  Snapshots hold the interior of p. */
FOMO_API int fomo_acoustic2d(fomo_ctx* ctx, const fomo_grid2d* g, const float* vp, const float* rho,
                    const fomo_acq* acq, int32_t snap_interval, float* seis_p, float* seis_vx,
                    float* seis_vz, float* snaps, const fomo_opts* opts, fomo_stats* stats);

/* acoustic2d_batch (equations/acoustic2d/batch.jl:180-261): n_shots shots of
 * n_src sources each on one shared model. */
FOMO_API int fomo_acoustic2d_batch(fomo_ctx* ctx, const fomo_grid2d* g, const float* vp, const float* rho,
                          const fomo_acq* acq, float* seis_p, float* seis_vx, float* seis_vz,
                          const fomo_opts* opts, fomo_stats* stats);

/* elastic2d (equations/elastic2d/elastic2d.jl:45-163; loops fused_kernels.jl:200-240,
 * loop_graph.jl:12-75).  Sources inject into txx and tzz; snapshots hold vz. */
FOMO_API int fomo_elastic2d(fomo_ctx* ctx, const fomo_grid2d* g, const float* vp, const float* vs,
                   const float* rho, const fomo_acq* acq, int32_t snap_interval, float* seis_vx,
                   float* seis_vz, float* snaps, const fomo_opts* opts, fomo_stats* stats);

/* elastic2d_batch (equations/elastic2d/batch.jl:197-261). */
FOMO_API int fomo_elastic2d_batch(fomo_ctx* ctx, const fomo_grid2d* g, const float* vp, const float* vs,
                         const float* rho, const fomo_acq* acq, float* seis_vx, float* seis_vz,
                         const fomo_opts* opts, fomo_stats* stats);

/* scalar2d (equations/scalar2d/scalar2d.jl:104-189).  The wavelet matrix is
 * already scaled as `source_scale` asks (the shim does :v2dt2 / :dt). */
FOMO_API int fomo_scalar2d(fomo_ctx* ctx, const fomo_grid2d* g, const float* vp, const fomo_acq* acq,
                  float* seis_u, const fomo_opts* opts, fomo_stats* stats);

/* ---- uneven-size batch -----------------------------------------------------
 * No single counterpart in the reference: acoustic2d_batch
 * (equations/acoustic2d/batch.jl:180-261) needs one shared model, so shots on
 * grids of different size are separate acoustic2d calls there.  Here each
 * shot brings its own model and acquisition and all shots step together in
 * one graph-captured run.  Every shot's seismograms equal a single
 * fomo_acoustic2d run of that shot bit for bit. */
typedef struct fomo_shot2d {
  int32_t nx, nz;        /* interior grid of this shot                          */
  const float* vp;       /* (nx, nz) host arrays                                */
  const float* rho;
  int32_t n_src;         /* sources firing together                             */
  const int32_t* sx;     /* (n_src), 1-based interior indices                   */
  const int32_t* sz;
  const float* wavelet;  /* (n_src, nt), injected raw                           */
  int32_t n_rec;
  const int32_t* rx;     /* (n_rec), 1-based interior indices                   */
  const int32_t* rz;
  float v_ref;           /* <= 0 selects min(vp > 0) of this shot               */
  float* seis_p;         /* (n_rec, nt) host outputs, each may be NULL          */
  float* seis_vx;
  float* seis_vz;
} fomo_shot2d;

/* Host arrays only (FOMO_F_DEVICE_PTRS returns FOMO_EUNSUPPORTED); FP32.
 * stats->sweep_config = tile width * 1000 + tile height of the chosen tiles. */
FOMO_API int fomo_acoustic2d_uneven(fomo_ctx* ctx, float dh, float dt, int32_t nt, int32_t nbc,
                                    int32_t fd_order, int32_t n_shots, const fomo_shot2d* shots,
                                    const fomo_opts* opts, fomo_stats* stats);

/* ---- 3D solvers ------------------------------------------------------------ */
typedef struct fomo_grid3d {
  int32_t nx, ny, nz; /* interior grid                                          */
  float dh, dt;
  int32_t nt, nbc, fd_order;
  float v_ref;        /* <= 0 selects min(vp > 0)                               */
} fomo_grid3d;

typedef struct fomo_acq3d {
  int32_t n_src;        /* sources (fire together)                              */
  const int32_t* sx;    /* (n_src), 1-based interior indices                    */
  const int32_t* sy;
  const int32_t* sz;
  const float* wavelet; /* (n_src, nt), injected raw                            */
  int32_t n_rec;
  const int32_t* rx;    /* (n_rec), 1-based interior indices                    */
  const int32_t* ry;
  const int32_t* rz;
} fomo_acq3d;

/* acoustic3d (equations/acoustic3d/acoustic3d.jl:37-185) and elastic3d
 * (equations/elastic3d/elastic3d.jl:37-162).  Seismograms (n_rec, nt) of vx,
 * vy, vz.  Snapshots every snap_interval steps of p (acoustic) or vz (elastic)
 * on the plane snap_plane (0 :xz at y = snap_index, 1 :xy at z, 2 :yz at x;
 * snap_index 1-based, 0 selects ny/2 as the reference does), laid out
 * (nx, nz) / (nx, ny) / (ny, nz) per snapshot, nt / snap_interval of them.
 * The HABC is the reference's 3D Higdon formula (boundary/habc/kernels_3d.jl)
 * evaluated two-pass, so results are deterministic.  FP32 only.
 * opts->final_state receives (nxp, nyp, nzp, nfield) padded fields:
 * acoustic vx,vy,vz,p; elastic vx,vy,vz,txx,tyy,tzz,txy,txz,tyz. */
FOMO_API int fomo_acoustic3d(fomo_ctx* ctx, const fomo_grid3d* g, const float* vp, const float* rho,
                             const fomo_acq3d* acq, int32_t snap_interval, int32_t snap_plane,
                             int32_t snap_index, float* seis_vx, float* seis_vy, float* seis_vz,
                             float* snaps, const fomo_opts* opts, fomo_stats* stats);
FOMO_API int fomo_elastic3d(fomo_ctx* ctx, const fomo_grid3d* g, const float* vp, const float* vs,
                            const float* rho, const fomo_acq3d* acq, int32_t snap_interval,
                            int32_t snap_plane, int32_t snap_index, float* seis_vx, float* seis_vy,
                            float* seis_vz, float* snaps, const fomo_opts* opts, fomo_stats* stats);

/* ---- z-slab decomposition of one 3D model ------------------------------------
 * No reference counterpart: Fomo advances a 3D model on one device
 * (equations/elastic3d/elastic3d.jl:37-162, acoustic3d/acoustic3d.jl:37-185).
 * Here a model may be split into z-slabs, one per GPU.  Each slab advances
 * with the fused half steps; between half steps the caller exchanges halo
 * planes with the neighbouring slabs (contiguous plane blocks: NCCL send/recv,
 * or device copies when several slabs share a device).  Every slab's owned
 * planes and seismograms then equal the single-device run's bit for bit.
 *
 * Planes are global padded z indices 0 .. nzp-1 (nzp = nz + 2 (nbc + fd_order/2)).
 * A slab owns [z_lo, z_hi) and holds [z_base, z_base + nz_local) =
 * [max(z_lo - halo, 0), min(z_hi + halo, nzp)), halo = fd_order / 2.  Cuts
 * between slabs lie in [cut_min, cut_max] = [pad + 1, nzp - pad - 1]
 * (pad = nbc + fd_order / 2): clear of the z bands of the Higdon boundary and
 * of the plane each band's z terms read, which would otherwise need the
 * neighbour's half-step values.  A slab with a neighbour owns at least `halo`
 * planes.
 *
 * Halo exchange after each half step of step it (1-based), set B = it % 2:
 *   half 0 (velocity): elastic fields 0 1 2 (vx vy vz), acoustic field 2 (vz);
 *   half 1 (stress / pressure, after injection and recording): elastic 7 8 5
 *     (txz tyz tzz), acoustic 3 (p).
 * Field f of set s is the volume state + (s * nfield + f) * plane * nz_local.
 * A slab sends its first / last `halo` owned planes to the slab above / below
 * and receives the `halo` planes next to its owned range.
 *
 * fomo_slab3d_layout_of: the slab's layout, or FOMO_EARG (message on ctx,
 * which may be NULL) when the cut is not allowed.
 * fomo_slab3d_create: vp, vs (elastic only), rho are the full HOST raw models
 * (nx, ny, nz), of which the slab uploads the planes it needs; acq is the full
 * HOST acquisition (points outside the owned planes are left to other slabs);
 * g->v_ref <= 0 scans vp for min(vp > 0) as fomo_elastic3d does.  `state` is
 * caller device memory of layout.state_floats floats (16-byte aligned), which
 * the slab zeroes and keeps using until it is destroyed.  Kernels run on the
 * context's stream (fomo_set_stream); ctx must outlive the slab.
 * fomo_slab3d_step: half 0 velocity, half 1 stress / pressure then injection
 * and recording, for step it (1..nt).
 * fomo_slab3d_seismograms: waits for the stream, then copies the (n_rec, nt)
 * seismograms to HOST arrays (receivers of other slabs read 0) and sets
 * owned[r] = 1 for the receivers this slab records.  Reports FOMO_ECUDA if a
 * bounded wait inside a half step timed out. */
typedef struct fomo_slab3d fomo_slab3d;
typedef struct fomo_slab3d_layout {
  int32_t nxp, nyp, nzp;    /* padded global grid                             */
  int32_t ld;               /* x pitch (floats)                               */
  int64_t plane;            /* floats per plane (ld * nyp)                    */
  int32_t z_lo, z_hi;       /* owned planes                                   */
  int32_t z_base, nz_local; /* planes held                                    */
  int32_t halo;             /* halo depth (fd_order / 2)                      */
  int32_t nfield;           /* fields per set: 9 elastic, 4 acoustic          */
  int32_t cut_min, cut_max; /* allowed cut planes                             */
  int64_t state_floats;     /* 2 * nfield * plane * nz_local                  */
} fomo_slab3d_layout;

FOMO_API int fomo_slab3d_layout_of(fomo_ctx* ctx, int32_t elastic, const fomo_grid3d* g,
                                   int32_t z_lo, int32_t z_hi, fomo_slab3d_layout* out);
FOMO_API int fomo_slab3d_create(fomo_ctx* ctx, int32_t elastic, const fomo_grid3d* g,
                                const float* vp, const float* vs, const float* rho,
                                const fomo_acq3d* acq, int32_t z_lo, int32_t z_hi, float* state,
                                fomo_slab3d** out);
FOMO_API int fomo_slab3d_step(fomo_slab3d* slab, int32_t it, int32_t half);
FOMO_API int fomo_slab3d_seismograms(fomo_slab3d* slab, float* seis_vx, float* seis_vy,
                                     float* seis_vz, uint8_t* owned);
FOMO_API void fomo_slab3d_destroy(fomo_slab3d* slab);

/* ---- learned coarse-grid corrector ------------------------------------------
 * No reference counterpart.  A 3-layer 3x3 CNN (6 -> 16 -> 16 -> 1 channels,
 * bias-free, ReLU between layers; BF16 tensor-core implicit GEMM with FP32
 * accumulation) predicts a per-step correction of u^{n+1} on a coarse grid
 * from the features (u^n, u^{n-1}, c2 u^n, c2^2 u^n, s^{n+1}, s^n), with
 * c2 = (vp dt / dh)^2 and s the values injected at the source cells.
 * Parameters: fomo_corr_param_count() FP32 values, W1[9][6][16] then
 * W2[9][16][16] then W3[9][16], index [tap = 3*dz + dx][in][out].
 * Images are (n, h, w) with x fastest; features are BF16 (n, h, w, 16).
 * All pointers of the fomo_corr_* calls are DEVICE pointers on the
 * context's stream. */
FOMO_API int fomo_corr_param_count(void);
/* Features of n windows (h x w, row pitch ld) of the wavefields: window k
 * starts at u_off[k] (or k*u_stride when u_off is NULL) in u and in u_prev,
 * at c2_off[k] (or k*c2_stride) in c2; values are multiplied by scale[k]
 * (NULL = 1).  Window k holds n_src source cells (x, z) at src[2(k n_src + q)]
 * (window coordinates) that received inj_next[k n_src + q] in this step and
 * inj_prev[k n_src + q] in the previous one (either may be NULL = 0). */
FOMO_API int fomo_corr_features(fomo_ctx* ctx, int32_t n, int32_t h, int32_t w, const float* u,
                                const float* u_prev, const float* c2, int64_t ld,
                                const int64_t* u_off, int64_t u_stride, const int64_t* c2_off,
                                int64_t c2_stride, const float* scale, int32_t n_src,
                                const int32_t* src, const float* inj_next, const float* inj_prev,
                                uint16_t* feat);
/* Training target of the same windows: scale[k] * (u_next - (scalar2d step of
 * (u, u_prev) + inj[k] at the window cell src[2k], src[2k+1])), using the
 * solver's own arithmetic; mask = 0 (target 0) within max(fd_order/2, 3) of
 * the window edge and within src_r of the source, else 1. */
FOMO_API int fomo_corr_target(fomo_ctx* ctx, int32_t n, int32_t h, int32_t w, int32_t fd_order,
                              const float* u, const float* u_prev, const float* u_next,
                              const float* c2, int64_t ld, const int64_t* u_off, int64_t u_stride,
                              const int64_t* c2_off, int64_t c2_stride, const float* scale,
                              const int32_t* src, const float* inj, int32_t src_r, float* target,
                              float* mask);
FOMO_API int fomo_corr_forward(fomo_ctx* ctx, int32_t n, int32_t h, int32_t w,
                               const uint16_t* feat, const float* params, float* y);
/* loss = mean over pixels of (mask * (y - target))^2 (mask may be NULL) and its
 * gradient with respect to the parameters; w % 16 == 0; y_out may be NULL. */
FOMO_API int fomo_corr_gradients(fomo_ctx* ctx, int32_t n, int32_t h, int32_t w,
                                 const uint16_t* feat, const float* target, const float* mask,
                                 const float* params, float* grad, float* loss, float* y_out);
FOMO_API int fomo_corr_adam(fomo_ctx* ctx, int32_t count, float* params, const float* grad,
                            float* m, float* v, float lr, float beta1, float beta2, float eps,
                            int32_t step);

/* scalar2d that also writes the interior wavefield every snap_every steps from
 * step snap_from on, sampled every `stride` cells from interior (1,1), as
 * (ceil(nx/stride), ceil(nz/stride), count) into `snaps`.  Requires
 * FOMO_F_DEVICE_PTRS.  Produces the training pairs of the corrector. */
FOMO_API int fomo_scalar2d_snapshots(fomo_ctx* ctx, const fomo_grid2d* g, const float* vp,
                                     const fomo_acq* acq, int32_t snap_from, int32_t snap_every,
                                     int32_t stride, float* snaps, float* seis_u,
                                     const fomo_opts* opts, fomo_stats* stats);
/* scalar2d with the corrector applied to the interior after every step and
 * injection (before recording); params as for fomo_corr_* (host pointer
 * unless FOMO_F_DEVICE_PTRS).  The network sees the interior plus 3 cells of
 * the absorbing zone; the correction is added to interior cells farther than
 * 3 cells from every source.  All-zero parameters give fomo_scalar2d's result
 * bit for bit. */
FOMO_API int fomo_scalar2d_corrected(fomo_ctx* ctx, const fomo_grid2d* g, const float* vp,
                                     const fomo_acq* acq, const float* params, float* seis_u,
                                     const fomo_opts* opts, fomo_stats* stats);

/* ---- allocation-free entry -------------------------------------------------
 * No counterpart in the reference.  scalar2d for callers that cannot allocate
 * device memory (a plugin inside a framework whose allocator owns all device
 * memory, a fixed-budget service): every working buffer lives in one static
 * 32 MiB device array that each GPU loading this library holds until exit, so
 * this call makes no cudaMalloc/cudaFree.  Every array argument (vp, acq's
 * sx/sz/wavelet/rx/rz, seis_u) is a DEVICE pointer; g->v_ref must be > 0;
 * acq->n_shots must be 1; the wavelet is pre-scaled as for fomo_scalar2d.
 * Runs on the calling thread's current device, on `stream` (NULL = default),
 * and returns after the stream has finished the run.  Problems whose working
 * set exceeds the array return FOMO_EARG.  All calls share the array (it keeps
 * the previous call's contents; the wavefields are cleared at each start), so
 * calls that overlap on the GPU race.  Each call looks up the array's address
 * in the current device and context (this allocates nothing), and returns only
 * once the run has finished (synchronous).  As with the other entry points,
 * the reference's time-step checks (centered CFL, utils/checks.jl:61-70) and
 * dispersion warning are the caller's: an unstable dt is not rejected here.
 * `err` (may be NULL) receives a message of at most err_len bytes. */
FOMO_API int fomo_scalar2d_noalloc(const fomo_grid2d* g, const float* vp, const fomo_acq* acq,
                                   float* seis_u, void* stream, char* err, int32_t err_len);

/* ---- coupled P-S potentials -------------------------------------------- */
/* coupled2d (equations/coupled2d/coupled2d.jl:53-171): constant-density coupled
 * P and S potentials on a regular grid with centered differences.  g->v_ref is
 * v_ref_p and v_ref_s the S field's HABC velocity (<= 0: minimum of the
 * positive vp, resp. vs).  smooth_sigma: Gaussian smoothing in grid points of
 * alpha = vp^2 and beta = vs^2 before their derivatives (<= 0: none; radius
 * ceil(3 sigma) <= 1024).  The wavelet (n_src, nt) is added to P.  Host arrays
 * only; FP32; HABC only (the reference's racy HABC in deterministic form).
 * seis_P, seis_S: (n_rec, nt); snaps_P, snaps_S: (nx, nz, nt / snap_interval)
 * or NULL.  acq->n_shots must be 1. */
FOMO_API int fomo_coupled2d(fomo_ctx* ctx, const fomo_grid2d* g, const float* vp,
                            const float* vs, float v_ref_s, double smooth_sigma,
                            const fomo_acq* acq, int32_t snap_interval, float* seis_P,
                            float* seis_S, float* snaps_P, float* snaps_S,
                            const fomo_opts* opts, fomo_stats* stats);

/* ---- diagnostics -------------------------------------------------------- */
/* coupled2d's device medium (coupled2d/medium.jl:46-107) downloaded to `out`,
 * (nx + 2 pad, nz + 2 pad, 8) column-major with pad = nbc + fd_order / 2:
 * alpha, beta, d alpha/dx, d alpha/dz, d beta/dx, d beta/dz, lap alpha, lap beta. */
FOMO_API int fomo_debug_coupled_medium(fomo_ctx* ctx, int32_t nx, int32_t nz, int32_t nbc,
                                       int32_t fd_order, float dh, double smooth_sigma,
                                       const float* vp, const float* vs, float* out);
/* Device-side medium preparation, downloaded to `out` (padded, column-major):
 * kind 0 elastic -> bx,bz,lam,lam2mu,mu_txz; 1 acoustic -> bx,bz,kappa;
 * 2 scalar -> c2.  Mirrors utils/pad_array.jl and equations/<eq>/medium.jl. */
FOMO_API int fomo_debug_medium2d(fomo_ctx* ctx, int32_t kind, int32_t nx, int32_t nz, int32_t pad,
                        float dt, float dh, const float* vp, const float* vs, const float* rho,
                        float* out);

#ifdef __cplusplus
}
#endif

#endif /* FOMO_B200_H */
