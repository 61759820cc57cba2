/*
 * gnss_b200.h -- C ABI of the B200-native pseudospectral temporal-jet step.
 *
 * Drop-in for the operator surface of the reference solver (mfkiwl/gnss-1):
 * the 3D transforms of fftfuncs.cu and the spectral / physical operators and
 * time step of solver.cu.  Every entry point cites the reference function it
 * replaces.  Buffers use the reference's layouts:
 *
 *   spectral field  complex [ny][nx][nz2], index kz + nz2*(x + nx*y)   (solver.cu:25)
 *   physical field  real    [nx][ny][2*nz2], index z + 2*nz2*(y + ny*x) (cudafuncs.cu:14-17)
 *
 * with nz2 = nz/2 + 1; a field buffer holds nx*ny*nz2 complex values and is
 * used in place for both views, exactly like the reference.  Element type is
 * double (GNSS_FP64) or float (GNSS_FP32) per the context's precision.
 * Device pointers must be aligned to one complex element (16 bytes for FP64,
 * 8 for FP32); misaligned pointers are rejected with GNSS_ERR_INVALID.
 *
 * Differences from the reference, all deliberate:
 *   - sizes and parameters are runtime values (gnss_config) instead of the
 *     compile-time macros of dnsparams.h;
 *   - every call takes an explicit CUDA stream (cudaStream_t passed as void*,
 *     NULL = legacy default stream) and returns a gnss_status instead of
 *     printing and returning void;
 *   - scratch memory (the reference's fft.temp / fft.wspace / rhs / temp
 *     buffers) is owned by the context.
 *
 * Thread safety: a context may be used by one host thread at a time; calls
 * on one context are ordered on the stream they are given.
 */
#ifndef GNSS_B200_H
#define GNSS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int gnss_status;
#define GNSS_OK 0
#define GNSS_ERR_INVALID 1       /* bad argument, unsupported size or configuration */
#define GNSS_ERR_CUDA 2          /* a CUDA runtime call or kernel launch failed       */
#define GNSS_ERR_NOMEM 3         /* device or pinned allocation failed                */
#define GNSS_ERR_UNSUPPORTED 4   /* operation not available for this configuration    */
#define GNSS_ERR_TIMEOUT 5       /* a bounded device-side wait gave up (see gnss_check) */

#define GNSS_SCHEME_CNAB2 0      /* reference scheme: Euler/CN first step, AB2/CN after (solver.cu:547-616) */
#define GNSS_SCHEME_RK3IF 1      /* low-storage RK3 (Wray) with integrating factor exp(-nu k^2 dt)          */

#define GNSS_FP64 0
#define GNSS_FP32 1

typedef struct gnss_config {
    int nx, ny, nz;          /* grid; each 2^a 3^b, even, 8..512                                */
    double lx, ly, lz;       /* box lengths (reference LX, LY, LZ)                              */
    double re;               /* velocity diffusivity 1/re (reference Re)                        */
    double sc;               /* scalar s diffusivity 1/(re*sc) (reference Sc)                   */
    double sc_c;             /* scalar c diffusivity 1/(re*sc_c) (reference Sc_c)               */
    double alpha;            /* drift coefficient of c (reference alpha)                        */
    double dt;               /* time step (reference dt)                                        */
    double alias_filter;     /* modes with k^2 > (alias_filter*nx*pi/lx)^2 are zeroed           */
    double nu_stats;         /* viscosity used by the statistics (reference nu = H/Re)          */
    int n_scalars;           /* 1: s only; 2: s and c                                          */
    int scheme;              /* GNSS_SCHEME_*                                                   */
    int precision;           /* GNSS_FP64 or GNSS_FP32                                          */
    int device;              /* CUDA device ordinal                                             */
} gnss_config;

/* Device pointers to the spectral fields of one state (or one set of RHS /
 * history fields).  c may be NULL when n_scalars == 1. */
typedef struct gnss_fields {
    void *u, *v, *w, *s, *c;
} gnss_fields;

typedef struct gnss_ctx gnss_ctx;

/* Statistics written by gnss_stats (statistics.cu:1494-1845 definitions). */
#define GNSS_STAT_KE 0       /* 1/2 sum |u_hat|^2 / NN^2             (calcVrms, statistics.cu:1549)            */
#define GNSS_STAT_VRMS2 1    /* sum |u_hat|^2 / (3 NN^2)             (calcVrms, statistics.cu:1551)            */
#define GNSS_STAT_EPS 2      /* nu_stats sum k^2 |u_hat|^2 / NN^2    (calcEpsilonKernel, statistics.cu:1637)   */
#define GNSS_STAT_CHI_S 3    /* 2 nu_stats/sc sum k^2|s_hat|^2/NN^2  (calcScalarDissipation, statistics.cu:1813) */
#define GNSS_STAT_CHI_C 4    /* same for c with sc_c                                                              */
#define GNSS_STAT_VAR_S 5    /* sum_{k != 0} |s_hat|^2 / NN^2        (scalar variance; not in the reference)     */
#define GNSS_STAT_VAR_C 6
#define GNSS_NSTATS 7

/* Create a context: validates the configuration, builds twiddle tables and
 * wavenumber constants.  Replaces plan1dFFT / plan2dFFT (fftfuncs.cu:133-231)
 * and initializeWaveNumbers (initialize.cu:693-707). */
gnss_status gnss_create(const gnss_config *cfg, gnss_ctx **out);
/* Release a context and all memory it owns (cufftDestroy in allocate.cu:297-301). */
gnss_status gnss_destroy(gnss_ctx *ctx);
/* The configuration a context was created with. */
gnss_status gnss_get_config(const gnss_ctx *ctx, gnss_config *out);
/* Bytes of one field buffer (nx*ny*nz2 complex of the context's precision). */
size_t gnss_field_bytes(const gnss_ctx *ctx);
/* Bytes of device memory the context owns right now. */
size_t gnss_workspace_bytes(const gnss_ctx *ctx);
const char *gnss_status_string(gnss_status st);
/* Human-readable description of the last error seen by this context. */
const char *gnss_last_error(const gnss_ctx *ctx);

/* 3D transforms, in place on one field buffer.
 * forward: physical -> spectral, unnormalised   (forwardTransform, fftfuncs.cu:288-320)
 * inverse: spectral -> physical, scaled by 1/(nx ny nz) (inverseTransform, fftfuncs.cu:322-359) */
gnss_status gnss_forward(gnss_ctx *ctx, void *field, void *stream);
gnss_status gnss_inverse(gnss_ctx *ctx, void *field, void *stream);

/* Spectral operators on spectral fields. */
gnss_status gnss_dealias(gnss_ctx *ctx, void *field, void *stream);                 /* deAliasKernel_mgpu, solver.cu:17-42  */
gnss_status gnss_vorticity(gnss_ctx *ctx, const void *uh, const void *vh, const void *wh,
                           void *o1, void *o2, void *o3, void *stream);             /* vorticity, solver.cu:68-137           */
gnss_status gnss_gradient(gnss_ctx *ctx, const void *fh, void *fx, void *fy, void *fz,
                          void *stream);                                              /* gradient, solver.cu:233-273           */
gnss_status gnss_divergence(gnss_ctx *ctx, const void *fx, const void *fy, const void *fz,
                            void *out, void *stream);                                 /* divergence, solver.cu:275-307         */
gnss_status gnss_make_rhs(gnss_ctx *ctx, void *ru, void *rv, void *rw, void *rs, void *rc,
                          void *stream);                                              /* makeRHS, solver.cu:461-544            */
/* CN time update of every field of `state` from `rhs` (and `rhs_old` when
 * euler == 0) (timestep, solver.cu:547-616). */
gnss_status gnss_timestep(gnss_ctx *ctx, int euler, const gnss_fields *state, const gnss_fields *rhs,
                          const gnss_fields *rhs_old, void *stream);
/* rhs_old <- rhs; rhs <- 0 (update, solver.cu:618-657). */
gnss_status gnss_update(gnss_ctx *ctx, const gnss_fields *rhs, const gnss_fields *rhs_old, void *stream);

/* Physical-space operators on physical (real, padded) fields. */
gnss_status gnss_cross_product(gnss_ctx *ctx, const void *u, const void *v, const void *w,
                               void *o1, void *o2, void *o3, void *stream);       /* crossProduct: o <- o x u, solver.cu:139-185 */
gnss_status gnss_dot_product(gnss_ctx *ctx, const void *a1, const void *a2, const void *a3,
                             const void *b1, const void *b2, const void *b3, void *out,
                             void *stream);                                          /* dotProduct, solver.cu:342-372 */
gnss_status gnss_colloid_advection(gnss_ctx *ctx, const void *u, const void *v, const void *w,
                                   const void *c, const void *cx, const void *cy, const void *cz,
                                   const void *sx, const void *sy, const void *sz, void *lap_s_inout,
                                   void *stream);                                    /* colloidAdvection, solver.cu:374-405 */

/* One full time step of the fused B200 path (solver_ps, solver.cu:700-765).
 * The transforms are pruned to the dealiasing truncation: state modes whose
 * wavenumber along any axis exceeds the truncation radius are neither read
 * nor written, so they must be zero on entry (gnss_dealias does that, as the
 * reference does once before its loop, main.cu:156, and at the start of
 * every step, solver.cu:704).  Within the kept box the spherical mask is
 * applied on input, so masked modes of the state never enter the step.  The
 * Euler step (euler != 0) writes exact zeros to the masked modes of state and
 * history inside the box; the other steps update only the modes inside the
 * sphere and leave the masked ones as they are (zero, for a dealiased state
 * and a history written by an earlier step).
 * state: spectral u, v, w, s (and c).  hist: for GNSS_SCHEME_CNAB2 the
 * previous RHS (the reference's rhs_old; read when euler == 0, always
 * written); unused (may be NULL) for GNSS_SCHEME_RK3IF.  euler selects the
 * reference's first-step Euler/CN update (main.cu:181-186). */
gnss_status gnss_step(gnss_ctx *ctx, const gnss_fields *state, const gnss_fields *hist, int euler, void *stream);

/* Spectral statistics of a state; writes GNSS_NSTATS doubles to host memory
 * and synchronises the stream (calcVrms, calcDissipationRate,
 * calcScalarDissipationRate: statistics.cu:1494-1845). */
gnss_status gnss_stats(gnss_ctx *ctx, const gnss_fields *state, double *out, void *stream);

/* Turbulence statistics of a state (calcTurbStats_mgpu, statistics.cu:2039-2156),
 * with the reference's definitions (nu = cfg.nu_stats):
 *   vrms     sqrt(sum |u_hat|^2 / (3 NN^2))                     (calcVrms, :1551, 1582)
 *   ke       1/2 sum |u_hat|^2 / NN^2                           (:1549)
 *   epsilon  nu sum k^2 |u_hat|^2 / NN^2                        (calcEpsilonKernel_mgpu)
 *   eta      (nu^3 / epsilon)^(1/4)                             (:2149)
 *   l        3 pi/4 sum_{k != 0} |u_hat|^2/(2 |k| NN^2) / ke    (calcIntegralLength, :2150)
 *   lambda   sqrt(15 nu vrms^2 / epsilon)                       (:2148)
 *   chi      2 nu/sc sum k^2 |s_hat|^2 / NN^2                    (calcScalarDissipationRate)
 *   omega    volume average of |curl u|                         (:2097-2106)
 *   omega_x, omega_y, omega_z  rms of each vorticity component (:2103-2105)
 * Spectral sums run over the full spectrum (kz mirror), the vorticity
 * statistics over the grid points, both in a fixed order.  yprof (may
 * be NULL) receives 5 x ny doubles: the mean profiles along y (averages over
 * x and z) of u, v, w, s, c (zeros for a missing c) (calcYprof, :1943-2003).
 * Uses four scratch fields of the context; synchronises the stream. */
typedef struct gnss_turb {
    double vrms, ke, epsilon, eta, l, lambda, chi, omega, omega_x, omega_y, omega_z;
} gnss_turb;
gnss_status gnss_turb_stats(gnss_ctx *ctx, const gnss_fields *state, gnss_turb *out, double *yprof, void *stream);

/* gnss_step (solver_ps, solver.cu:700-765) together with gnss_turb_stats of
 * the state the step starts from (calcTurbStats_mgpu, statistics.cu:2039-2156,
 * which the reference calls on the state between steps).  Where the register
 * z kernel serves the context, the vorticity statistics are summed by the
 * step's own z kernel from the physical vorticity it forms for the nonlinear
 * term, so they cost no transforms; elsewhere they come from three inverse
 * transforms before the step, as in gnss_turb_stats.  For a dealiased state
 * (the precondition of the step) the statistics equal gnss_turb_stats to
 * round-off and the new state equals gnss_step's.  Synchronises the stream. */
gnss_status gnss_step_turb(gnss_ctx *ctx, const gnss_fields *state, const gnss_fields *hist, int euler,
                           gnss_turb *out, double *yprof, void *stream);

/* End-to-end call with host buffers: copies the packed host state
 * (3 + n_scalars spectral fields back to back) to context-owned device
 * buffers, dealiases it (main.cu:156), runs n_steps steps (the first one
 * Euler when first_euler != 0 for
 * GNSS_SCHEME_CNAB2; hist starts at zero), records the statistics after each
 * step into stats_out (n_steps * GNSS_NSTATS doubles, may be NULL) and copies
 * the final state back into host_state_out (may alias host_state_in).
 * Only the modes a dealias can keep (the box |kx|, |ky|, |kz| <= the
 * truncation radius) are read from host_state_in; the result is the same as
 * uploading everything.  The modes outside that box, zero after the dealias,
 * are written to host_state_out on a second stream while the steps run, the
 * box after the last step.  The statistics are summed by the update kernel of
 * each step and read back once, after the last step; they equal gnss_stats
 * of the same state to round-off.  Synchronises the stream before returning. */
gnss_status gnss_run_host(gnss_ctx *ctx, const void *host_state_in, void *host_state_out, int n_steps,
                          int first_euler, double *stats_out, void *stream);

/* State bytes one gnss_run_host call copies host-to-device (the kept box of
 * every field) and device-to-host (the whole packed state), statistics
 * excluded.  No counterpart in the reference. */
gnss_status gnss_run_host_bytes(gnss_ctx *ctx, size_t *h2d_bytes, size_t *d2h_bytes);

/* Synchronises the stream and reports GNSS_ERR_TIMEOUT if any kernel of this
 * context gave up a bounded wait since the last check (the flag is then
 * cleared).  No counterpart in the reference, which has no device-side waits.
 * gnss_stats and gnss_run_host perform this check themselves. */
gnss_status gnss_check(gnss_ctx *ctx, void *stream);

/* Instrumentation (no counterpart in the reference, which only brackets its
 * loop with cudaProfilerStart/Stop, main.cu:171,249).
 * gnss_launch_count: kernels this context has launched so far.
 * gnss_profile_enable: when on, gnss_step records CUDA events around each of
 * its stages (x inverse, y inverse, z physical, y forward, x forward,
 * spectral update) on the step's stream.
 * gnss_profile_read: synchronises, then returns for each stage the summed
 * device time in ms and the number of launches since profiling was enabled
 * (arrays of GNSS_NSTAGES entries), and clears the record. */
#define GNSS_NSTAGES 6
long long gnss_launch_count(const gnss_ctx *ctx);
/* Algorithmic HBM bytes of one launch of each stage of gnss_step (the
 * compulsory reads and writes of the pruned layouts; GNSS_NSTAGES doubles),
 * for roofline accounting. */
gnss_status gnss_stage_bytes(const gnss_ctx *ctx, double *bytes);
gnss_status gnss_profile_enable(gnss_ctx *ctx, int on);
gnss_status gnss_profile_read(gnss_ctx *ctx, double *ms, long long *launches);

/* Kernel variant options of a context (the knobs the autotuner sets; no
 * counterpart in the reference, which has one cuFFT plan per size).
 * GNSS_OPT_ZVARIANT picks the kernel of the fused z stage, GNSS_OPT_PVARIANT
 * the kernel of the strided x and y passes (of the step and of the 3D
 * transforms):
 *   GNSS_VARIANT_AUTO      the kernel measured fastest on B200: register-
 *                          resident transforms where they fit (z: every N
 *                          below, with separate inverse and forward warps
 *                          in FP64 where that kernel exists; x / y passes:
 *                          N = 96 .. 512 in FP32, 256 and 512 in FP64),
 *                          staged otherwise;
 *   GNSS_VARIANT_REGISTER  register-resident transforms where they exist
 *                          (N = 64, 96, 128, 192 with lane shuffles only;
 *                          N = 256, 512 with one transpose) and fit (a
 *                          request, not a guarantee);
 *   GNSS_VARIANT_STAGED    per-radix-stage transforms through shared memory;
 *   GNSS_VARIANT_WARPSPEC  (GNSS_OPT_ZVARIANT only) the register z kernel
 *                          with separate inverse and forward warps, where it
 *                          exists (z length 256 or 512, no colloid term; FP32
 *                          with one scalar, FP64 with one or two); the
 *                          register kernel otherwise;
 *   GNSS_VARIANT_TENSOR    (GNSS_OPT_PVARIANT only) line transforms on the
 *                          tensor cores as split-TF32 DFT-matrix GEMMs
 *                          (tcgen05, three TF32 products per GEMM with FP32
 *                          accumulation) where they exist: FP32, x / y
 *                          lengths 256 and 512; the AUTO choice elsewhere.
 * Every variant computes the same step to round-off (the tensor-core
 * variant to FP32 accuracy: it replaces the butterflies' rounding with the
 * 2^-22 relative error of the split products). */
#define GNSS_OPT_ZVARIANT 0
#define GNSS_OPT_PVARIANT 1
#define GNSS_OPT_ZKERNEL 2   /* read-only (gnss_get_option): the z kernel the options select for this
                              * context, GNSS_VARIANT_WARPSPEC, _REGISTER or _STAGED */
#define GNSS_OPT_TEST_WAIT 3 /* test of the bounded device waits, 0 (default) = off.  A value v > 0 caps
                              * every wait of the fused z kernels at v polls, and the first block withholds
                              * the copies of its first line pair (the mbarrier phase is armed, no copy is
                              * issued), so its wait runs out with nothing in flight: the block stops, the
                              * step's result is incomplete, and the next gnss_check (or gnss_stats,
                              * gnss_run_host) returns GNSS_ERR_TIMEOUT.  For tests of that path only. */
#define GNSS_VARIANT_AUTO 0
#define GNSS_VARIANT_REGISTER 1
#define GNSS_VARIANT_STAGED 2
#define GNSS_VARIANT_WARPSPEC 3
#define GNSS_VARIANT_TENSOR 4
#define GNSS_ZVARIANT_AUTO GNSS_VARIANT_AUTO
#define GNSS_ZVARIANT_REGISTER GNSS_VARIANT_REGISTER
#define GNSS_ZVARIANT_STAGED GNSS_VARIANT_STAGED
gnss_status gnss_set_option(gnss_ctx *ctx, int key, int value);
gnss_status gnss_get_option(const gnss_ctx *ctx, int key, int *value);

/* Scratch of a context.  gnss_scratch_bytes: the device bytes every
 * operation of the context can ask for (the fused step's intermediates, or
 * one field for the transforms).  gnss_attach_scratch: use caller memory
 * (256-byte aligned, at least gnss_scratch_bytes) instead of the context's
 * own; the context frees its own scratch and never frees the attached one.
 * Contexts whose work is ordered on one stream may share one buffer.  No
 * counterpart in the reference (fft.temp / fft.wspace, allocate.cu:9-225). */
size_t gnss_scratch_bytes(const gnss_ctx *ctx);
gnss_status gnss_attach_scratch(gnss_ctx *ctx, void *scratch, size_t bytes);

/* ---------------------------------------------------------------- batching
 * An ensemble of independent jets (uneven grids, Reynolds and Schmidt
 * numbers) stepped together.  The library owns every member's state and
 * history.  Members of one geometry (grid, box, precision, scalar count,
 * scheme, dealiasing, drift coefficient) form groups of up to 16 whose state,
 * history and scratch lie at fixed strides in one buffer per group.  A group
 * steps member by member, each member with its own launches, or, where its
 * kernels allow (CN/AB2, the register z kernel and register lengths), as ONE
 * batched launch per stage for the whole group, each member keeping its own
 * Reynolds and Schmidt numbers and time step (gnss_ensemble_set_batching, or
 * the autotuner per group).  The units (batched groups and members stepping
 * on their own) are spread over n_branches streams (largest first, each to
 * the least-loaded branch).  gnss_ensemble_step runs n_steps steps of every
 * member: the first step of a run (Euler, for GNSS_SCHEME_CNAB2) is launched
 * directly, and the rest as ONE CUDA graph launch that holds every unit's
 * steps in parallel branches (captured on first use for that step count,
 * replayed afterwards).  A member's result is bit-identical to stepping it
 * alone with gnss_step, in either form.  No counterpart in the reference
 * (one jet per program). */
typedef struct gnss_ensemble gnss_ensemble;
gnss_status gnss_ensemble_create(const gnss_config *cfgs, int n_members, int n_branches, gnss_ensemble **out);
gnss_status gnss_ensemble_destroy(gnss_ensemble *e);
int gnss_ensemble_size(const gnss_ensemble *e);
/* Member i: its context (owned by the ensemble) and its device state and
 * history (zeroed at creation; upload and dealias the state before the first
 * step, e.g. with cudaMemcpy + gnss_dealias). */
gnss_status gnss_ensemble_member(gnss_ensemble *e, int i, gnss_ctx **ctx, gnss_fields *state, gnss_fields *hist);
/* Copy member i's state from / to packed host memory (3 + n_scalars fields
 * back to back, pinned for asynchronous copies).  Upload also zeroes the
 * member's history and dealiases the state (main.cu:156); upload every
 * member before the first step.  Download synchronises the stream. */
gnss_status gnss_ensemble_upload(gnss_ensemble *e, int i, const void *host_state, void *stream);
gnss_status gnss_ensemble_download(gnss_ensemble *e, int i, void *host_state, void *stream);
gnss_status gnss_ensemble_step(gnss_ensemble *e, int n_steps, void *stream);
/* Kernels launched per step of the whole ensemble (for launch accounting). */
long long gnss_ensemble_launches_per_step(const gnss_ensemble *e);
/* on != 0: every group whose kernels allow it steps as one batched launch per
 * stage; 0 (the state after creation): every member steps with its own
 * launches.  No counterpart in the reference. */
gnss_status gnss_ensemble_set_batching(gnss_ensemble *e, int on);
/* 1 when member i's group steps as batched launches, 0 when it steps member by
 * member, -1 for a bad argument. */
int gnss_ensemble_batched(const gnss_ensemble *e, int i);
/* Autotuner: for every group, time each kernel variant (GNSS_OPT_*) over
 * `steps` steps of the group as the ensemble runs it, member by member on the
 * branch streams and, where the kernels allow it, as batched launches, on the
 * members' own buffers (which are zeroed afterwards, so tune before uploading
 * states), and keep the fastest form with the fastest of the z variants
 * REGISTER, STAGED, WARPSPEC by the pass variants REGISTER, STAGED and, where
 * it exists (FP32, an x or y length of 256 or 512), TENSOR.  choices (may be
 * NULL) receives, per member, the chosen GNSS_OPT_ZVARIANT value + 4 * the
 * GNSS_OPT_PVARIANT value; gnss_ensemble_batched reports the form. */
gnss_status gnss_ensemble_autotune(gnss_ensemble *e, int steps, int *choices);

/* ---------------------------------------------------------------- serving
 * A request loop with continuous batching.  Requests (a configuration, a
 * packed host state of 3 + n_scalars spectral fields, a step count) are
 * queued by gnss_server_submit from any host thread.  A scheduler thread
 * admits them in arrival order as soon as an active slot and enough of the
 * device-memory budget are free (state, history and scratch are reserved at
 * admission and stay on the device until the request ends), uploads and
 * dealiases the state, and advances every active request on its own stream
 * in chunks of steps_per_launch steps (one CUDA graph launch per chunk), so
 * the work of requests in flight overlaps on the device.  A finished request
 * keeps its final state and statistics until gnss_server_result.  A
 * request's result is bit-identical to gnss_run_host on the same input,
 * whatever else is in flight.  Times are seconds since the server started. */
typedef struct gnss_server gnss_server;
typedef struct gnss_server_config {
    size_t budget_bytes;     /* device memory the server may reserve for requests  */
    int max_active;          /* requests in flight at most                          */
    int steps_per_launch;    /* steps per graph launch of one request               */
    int device;              /* CUDA device ordinal                                 */
} gnss_server_config;
typedef struct gnss_server_report {
    long long submitted, admitted, completed, failed;
    size_t bytes_reserved;       /* now                                             */
    size_t bytes_reserved_max;   /* the most reserved at any time                   */
    int active_max;              /* the most requests in flight at any time         */
    double point_steps;          /* sum over completed requests of nx*ny*nz*steps   */
    double busy_seconds;         /* wall time with at least one request in flight    */
} gnss_server_report;
gnss_status gnss_server_create(const gnss_server_config *cfg, gnss_server **out);
/* Stops the scheduler after the requests in flight end; pending requests are
 * dropped. */
gnss_status gnss_server_destroy(gnss_server *srv);
gnss_status gnss_server_submit(gnss_server *srv, const gnss_config *cfg, const void *host_state, int n_steps,
                               long long *id);
/* Blocks until request id has ended (GNSS_ERR_TIMEOUT after timeout_s). */
gnss_status gnss_server_wait(gnss_server *srv, long long id, double timeout_s);
/* Final state (packed like the input; may be NULL), statistics after the last
 * step (GNSS_NSTATS doubles; may be NULL) and times {submitted, admitted,
 * finished} (may be NULL) of an ended request, which is then forgotten.
 * Returns the request's own status (GNSS_ERR_* if it failed). */
gnss_status gnss_server_result(gnss_server *srv, long long id, void *host_state_out, double *stats, double *times);
gnss_status gnss_server_report_get(gnss_server *srv, gnss_server_report *out);

/* ---------------------------------------------------------------- files
 * The reference's file formats (iofuncs.cu) and an exact checkpoint.
 * Physical fields are host arrays of doubles in the padded in-place layout
 * [nx][ny][2 (nz/2+1)] of the reference. */
#define GNSS_PLANE_XY 0   /* fixed z (writexyfields, iofuncs.cu:187-209) */
#define GNSS_PLANE_XZ 1   /* fixed y (writexzfields, iofuncs.cu:211-233) */
#define GNSS_PLANE_YZ 2   /* fixed x (writeyzfields, iofuncs.cu:235-257) */
/* 3D field file: one double holding the byte count 8 nx ny nz, then the
 * values in [x][y][z] order (write3Dfields_mgpu, iofuncs.cu:329-358). */
gnss_status gnss_io_write_field(int nx, int ny, int nz, const double *phys, const char *path);
/* Reads a 3D field file into the padded layout, leaving the padding as it
 * was (loadData, iofuncs.cu:462-497); GNSS_ERR_INVALID when the byte count
 * in the file does not match nx ny nz. */
gnss_status gnss_io_read_field(int nx, int ny, int nz, const char *path, double *phys);
/* One plane of a 3D field: the byte count as a double, then the values
 * (x then y for xy; x then z for xz; y then z for yz). */
gnss_status gnss_io_write_slice(int nx, int ny, int nz, const double *phys, int plane, int index, const char *path);
/* One statistics record, a raw double; the file is created when append == 0
 * and appended to otherwise (writeStats, iofuncs.cu:128-146). */
gnss_status gnss_io_write_stat(const char *path, double value, int append);
/* A mean profile: ny raw doubles (writeYprofs, iofuncs.cu:78-98). */
gnss_status gnss_io_write_profile(int ny, const double *prof, const char *path);
/* A state in the reference's files <dir>/u.<iter>, v, w, z (the scalar s), c
 * (save3Dfields, iofuncs.cu:360-432).  Each field is transformed to physical
 * space in a temporary buffer, so the state itself is untouched (the
 * reference transforms in place and back); FP32 values are widened; c is
 * written as zeros with one scalar.  Synchronises the stream. */
gnss_status gnss_save_state(gnss_ctx *ctx, const gnss_fields *state, const char *dir, int iter, void *stream);
/* Reads such files and forward-transforms them into the state
 * (importVelocity / importScalar, iofuncs.cu:499-535, then main.cu:149-153).
 * A missing scalar file leaves that field zero.  Synchronises the stream. */
gnss_status gnss_load_state(gnss_ctx *ctx, const char *dir, int iter, const gnss_fields *state, void *stream);
/* Exact checkpoint (no counterpart in the reference, whose restart goes
 * through physical space): the grid, precision, scalar count, scheme, a step
 * counter and the spectral state and history bit for bit.  hist may be NULL
 * (GNSS_SCHEME_RK3IF keeps none); loading checks the file against the
 * context.  Both synchronise the stream. */
gnss_status gnss_checkpoint_save(gnss_ctx *ctx, const gnss_fields *state, const gnss_fields *hist, long long step,
                                 const char *path, void *stream);
gnss_status gnss_checkpoint_load(gnss_ctx *ctx, const char *path, const gnss_fields *state, const gnss_fields *hist,
                                 long long *step, void *stream);

/* The reference's initial temporal jet (initializeJet, initialize.cu:615-641)
 * followed by forward transforms and dealiasing (main.cu:149-156), written
 * into the spectral state.  u = 0.5 - 0.5 tanh(h/(4 theta)(2|y|/h - 1)) plus
 * pert_amp times solenoidal noise with the reference's Gaussian spectrum
 * (generateNoise, initialize.cu:303-612), v and w the noise alone, s the same
 * profile with theta, c with theta_c; y = -ly/2 + j ly/ny.  The noise draws
 * come from the C library's rand() generator seeded with
 * srand(666*37 + 37*13) as in the reference (seed 0), or with `seed`,
 * through a private state, in the reference's loop order on the host; the
 * transforms and profiles run on the device.  Synchronises the stream. */
typedef struct gnss_jet_params {
    double h;          /* jet width H (dnsparams.h)                         */
    double theta;      /* momentum thickness of u and s (theta)             */
    double theta_c;    /* thickness of the c profile (theta_c)              */
    double pert_amp;   /* noise amplitude (pert_amp)                        */
    unsigned seed;     /* 0: the reference's seed                           */
} gnss_jet_params;
gnss_status gnss_initial_jet(gnss_ctx *ctx, const gnss_jet_params *p, const gnss_fields *state, void *stream);

/* Forward transform that allocates nothing.  No counterpart in the
 * reference.  For callers that may not allocate device memory: code running
 * under a memory manager that owns the whole device (a framework's caching
 * allocator, a fixed budget) and latency-critical loops where cudaMalloc or
 * cudaFree would synchronise the device.  Same result as gnss_forward on the
 * same configuration, but without a context: twiddles and the one-field
 * scratch live in a static device array of the library (about 18 MB, held on
 * every GPU that loads the library until the process exits), so the field
 * must satisfy nx*ny*(nz/2+1) <= GNSS_NOALLOC_MAX_ELEMS (128^3 fits);
 * larger sizes, like other bad arguments, return GNSS_ERR_INVALID.  The first
 * call on a device looks up the array's device address; make that first call
 * before any stream capture.  All calls share the array and keep the last
 * call's contents in it; calls that overlap on the GPU (any stream, any
 * thread) race and must be serialised by the caller.  Only cfg's sizes, box
 * lengths, precision and device are used.  The twiddle tables reach the
 * device as launch parameters of a small kernel, not through a host buffer.
 * With no context to hold a message, a failure other than a rejected
 * argument prints its reason to stderr. */
#define GNSS_NOALLOC_MAX_ELEMS 1114112
gnss_status gnss_forward_noalloc(const gnss_config *cfg, void *field, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* GNSS_B200_H */
