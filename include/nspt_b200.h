/*
 * nspt_b200.h -- C ABI of the B200 NSPT Langevin engine.
 *
 * The reference (PRlgt2020) has no FFI layer: its hot path is the C++
 * function set of nspt.h:55-94, operating on a ptGluon_fld plus file-scope
 * globals (defined in Quenched.cc:42-81).  This header is the drop-in
 * boundary a host driver calls instead; every entry point names the
 * reference function it replaces.  No torch or CUDA types cross it: plain
 * pointers, sizes and int status codes (0 = success, as Quenched.cc:776 and
 * the reference's load/save helpers, QCDenvNODEpt_test.h:359-374).
 *
 * Field layout on the host side is the reference's own (ptGluon,
 * QCDpt.h:249-252; ptSU3, QCDpt.h:42-50): site-major (t fastest,
 * lattice.h:37), then mu = 0..3, then one series of 1 + 9*allocORD complex
 * doubles {flag, order 1 [3x3 row major], ..., order allocORD}.  On the
 * device the engine keeps structure-of-arrays planes (mu, order, colour
 * component, site) of complex doubles.
 *
 * Threading: one context per host thread; each context owns one CUDA stream
 * and all of its device memory.  Calls are synchronous unless noted.
 */
#ifndef NSPT_B200_H
#define NSPT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define NSPT_OK 0
#define NSPT_ERR_ARG 1       /* invalid argument */
#define NSPT_ERR_ORDER 2     /* perturbative order outside [1, NSPT_MAX_ORDER] */
#define NSPT_ERR_NOMEM 3     /* device or host allocation failed */
#define NSPT_ERR_CUDA 4      /* CUDA runtime error */
#define NSPT_ERR_NODEVICE 5  /* no CUDA device */
#define NSPT_ERR_STATE 6     /* call out of sequence (e.g. no noise set) */
#define NSPT_ERR_IO 7        /* file I/O error */
#define NSPT_ERR_TIMEOUT 8   /* device work still running at the time limit
                                (nspt_set_timeout); the work is not cancelled */

#define NSPT_MAX_ORDER 48

/* ---- nspt_create flags (choices.h:42-89 as run-time options) ---- */
#define NSPT_TWIST_Y (1u << 1)   /* twisted y boundary (choices.h:47) */
#define NSPT_TWIST_Z (1u << 2)   /* twisted z boundary (choices.h:48) */
#define NSPT_TWIST_T (1u << 3)   /* twisted t boundary (choices.h:49) */
#define NSPT_ZEROMODE (1u << 4)  /* REMOVE_GLUON_ZEROMOM (choices.h:82-84) */
#define NSPT_GF_FA (1u << 5)     /* Fourier-accelerated gauge fixing */
#define NSPT_GF_LOCAL (1u << 6)  /* local stochastic gauge fixing (the reference's
                                    default without __FA_GAUGE_FIXING__) */
/* improved gauge actions (GAUGE_ACTION, choices.h:110; c1 of Quenched.cc:
 * 311-322), periodic boundaries only; at most one */
#define NSPT_ACTION_TLSYM (1u << 7)  /* tree-level Symanzik, c1 = -1/12 */
#define NSPT_ACTION_IWA (1u << 8)    /* Iwasaki, c1 = -0.331 */
#define NSPT_ACTION_DBW2 (1u << 9)   /* DBW2, c1 = -1.4088 */
/* Float-float Cauchy products in the Wilson sweep: the staple and
 * U*staples products run in compensated FP32 pairs (48 significant bits)
 * with a per-order scale 2^(e k); exp, log, exp*U, the force, the
 * accumulations and everything else stay FP64.  No reference counterpart
 * (the reference multiplies in double, QCDpt.h operator*); Wilson action. */
#define NSPT_PRECISION_FF (1u << 10)
/* UPDATE_ONTHEFLY (choices.h:61), the reference's default: gauge_wilson
 * updates every link in place, U = exp(W1) U (nspt.cc:427), in the order of
 * the OpenMP thread grid set by nspt_set_gf_grid (each thread walks its
 * block lexicographically, mu inner; barriers as nspt.cc:440-460), so that
 * a link's staples see the links updated before it.  With twisted
 * boundaries a read across a twisted face sees the field of the step's
 * start, as the reference's copy sites do until twist_boundary
 * (nspt_twist_boundary; nspt_step calls it at the end of every step).
 * Without the flag: the Jacobi update (F = exp(W1) U, then U = F).
 * FP64 only (not with NSPT_PRECISION_FF). */
#define NSPT_UPDATE_ONTHEFLY (1u << 11)

typedef struct nspt_ctx nspt_ctx;

/* Create a context for an L[0] x L[1] x L[2] x L[3] lattice (lattice.h:139)
 * with N perturbative orders (PTORD; allocORD == N on the device).
 * alpha is the gauge-fixing parameter act_pars.alpha (input.h:58).
 * Allocates both link fields (Jacobi update) on the current device. */
int nspt_create(const int L[4], int N, unsigned flags, double alpha,
                nspt_ctx **out);
int nspt_destroy(nspt_ctx *ctx);
const char *nspt_error_string(int code);
const char *nspt_last_error(nspt_ctx *ctx);

/* Device and memory footprint of a context (bytes). */
size_t nspt_device_bytes(const nspt_ctx *ctx);

/* Replace ptGluon_fld::load / save (QCDenvNODEpt_test.h:342-374):
 * copy a host field in the reference's AoS layout (allocORD orders per
 * series, allocORD >= N; orders above N are ignored on upload and written
 * as zero on download). */
int nspt_upload_links(nspt_ctx *ctx, const void *aos, int allocORD);
int nspt_download_links(nspt_ctx *ctx, void *aos, int allocORD);
/* Cold start, Quenched.cc:596-603 (flag 1, all orders zero). */
int nspt_cold_start(nspt_ctx *ctx);

/* Noise.  Either inject the 8 Gaussians SU3rand draws per link
 * (MyMath.cc:256-292) for the next sweep -- eta[V][4][8], site-major as
 * the reference draws them (nspt.cc:365-423) -- or seed the device
 * counter-based generator (Philox-4x32-10) used when nothing is injected.
 * Injected noise is consumed by exactly one sweep. */
int nspt_set_noise(nspt_ctx *ctx, const double *eta);
int nspt_seed(nspt_ctx *ctx, uint64_t seed, uint64_t counter);
/* The device generator's seed and its counter: the number of sweeps whose
 * noise has been drawn since nspt_seed.  Saved beside a configuration, they
 * let a resumed run continue the same noise stream (nspt_seed with both). */
int nspt_get_seed(nspt_ctx *ctx, uint64_t *seed, uint64_t *counter);

/* NsptEvolve (nspt.cc:953-1039) with Beat = nsteps and dt = tau_g of
 * Quench.cfg (before the /(-2 NC) of Quenched.cc:584-589): per step a
 * Langevin sweep (Jacobi, or on the fly with NSPT_UPDATE_ONTHEFLY), then the
 * zero-mode subtraction and the gauge fixing (NSPT_GF_FA or NSPT_GF_LOCAL,
 * with the alpha given at creation) selected at creation, then
 * twist_boundary.  Twisted boundaries are applied inside every neighbour
 * read (no copy sites).  gf_every > 1 gauge-fixes only every gf_every-th
 * step (0 = never). */
int nspt_step(nspt_ctx *ctx, double dt, int nsteps, int gf_every);

/* The three pieces of NsptEvolve, separately:
 * gauge_wilson (nspt.cc:258-600, the Jacobi or the on-the-fly branch as
 * selected at creation; also accumulates the zero mode when the context has
 * NSPT_ZEROMODE); zero_modes_subtraction
 * (nspt.cc:605-654); FAstochastic_gauge_fixing (nspt.cc:866-948). */
int nspt_gauge_wilson(nspt_ctx *ctx, double dt);
int nspt_zero_modes_subtraction(nspt_ctx *ctx);
int nspt_fa_gauge_fixing(nspt_ctx *ctx, double alpha);

/* stochastic_gauge_fixing (nspt.cc:660-862): the local, in-place gauge
 * transformation site by site, with twisted boundaries where the context has
 * them.  The result depends on the order of the sites, which the reference
 * fixes by its OpenMP thread grid (ntt, ntx, nty, ntz of choices.h:124-128,
 * blocks set up at Quenched.cc:518-531): the engine reproduces the
 * reference built with the grid set by nspt_set_gf_grid.  The default grid
 * is the finest one the reference accepts: blocks of 2 sites along every
 * even extent (1 thread along odd ones).  {1,1,1,1} is the sequential sweep
 * and runs one site at a time. */
int nspt_local_gauge_fixing(nspt_ctx *ctx, double alpha);
/* twist_boundary (nspt.cc:163-255): the engine applies twists inside every
 * neighbour read, so this only matters after an on-the-fly gauge_wilson
 * (NSPT_UPDATE_ONTHEFLY) on twisted boundaries, whose reads across a
 * twisted face, and those of a local gauge fixing after it, see the step's
 * start field until this call.  A no-op otherwise. */
int nspt_twist_boundary(nspt_ctx *ctx);
/* grid[d] threads along direction d; every L[d] % grid[d] == 0 and
 * L[d] / grid[d] >= 2 where grid[d] > 1 (>= 3 for an improved action with
 * NSPT_UPDATE_ONTHEFLY, whose rectangles reach two sites), else
 * NSPT_ERR_ARG. */
int nspt_set_gf_grid(nspt_ctx *ctx, const int grid[4]);
/* Which kernels run the work ordered by the thread grid -- the local gauge
 * fixing and the on-the-fly sweep; both forms visit the sites in the grid's
 * order and give the same links.  NSPT_LGF_GROUP: one 9-lane link group per
 * reference thread.  NSPT_LGF_TEAM: a warp of three groups per thread (the
 * gauge fixing's stagings and link products, or the sweep's three planes of
 * staples, spread over them: shorter latency for grids with few threads;
 * the on-the-fly team form needs one site per thread and barrier step).
 * NSPT_LGF_AUTO (the default): the team form when all the barrier step's
 * teams fit on the GPU at once.  Anything else: NSPT_ERR_ARG. */
#define NSPT_LGF_AUTO 0
#define NSPT_LGF_GROUP 1
#define NSPT_LGF_TEAM 2
int nspt_set_local_gf_form(nspt_ctx *ctx, int form);

/* Observables of the last sweep, normalised as nspt.cc:570-597:
 * plaq[(N+1)*2] (/72V), norm[N] (/12V), trU[4*N*2] (/3V, mu major).
 * Any pointer may be NULL. */
int nspt_observables(nspt_ctx *ctx, double *plaq, double *norm, double *trU);

/* Improved actions: the rectangle traces w2 of the last sweep, per order
 * 0..N, /72V as nspt.cc:586-597 prints them (NSPT_ERR_STATE for the Wilson
 * action).  The reference never resets w2[PTORD] between steps
 * (nspt.cc:972-985), so its printed top order is a running sum; this one is
 * the sweep's own value. */
int nspt_rect_observables(nspt_ctx *ctx, double *w2);

/* plaquette_measure (nspt.cc:1316-1406): static plaquette of the current
 * field, plaq[(N+1)*2]. */
int nspt_plaquette_measure(nspt_ctx *ctx, double *plaq);

/* ComputeLoops (nspt.cc:1148-1312), periodic boundaries: traces per order
 * 0..N of the 1x2 (both orientations), 2x2, 2x4 (both) and 4x4 Wilson loops
 * summed over all planes and sites, loops[4][(N+1)*2] in that order,
 * normalised as the reference prints them (1/(18V), halved for 1x2 and
 * 2x4; it prints the real parts of the even orders).  NSPT_ERR_STATE with
 * twisted boundaries. */
int nspt_wilson_loops(nspt_ctx *ctx, double *loops);

/* WL2x2 (nspt.cc:1064-1140, __WILLOOP_2x2__, periodic boundaries): trace of
 * the 2x2 Wilson loop summed over all planes and sites, per order 0..N,
 * loop[(N+1)*2], normalised by 1/(18V); the reference prints the real parts
 * of orders 2, 4, ... (its ptU[1], ptU[3], ...).  NSPT_ERR_STATE with
 * twisted boundaries. */
int nspt_wl2x2(nspt_ctx *ctx, double *loop);

/* Host-side watchdog: the calls that wait for their device work (the step,
 * sweep, gauge-fixing, zero-mode and loop calls) wait at most `seconds`
 * (0, the default: without limit) and then return NSPT_ERR_TIMEOUT.  The
 * device work is not interrupted and stays queued in order; the next such
 * call waits for it first, so the context stays usable.  No kernel of the
 * engine spins on a flag, so only slow work can reach the limit. */
int nspt_set_timeout(nspt_ctx *ctx, double seconds);

/* Per-order scale of the float-float products (NSPT_PRECISION_FF): with
 * automatic != 0 (the default) each sweep fits e to the field, so that
 * 2^(e k) max|U_k| is about the same for every order k; otherwise e is
 * fixed (|e| N <= 1000).  nspt_get_ff_scale gives the e of the last sweep. */
int nspt_set_ff_scale(nspt_ctx *ctx, int automatic, int e);
int nspt_get_ff_scale(nspt_ctx *ctx, int *e);

/* Configuration files in the reference's binary format
 * (QCDenvNODEpt_test.h:359-374: field, then (allocORD+1) complex plaquette).
 * save writes plaquette_measure of the current field as the trailer. */
int nspt_save_config(nspt_ctx *ctx, const char *path, int allocORD);
int nspt_load_config(nspt_ctx *ctx, const char *path, int allocORD,
                     double *plaq_trailer);
/* loadlowerorder (ptGluon_fld::loadlowerorder, QCDenvNODEpt_test.h:376-426):
 * start a run at N orders from a configuration file saved with loworder <=
 * N orders (reference format: V*4 series of 1 + 9*loworder complex, then
 * loworder + 1 complex plaquette values).  Orders 1..loworder come from the
 * file, every order above is zero, and each link is then unitarised, U =
 * exp(reH(log U)) with flag 1.  plaq_trailer (may be NULL) receives the
 * file's (loworder + 1) * 2 plaquette doubles.  loworder outside 1..N:
 * NSPT_ERR_ORDER; a missing file or a byte count that does not match:
 * NSPT_ERR_IO.  (The reference's zeroing loop starts at ptU[loworder+1], so
 * there order loworder + 1 keeps whatever the field held, zero after a cold
 * start; here it is always zero.) */
int nspt_load_lower_order(nspt_ctx *ctx, const char *path, int loworder,
                          double *plaq_trailer);

/* Device time of the last nspt_step, nspt_gauge_wilson,
 * nspt_zero_modes_subtraction, nspt_fa_gauge_fixing,
 * nspt_local_gauge_fixing, nspt_wilson_loops or nspt_wl2x2 call (CUDA
 * events on the context's stream around all of its launches), milliseconds. */
double nspt_last_step_ms(const nspt_ctx *ctx);
/* Average device time of one sweep-kernel launch in the last nspt_step or
 * nspt_gauge_wilson call (CUDA events around each of the first 64
 * launches), milliseconds: the duration the sweep's roofline divides by. */
double nspt_last_kernel_ms(const nspt_ctx *ctx);

/* Measured FP64 FMA throughput of the current device (independent FMA
 * chains on every SM), TFLOP/s.  Roofline denominator for the sweep. */
int nspt_measure_fp64_peak(double *tflops);

/* ---- batches of independent replicas ----
 * The reference runs one lattice per process; studies such as the dt -> 0
 * extrapolation run many (seeds x time steps x volumes).  A batch holds nrep
 * replicas -- each an ordinary context: extents L[4r..4r+3], its own time
 * step dt[r] and noise seed seeds[r] (Philox counter 0), the same N, flags
 * and alpha -- and advances all of them per step with one CUDA graph in
 * which the replicas' kernels run side by side.  Replica r after k batch
 * steps is bit-identical to a context created and seeded alike and advanced
 * by nspt_step(ctx, dt[r], k, gf_every). */
typedef struct nspt_batch nspt_batch;
int nspt_batch_create(int nrep, const int *L, int N, unsigned flags, double alpha,
                      const double *dt, const uint64_t *seeds, nspt_batch **out);
int nspt_batch_destroy(nspt_batch *b);
/* Replica r's context, owned by the batch (upload, download, observables,
 * plaquette, save/load all apply; do not destroy it). */
int nspt_batch_context(nspt_batch *b, int r, nspt_ctx **ctx);
/* nsteps Langevin steps of every replica (nspt_step's body, device noise):
 * nsteps must be a multiple of the graph length, 2 for gf_every <= 1, else
 * the even multiple of gf_every (gf_every, or 2 gf_every when odd).  The
 * first call captures the graph; later calls replay it.  NSPT_ERR_STATE if
 * a replica has injected noise pending. */
int nspt_batch_step(nspt_batch *b, int nsteps, int gf_every);
/* Device time of the last nspt_batch_step (CUDA events), milliseconds. */
double nspt_batch_last_step_ms(const nspt_batch *b);
/* Plaquette series of every replica's last sweep: plaq[nrep][(N+1)*2]. */
int nspt_batch_observables(nspt_batch *b, double *plaq);
/* Autotuner over the tile shape of the series kernels: orders per lane and
 * pass (8, or 4 where N <= 12; in the paired-run product the run length is
 * half of it) and the sweep's warps per CTA (3 links each).  Every candidate
 * is timed on the batch step itself and the fastest kept: *warps_out,
 * *mo_out (orders per lane and pass); ms_table (may be NULL) gets [2][8]
 * times, row 0 for 8 orders per lane, row 1 for 4, column w-1 for w warps,
 * 0 where a candidate does not exist.  The trial steps are undone (every
 * replica back to a cold start with its seed).  Call before stepping. */
int nspt_batch_tune_shape(nspt_batch *b, int gf_every, int *warps_out, int *mo_out,
                          float *ms_table);
/* nspt_batch_tune_shape reporting the warps only. */
int nspt_batch_tune(nspt_batch *b, int gf_every, int *warps_out);

/* Static plaquette of a field the caller already holds in device memory,
 * without a context and without allocating anything.  This entry point has
 * no counterpart in the reference.  It computes what nspt_plaquette_measure
 * computes (plaquette_measure, nspt.cc:1316-1406): plaq[(N+1)*2], per order
 * sum Tr(U * staples) / 72V.
 *
 * Who needs it: a program that keeps its own device copy of a
 * configuration.  Examples: a driver that moved it with its own copies, a
 * framework with a fixed memory pool, or a job whose device memory is
 * already spent on evolution fields.  nspt_create would allocate two more
 * field-sized buffers (29 GB at 32^4 x 24) just to look at one number.  The
 * caller may not have that memory, or may not be allowed to allocate at that
 * point without synchronising the device or breaking its memory plan.
 *
 * links_dev: the reference's AoS layout (site-major, mu, {flag, allocORD x
 * 9 complex}), 16-byte aligned, in device memory of the current device.
 * flags: NSPT_TWIST_Y | NSPT_TWIST_Z | NSPT_TWIST_T only.  stream: a
 * cudaStream_t (NULL = the default stream); the call waits for it.
 *
 * Scratch: a fixed static device array of 803,600 bytes (1024 partial rows
 * plus one result row of NSPT_MAX_ORDER + 1 complex doubles).  Its address
 * is looked up once per device on the first call, with that device
 * current; make that first call before any stream capture.  That set-up
 * (the address, and the twist matrices it uploads) is kept for the life of
 * the process: a cudaDeviceReset of that device after the first call is not
 * supported, since the module reloads and the kept values go stale.  No call relies
 * on the array's earlier contents.  Calls that overlap on one device share
 * the array and race: serialise them.  N > NSPT_MAX_ORDER (more orders than
 * the scratch rows hold) returns NSPT_ERR_ORDER; N > allocORD, a bad flag,
 * a misaligned pointer or a volume above 2^29 sites returns NSPT_ERR_ARG. */
int nspt_plaquette_measure_noalloc(const void *links_dev, int allocORD,
                                   const int L[4], int N, unsigned flags,
                                   double *plaq, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* NSPT_B200_H */
