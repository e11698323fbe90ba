// engine.cu -- host side of the C ABI declared in include/nspt_b200.h.
//
// One context = one lattice on one device with its own stream.  nspt_step
// mirrors NsptEvolve (nspt.cc:953-1039) with the reference's Jacobi option:
//   sweep (U -> F, observables, per-link log F)   gauge_wilson
//   swap U <-> F                                  Umu = Fmu   (nspt.cc:992)
//   zero-mode reduction + subtraction             zero_modes_subtraction
//   Fourier-accelerated gauge fixing              FAstochastic_gauge_fixing
// Twisted boundaries are applied inside every neighbour read.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/nspt_b200.h"
#include "kernels.cuh"
#include "fft.cuh"
#include "loops.cuh"

using namespace nspt;

struct KernelShape {
  int warps;  // warps per CTA (3 link groups of 9 lanes each)
  int slots;  // shared series slots per group
};

struct nspt_ctx {
  int L[4];
  int N;
  unsigned flags;
  double alpha;
  long V;
  int dev, nsm;
  size_t smem_optin;
  cudaStream_t st;
  cudaEvent_t ev0, ev1;
  float last_ms;
  // CUDA events around the first KEV sweep-kernel launches of a call
  static constexpr int KEV = 64;
  cudaEvent_t kev[2 * KEV];
  int kcount;
  double last_kernel_ms;  // average sweep-kernel launch of the last call
  Geo geo;
  int SS;  // slot stride (double2)
  double2 *U, *Uf, *F, *Ff;
  double2 *Lg;       // per-link logs (zero modes, FA)
  bool snap_valid;   // on the fly, twisted: F holds the step's start field, which reads
                     // across a twisted face see until twist_boundary
  bool lg_current;   // Lg holds log U of the current field (after a sweep with
                     // zero modes and after the zero-mode subtraction)
  double2 *Wg, *Gx;  // FA work planes
  double2 *obs_tr, *obs_tru;
  double *obs_norm;
  double2 *red2;  // [(N+1) + 4N + 4*9N] reduced sums
  double *red1;   // [N]
  double *p2;     // lattice momenta p2hat[4][128] of this context's extents
  double2 *ftw;   // FFT twiddles exp(-2 pi i t / L_d), [4][128] (FA only)
  int gf_grid[4]; // local gauge fixing: the reference's thread grid (ntt, ntx, nty, ntz)
  int gf_form;    // local gauge fixing kernel: NSPT_LGF_AUTO, NSPT_LGF_GROUP or NSPT_LGF_TEAM
  unsigned long long *dcounter;  // Philox step counter on the device (advanced by k_inc)
  int sweep_warps;               // warps per CTA of the sweep, 0 = as many as fit
  // orders per lane and pass of the series kernels: 0 = by N (the low-order
  // shape, MO_LOW, for N <= 3 MO_LOW), MO = the 24-order shape everywhere,
  // MO_LOW = the low-order shape (only where N <= 3 MO_LOW)
  int shape_mo;
  double c1;                     // improved action weight (0: Wilson), c0 = 1 - 8 c1
  double2 *obs_tr2;              // [(N+1)][4V] rectangle traces (improved actions)
  int *ff_e;                     // float-float scale exponent used by the sweep (device)
  unsigned long long *ff_mx;     // [N] per-order max |U_k| (bit patterns)
  bool ff_auto;                  // fit the exponent each sweep
  double timeout_s;              // host-side limit on waiting for a call's device work (0: none)
  bool busy;                     // a call returned NSPT_ERR_TIMEOUT; its work may still run
  double2 *loop_part;            // Wilson loops: per-CTA rows and the summed row
  size_t loop_part_n;
  double *noise;  // injected noise
  bool noise_pending;
  bool have_obs;
  uint64_t seed, counter;
  // bumped by every setter that changes what a step launches or the values
  // its kernels take by argument (seed, gauge-fixing grid, sweep shape,
  // float-float scale mode); a CUDA graph captured under another value is
  // stale (batch.cuh)
  uint64_t launch_gen;
  size_t bytes;
  std::string err;
};

static const char *kErr[] = {"ok",
                             "invalid argument",
                             "perturbative order outside the supported range",
                             "allocation failed",
                             "CUDA runtime error",
                             "no CUDA device",
                             "call out of sequence",
                             "file I/O error",
                             "device work still running at the time limit"};

extern "C" const char *nspt_error_string(int code) {
  if (code < 0 || code > 8) return "unknown error";
  return kErr[code];
}

extern "C" const char *nspt_last_error(nspt_ctx *ctx) {
  return ctx ? ctx->err.c_str() : "null context";
}

#define CK(call)                                                              \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      if (ctx) ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_); \
      return NSPT_ERR_CUDA;                                                   \
    }                                                                         \
  } while (0)

// ---------------- kernel shapes ----------------

// per-group shared memory: `slots` series slots plus `extra` double2
static size_t group_bytes(const nspt_ctx *ctx, int slots, int extra) {
  return ((size_t)slots * ctx->SS + extra) * sizeof(double2);
}

// the low-order kernel shape (MO_LOW orders per lane and pass, 6-warp CTAs,
// two per SM) for this context's series kernels
static bool use_low(const nspt_ctx *ctx) {
  if (ctx->N > 3 * MO_LOW) return false;
  return ctx->shape_mo != MO;
}

static KernelShape choose_shape(const nspt_ctx *ctx, int slots, long units, int extra = 0,
                                int max_warps = 8, int ctas_per_sm = 1) {
  KernelShape k;
  k.slots = slots;
  const size_t per_warp = (size_t)LPW * group_bytes(ctx, slots, extra);
  // shared memory per SM: 228 KB, of which up to smem_optin for one CTA
  const size_t budget = ctas_per_sm > 1 ? (size_t)228 * 1024 / ctas_per_sm - 1024 : ctx->smem_optin;
  int wmax = (int)std::min<size_t>(max_warps, std::min(budget, ctx->smem_optin) / per_warp);
  if (wmax < 1) wmax = 1;
  // spread small lattices over the SMs: about two CTAs per SM if possible
  const long want = (units + (long)LPW * 2 * ctx->nsm - 1) / ((long)LPW * 2 * ctx->nsm);
  k.warps = (int)std::max<long>(1, std::min<long>(wmax, want));
  return k;
}

template <bool MEASURE, bool FF, bool LOW = false>
static void sweep_kernel(dim3 grid, dim3 blk, size_t smem, cudaStream_t st, const SweepArgs &a) {
  cudaFuncSetAttribute(k_sweep<MEASURE, FF, LOW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smem);
  k_sweep<MEASURE, FF, LOW><<<grid, blk, smem, st>>>(a);
}

static int launch_sweep(nspt_ctx *ctx, const SweepArgs &a0, bool measure) {
  const long nl = 4 * ctx->V;
  const bool ff = (ctx->flags & NSPT_PRECISION_FF) != 0;
  // low orders: the lighter variant, two CTAs per SM
  const bool low = !measure && !ff && use_low(ctx);
  const int max_warps = (low ? SWEEP_THREADS_LOW : SWEEP_THREADS) / 32;
  KernelShape k = choose_shape(ctx, SWEEP_SLOTS, nl, 0,
                               ctx->sweep_warps > 0 ? std::min(ctx->sweep_warps, max_warps)
                                                    : max_warps,
                               low ? 2 : 1);
  int warps = k.warps, gpc = k.warps * LPW;
  if (!low && ctx->sweep_warps == 0 && k.warps < max_warps) {
    // shared memory, not the lattice, limits the CTA: as many link groups
    // as it holds, over all max_warps warps (sweep_group), where that keeps
    // at least 2.5 groups per warp.  Measured at 32^4 x 24: 22 groups as 8
    // warps 511 ms, 21 as 7 full warps 538 ms; at 24^4 x 40, 13 groups as 8
    // warps 732 ms, 12 as 4 full warps 671 ms.
    const size_t per_group = group_bytes(ctx, SWEEP_SLOTS, 0);
    const long fit = std::min<long>((long)(ctx->smem_optin / per_group), (long)max_warps * LPW);
    const long want = (nl + 2L * ctx->nsm - 1) / (2L * ctx->nsm);  // about two CTAs per SM
    if (fit > gpc && want >= fit && 2 * fit >= 5L * max_warps) {
      gpc = (int)fit;
      warps = max_warps;
    }
  }
  SweepArgs a = a0;
  a.gpc = gpc;
  const size_t smem = (size_t)gpc * group_bytes(ctx, SWEEP_SLOTS, 0);
  const unsigned grid = (unsigned)((nl + gpc - 1) / gpc);
  const dim3 blk(32 * warps);
  if (measure)
    sweep_kernel<true, false>(grid, blk, smem, ctx->st, a);
  else if (ff)
    sweep_kernel<false, true>(grid, blk, smem, ctx->st, a);
  else if (low)
    sweep_kernel<false, false, true>(grid, blk, smem, ctx->st, a);
  else
    sweep_kernel<false, false>(grid, blk, smem, ctx->st, a);
  CK(cudaGetLastError());
  return NSPT_OK;
}

static int launch_sweep_imp(nspt_ctx *ctx, const SweepArgs &a) {
  const long nl = 4 * ctx->V;
  const bool low = use_low(ctx);
  KernelShape k = low ? choose_shape(ctx, IMP_SLOTS, nl, 0, SWEEP_THREADS_LOW / 32, 2)
                      : choose_shape(ctx, IMP_SLOTS, nl, 0);
  const size_t smem = (size_t)k.warps * LPW * group_bytes(ctx, IMP_SLOTS, 0);
  const long per_cta = (long)k.warps * LPW;
  const unsigned grid = (unsigned)((nl + per_cta - 1) / per_cta);
  if (low) {
    cudaFuncSetAttribute(k_sweep_imp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_sweep_imp<true><<<grid, 32 * k.warps, smem, ctx->st>>>(a);
  } else {
    cudaFuncSetAttribute(k_sweep_imp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_sweep_imp<false><<<grid, 32 * k.warps, smem, ctx->st>>>(a);
  }
  CK(cudaGetLastError());
  return NSPT_OK;
}

// Launch a per-link (or per-site) group kernel with `slots` series per group.
// low: the kernel's low-order instantiation (N <= 3 MO_LOW; 6-warp CTAs,
// two per SM).
template <class Fn>
static int launch_groups(nspt_ctx *ctx, const void *fn, int slots, long units, Fn launch,
                         const char *what, int extra = 0, bool low = false) {
  KernelShape k = low ? choose_shape(ctx, slots, units, extra, SWEEP_THREADS_LOW / 32, 2)
                      : choose_shape(ctx, slots, units, extra);
  const size_t smem = (size_t)k.warps * LPW * group_bytes(ctx, slots, extra);
  const long per_cta = (long)k.warps * LPW;
  const unsigned grid = (unsigned)((units + per_cta - 1) / per_cta);
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  launch(grid, dim3(32 * k.warps), smem);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    ctx->err = std::string(what) + ": " + cudaGetErrorString(e);
    return NSPT_ERR_CUDA;
  }
  return NSPT_OK;
}

// ---------------- reductions ----------------

// rectangle traces of the improved actions sit after the MM area of red2
static size_t w2_offset(int N) { return (size_t)(N + 1) + 4 * N + 36 * N; }

static int reduce_sweep_obs(nspt_ctx *ctx) {
  const int N = ctx->N;
  const long nl = 4 * ctx->V;
  if (ctx->c1 != 0.0)
    k_rowsum<double2><<<N + 1, 256, 0, ctx->st>>>(ctx->obs_tr2, (size_t)nl, nl,
                                                   ctx->red2 + w2_offset(N));
  k_rowsum<double2><<<N + 1, 256, 0, ctx->st>>>(ctx->obs_tr, (size_t)nl, nl, ctx->red2);
  k_rowsum<double2><<<4 * N, 256, 0, ctx->st>>>(ctx->obs_tru, (size_t)ctx->V, ctx->V,
                                                   ctx->red2 + (N + 1));
  k_rowsum<double><<<N, 256, 0, ctx->st>>>(ctx->obs_norm, (size_t)nl, nl, ctx->red1);
  CK(cudaGetLastError());
  return NSPT_OK;
}

// The reference's OpenMP thread grid (the context's gf_grid) as the kernels
// walk it: steps = the number of barrier steps.
static LgfGrid thread_grid(const nspt_ctx *ctx, long &steps) {
  LgfGrid gr;
  gr.dmax = -1;
  gr.nthr = 1;
  gr.seg = 1;
  for (int d = 0; d < 4; d++) {
    gr.n[d] = ctx->gf_grid[d];
    gr.bs[d] = ctx->L[d] / gr.n[d];
    gr.nthr *= gr.n[d];
    if (gr.n[d] > 1) gr.dmax = d;
  }
  steps = 1;
  for (int d = 0; d < 4; d++) {
    if (d <= gr.dmax)
      steps *= gr.bs[d];
    else
      gr.seg *= ctx->L[d];
  }
  return gr;
}

// gauge_wilson on the fly (UPDATE_ONTHEFLY, nspt.cc:355-460): one launch per
// barrier step of the thread grid, one group per reference thread.
static int launch_sweep_otf(nspt_ctx *ctx, const SweepArgs &a0) {
  long steps;
  const LgfGrid gr = thread_grid(ctx, steps);
  const bool low = use_low(ctx);
  const int max_warps = (low ? SWEEP_THREADS_LOW : SWEEP_THREADS) / 32;
  const KernelShape k = choose_shape(ctx, SWEEP_SLOTS, gr.nthr, 0, max_warps, low ? 2 : 1);
  int warps = k.warps;
  SweepArgs a = a0;
  a.gpc = k.warps * LPW;
  if (!low && k.warps < max_warps) {
    // as the Jacobi sweep: as many groups as shared memory holds, dealt over
    // all max_warps warps (sweep_group), where that keeps >= 2.5 per warp
    const long fit = std::min<long>((long)(ctx->smem_optin / group_bytes(ctx, SWEEP_SLOTS, 0)),
                                    (long)max_warps * LPW);
    const long want = (gr.nthr + 2L * ctx->nsm - 1) / (2L * ctx->nsm);
    if (fit > a.gpc && want >= fit && 2 * fit >= 5L * max_warps) {
      a.gpc = (int)fit;
      warps = max_warps;
    }
  }
  const size_t smem = (size_t)a.gpc * group_bytes(ctx, SWEEP_SLOTS, 0);
  const unsigned grid = (unsigned)((gr.nthr + a.gpc - 1) / a.gpc);
  // a warp of three groups per reference thread (the three planes' staples
  // side by side) where every team of a barrier step fits on the GPU at once
  const size_t team_bytes = (size_t)LPW * SWEEP_SLOTS * ctx->SS * sizeof(double2);
  int team_warps = 4;
  while (team_warps > 1 && (size_t)team_warps * team_bytes > ctx->smem_optin) team_warps /= 2;
  bool team = gr.seg == 1 && team_bytes <= ctx->smem_optin && ctx->gf_form != NSPT_LGF_GROUP;
  if (team && ctx->gf_form == NSPT_LGF_AUTO) {
    const long per_sm = std::min<long>((long)((size_t)228 * 1024 / team_bytes), low ? 12 : 8);
    team = gr.nthr <= per_sm * ctx->nsm;
  }
  if (team) {
    const size_t tsmem = (size_t)team_warps * team_bytes;
    const void *fn =
        low ? (const void *)k_sweep_otf1_team<true> : (const void *)k_sweep_otf1_team<false>;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsmem);
    const unsigned tgrid = (unsigned)((gr.nthr + team_warps - 1) / team_warps);
    for (long p = 0; p < steps; p++)
      for (int mu = 0; mu < 4; mu++) {
        if (low)
          k_sweep_otf1_team<true><<<tgrid, 32 * team_warps, tsmem, ctx->st>>>(a, gr, p, mu);
        else
          k_sweep_otf1_team<false><<<tgrid, 32 * team_warps, tsmem, ctx->st>>>(a, gr, p, mu);
      }
  } else if (gr.seg == 1) {
    // one site per thread and barrier step: a launch per (step, mu), the
    // link update inline without a loop around it
    const void *fn = low ? (const void *)k_sweep_otf1<true> : (const void *)k_sweep_otf1<false>;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    for (long p = 0; p < steps; p++)
      for (int mu = 0; mu < 4; mu++) {
        if (low)
          k_sweep_otf1<true><<<grid, 32 * warps, smem, ctx->st>>>(a, gr, p, mu);
        else
          k_sweep_otf1<false><<<grid, 32 * warps, smem, ctx->st>>>(a, gr, p, mu);
      }
  } else {
    const void *fn = low ? (const void *)k_sweep_otf<true> : (const void *)k_sweep_otf<false>;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    for (long p = 0; p < steps; p++) {
      if (low)
        k_sweep_otf<true><<<grid, 32 * warps, smem, ctx->st>>>(a, gr, p);
      else
        k_sweep_otf<false><<<grid, 32 * warps, smem, ctx->st>>>(a, gr, p);
    }
  }
  CK(cudaGetLastError());
  return NSPT_OK;
}

// The improved-action sweep on the fly (periodic boundaries only): one
// launch per barrier step, or per (barrier step, mu) where every thread owns
// one site per barrier step.
static int launch_sweep_imp_otf(nspt_ctx *ctx, const SweepArgs &a) {
  long steps;
  const LgfGrid gr = thread_grid(ctx, steps);
  const bool low = use_low(ctx);
  const int max_warps = low ? SWEEP_THREADS_LOW / 32 : 8;
  const KernelShape k = choose_shape(ctx, IMP_SLOTS, gr.nthr, 0, max_warps, low ? 2 : 1);
  const size_t smem = (size_t)k.warps * LPW * group_bytes(ctx, IMP_SLOTS, 0);
  const long per_cta = (long)k.warps * LPW;
  const unsigned grid = (unsigned)((gr.nthr + per_cta - 1) / per_cta);
  if (gr.seg == 1) {
    const void *fn =
        low ? (const void *)k_sweep_imp_otf1<true> : (const void *)k_sweep_imp_otf1<false>;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    for (long p = 0; p < steps; p++)
      for (int mu = 0; mu < 4; mu++) {
        if (low)
          k_sweep_imp_otf1<true><<<grid, 32 * k.warps, smem, ctx->st>>>(a, gr, p, mu);
        else
          k_sweep_imp_otf1<false><<<grid, 32 * k.warps, smem, ctx->st>>>(a, gr, p, mu);
      }
  } else {
    const void *fn =
        low ? (const void *)k_sweep_imp_otf<true> : (const void *)k_sweep_imp_otf<false>;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    for (long p = 0; p < steps; p++) {
      if (low)
        k_sweep_imp_otf<true><<<grid, 32 * k.warps, smem, ctx->st>>>(a, gr, p, 0, 4);
      else
        k_sweep_imp_otf<false><<<grid, 32 * k.warps, smem, ctx->st>>>(a, gr, p, 0, 4);
    }
  }
  CK(cudaGetLastError());
  return NSPT_OK;
}

static int do_sweep(nspt_ctx *ctx, double dt, bool use_noise) {
  SweepArgs a;
  a.U = ctx->U;
  a.Uf = ctx->Uf;
  a.F = ctx->F;
  a.Ff = ctx->Ff;
  a.Lg = (ctx->flags & NSPT_ZEROMODE) ? ctx->Lg : nullptr;
  a.obs_tr = ctx->obs_tr;
  a.obs_norm = ctx->obs_norm;
  a.obs_tru = ctx->obs_tru;
  a.noise = use_noise ? ctx->noise : nullptr;
  a.seed = ctx->seed;
  a.step = ctx->counter;
  a.stepp = ctx->dcounter;
  a.obs_tr2 = ctx->obs_tr2;
  a.c1 = ctx->c1;
  a.c0 = 1. - 8. * ctx->c1;
  a.ff_scale = ctx->ff_e;
  // QuenchedAllocate: stau = sqrt(tau_g); tau_g /= -(2 NC)  (Quenched.cc:584-589)
  a.stau = sqrt(dt);
  double tg = dt;
  tg /= -(2 * 3);
  a.tau_g = tg;
  a.N = ctx->N;
  a.SS = ctx->SS;
  a.g = ctx->geo;
  a.Ut = ctx->U;
  a.Utf = ctx->Uf;
  const bool otf = (ctx->flags & NSPT_UPDATE_ONTHEFLY) != 0;
  if (otf) {
    // in place; with twisted boundaries F keeps the step's start field for
    // the reads across a twisted face (the reference's copy sites)
    a.F = ctx->U;
    a.Ff = ctx->Uf;
    if (ctx->geo.twist) {
      if (!ctx->snap_valid) {
        const size_t nb = (size_t)4 * 9 * ctx->N * ctx->V * sizeof(double2);
        CK(cudaMemcpyAsync(ctx->F, ctx->U, nb, cudaMemcpyDeviceToDevice, ctx->st));
        CK(cudaMemcpyAsync(ctx->Ff, ctx->Uf, (size_t)4 * ctx->V * sizeof(double2),
                           cudaMemcpyDeviceToDevice, ctx->st));
        ctx->snap_valid = true;
      }
      a.Ut = ctx->F;
      a.Utf = ctx->Ff;
    }
  }
  if ((ctx->flags & NSPT_PRECISION_FF) && ctx->ff_auto) {
    // per-order scale of the float-float products, fitted to this field
    CK(cudaMemsetAsync(ctx->ff_mx, 0, ctx->N * sizeof(unsigned long long), ctx->st));
    k_order_absmax<<<dim3(2 * ctx->nsm, ctx->N), 256, 0, ctx->st>>>(ctx->U, ctx->N,
                                                                    (size_t)ctx->V, ctx->ff_mx);
    k_ff_fit<<<1, 1, 0, ctx->st>>>(ctx->ff_mx, ctx->N, ctx->ff_e);
    CK(cudaGetLastError());
  }
  const bool timed = ctx->kcount < nspt_ctx::KEV;
  if (timed) CK(cudaEventRecord(ctx->kev[2 * ctx->kcount], ctx->st));
  int rc = otf && ctx->c1 != 0.0 ? launch_sweep_imp_otf(ctx, a)
           : otf                 ? launch_sweep_otf(ctx, a)
           : ctx->c1 != 0.0      ? launch_sweep_imp(ctx, a)
                                 : launch_sweep(ctx, a, false);
  if (rc) return rc;
  if (timed) {
    CK(cudaEventRecord(ctx->kev[2 * ctx->kcount + 1], ctx->st));
    ctx->kcount++;
  }
  rc = reduce_sweep_obs(ctx);
  if (rc) return rc;
  k_inc<<<1, 1, 0, ctx->st>>>(ctx->dcounter);
  CK(cudaGetLastError());
  if (!otf) {
    std::swap(ctx->U, ctx->F);
    std::swap(ctx->Uf, ctx->Ff);
  }
  ctx->counter++;
  ctx->have_obs = true;
  ctx->lg_current = a.Lg != nullptr;  // the sweep stored log U' per link
  return NSPT_OK;
}

static int do_zero_modes(nspt_ctx *ctx) {
  const int N = ctx->N;
  double2 *MM = ctx->red2 + (N + 1) + 4 * N;
  k_rowsum<double2><<<4 * 9 * N, 256, 0, ctx->st>>>(ctx->Lg, (size_t)ctx->V, ctx->V, MM);
  k_scale_mm<<<(36 * N + 127) / 128, 128, 0, ctx->st>>>(MM, 36 * N, 1.0 / (double)ctx->V);
  CK(cudaGetLastError());
  const long nl = 4 * ctx->V;
  double2 *U = ctx->U, *Uf = ctx->Uf;
  double2 *Lg = ctx->Lg;
  const int SS = ctx->SS;
  const Geo geo = ctx->geo;
  cudaStream_t st = ctx->st;
  const bool low = use_low(ctx);
  const int rc = launch_groups(
      ctx, low ? (const void *)k_zero_modes<true> : (const void *)k_zero_modes<false>, 3, nl,
      [&](unsigned g, dim3 b, size_t sm) {
        if (low)
          k_zero_modes<true><<<g, b, sm, st>>>(U, Uf, Lg, MM, N, SS, geo);
        else
          k_zero_modes<false><<<g, b, sm, st>>>(U, Uf, Lg, MM, N, SS, geo);
      },
      "zero modes", 0, low);
  if (rc == NSPT_OK) ctx->lg_current = true;  // Lg = the new field's log
  return rc;
}

static int fft4d(nspt_ctx *ctx, double2 *data, int sign) {
  const int N = ctx->N;
  const size_t V = (size_t)ctx->V;
  const int strides[4] = {ctx->geo.s0, ctx->geo.s1, ctx->geo.s2, 1};
  for (int d = 3; d >= 0; d--) {
    const int n = ctx->L[d];
    const long nlines = (long)9 * N * (long)(V / n);
    const unsigned grid = (unsigned)((nlines + 127) / 128);
    switch (n) {
      case 2: k_fft_pow2<2><<<grid, 128, 0, ctx->st>>>(data, nlines, strides[d], V, sign); break;
      case 4: k_fft_pow2<4><<<grid, 128, 0, ctx->st>>>(data, nlines, strides[d], V, sign); break;
      case 8: k_fft_pow2<8><<<grid, 128, 0, ctx->st>>>(data, nlines, strides[d], V, sign); break;
      case 16: k_fft_pow2<16><<<grid, 128, 0, ctx->st>>>(data, nlines, strides[d], V, sign); break;
      case 32: k_fft_pow2<32><<<grid, 128, 0, ctx->st>>>(data, nlines, strides[d], V, sign); break;
      case 64: k_fft_pow2<64><<<grid, 128, 0, ctx->st>>>(data, nlines, strides[d], V, sign); break;
      default:
        k_fft_direct<<<grid, 128, 0, ctx->st>>>(data, nlines, n, strides[d], V, sign);
    }
    CK(cudaGetLastError());
  }
  return NSPT_OK;
}

// Extents with a compile-time FFT plan (fft.cuh); others use fft4d.
#define NSPT_FFT_SIZES(X) X(2) X(3) X(4) X(5) X(6) X(8) X(10) X(12) X(16) X(20) X(24) X(32)

static bool fft_planned(int n) {
#define NSPT_FFT_CASE(n_) if (n == n_) return true;
  NSPT_FFT_SIZES(NSPT_FFT_CASE)
#undef NSPT_FFT_CASE
  return false;
}

template <int n>
static void fft_t_launch(nspt_ctx *ctx, double2 *data, const double2 *Lg, bool div, int inv) {
  const long nlines = (long)9 * ctx->N * (ctx->V / n);
  const unsigned grid = (unsigned)((nlines + 127) / 128);
  const size_t smem = (size_t)128 * (n | 1) * sizeof(double2);
  if (div) {
    cudaFuncSetAttribute(k_fft_t<n, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_fft_t<n, true><<<grid, 128, smem, ctx->st>>>(data, Lg, nlines, 9 * ctx->N, ctx->geo,
                                                   ctx->ftw + 3 * 128, inv);
  } else {
    cudaFuncSetAttribute(k_fft_t<n, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_fft_t<n, false><<<grid, 128, smem, ctx->st>>>(data, Lg, nlines, 9 * ctx->N, ctx->geo,
                                                    ctx->ftw + 3 * 128, inv);
  }
}

template <int n>
static void fft_strided_launch(nspt_ctx *ctx, double2 *data, int d, int inv) {
  const long nlines = (long)9 * ctx->N * (ctx->V / n);
  const int st = d == 0 ? ctx->geo.s0 : d == 1 ? ctx->geo.s1 : ctx->geo.s2;
  k_fft_strided<n><<<(unsigned)((nlines + 127) / 128), 128, 0, ctx->st>>>(
      data, nlines, st, (size_t)ctx->V, ctx->ftw + d * 128, inv);
}

template <int n>
static void fft_x_launch(nspt_ctx *ctx, double2 *data, double alpha) {
  const long nlines = (long)9 * ctx->N * (ctx->V / n);
  k_fft_x_scale<n><<<(unsigned)((nlines + 127) / 128), 128, 0, ctx->st>>>(
      data, nlines, ctx->geo, ctx->ftw, alpha, ctx->p2);
}

// Wg = iFFT(-alpha / p^2 FFT(div log U)) in seven passes (fft.cuh), or
// NSPT_ERR_ARG when an extent has no compile-time plan.
static int fa_fft_fused(nspt_ctx *ctx, double alpha) {
  for (int d = 0; d < 4; d++)
    if (!fft_planned(ctx->L[d])) return NSPT_ERR_ARG;
  double2 *Wg = ctx->Wg;
  const double2 *Lg = ctx->Lg;
  auto t_pass = [&](bool div, int inv) {
    switch (ctx->L[3]) {
#define NSPT_FFT_CASE(n_) case n_: fft_t_launch<n_>(ctx, Wg, Lg, div, inv); break;
      NSPT_FFT_SIZES(NSPT_FFT_CASE)
#undef NSPT_FFT_CASE
    }
  };
  auto s_pass = [&](int d, int inv) {
    switch (ctx->L[d]) {
#define NSPT_FFT_CASE(n_) case n_: fft_strided_launch<n_>(ctx, Wg, d, inv); break;
      NSPT_FFT_SIZES(NSPT_FFT_CASE)
#undef NSPT_FFT_CASE
    }
  };
  t_pass(true, 0);  // divergence + forward t
  s_pass(2, 0);
  s_pass(1, 0);
  switch (ctx->L[0]) {  // forward x, -alpha / p^2, backward x
#define NSPT_FFT_CASE(n_) case n_: fft_x_launch<n_>(ctx, Wg, alpha); break;
    NSPT_FFT_SIZES(NSPT_FFT_CASE)
#undef NSPT_FFT_CASE
  }
  s_pass(1, 1);
  s_pass(2, 1);
  t_pass(false, 1);
  CK(cudaGetLastError());
  return NSPT_OK;
}

static int do_fa(nspt_ctx *ctx, double alpha) {
  const int N = ctx->N, SS = ctx->SS;
  const long nl = 4 * ctx->V;
  const Geo geo = ctx->geo;
  cudaStream_t st = ctx->st;
  double2 *U = ctx->U, *Uf = ctx->Uf, *F = ctx->F, *Ff = ctx->Ff, *Lg = ctx->Lg, *Wg = ctx->Wg,
          *Gx = ctx->Gx;
  const bool low = use_low(ctx);
  // log U per link (nspt.cc:874-875); after the zero-mode subtraction Lg
  // already holds it (k_zero_modes)
  int rc = NSPT_OK;
  if (!ctx->lg_current) {
    rc = launch_groups(
      ctx, low ? (const void *)k_log_links<true> : (const void *)k_log_links<false>, 3, nl,
      [&](unsigned g, dim3 b, size_t sm) {
        if (low)
          k_log_links<true><<<g, b, sm, st>>>(U, Uf, Lg, N, SS, geo);
        else
          k_log_links<false><<<g, b, sm, st>>>(U, Uf, Lg, N, SS, geo);
      },
      "FA logs", 0, low);
    if (rc) return rc;
  }
  rc = fa_fft_fused(ctx, alpha);
  if (rc == NSPT_ERR_ARG) {  // an extent without a compile-time FFT plan
    const size_t tot = (size_t)9 * N * ctx->V;
    const unsigned eg = (unsigned)std::min<size_t>((tot + 255) / 256, (size_t)ctx->nsm * 32);
    k_fa_div<<<eg, 256, 0, st>>>(Lg, Wg, N, geo);
    CK(cudaGetLastError());
    if ((rc = fft4d(ctx, Wg, -1))) return rc;
    k_fa_scale<<<eg, 256, 0, st>>>(Wg, N, geo, alpha, ctx->p2);
    CK(cudaGetLastError());
    if ((rc = fft4d(ctx, Wg, +1))) return rc;
  } else if (rc) {
    return rc;
  }
  rc = launch_groups(
      ctx, low ? (const void *)k_fa_gt<true> : (const void *)k_fa_gt<false>, 3, ctx->V,
      [&](unsigned g, dim3 b, size_t sm) {
        if (low)
          k_fa_gt<true><<<g, b, sm, st>>>(Wg, Gx, N, SS, geo);
        else
          k_fa_gt<false><<<g, b, sm, st>>>(Wg, Gx, N, SS, geo);
      },
      "FA gauge transform", 0, low);
  if (rc) return rc;
  rc = launch_groups(
      ctx, low ? (const void *)k_fa_apply<true> : (const void *)k_fa_apply<false>, 2, nl,
      [&](unsigned g, dim3 b, size_t sm) {
        if (low)
          k_fa_apply<true><<<g, b, sm, st>>>(U, Uf, Gx, F, Ff, N, SS, geo);
        else
          k_fa_apply<false><<<g, b, sm, st>>>(U, Uf, Gx, F, Ff, N, SS, geo);
      },
      "FA apply", 0, low);
  if (rc) return rc;
  std::swap(ctx->U, ctx->F);
  std::swap(ctx->Uf, ctx->Ff);
  ctx->lg_current = false;
  return NSPT_OK;
}

// stochastic_gauge_fixing (nspt.cc:660-862) with the context's thread
// grid: one launch per barrier step, one group per reference thread.
static int do_local_gf(nspt_ctx *ctx, double alpha) {
  long steps;
  const LgfGrid gr = thread_grid(ctx, steps);
  const int N = ctx->N, SS = ctx->SS;
  const Geo geo = ctx->geo;
  cudaStream_t st = ctx->st;
  double2 *U = ctx->U, *Uf = ctx->Uf;
  // reads across a twisted face: the step's start field after an on-the-fly
  // sweep (the reference's copy sites before twist_boundary)
  const double2 *Ut = ctx->snap_valid ? ctx->F : U, *Utf = ctx->snap_valid ? ctx->Ff : Uf;
  const bool low = use_low(ctx);
  ctx->lg_current = false;
  // The team form (a warp of three groups per reference thread) shortens
  // each thread's chain of dependent stagings and products about threefold
  // but keeps a third of its lanes idle in the exps: automatic choice takes
  // it when every team of the barrier step is resident at once.
  const size_t team_bytes = (size_t)LGF_TEAM_SLOTS * SS * sizeof(double2);
  const int team_warps = 2 * team_bytes <= ctx->smem_optin ? 2 : 1;
  bool team = team_bytes <= ctx->smem_optin && ctx->gf_form != NSPT_LGF_GROUP;
  if (team && ctx->gf_form == NSPT_LGF_AUTO) {
    const long per_sm = std::min<long>((long)((size_t)228 * 1024 / team_bytes), low ? 12 : 8);
    team = gr.nthr <= per_sm * ctx->nsm;
  }
  if (team) {
    const size_t smem = (size_t)team_warps * team_bytes;
    const void *fn = low ? (const void *)k_local_gf_team<true> : (const void *)k_local_gf_team<false>;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const unsigned grid = (unsigned)((gr.nthr + team_warps - 1) / team_warps);
    for (long p = 0; p < steps; p++) {
      if (low)
        k_local_gf_team<true><<<grid, 32 * team_warps, smem, st>>>(U, Uf, Ut, Utf, N, SS, geo,
                                                                    alpha, gr, p);
      else
        k_local_gf_team<false><<<grid, 32 * team_warps, smem, st>>>(U, Uf, Ut, Utf, N, SS, geo,
                                                                     alpha, gr, p);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      ctx->err = std::string("local gauge fixing: ") + cudaGetErrorString(e);
      return NSPT_ERR_CUDA;
    }
    return NSPT_OK;
  }
  for (long p = 0; p < steps; p++) {
    int rc = launch_groups(
        ctx, low ? (const void *)k_local_gf<true> : (const void *)k_local_gf<false>, 4, gr.nthr,
        [&](unsigned g, dim3 b, size_t sm) {
          if (low)
            k_local_gf<true><<<g, b, sm, st>>>(U, Uf, Ut, Utf, N, SS, geo, alpha, gr, p);
          else
            k_local_gf<false><<<g, b, sm, st>>>(U, Uf, Ut, Utf, N, SS, geo, alpha, gr, p);
        },
        "local gauge fixing", 0, low);
    if (rc) return rc;
  }
  return NSPT_OK;
}

// minb: the smallest block along a split direction.  The reference needs 2
// (threads of one barrier step then share no link); an on-the-fly sweep of
// an improved action needs 3, because its rectangles reach two sites: with
// blocks of 2 the reference's own threaded run races and differs from run
// to run.
static bool grid_ok(const int L[4], const int grid[4], int minb = 2) {
  for (int d = 0; d < 4; d++) {
    if (grid[d] < 1 || L[d] % grid[d]) return false;
    if (grid[d] > 1 && L[d] / grid[d] < minb) return false;
  }
  return true;
}

static int grid_min_block(const nspt_ctx *ctx) {
  return (ctx->flags & NSPT_UPDATE_ONTHEFLY) && ctx->c1 != 0.0 ? 3 : 2;
}

// ---------------- context ----------------

static int upload_constants(nspt_ctx *ctx) {
  double2 om[4][9], omd[4][9];
  memset(om, 0, sizeof(om));
  for (int d = 0; d < 4; d++)
    for (int e = 0; e < 9; e += 4) om[d][e] = make_double2(1.0, 0.0);
  // twistmatrices.h:158-240
  om[1][0] = make_double2(cos(-2. * M_PI / 3.), sin(-2. * M_PI / 3.));
  om[1][8] = make_double2(cos(2. * M_PI / 3.), sin(2. * M_PI / 3.));
  for (int e = 0; e < 9; e++) om[2][e] = make_double2(0, 0), om[3][e] = make_double2(0, 0);
  om[2][1] = om[2][5] = om[2][6] = make_double2(1.0, 0.0);
  om[3][1] = make_double2(cos(-2. * M_PI / 3.), sin(-2. * M_PI / 3.));
  om[3][5] = make_double2(1.0, 0.0);
  om[3][6] = make_double2(cos(2. * M_PI / 3.), sin(2. * M_PI / 3.));
  for (int d = 0; d < 4; d++)
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) omd[d][3 * i + j] = make_double2(om[d][3 * j + i].x, -om[d][3 * j + i].y);
  CK(cudaMemcpyToSymbol(c_om, om, sizeof(om)));
  CK(cudaMemcpyToSymbol(c_omd, omd, sizeof(omd)));
  double p2[4][128];
  memset(p2, 0, sizeof(p2));
  for (int d = 0; d < 4; d++)
    for (int i = 0; i < ctx->L[d]; i++) {  // lattice.h:1144-1169
      double p = 2 * M_PI * i / ctx->L[d];
      double h = sin(p * 0.5);
      h *= 4 * h;
      p2[d][i] = h;
    }
  CK(cudaMemcpy(ctx->p2, p2, sizeof(p2), cudaMemcpyHostToDevice));
  double2 tw[64];
  for (int k = 0; k < 64; k++) {
    double ang = -1.0 * 2.0 * M_PI * (double)k / 64.0;
    tw[k] = make_double2(cos(ang), sin(ang));
  }
  CK(cudaMemcpyToSymbol(c_tw64, tw, sizeof(tw)));
  if (ctx->ftw) {
    std::vector<double2> ftw(4 * 128, make_double2(0.0, 0.0));
    for (int d = 0; d < 4; d++)
      for (int t = 0; t < ctx->L[d]; t++) {
        const double ang = -2.0 * M_PI * (double)t / (double)ctx->L[d];
        ftw[d * 128 + t] = make_double2(cos(ang), sin(ang));
      }
    CK(cudaMemcpy(ctx->ftw, ftw.data(), ftw.size() * sizeof(double2), cudaMemcpyHostToDevice));
  }
  return NSPT_OK;
}

static void free_all(nspt_ctx *ctx) {
  void *ptrs[] = {ctx->U, ctx->Uf, ctx->F, ctx->Ff, ctx->Lg, ctx->Wg, ctx->Gx, ctx->p2, ctx->ftw,
                  ctx->dcounter,
                  ctx->loop_part, ctx->obs_tr2, ctx->ff_e, ctx->ff_mx,
                  ctx->obs_tr, ctx->obs_tru, ctx->obs_norm, ctx->red2, ctx->red1, ctx->noise};
  for (void *p : ptrs)
    if (p) cudaFree(p);
}

extern "C" int nspt_create(const int L[4], int N, unsigned flags, double alpha, nspt_ctx **out) {
  nspt_ctx *ctx = nullptr;
  if (!out || !L) return NSPT_ERR_ARG;
  *out = nullptr;
  if (N < 1 || N > NSPT_MAX_ORDER) return NSPT_ERR_ORDER;
  const unsigned actions = NSPT_ACTION_TLSYM | NSPT_ACTION_IWA | NSPT_ACTION_DBW2;
  const unsigned known = NSPT_TWIST_Y | NSPT_TWIST_Z | NSPT_TWIST_T | NSPT_ZEROMODE | NSPT_GF_FA |
                         NSPT_GF_LOCAL | actions | NSPT_PRECISION_FF | NSPT_UPDATE_ONTHEFLY;
  if (flags & ~known) return NSPT_ERR_ARG;
  // the on-the-fly update is built for the FP64 sweeps
  if ((flags & NSPT_UPDATE_ONTHEFLY) && (flags & NSPT_PRECISION_FF)) return NSPT_ERR_ARG;
  // float-float products are built into the Wilson sweep only
  if ((flags & NSPT_PRECISION_FF) && (flags & actions)) return NSPT_ERR_ARG;
  if (__builtin_popcount(flags & actions) > 1) return NSPT_ERR_ARG;
  // the reference has improved actions with periodic boundaries only (choices.h:110)
  if ((flags & actions) && (flags & (NSPT_TWIST_Y | NSPT_TWIST_Z | NSPT_TWIST_T)))
    return NSPT_ERR_ARG;
  if ((flags & NSPT_GF_FA) && (flags & NSPT_GF_LOCAL)) return NSPT_ERR_ARG;
  long V = 1;
  for (int d = 0; d < 4; d++) {
    if (L[d] < 2 || L[d] > 128) return NSPT_ERR_ARG;
    V *= L[d];
  }
  // the reference defines zero modes and FA only with periodic boundaries
  if ((flags & (NSPT_TWIST_Y | NSPT_TWIST_Z | NSPT_TWIST_T)) && (flags & (NSPT_ZEROMODE | NSPT_GF_FA)))
    return NSPT_ERR_ARG;
  if (V * 4 * 9L * N > (1L << 40)) return NSPT_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return NSPT_ERR_NODEVICE;
  ctx = new nspt_ctx();
  memset(ctx->L, 0, sizeof(ctx->L));
  for (int d = 0; d < 4; d++) ctx->L[d] = L[d];
  ctx->N = N;
  ctx->flags = flags;
  ctx->alpha = alpha;
  ctx->V = V;
  ctx->U = ctx->Uf = ctx->F = ctx->Ff = ctx->Lg = ctx->Wg = ctx->Gx = nullptr;
  ctx->p2 = nullptr;
  ctx->ftw = nullptr;
  ctx->dcounter = nullptr;
  ctx->sweep_warps = 0;
  ctx->shape_mo = 0;
  ctx->lg_current = false;
  ctx->snap_valid = false;
  ctx->launch_gen = 0;
  ctx->loop_part = nullptr;
  ctx->loop_part_n = 0;
  ctx->timeout_s = 0.0;
  ctx->busy = false;
  ctx->obs_tr2 = nullptr;
  ctx->ff_e = nullptr;
  ctx->ff_mx = nullptr;
  ctx->ff_auto = true;
  // improved action parameters, Quenched.cc:311-322
  ctx->c1 = (flags & NSPT_ACTION_TLSYM) ? -1.0 / 12.0
          : (flags & NSPT_ACTION_IWA)   ? -0.331
          : (flags & NSPT_ACTION_DBW2)  ? -1.4088
                                        : 0.0;
  // the finest thread grid the reference accepts: blocks of 2 sites where L
  // is even, one thread along odd extents (for an improved action on the
  // fly: blocks of the smallest size >= 3 dividing L)
  for (int d = 0; d < 4; d++) {
    if (grid_min_block(ctx) == 2) {
      ctx->gf_grid[d] = (L[d] % 2 == 0) ? L[d] / 2 : 1;
    } else {
      int b = 3;
      while (L[d] % b) b++;
      ctx->gf_grid[d] = L[d] / b;
    }
  }
  ctx->gf_form = NSPT_LGF_AUTO;
  ctx->obs_tr = ctx->obs_tru = ctx->red2 = nullptr;
  ctx->obs_norm = ctx->red1 = ctx->noise = nullptr;
  ctx->noise_pending = false;
  ctx->have_obs = false;
  ctx->seed = 0x5eed5eedULL;
  ctx->counter = 0;
  ctx->last_ms = 0.f;
  ctx->bytes = 0;
  auto fail = [&](int code) {
    free_all(ctx);
    delete ctx;
    return code;
  };
  if (cudaGetDevice(&ctx->dev) != cudaSuccess) return fail(NSPT_ERR_CUDA);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, ctx->dev) != cudaSuccess) return fail(NSPT_ERR_CUDA);
  ctx->nsm = prop.multiProcessorCount;
  ctx->smem_optin = prop.sharedMemPerBlockOptin;
  Geo &g = ctx->geo;
  for (int d = 0; d < 4; d++) g.L[d] = L[d];
  g.V = (int)V;
  g.s2 = L[3];
  g.s1 = L[2] * L[3];
  g.s0 = L[1] * L[2] * L[3];
  g.twist = 0;
  // the sweep's site tiles (sweep_link): 4 x 4 x 4 where the extents allow
  // (measured at 16^4 x 24: DRAM traffic 1.68x the algorithmic bytes, against
  // 2.89x for 4 x 4 x L2 and 3.98x untiled; the same kernel time)
  g.t0 = L[0] % 4 == 0 ? 4 : L[0] % 2 == 0 ? 2 : 1;
  g.t1 = L[1] % 4 == 0 ? 4 : L[1] % 2 == 0 ? 2 : 1;
  g.t2 = L[2] % 4 == 0 ? 4 : L[2] % 2 == 0 ? 2 : 1;
  if (flags & NSPT_TWIST_Y) g.twist |= 2u;
  if (flags & NSPT_TWIST_Z) g.twist |= 4u;
  if (flags & NSPT_TWIST_T) g.twist |= 8u;
  // slot stride = 3 (mod 8) 16-byte quads: see series.cuh on bank quads
  ctx->SS = 1 + 9 * N;
  while (ctx->SS % 8 != 3) ctx->SS++;
  // one warp (3 link groups of 3 slots) must fit in a CTA
  if ((size_t)LPW * group_bytes(ctx, SWEEP_SLOTS, 0) > ctx->smem_optin) return fail(NSPT_ERR_ORDER);
  if (ctx->c1 != 0.0 && (size_t)LPW * group_bytes(ctx, IMP_SLOTS, 0) > ctx->smem_optin)
    return fail(NSPT_ERR_ORDER);
  if (cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking) != cudaSuccess) return fail(NSPT_ERR_CUDA);
  cudaEventCreate(&ctx->ev0);
  cudaEventCreate(&ctx->ev1);
  for (int i = 0; i < 2 * nspt_ctx::KEV; i++) cudaEventCreate(&ctx->kev[i]);
  ctx->kcount = 0;
  ctx->last_kernel_ms = 0.0;
  const size_t field = (size_t)4 * 9 * N * V * sizeof(double2);
  const size_t flagb = (size_t)4 * V * sizeof(double2);
  const size_t nl = (size_t)4 * V;
  auto alloc = [&](void **p, size_t n) {
    if (cudaMalloc(p, n) != cudaSuccess) return false;
    ctx->bytes += n;
    return true;
  };
  bool ok = alloc((void **)&ctx->U, field) && alloc((void **)&ctx->F, field) &&
            alloc((void **)&ctx->Uf, flagb) && alloc((void **)&ctx->Ff, flagb) &&
            alloc((void **)&ctx->obs_tr, (N + 1) * nl * sizeof(double2)) &&
            alloc((void **)&ctx->obs_tru, N * nl * sizeof(double2)) &&
            alloc((void **)&ctx->obs_norm, N * nl * sizeof(double)) &&
            alloc((void **)&ctx->red2, (2 * (N + 1) + 4 * N + 36 * N) * sizeof(double2)) &&
            alloc((void **)&ctx->red1, N * sizeof(double)) &&
            alloc((void **)&ctx->p2, 4 * 128 * sizeof(double)) &&
            alloc((void **)&ctx->dcounter, sizeof(unsigned long long));
  if (ok && (flags & (NSPT_ZEROMODE | NSPT_GF_FA))) ok = alloc((void **)&ctx->Lg, field);
  if (ok && ctx->c1 != 0.0) ok = alloc((void **)&ctx->obs_tr2, (N + 1) * nl * sizeof(double2));
  if (ok && (flags & NSPT_PRECISION_FF))
    ok = alloc((void **)&ctx->ff_e, sizeof(int)) &&
         alloc((void **)&ctx->ff_mx, N * sizeof(unsigned long long));
  if (ok && (flags & NSPT_GF_FA))
    ok = alloc((void **)&ctx->Wg, field / 4) && alloc((void **)&ctx->Gx, field / 4) &&
         alloc((void **)&ctx->ftw, 4 * 128 * sizeof(double2));
  if (!ok) {
    cudaGetLastError();
    cudaStreamDestroy(ctx->st);
    return fail(NSPT_ERR_NOMEM);
  }
  if (upload_constants(ctx) != NSPT_OK) return fail(NSPT_ERR_CUDA);
  if (cudaMemsetAsync(ctx->dcounter, 0, sizeof(unsigned long long), ctx->st) != cudaSuccess ||
      (ctx->ff_e && cudaMemsetAsync(ctx->ff_e, 0, sizeof(int), ctx->st) != cudaSuccess)) {
    cudaStreamDestroy(ctx->st);
    return fail(NSPT_ERR_CUDA);
  }
  *out = ctx;
  return nspt_cold_start(ctx);
}

extern "C" int nspt_destroy(nspt_ctx *ctx) {
  if (!ctx) return NSPT_ERR_ARG;
  cudaStreamSynchronize(ctx->st);
  free_all(ctx);
  cudaEventDestroy(ctx->ev0);
  cudaEventDestroy(ctx->ev1);
  for (int i = 0; i < 2 * nspt_ctx::KEV; i++) cudaEventDestroy(ctx->kev[i]);
  cudaStreamDestroy(ctx->st);
  delete ctx;
  return NSPT_OK;
}

extern "C" size_t nspt_device_bytes(const nspt_ctx *ctx) { return ctx ? ctx->bytes : 0; }

extern "C" int nspt_cold_start(nspt_ctx *ctx) {
  if (!ctx) return NSPT_ERR_ARG;
  ctx->lg_current = false;
  ctx->snap_valid = false;  // a new field: no stale twisted reads
  const size_t nU = (size_t)4 * 9 * ctx->N * ctx->V, nF = (size_t)4 * ctx->V;
  k_cold<<<ctx->nsm * 8, 256, 0, ctx->st>>>(ctx->U, ctx->Uf, nU, nF);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->st));
  return NSPT_OK;
}

static const size_t kChunkBytes = 64u << 20;

extern "C" int nspt_upload_links(nspt_ctx *ctx, const void *aos, int A) {
  if (!ctx || !aos || A < ctx->N) return NSPT_ERR_ARG;
  ctx->lg_current = false;
  ctx->snap_valid = false;  // a new field: no stale twisted reads
  const size_t per_site = (size_t)4 * (1 + 9 * A) * sizeof(double2);
  const int cs = (int)std::max<size_t>(1, std::min<size_t>(kChunkBytes / per_site, ctx->V));
  double2 *buf = nullptr;
  CK(cudaMalloc(&buf, per_site * cs));
  int rc = NSPT_OK;
  for (long s0 = 0; s0 < ctx->V; s0 += cs) {
    const int n = (int)std::min<long>(cs, ctx->V - s0);
    cudaError_t e = cudaMemcpyAsync(buf, (const char *)aos + per_site * s0, per_site * n,
                                    cudaMemcpyHostToDevice, ctx->st);
    if (e == cudaSuccess) {
      k_unpack<<<ctx->nsm * 8, 256, 0, ctx->st>>>(buf, A, (int)s0, n, ctx->U, ctx->Uf, ctx->N,
                                                  (size_t)ctx->V);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
      ctx->err = std::string("upload: ") + cudaGetErrorString(e);
      rc = NSPT_ERR_CUDA;
      break;
    }
  }
  cudaStreamSynchronize(ctx->st);
  cudaFree(buf);
  return rc;
}

extern "C" int nspt_download_links(nspt_ctx *ctx, void *aos, int A) {
  if (!ctx || !aos || A < ctx->N) return NSPT_ERR_ARG;
  const size_t per_site = (size_t)4 * (1 + 9 * A) * sizeof(double2);
  const int cs = (int)std::max<size_t>(1, std::min<size_t>(kChunkBytes / per_site, ctx->V));
  double2 *buf = nullptr;
  CK(cudaMalloc(&buf, per_site * cs));
  int rc = NSPT_OK;
  for (long s0 = 0; s0 < ctx->V; s0 += cs) {
    const int n = (int)std::min<long>(cs, ctx->V - s0);
    k_pack<<<ctx->nsm * 8, 256, 0, ctx->st>>>(buf, A, (int)s0, n, ctx->U, ctx->Uf, ctx->N,
                                              (size_t)ctx->V);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync((char *)aos + per_site * s0, buf, per_site * n, cudaMemcpyDeviceToHost,
                          ctx->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
    if (e != cudaSuccess) {
      ctx->err = std::string("download: ") + cudaGetErrorString(e);
      rc = NSPT_ERR_CUDA;
      break;
    }
  }
  cudaFree(buf);
  return rc;
}

extern "C" int nspt_set_noise(nspt_ctx *ctx, const double *eta) {
  if (!ctx || !eta) return NSPT_ERR_ARG;
  const size_t n = (size_t)ctx->V * 4 * 8 * sizeof(double);
  if (!ctx->noise) {
    if (cudaMalloc(&ctx->noise, n) != cudaSuccess) {
      cudaGetLastError();
      ctx->noise = nullptr;
      return NSPT_ERR_NOMEM;
    }
    ctx->bytes += n;
  }
  CK(cudaMemcpyAsync(ctx->noise, eta, n, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  ctx->noise_pending = true;
  return NSPT_OK;
}

extern "C" int nspt_seed(nspt_ctx *ctx, uint64_t seed, uint64_t counter) {
  if (!ctx) return NSPT_ERR_ARG;
  ctx->seed = seed;
  ctx->counter = counter;
  ctx->launch_gen++;
  const unsigned long long c = counter;
  CK(cudaMemcpyAsync(ctx->dcounter, &c, sizeof(c), cudaMemcpyHostToDevice, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return NSPT_OK;
}

extern "C" int nspt_get_seed(nspt_ctx *ctx, uint64_t *seed, uint64_t *counter) {
  if (!ctx || !seed || !counter) return NSPT_ERR_ARG;
  *seed = ctx->seed;
  *counter = ctx->counter;
  return NSPT_OK;
}

// Device time of a call: events on the context's stream around its launches.
// Wait for the context's stream, at most timeout_s seconds when a limit is
// set: the device work itself is never interrupted; past the limit the call
// returns NSPT_ERR_TIMEOUT and the next call waits for that work first.
static int wait_stream(nspt_ctx *ctx, cudaEvent_t done) {
  if (ctx->timeout_s <= 0.0) {
    CK(cudaEventSynchronize(done));
    ctx->busy = false;
    return NSPT_OK;
  }
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t e = cudaEventQuery(done);
    if (e == cudaSuccess) break;
    if (e != cudaErrorNotReady) CK(e);
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (el > ctx->timeout_s) {
      ctx->busy = true;
      char msg[96];
      snprintf(msg, sizeof(msg), "device work still running after %.3g s", el);
      ctx->err = msg;
      return NSPT_ERR_TIMEOUT;
    }
  }
  ctx->busy = false;
  return NSPT_OK;
}

static int timed_begin(nspt_ctx *ctx) {
  if (ctx->busy) {  // the work a timed-out call left behind
    CK(cudaEventRecord(ctx->ev1, ctx->st));
    int rc = wait_stream(ctx, ctx->ev1);
    if (rc) return rc;
  }
  ctx->kcount = 0;
  CK(cudaEventRecord(ctx->ev0, ctx->st));
  return NSPT_OK;
}
static int timed_end(nspt_ctx *ctx) {
  CK(cudaEventRecord(ctx->ev1, ctx->st));
  int rc = wait_stream(ctx, ctx->ev1);
  if (rc) return rc;
  cudaEventElapsedTime(&ctx->last_ms, ctx->ev0, ctx->ev1);
  double sum = 0.0;
  for (int i = 0; i < ctx->kcount; i++) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->kev[2 * i], ctx->kev[2 * i + 1]);
    sum += ms;
  }
  ctx->last_kernel_ms = ctx->kcount ? sum / ctx->kcount : 0.0;
  return NSPT_OK;
}

extern "C" int nspt_gauge_wilson(nspt_ctx *ctx, double dt) {
  if (!ctx || !(dt >= 0.0)) return NSPT_ERR_ARG;
  int rc = timed_begin(ctx);
  if (rc) return rc;
  const bool use = ctx->noise_pending;
  rc = do_sweep(ctx, dt, use);
  ctx->noise_pending = false;
  if (rc) return rc;
  return timed_end(ctx);
}

extern "C" int nspt_zero_modes_subtraction(nspt_ctx *ctx) {
  if (!ctx) return NSPT_ERR_ARG;
  if (!(ctx->flags & NSPT_ZEROMODE) || !ctx->have_obs) return NSPT_ERR_STATE;
  int rc = timed_begin(ctx);
  if (rc || (rc = do_zero_modes(ctx))) return rc;
  return timed_end(ctx);
}

extern "C" int nspt_fa_gauge_fixing(nspt_ctx *ctx, double alpha) {
  if (!ctx) return NSPT_ERR_ARG;
  if (!(ctx->flags & NSPT_GF_FA)) return NSPT_ERR_STATE;
  int rc = timed_begin(ctx);
  if (rc || (rc = do_fa(ctx, alpha))) return rc;
  return timed_end(ctx);
}

// Sums over planes and sites of the 1x2, 2x2, 2x4 and 4x4 loop traces,
// h[q * (N+1) + k], un-normalised (k_loops, then its per-CTA rows summed)
static int loop_sums(nspt_ctx *ctx, std::vector<double2> &h) {
  const int N = ctx->N, row = 4 * (N + 1);
  const size_t gb = ((size_t)LOOP_SLOTS * ctx->SS + row) * sizeof(double2);
  const int warps = (int)std::min<size_t>(8, ctx->smem_optin / (LPW * gb));
  if (warps < 1) return NSPT_ERR_ORDER;
  const long units = 6L * ctx->V;
  const long per_cta = (long)warps * LPW;
  const int grid = (int)std::min<long>((units + per_cta - 1) / per_cta, 8L * ctx->nsm);
  const size_t need = (size_t)(grid + 1) * row;
  if (need > ctx->loop_part_n) {
    if (ctx->loop_part) cudaFree(ctx->loop_part);
    ctx->loop_part = nullptr;
    ctx->loop_part_n = 0;
    if (cudaMalloc(&ctx->loop_part, need * sizeof(double2)) != cudaSuccess) {
      cudaGetLastError();
      return NSPT_ERR_NOMEM;
    }
    ctx->loop_part_n = need;
  }
  double2 *part = ctx->loop_part, *res = ctx->loop_part + (size_t)grid * row;
  const size_t smem = (size_t)warps * LPW * gb;
  int rc = timed_begin(ctx);
  if (rc) return rc;
  CK(cudaFuncSetAttribute(k_loops, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_loops<<<grid, 32 * warps, smem, ctx->st>>>(ctx->U, ctx->Uf, N, ctx->SS, ctx->geo, part);
  CK(cudaGetLastError());
  k_rows_sum<<<(row + 127) / 128, 128, 0, ctx->st>>>(part, grid, row, res);
  CK(cudaGetLastError());
  h.resize(row);
  CK(cudaMemcpyAsync(h.data(), res, row * sizeof(double2), cudaMemcpyDeviceToHost, ctx->st));
  return timed_end(ctx);
}

extern "C" int nspt_wilson_loops(nspt_ctx *ctx, double *loops) {
  if (!ctx || !loops) return NSPT_ERR_ARG;
  if (ctx->geo.twist) return NSPT_ERR_STATE;  // the reference has them with periodic bc only
  const int N = ctx->N;
  std::vector<double2> h;
  int rc = loop_sums(ctx, h);
  if (rc) return rc;
  // loopNorm = 1/(3*2*3*V), halved for 1x2 and 2x4 (nspt.cc:1280-1306)
  const double norm = 1. / (3 * 2 * 3 * (double)ctx->V);
  const double fac[4] = {.5 * norm, norm, .5 * norm, norm};
  for (int q = 0; q < 4; q++)
    for (int k = 0; k <= N; k++) {
      loops[2 * (q * (N + 1) + k)] = h[q * (N + 1) + k].x * fac[q];
      loops[2 * (q * (N + 1) + k) + 1] = h[q * (N + 1) + k].y * fac[q];
    }
  return NSPT_OK;
}

extern "C" int nspt_wl2x2(nspt_ctx *ctx, double *loop) {
  if (!ctx || !loop) return NSPT_ERR_ARG;
  if (ctx->geo.twist) return NSPT_ERR_STATE;  // __WILLOOP_2x2__ is periodic only (choices.h:75-78)
  const int N = ctx->N;
  std::vector<double2> h;
  int rc = loop_sums(ctx, h);
  if (rc) return rc;
  // WL2x2 walks each plane's 2x2 loop the other way round from ComputeLoops'
  // 2x2 (mu > nu, along mu first): its trace is the complex conjugate.
  // Normalisation rVol * D18 (nspt.cc:1121).
  const double norm = 1. / (18. * (double)ctx->V);
  for (int k = 0; k <= N; k++) {
    loop[2 * k] = h[(N + 1) + k].x * norm;
    loop[2 * k + 1] = -h[(N + 1) + k].y * norm;
  }
  return NSPT_OK;
}

extern "C" int nspt_local_gauge_fixing(nspt_ctx *ctx, double alpha) {
  if (!ctx) return NSPT_ERR_ARG;
  int rc = timed_begin(ctx);
  if (rc || (rc = do_local_gf(ctx, alpha))) return rc;
  return timed_end(ctx);
}

extern "C" int nspt_set_gf_grid(nspt_ctx *ctx, const int grid[4]) {
  if (!ctx || !grid || !grid_ok(ctx->L, grid, grid_min_block(ctx))) return NSPT_ERR_ARG;
  for (int d = 0; d < 4; d++) ctx->gf_grid[d] = grid[d];
  ctx->launch_gen++;
  return NSPT_OK;
}

extern "C" int nspt_set_local_gf_form(nspt_ctx *ctx, int form) {
  if (!ctx) return NSPT_ERR_ARG;
  if (form != NSPT_LGF_AUTO && form != NSPT_LGF_GROUP && form != NSPT_LGF_TEAM) return NSPT_ERR_ARG;
  ctx->gf_form = form;
  ctx->launch_gen++;
  return NSPT_OK;
}

extern "C" int nspt_step(nspt_ctx *ctx, double dt, int nsteps, int gf_every) {
  if (!ctx || nsteps < 0 || !(dt >= 0.0) || gf_every < 0) return NSPT_ERR_ARG;
  int rc0 = timed_begin(ctx);
  if (rc0) return rc0;
  for (int s = 0; s < nsteps; s++) {
    const bool use = ctx->noise_pending;
    int rc = do_sweep(ctx, dt, use);
    ctx->noise_pending = false;
    if (rc) return rc;
    if (ctx->flags & NSPT_ZEROMODE)
      if ((rc = do_zero_modes(ctx))) return rc;
    if ((ctx->flags & NSPT_GF_FA) && gf_every > 0 && ((ctx->counter % gf_every) == 0))
      if ((rc = do_fa(ctx, ctx->alpha))) return rc;
    if ((ctx->flags & NSPT_GF_LOCAL) && gf_every > 0 && ((ctx->counter % gf_every) == 0))
      if ((rc = do_local_gf(ctx, ctx->alpha))) return rc;
    ctx->snap_valid = false;  // twist_boundary ends the step (nspt.cc:1025-1027)
  }
  return timed_end(ctx);
}

extern "C" int nspt_twist_boundary(nspt_ctx *ctx) {
  if (!ctx) return NSPT_ERR_ARG;
  ctx->snap_valid = false;
  return NSPT_OK;
}

extern "C" double nspt_last_step_ms(const nspt_ctx *ctx) { return ctx ? ctx->last_ms : 0.0; }
extern "C" double nspt_last_kernel_ms(const nspt_ctx *ctx) {
  return ctx ? ctx->last_kernel_ms : 0.0;
}

extern "C" int nspt_observables(nspt_ctx *ctx, double *plaq, double *norm, double *trU) {
  if (!ctx) return NSPT_ERR_ARG;
  if (!ctx->have_obs) return NSPT_ERR_STATE;
  const int N = ctx->N;
  std::vector<double2> r2((N + 1) + 4 * N);
  std::vector<double> r1(N);
  CK(cudaMemcpyAsync(r2.data(), ctx->red2, r2.size() * sizeof(double2), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaMemcpyAsync(r1.data(), ctx->red1, r1.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  const double V = (double)ctx->V;
  (void)V;
  if (plaq)
    for (int k = 0; k <= N; k++) {  // nspt.cc:570-597
      plaq[2 * k] = r2[k].x / (double)(72 * ctx->V);
      plaq[2 * k + 1] = r2[k].y / (double)(72 * ctx->V);
    }
  if (norm)
    for (int k = 0; k < N; k++) norm[k] = r1[k] / (double)(12 * ctx->V);
  if (trU)
    for (int k = 0; k < N; k++)
      for (int mu = 0; mu < 4; mu++) {
        const double2 t = r2[(N + 1) + 4 * k + mu];
        trU[2 * (mu * N + k)] = t.x / (double)(3 * ctx->V);
        trU[2 * (mu * N + k) + 1] = t.y / (double)(3 * ctx->V);
      }
  return NSPT_OK;
}

extern "C" int nspt_set_timeout(nspt_ctx *ctx, double seconds) {
  if (!ctx || !(seconds >= 0.0)) return NSPT_ERR_ARG;
  ctx->timeout_s = seconds;
  return NSPT_OK;
}

extern "C" int nspt_set_ff_scale(nspt_ctx *ctx, int automatic, int e) {
  if (!ctx) return NSPT_ERR_ARG;
  if (!(ctx->flags & NSPT_PRECISION_FF)) {
    ctx->err = "float-float scale: context created without NSPT_PRECISION_FF";
    return NSPT_ERR_STATE;
  }
  ctx->launch_gen++;
  if (automatic) {
    ctx->ff_auto = true;
    return NSPT_OK;
  }
  if ((long)std::abs(e) * ctx->N > 1000) {
    ctx->err = "float-float scale: |e| N above 1000";
    return NSPT_ERR_ARG;
  }
  ctx->ff_auto = false;
  CK(cudaMemcpyAsync(ctx->ff_e, &e, sizeof(int), cudaMemcpyHostToDevice, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return NSPT_OK;
}

extern "C" int nspt_get_ff_scale(nspt_ctx *ctx, int *e) {
  if (!ctx || !e) return NSPT_ERR_ARG;
  if (!(ctx->flags & NSPT_PRECISION_FF)) {
    ctx->err = "float-float scale: context created without NSPT_PRECISION_FF";
    return NSPT_ERR_STATE;
  }
  CK(cudaMemcpyAsync(e, ctx->ff_e, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return NSPT_OK;
}

extern "C" int nspt_rect_observables(nspt_ctx *ctx, double *w2) {
  if (!ctx || !w2) return NSPT_ERR_ARG;
  if (ctx->c1 == 0.0 || !ctx->have_obs) return NSPT_ERR_STATE;
  const int N = ctx->N;
  std::vector<double2> r(N + 1);
  CK(cudaMemcpyAsync(r.data(), ctx->red2 + w2_offset(N), r.size() * sizeof(double2),
                     cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  for (int k = 0; k <= N; k++) {  // nspt.cc:586-597
    w2[2 * k] = r[k].x / (double)(72 * ctx->V);
    w2[2 * k + 1] = r[k].y / (double)(72 * ctx->V);
  }
  return NSPT_OK;
}

extern "C" int nspt_plaquette_measure(nspt_ctx *ctx, double *plaq) {
  if (!ctx || !plaq) return NSPT_ERR_ARG;
  SweepArgs a;
  memset(&a, 0, sizeof(a));
  a.U = ctx->U;
  a.Uf = ctx->Uf;
  a.obs_tr = ctx->obs_tr;
  a.N = ctx->N;
  a.SS = ctx->SS;
  a.g = ctx->geo;
  int rc = launch_sweep(ctx, a, true);
  if (rc) return rc;
  const int N = ctx->N;
  const long nl = 4 * ctx->V;
  double2 *tmp = ctx->red2 + (N + 1) + 4 * N;  // MM area, free outside zero modes
  k_rowsum<double2><<<N + 1, 256, 0, ctx->st>>>(ctx->obs_tr, (size_t)nl, nl, tmp);
  CK(cudaGetLastError());
  std::vector<double2> r(N + 1);
  CK(cudaMemcpyAsync(r.data(), tmp, r.size() * sizeof(double2), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  ctx->have_obs = false;  // the trace buffer now holds the static measurement
  for (int k = 0; k <= N; k++) {  // nspt.cc:1398-1404
    plaq[2 * k] = r[k].x / (double)(ctx->V * 72);
    plaq[2 * k + 1] = r[k].y / (double)(ctx->V * 72);
  }
  return NSPT_OK;
}

extern "C" int nspt_save_config(nspt_ctx *ctx, const char *path, int A) {
  if (!ctx || !path || A < ctx->N) return NSPT_ERR_ARG;
  std::vector<double> host((size_t)ctx->V * 4 * (1 + 9 * A) * 2);
  int rc = nspt_download_links(ctx, host.data(), A);
  if (rc) return rc;
  std::vector<double> plaq(2 * (ctx->N + 1));
  rc = nspt_plaquette_measure(ctx, plaq.data());
  if (rc) return rc;
  std::vector<double> trailer(2 * (A + 1), 0.0);
  std::copy(plaq.begin(), plaq.end(), trailer.begin());
  FILE *f = fopen(path, "wb");
  if (!f) return NSPT_ERR_IO;
  bool ok = fwrite(host.data(), sizeof(double), host.size(), f) == host.size() &&
            fwrite(trailer.data(), sizeof(double), trailer.size(), f) == trailer.size();
  ok = (fclose(f) == 0) && ok;
  return ok ? NSPT_OK : NSPT_ERR_IO;
}

extern "C" int nspt_load_config(nspt_ctx *ctx, const char *path, int A, double *plaq_trailer) {
  if (!ctx || !path || A < ctx->N) return NSPT_ERR_ARG;
  FILE *f = fopen(path, "rb");
  if (!f) return NSPT_ERR_IO;
  std::vector<double> host((size_t)ctx->V * 4 * (1 + 9 * A) * 2);
  std::vector<double> trailer(2 * (A + 1));
  // io::load checks the byte count (QCDenvNODEpt_test.h:370-374)
  fseek(f, 0, SEEK_END);
  const long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  const long want = (long)((host.size() + trailer.size()) * sizeof(double));
  bool ok = sz == want && fread(host.data(), sizeof(double), host.size(), f) == host.size() &&
            fread(trailer.data(), sizeof(double), trailer.size(), f) == trailer.size();
  fclose(f);
  if (!ok) return NSPT_ERR_IO;
  if (plaq_trailer) std::copy(trailer.begin(), trailer.end(), plaq_trailer);
  return nspt_upload_links(ctx, host.data(), A);
}

extern "C" int nspt_load_lower_order(nspt_ctx *ctx, const char *path, int loworder,
                                     double *plaq_trailer) {
  if (!ctx || !path) return NSPT_ERR_ARG;
  // QCDenvNODEpt_test.h:377-380: no more orders than the field holds
  if (loworder < 1 || loworder > ctx->N) return NSPT_ERR_ORDER;
  const int lo = loworder, N = ctx->N;
  FILE *f = fopen(path, "rb");
  if (!f) return NSPT_ERR_IO;
  const size_t ser_lo = 2 * (1 + 9 * (size_t)lo), ser_n = 2 * (1 + 9 * (size_t)N);
  std::vector<double> file((size_t)ctx->V * 4 * ser_lo);
  std::vector<double> trailer(2 * (lo + 1));
  // the exact byte count of a loworder file (QCDenvNODEpt_test.h:387-390)
  fseek(f, 0, SEEK_END);
  const long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  const long want = (long)((file.size() + trailer.size()) * sizeof(double));
  bool ok = sz == want && fread(file.data(), sizeof(double), file.size(), f) == file.size() &&
            fread(trailer.data(), sizeof(double), trailer.size(), f) == trailer.size();
  fclose(f);
  if (!ok) return NSPT_ERR_IO;
  // orders 1..lo from the file, every order above zero (QCDenvNODEpt_test.h:396-411)
  std::vector<double> host((size_t)ctx->V * 4 * ser_n, 0.0);
  for (size_t l = 0; l < (size_t)ctx->V * 4; l++)
    std::copy(file.begin() + l * ser_lo, file.begin() + (l + 1) * ser_lo, host.begin() + l * ser_n);
  std::vector<double>().swap(file);
  int rc = nspt_upload_links(ctx, host.data(), N);
  if (rc) return rc;
  // U = exp(reH(log U)) per link (QCDenvNODEpt_test.h:414-417)
  double2 *U = ctx->U, *Uf = ctx->Uf;
  const int SS = ctx->SS;
  const Geo geo = ctx->geo;
  cudaStream_t st = ctx->st;
  const bool low = use_low(ctx);
  rc = launch_groups(
      ctx, low ? (const void *)k_unitarise<true> : (const void *)k_unitarise<false>, 3, 4 * ctx->V,
      [&](unsigned g, dim3 b, size_t sm) {
        if (low)
          k_unitarise<true><<<g, b, sm, st>>>(U, Uf, N, SS, geo);
        else
          k_unitarise<false><<<g, b, sm, st>>>(U, Uf, N, SS, geo);
      },
      "unitarise", 0, low);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->st));
  ctx->have_obs = false;
  if (plaq_trailer) std::copy(trailer.begin(), trailer.end(), plaq_trailer);
  return NSPT_OK;
}

extern "C" int nspt_measure_fp64_peak(double *tflops) {
  nspt_ctx *ctx = nullptr;
  if (!tflops) return NSPT_ERR_ARG;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, dev));
  double *out = nullptr;
  CK(cudaMalloc(&out, sizeof(double)));
  const int blocks = prop.multiProcessorCount * 8, threads = 256, iters = 4096;
  k_fp64_peak<<<blocks, threads>>>(out, 64, 1.0);  // warm-up
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  k_fp64_peak<<<blocks, threads>>>(out, iters, 1.0);
  cudaEventRecord(e1);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (e != cudaSuccess) return NSPT_ERR_CUDA;
  const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return NSPT_OK;
}

// allocation-free plaquette of a caller-owned device field
#include "noalloc.cuh"

// batches of replicas in one CUDA graph
#include "batch.cuh"
