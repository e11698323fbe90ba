// Batches of independent replicas advanced in one CUDA graph.
//
// A replica is an ordinary context (its own fields, noise seed and time
// step).  A batch step captures, once, the launches of every replica's
// Langevin step on its own stream -- forked from the batch stream and joined
// back -- so the replicas' kernels are independent graph nodes that run side
// by side on the SMs a small lattice alone would leave idle; every later
// step replays the graph.  Three things make a replay equal to a fresh
// launch: the Philox step counter lives in device memory and is advanced by
// a kernel (k_inc); the graph covers an even number of steps, so the Jacobi
// swap of the two fields brings every replica back to the pointers the graph
// was captured with; and the gauge fixing schedule (every gf_every steps)
// repeats with the graph's length.  A replica stepped on its own in between
// (an odd number of steps) changes its pointers; the next batch step sees
// that and captures again.  The captured kernels also hold values taken by
// argument (the noise seed, the gauge-fixing grid, the float-float scale
// mode): a replica context whose setters ran since the capture (its
// launch_gen moved) is stale too, and the graph is captured again.
#pragma once

#include <vector>

struct nspt_batch {
  int nrep = 0, N = 0;
  std::vector<nspt_ctx *> ctx;
  std::vector<double> dt;
  std::vector<uint64_t> seed;
  cudaStream_t st = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t exec = nullptr;
  int graph_steps = 0, graph_gf_every = -1;
  std::vector<const void *> graph_U;
  std::vector<uint64_t> graph_phase;
  std::vector<uint64_t> graph_gen;
  float last_ms = 0.f;
  int warps = 0;
};

namespace {

// One Langevin step of a context (the body of nspt_step's loop).
int step_body(nspt_ctx *ctx, double dt, int gf_every) {
  int rc = do_sweep(ctx, dt, false);
  if (rc) return rc;
  if (ctx->flags & NSPT_ZEROMODE)
    if ((rc = do_zero_modes(ctx))) return rc;
  if ((ctx->flags & NSPT_GF_FA) && gf_every > 0 && (ctx->counter % gf_every) == 0)
    if ((rc = do_fa(ctx, ctx->alpha))) return rc;
  if ((ctx->flags & NSPT_GF_LOCAL) && gf_every > 0 && (ctx->counter % gf_every) == 0)
    if ((rc = do_local_gf(ctx, ctx->alpha))) return rc;
  ctx->snap_valid = false;  // twist_boundary ends the step (nspt.cc:1025-1027)
  return NSPT_OK;
}

int graph_length(int gf_every) {
  if (gf_every <= 1) return 2;
  return gf_every % 2 ? 2 * gf_every : gf_every;
}

void drop_graph(nspt_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
  b->graph_steps = 0;
  b->graph_gf_every = -1;
}

bool graph_current(const nspt_batch *b, int P, int gf_every) {
  if (!b->exec || b->graph_steps != P || b->graph_gf_every != gf_every) return false;
  for (int r = 0; r < b->nrep; r++) {
    if (b->graph_U[r] != b->ctx[r]->U) return false;
    if (b->graph_phase[r] != b->ctx[r]->counter % (uint64_t)P) return false;
    if (b->graph_gen[r] != b->ctx[r]->launch_gen) return false;
  }
  return true;
}

int capture(nspt_batch *b, int P, int gf_every) {
  drop_graph(b);
  std::vector<uint64_t> counter(b->nrep);
  for (int r = 0; r < b->nrep; r++) {
    counter[r] = b->ctx[r]->counter;
    b->ctx[r]->kcount = nspt_ctx::KEV;  // no timing events inside the graph
  }
  if (cudaStreamBeginCapture(b->st, cudaStreamCaptureModeRelaxed) != cudaSuccess)
    return NSPT_ERR_CUDA;
  int rc = NSPT_OK;
  if (cudaEventRecord(b->fork, b->st) != cudaSuccess) rc = NSPT_ERR_CUDA;
  for (int r = 0; r < b->nrep && !rc; r++) {
    nspt_ctx *c = b->ctx[r];
    if (cudaStreamWaitEvent(c->st, b->fork, 0) != cudaSuccess) {
      rc = NSPT_ERR_CUDA;
      break;
    }
    for (int s = 0; s < P && !rc; s++) rc = step_body(c, b->dt[r], gf_every);
    if (!rc && (cudaEventRecord(b->join[r], c->st) != cudaSuccess ||
                cudaStreamWaitEvent(b->st, b->join[r], 0) != cudaSuccess))
      rc = NSPT_ERR_CUDA;
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->st, &graph);
  for (int r = 0; r < b->nrep; r++) b->ctx[r]->counter = counter[r];  // nothing ran yet
  if (rc || e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return rc ? rc : NSPT_ERR_CUDA;
  }
  const cudaError_t ei = cudaGraphInstantiate(&b->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ei != cudaSuccess) {
    b->exec = nullptr;
    return NSPT_ERR_CUDA;
  }
  b->graph_steps = P;
  b->graph_gf_every = gf_every;
  for (int r = 0; r < b->nrep; r++) {
    b->graph_U[r] = b->ctx[r]->U;
    b->graph_phase[r] = counter[r] % (uint64_t)P;
    b->graph_gen[r] = b->ctx[r]->launch_gen;
  }
  return NSPT_OK;
}

}  // namespace

extern "C" int nspt_batch_destroy(nspt_batch *b) {
  if (!b) return NSPT_ERR_ARG;
  if (b->st) cudaStreamSynchronize(b->st);
  drop_graph(b);
  for (nspt_ctx *c : b->ctx)
    if (c) nspt_destroy(c);
  for (cudaEvent_t e : b->join)
    if (e) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
  return NSPT_OK;
}

extern "C" int nspt_batch_create(int nrep, const int *L, int N, unsigned flags, double alpha,
                                 const double *dt, const uint64_t *seeds, nspt_batch **out) {
  if (!out || !L || !dt || !seeds || nrep < 1) return NSPT_ERR_ARG;
  *out = nullptr;
  for (int r = 0; r < nrep; r++)
    if (!(dt[r] >= 0.0)) return NSPT_ERR_ARG;
  nspt_batch *b = new nspt_batch();
  b->nrep = nrep;
  b->N = N;
  b->ctx.assign(nrep, nullptr);
  b->join.assign(nrep, nullptr);
  b->graph_U.assign(nrep, nullptr);
  b->graph_phase.assign(nrep, 0);
  b->graph_gen.assign(nrep, 0);
  for (int r = 0; r < nrep; r++) {
    b->dt.push_back(dt[r]);
    b->seed.push_back(seeds[r]);
  }
  int rc = NSPT_OK;
  for (int r = 0; r < nrep && !rc; r++) {
    rc = nspt_create(L + 4 * r, N, flags, alpha, &b->ctx[r]);
    if (!rc) rc = nspt_seed(b->ctx[r], seeds[r], 0);
    if (!rc && cudaEventCreateWithFlags(&b->join[r], cudaEventDisableTiming) != cudaSuccess)
      rc = NSPT_ERR_CUDA;
  }
  if (!rc && (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
              cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
              cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess))
    rc = NSPT_ERR_CUDA;
  if (rc) {
    nspt_batch_destroy(b);
    return rc;
  }
  *out = b;
  return NSPT_OK;
}

extern "C" int nspt_batch_context(nspt_batch *b, int r, nspt_ctx **ctx) {
  if (!b || !ctx || r < 0 || r >= b->nrep) return NSPT_ERR_ARG;
  *ctx = b->ctx[r];
  return NSPT_OK;
}

extern "C" int nspt_batch_step(nspt_batch *b, int nsteps, int gf_every) {
  if (!b || nsteps < 0 || gf_every < 0) return NSPT_ERR_ARG;
  const int P = graph_length(gf_every);
  if (nsteps % P) return NSPT_ERR_ARG;
  for (nspt_ctx *c : b->ctx) {
    if (c->noise_pending) return NSPT_ERR_STATE;  // injected noise is for single steps
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return NSPT_ERR_CUDA;
  }
  if (!graph_current(b, P, gf_every)) {
    const int rc = capture(b, P, gf_every);
    if (rc) return rc;
  }
  if (cudaEventRecord(b->ev0, b->st) != cudaSuccess) return NSPT_ERR_CUDA;
  for (int i = 0; i < nsteps / P; i++)
    if (cudaGraphLaunch(b->exec, b->st) != cudaSuccess) return NSPT_ERR_CUDA;
  if (cudaEventRecord(b->ev1, b->st) != cudaSuccess) return NSPT_ERR_CUDA;
  if (cudaStreamSynchronize(b->st) != cudaSuccess) return NSPT_ERR_CUDA;
  cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
  for (nspt_ctx *c : b->ctx) {
    c->counter += (uint64_t)nsteps;
    if (nsteps) c->have_obs = true;
  }
  return NSPT_OK;
}

extern "C" double nspt_batch_last_step_ms(const nspt_batch *b) { return b ? b->last_ms : 0.0; }

extern "C" int nspt_batch_observables(nspt_batch *b, double *plaq) {
  if (!b || !plaq) return NSPT_ERR_ARG;
  for (int r = 0; r < b->nrep; r++) {
    const int rc = nspt_observables(b->ctx[r], plaq + (size_t)r * 2 * (b->N + 1), nullptr, nullptr);
    if (rc) return rc;
  }
  return NSPT_OK;
}

// Autotuner over the tile shape of the series kernels: orders per lane and
// pass (MO, or MO_LOW where N <= 3 MO_LOW; in the paired-run product this
// is the run length, MO/2) and, for the sweep, warps per CTA (3 links per
// warp: the links, i.e. sites x directions, per block).  Every candidate is
// captured and timed on the batch itself; the fastest is kept.  The trial
// steps change the fields, so every replica is put back to a cold start
// with its seed (counter 0) afterwards.  ms_table (may be NULL) receives
// [2][8] times: row 0 the MO shape, row 1 MO_LOW, column w-1 for w warps,
// 0 where the candidate does not exist.
extern "C" int nspt_batch_tune_shape(nspt_batch *b, int gf_every, int *warps_out, int *mo_out,
                                     float *ms_table) {
  if (!b) return NSPT_ERR_ARG;
  const int P = graph_length(gf_every);
  if (ms_table)
    for (int i = 0; i < 16; i++) ms_table[i] = 0.f;
  float best = 0.f;
  int best_w = 0, best_mo = 0;
  for (int row = 0; row < 2; row++) {
    const int mo = row == 0 ? MO : MO_LOW;
    if (mo == MO_LOW && b->N > 3 * MO_LOW) continue;
    const int wmax = (mo == MO ? SWEEP_THREADS : SWEEP_THREADS_LOW) / 32;
    for (int w = 1; w <= wmax; w++) {
      for (nspt_ctx *c : b->ctx) {
        c->sweep_warps = w;
        c->shape_mo = mo;
        c->launch_gen++;
      }
      drop_graph(b);
      int rc = nspt_batch_step(b, P, gf_every);  // capture + warm-up
      if (!rc) rc = nspt_batch_step(b, 2 * P, gf_every);
      if (rc) return rc;
      if (ms_table) ms_table[row * 8 + (w - 1)] = b->last_ms;
      if (!best_w || b->last_ms < best) {
        best = b->last_ms;
        best_w = w;
        best_mo = mo;
      }
    }
  }
  for (int r = 0; r < b->nrep; r++) {
    b->ctx[r]->sweep_warps = best_w;
    b->ctx[r]->shape_mo = best_mo;
    b->ctx[r]->launch_gen++;
    int rc = nspt_cold_start(b->ctx[r]);
    if (!rc) rc = nspt_seed(b->ctx[r], b->seed[r], 0);
    if (rc) return rc;
    b->ctx[r]->have_obs = false;
  }
  drop_graph(b);
  b->warps = best_w;
  if (warps_out) *warps_out = best_w;
  if (mo_out) *mo_out = best_mo;
  return NSPT_OK;
}

// The same tuner, reporting the warps only.
extern "C" int nspt_batch_tune(nspt_batch *b, int gf_every, int *warps_out) {
  return nspt_batch_tune_shape(b, gf_every, warps_out, nullptr, nullptr);
}
