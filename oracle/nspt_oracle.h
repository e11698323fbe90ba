/*
 * TEST INFRASTRUCTURE (oracle).  Plain-C restatement of the PRlgt2020
 * quenched SU(3) NSPT Langevin step.  Only tests/, the smoke check and the
 * CPU-baseline leg of bench.py use it, and only as the checker; the product
 * never links it.
 *
 * Data layout follows the reference's AoS field exactly (ptGluon_fld,
 * QCDenvNODEpt_test.h:331-338; ptSU3, QCDpt.h:42-50): per site, per mu, one
 * series of 1 + 9*N complex numbers = {flag, order 1 [9], ..., order N [9]},
 * each complex stored (re, im), each 3x3 row major.  With allocORD == N this
 * is byte-identical to the reference's configuration files (minus the
 * plaquette trailer, QCDenvNODEpt_test.h:359-366).
 */
#ifndef NSPT_ORACLE_H
#define NSPT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_ctx oracle_ctx;
typedef struct oracle_rng oracle_rng;

/* twist_mask bit d set: direction d has twisted boundary conditions with the
 * reference's matrix (twistmatrices.h:158-240); bit 0 (x) is rejected, as in
 * the reference where the x twist matrix is not defined. */
oracle_ctx *oracle_create(const int L[4], int N, int twist_mask);
void oracle_destroy(oracle_ctx *c);
/* V*4*(1+9N) complex doubles, reference AoS layout */
double *oracle_links(oracle_ctx *c);
long oracle_volume(oracle_ctx *c);
void oracle_cold_start(oracle_ctx *c);
/* order-k real components ~ N(0, sigma^k), then U = exp(reH(log U)) */
void oracle_random_start(oracle_ctx *c, long seed, double sigma);
/* U = exp(reH(log U)) per link (QCDenvNODEpt_test.h:414-417) */
void oracle_unitarise(oracle_ctx *c);

/* One Jacobi Langevin sweep (gauge_wilson, nspt.cc:258-600, Jacobi branch).
 * noise: V*4*8 Gaussians in the reference's draw order (site, mu, 8).
 * Outputs (any may be NULL), normalised as nspt.cc:570-597:
 *   plaq[(N+1)*2]   sum Tr(U * staples) / (72 V) per order 0..N
 *   norm[N]         sum Re Tr(U_k U_k^dag) / (12 V)
 *   tru[4*N*2]      sum Tr U_k per mu / (3 V)   (mu major)
 * If zero_modes, also accumulates MM[mu] = sum log(U') for the subtraction.
 */
void oracle_sweep(oracle_ctx *c, double dt, const double *noise, double *plaq,
                  double *norm, double *tru, int zero_modes);
/* gauge_wilson with UPDATE_ONTHEFLY (the reference's default, choices.h:61):
 * links updated in place, in the order of the OpenMP thread grid
 * grid = {ntt, ntx, nty, ntz}; same noise layout and outputs as
 * oracle_sweep.  With twisted boundaries, reads across a twisted face see
 * the field of the step's start (the reference's copy sites) until
 * oracle_twist_boundary.  -1 for a grid the reference rejects. */
int oracle_sweep_onthefly(oracle_ctx *c, double dt, const double *noise, const int *grid,
                          double *plaq, double *norm, double *tru, int zero_modes);
/* twist_boundary, nspt.cc:163-255: the copy sites refreshed */
void oracle_twist_boundary(oracle_ctx *c);
/* zero_modes_subtraction, nspt.cc:605-654 (uses MM from the last sweep) */
void oracle_zero_modes(oracle_ctx *c);
/* FAstochastic_gauge_fixing, nspt.cc:866-948 (periodic only) */
void oracle_fa_gauge_fix(oracle_ctx *c, double alpha);
/* stochastic_gauge_fixing, nspt.cc:660-862: sequential, in place */
void oracle_local_gauge_fix(oracle_ctx *c, double alpha);
/* the same as the reference built with OpenMP thread grid
 * grid = {ntt, ntx, nty, ntz} runs it; -1 for a grid the reference rejects */
int oracle_local_gauge_fix_grid(oracle_ctx *c, double alpha, const int *grid);
/* improved gauge action c1 (c0 = 1 - 8 c1), periodic only; -1 otherwise */
int oracle_set_action(oracle_ctx *c, double c1);
/* rectangle traces w2 of the last sweep, (N+1)*2, /72V */
void oracle_last_w2(oracle_ctx *c, double *out);
/* ComputeLoops (nspt.cc:1148-1312, periodic): traces of the summed 1x2,
 * 2x2, 2x4 and 4x4 loops, out[4][(N+1)*2], normalised as printed */
void oracle_wilson_loops(oracle_ctx *c, double *out);
/* plaquette_measure, nspt.cc:1316-1406 (OpenMP variant, /72V) */
void oracle_plaquette(oracle_ctx *c, double *plaq);

/* Series primitives on one series (2 + 18N doubles), for unit tests. */
void oracle_ser_mul(int N, const double *a, const double *b, double *out);
void oracle_ser_exp(int N, const double *a, double *out);
void oracle_ser_log(int N, const double *a, double *out);
void oracle_ser_reH(int N, double *a);
void oracle_ser_dag(int N, const double *a, double *out);

/* MyRand "rand55" generator (MyRand.cc:73-130, MyRand.h:81-91). */
oracle_rng *oracle_rng_create(long seed);
void oracle_rng_destroy(oracle_rng *r);
void oracle_rng_gauss(oracle_rng *r, double *out, long n);
/* SU3rand mapping of 8 Gaussians to a 3x3 complex (MyMath.cc:256-292) */
void oracle_su3rand(const double *g8, double *m18);

#ifdef __cplusplus
}
#endif
#endif
