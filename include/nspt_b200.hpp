/* nspt_b200.hpp -- C++ host API in the reference's vocabulary, over the C ABI
 * of nspt_b200.h.
 *
 * The reference's program is written against three headers: MyMath.h (Cplx,
 * SU3), QCDpt.h (the series link ptSU3, QCDpt.h:42-84) and nspt.h (the
 * Langevin function set, nspt.h:55-94, acting on a ptGluon_fld plus the
 * globals act_pars, w, norm, trU of Quenched.cc:42-81).  This header keeps
 * those names and byte layouts for C++ callers:
 *   Cplx, SU3, ptSU3<allocORD>   layout-identical host types (a field on the
 *                                host is an array of ptGluon<allocORD>);
 *   act_params_t                 the subset of input.h:56-66 the step uses;
 *   ptGluon_fld                  the field, resident on the device (one
 *                                context of the C ABI), with the
 *                                reference's load/save and AoS copies;
 *   gauge_wilson, zero_modes_subtraction, stochastic_gauge_fixing,
 *   FAstochastic_gauge_fixing, NsptEvolve, twist_boundary,
 *   plaquette_measure, ComputeLoops, WL2x2
 *                                the nspt.h functions, returning the C ABI's
 *                                status (0 = success) instead of void.
 * The reference fixes the boundary conditions, gauge fixing, zero modes and
 * action at compile time (choices.h); here they are the `choices` argument.
 * Nothing here computes on the host: every function calls the library.
 */
#ifndef NSPT_B200_HPP
#define NSPT_B200_HPP

#include <string>
#include <vector>

#include "nspt_b200.h"

namespace nspt_b200 {

/* MyMath.h:65-77 */
struct Cplx {
  double re = 0.0, im = 0.0;
};
/* MyMath.h:505-510: row-major 3x3 */
struct SU3 {
  Cplx whr[9];
};
/* QCDpt.h:42-50: order-0 flag, then orders 1..allocORD */
template <int allocORD>
struct ptSU3 {
  Cplx flag;
  SU3 ptU[allocORD];
};
/* QCDpt.h:249-252: the four links of a site */
template <int allocORD>
struct ptGluon {
  ptSU3<allocORD> U[4];
};
static_assert(sizeof(Cplx) == 16 && sizeof(SU3) == 144, "MyMath.h layout");
static_assert(sizeof(ptSU3<24>) == 16 * (1 + 9 * 24), "QCDpt.h layout");

/* input.h:56-66, the members the Langevin step reads */
struct act_params_t {
  int sz[4];     // lattice extents (taglia)
  double tau_g;  // Langevin time step as in Quench.cfg (the step forms -tau_g/6, sqrt(tau_g))
  double alpha;  // gauge-fixing parameter as in Quench.cfg
};

/* choices.h switches as run-time flags (NSPT_TWIST_*, NSPT_ZEROMODE,
 * NSPT_GF_FA, NSPT_GF_LOCAL, NSPT_ACTION_*, NSPT_PRECISION_FF,
 * NSPT_UPDATE_ONTHEFLY) */
using choices = unsigned;

/* QCDenvNODEpt_test.h:331-338: the gauge field, here on the device */
class ptGluon_fld {
 public:
  ptGluon_fld(const act_params_t &p, int PTORD, choices flags) : p_(p), N_(PTORD) {
    status_ = nspt_create(p.sz, PTORD, flags, p.alpha, &ctx_);
  }
  ~ptGluon_fld() {
    if (ctx_) nspt_destroy(ctx_);
  }
  ptGluon_fld(const ptGluon_fld &) = delete;
  ptGluon_fld &operator=(const ptGluon_fld &) = delete;

  /* 0 when the field was created; else the nspt_create status */
  int status() const { return status_; }
  int order() const { return N_; }
  long volume() const { return (long)p_.sz[0] * p_.sz[1] * p_.sz[2] * p_.sz[3]; }
  const act_params_t &params() const { return p_; }
  nspt_ctx *ctx() const { return ctx_; }
  std::string last_error() const { return ctx_ ? nspt_last_error(ctx_) : "no context"; }

  /* ptGluon_fld::load / save (QCDenvNODEpt_test.h:342-374): the reference's
   * configuration files, allocORD orders per link, plaquette trailer */
  int load(const char *path, int allocORD, Cplx *plaq_trailer) {
    return nspt_load_config(ctx_, path, allocORD, &plaq_trailer[0].re);
  }
  int save(const char *path, int allocORD) { return nspt_save_config(ctx_, path, allocORD); }
  /* ptGluon_fld::loadlowerorder (QCDenvNODEpt_test.h:376-426): a file with
   * loworder <= N orders, upper orders zero, links unitarised;
   * plaquette: loworder + 1 values */
  int loadlowerorder(const char *path, int loworder, Cplx *plaquette) {
    return nspt_load_lower_order(ctx_, path, loworder, plaquette ? &plaquette[0].re : nullptr);
  }

  /* the field in the reference's AoS bytes: V x ptGluon<allocORD> */
  template <int allocORD>
  int get(std::vector<ptGluon<allocORD>> &w) const {
    w.resize(volume());
    return nspt_download_links(ctx_, w.data(), allocORD);
  }
  template <int allocORD>
  int put(const std::vector<ptGluon<allocORD>> &w) {
    if ((long)w.size() != volume()) return NSPT_ERR_ARG;
    return nspt_upload_links(ctx_, w.data(), allocORD);
  }

  /* Cold start (Quenched.cc:596-603) and the noise: device Philox from a
   * seed, or the eight Gaussians per link of the reference's SU3rand draws
   * ([V][4][8], consumed by the next sweep) */
  int cold_start() { return nspt_cold_start(ctx_); }
  int seed(unsigned long long s, unsigned long long counter = 0) {
    return nspt_seed(ctx_, s, counter);
  }
  int set_noise(const double *eta) { return nspt_set_noise(ctx_, eta); }

 private:
  act_params_t p_;
  int N_;
  nspt_ctx *ctx_ = nullptr;
  int status_ = NSPT_ERR_STATE;
};

/* The per-sweep values gauge_wilson writes (nspt.cc:570-597): w[N+1]
 * (plaquette), norm[N], trU[4][N] */
struct sweep_observables {
  std::vector<Cplx> w, trU;
  std::vector<double> norm;
};

/* nspt.h:55-94 */
inline int gauge_wilson(ptGluon_fld &U) { return nspt_gauge_wilson(U.ctx(), U.params().tau_g); }
inline int zero_modes_subtraction(ptGluon_fld &U) { return nspt_zero_modes_subtraction(U.ctx()); }
inline int stochastic_gauge_fixing(ptGluon_fld &U) {
  return nspt_local_gauge_fixing(U.ctx(), U.params().alpha);
}
inline int FAstochastic_gauge_fixing(ptGluon_fld &U) {
  return nspt_fa_gauge_fixing(U.ctx(), U.params().alpha);
}
/* NsptEvolve (nspt.cc:953-1039) for Beat steps, gauge fixing every gf_every */
inline int NsptEvolve(ptGluon_fld &U, int beat = 1, int gf_every = 1) {
  return nspt_step(U.ctx(), U.params().tau_g, beat, gf_every);
}
/* twists are applied inside every neighbour read; this ends the stale
 * twisted reads an on-the-fly gauge_wilson leaves (the copy sites) */
inline int twist_boundary(ptGluon_fld &U) { return nspt_twist_boundary(U.ctx()); }
inline int plaquette_measure(ptGluon_fld &U, Cplx *w) {
  return nspt_plaquette_measure(U.ctx(), &w[0].re);
}
inline int observables(ptGluon_fld &U, sweep_observables &o) {
  const int N = U.order();
  o.w.assign(N + 1, Cplx{});
  o.norm.assign(N, 0.0);
  o.trU.assign(4 * N, Cplx{});
  return nspt_observables(U.ctx(), &o.w[0].re, o.norm.data(), &o.trU[0].re);
}
/* ComputeLoops (nspt.cc:1148-1312): loops[4 * (N+1)], 1x2 2x2 2x4 4x4 */
inline int ComputeLoops(ptGluon_fld &U, Cplx *loops) {
  return nspt_wilson_loops(U.ctx(), &loops[0].re);
}
/* WL2x2 (nspt.cc:1064-1140): loop[N+1] */
inline int WL2x2(ptGluon_fld &U, Cplx *loop) { return nspt_wl2x2(U.ctx(), &loop[0].re); }

}  // namespace nspt_b200

#endif
