// nspt_api_check -- a reference-style program written against the C++ API
// (include/nspt_b200.hpp): it loads a configuration in the reference's
// format, runs gauge_wilson sweeps on injected noise, prints each sweep's
// plaquette and the final plaquette_measure / WL2x2, checks the AoS round
// trip through ptGluon<allocORD>, and saves the field.
//
//   nspt_api_check L0 L1 L2 L3 N start.dat noise.bin steps dt out.dat
//
// noise.bin: steps x V x 4 x 8 doubles (SU3rand's draws, nspt.cc:365-423).
// Exit status 0 on success; the first failing call's status otherwise.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../include/nspt_b200.hpp"

using namespace nspt_b200;

namespace {

template <int ORD>
int roundtrip(ptGluon_fld &U) {
  std::vector<ptGluon<ORD>> a, b;
  int rc = U.get<ORD>(a);
  if (rc) return rc;
  if ((rc = U.put<ORD>(a))) return rc;
  if ((rc = U.get<ORD>(b))) return rc;
  for (size_t s = 0; s < a.size(); s++)
    for (int mu = 0; mu < 4; mu++)
      for (int k = 0; k < ORD; k++)
        for (int e = 0; e < 9; e++)
          if (a[s].U[mu].ptU[k].whr[e].re != b[s].U[mu].ptU[k].whr[e].re ||
              a[s].U[mu].ptU[k].whr[e].im != b[s].U[mu].ptU[k].whr[e].im)
            return NSPT_ERR_STATE;
  return NSPT_OK;
}

int fail(const char *what, int rc, const ptGluon_fld *U) {
  fprintf(stderr, "nspt_api_check: %s: %s (%s)\n", what, nspt_error_string(rc),
          U ? U->last_error().c_str() : "");
  return rc ? rc : 1;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 11) {
    fprintf(stderr, "usage: nspt_api_check L0 L1 L2 L3 N start.dat noise.bin steps dt out.dat\n");
    return 2;
  }
  act_params_t p;
  for (int d = 0; d < 4; d++) p.sz[d] = atoi(argv[1 + d]);
  const int N = atoi(argv[5]);
  const int steps = atoi(argv[8]);
  p.tau_g = atof(argv[9]);
  p.alpha = 0.0;
  ptGluon_fld U(p, N, 0u);  // periodic, Jacobi sweep only
  if (U.status()) return fail("ptGluon_fld", U.status(), nullptr);
  std::vector<Cplx> trailer(N + 1);
  int rc = U.load(argv[6], N, trailer.data());
  if (rc) return fail("load", rc, &U);
  const long V = U.volume();
  std::vector<double> eta(V * 32);
  FILE *fn = fopen(argv[7], "rb");
  if (!fn) return fail("noise file", NSPT_ERR_IO, &U);
  sweep_observables o;
  for (int t = 0; t < steps; t++) {
    if (fread(eta.data(), sizeof(double), eta.size(), fn) != eta.size()) {
      fclose(fn);
      return fail("noise file", NSPT_ERR_IO, &U);
    }
    if ((rc = U.set_noise(eta.data()))) return fail("set_noise", rc, &U);
    if ((rc = gauge_wilson(U))) return fail("gauge_wilson", rc, &U);
    if ((rc = twist_boundary(U))) return fail("twist_boundary", rc, &U);
    if ((rc = observables(U, o))) return fail("observables", rc, &U);
    printf("plaq");
    for (int k = 0; k <= N; k++) printf(" %.17e %.17e", o.w[k].re, o.w[k].im);
    printf("\n");
  }
  fclose(fn);
  std::vector<Cplx> w(N + 1), wl(N + 1);
  if ((rc = plaquette_measure(U, w.data()))) return fail("plaquette_measure", rc, &U);
  if ((rc = WL2x2(U, wl.data()))) return fail("WL2x2", rc, &U);
  printf("measure");
  for (int k = 0; k <= N; k++) printf(" %.17e %.17e", w[k].re, w[k].im);
  printf("\nwl2x2");
  for (int k = 0; k <= N; k++) printf(" %.17e %.17e", wl[k].re, wl[k].im);
  printf("\n");
  if (N == 4 && (rc = roundtrip<4>(U))) return fail("AoS round trip", rc, &U);
  if ((rc = U.save(argv[10], N))) return fail("save", rc, &U);
  return 0;
}
