/*
 * TEST INFRASTRUCTURE (oracle).  FFTW3 advanced-interface shim.
 *
 * Implements the two calls the reference makes (`fftw_plan_many_dft`,
 * Quenched.cc:827-838; `fftw_execute`, nspt.cc:879,897) for in-place
 * transforms with inembed == onembed == NULL: `howmany` rank-d transforms,
 * transform m starting at complex element m*idist with element stride
 * istride.  The arithmetic is oracle_dft_nd (oracle_dft.c).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"
#include "oracle_dft.h"

struct oracle_fftw_plan_s {
  int rank;
  int n[8];
  int howmany;
  double *data;
  int stride;
  int dist;
  int sign;
};

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany,
                             fftw_complex *in, const int *inembed,
                             int istride, int idist, fftw_complex *out,
                             const int *onembed, int ostride, int odist,
                             int sign, unsigned flags) {
  (void)flags;
  if (rank < 1 || rank > 8 || in != out || inembed || onembed ||
      istride != ostride || idist != odist) {
    fprintf(stderr, "fftw shim: unsupported plan\n");
    abort();
  }
  struct oracle_fftw_plan_s *p =
      (struct oracle_fftw_plan_s *)calloc(1, sizeof(*p));
  p->rank = rank;
  memcpy(p->n, n, sizeof(int) * (size_t)rank);
  p->howmany = howmany;
  p->data = (double *)in;
  p->stride = istride;
  p->dist = idist;
  p->sign = sign;
  return p;
}

void fftw_execute(const fftw_plan p) {
  for (int m = 0; m < p->howmany; m++)
    oracle_dft_nd(p->data + 2L * m * p->dist, p->rank, p->n, p->stride,
                  p->sign);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { (void)nthreads; }
