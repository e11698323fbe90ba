/*
 * TEST INFRASTRUCTURE (oracle).  Plain-C multi-dimensional complex DFT.
 *
 * Restates the transform FFTW3 computes for the reference's
 * Fourier-accelerated gauge fixing (nspt.cc:879 forward, nspt.cc:897
 * backward; plans at Quenched.cc:827-832): an unnormalised rank-d DFT over a
 * row-major array, sign -1 for FFTW_FORWARD and +1 for FFTW_BACKWARD.
 *
 * Power-of-two lengths use an iterative radix-2 Cooley-Tukey transform;
 * other lengths use the direct O(n^2) sum.  Twiddles are exp(sign*2*pi*i*k/n)
 * evaluated per k (no recurrence).  Used by the FFTW shim that the oracle
 * build of the reference links, and by the C restatement in nspt_oracle.c.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_dft.h"

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* In-place 1-D DFT of n complex values held contiguously in buf[2*n]. */
static void dft_1d(double *buf, int n, int sign, double *scratch) {
  if (n <= 1) return;
  if (is_pow2(n)) {
    /* bit reversal */
    for (int i = 1, j = 0; i < n; i++) {
      int bit = n >> 1;
      for (; j & bit; bit >>= 1) j ^= bit;
      j ^= bit;
      if (i < j) {
        double tr = buf[2 * i], ti = buf[2 * i + 1];
        buf[2 * i] = buf[2 * j];
        buf[2 * i + 1] = buf[2 * j + 1];
        buf[2 * j] = tr;
        buf[2 * j + 1] = ti;
      }
    }
    for (int len = 2; len <= n; len <<= 1) {
      int half = len >> 1;
      for (int k = 0; k < half; k++) {
        double ang = sign * 2.0 * M_PI * (double)k / (double)len;
        double wr = cos(ang), wi = sin(ang);
        for (int s = 0; s < n; s += len) {
          double *a = buf + 2 * (s + k), *b = buf + 2 * (s + k + half);
          double br = b[0] * wr - b[1] * wi;
          double bi = b[0] * wi + b[1] * wr;
          b[0] = a[0] - br;
          b[1] = a[1] - bi;
          a[0] += br;
          a[1] += bi;
        }
      }
    }
    return;
  }
  for (int k = 0; k < n; k++) {
    double sr = 0.0, si = 0.0;
    for (int x = 0; x < n; x++) {
      long m = ((long)k * x) % n;
      double ang = sign * 2.0 * M_PI * (double)m / (double)n;
      double wr = cos(ang), wi = sin(ang);
      sr += buf[2 * x] * wr - buf[2 * x + 1] * wi;
      si += buf[2 * x] * wi + buf[2 * x + 1] * wr;
    }
    scratch[2 * k] = sr;
    scratch[2 * k + 1] = si;
  }
  memcpy(buf, scratch, sizeof(double) * 2 * (size_t)n);
}

void oracle_dft_nd(double *data, int rank, const int *dims, long stride,
                   int sign) {
  long total = 1;
  int nmax = 1;
  for (int d = 0; d < rank; d++) {
    total *= dims[d];
    if (dims[d] > nmax) nmax = dims[d];
  }
  double *line = (double *)malloc(sizeof(double) * 2 * (size_t)nmax);
  double *scratch = (double *)malloc(sizeof(double) * 2 * (size_t)nmax);
  /* element stride (in complex units) of dimension d in the row-major array */
  for (int d = 0; d < rank; d++) {
    long inner = 1;
    for (int e = d + 1; e < rank; e++) inner *= dims[e];
    int n = dims[d];
    long outer = total / ((long)n * inner);
    for (long o = 0; o < outer; o++) {
      for (long in = 0; in < inner; in++) {
        long base = o * (long)n * inner + in;
        for (int x = 0; x < n; x++) {
          double *p = data + 2 * (base + (long)x * inner) * stride;
          line[2 * x] = p[0];
          line[2 * x + 1] = p[1];
        }
        dft_1d(line, n, sign, scratch);
        for (int x = 0; x < n; x++) {
          double *p = data + 2 * (base + (long)x * inner) * stride;
          p[0] = line[2 * x];
          p[1] = line[2 * x + 1];
        }
      }
    }
  }
  free(line);
  free(scratch);
}
