/*
 * TEST INFRASTRUCTURE (oracle).  Plain-C restatement of the PRlgt2020
 * quenched SU(3) NSPT Langevin step, used only as the checker for the CUDA
 * engine (tests/, smoke check, CPU-baseline leg of bench.py).
 *
 * Every function cites the reference code it restates.  Floating-point
 * operations follow the reference's evaluation order where that is natural
 * (left-to-right sums inside SU3::operator*, accumulation order of the
 * truncated Cauchy / exp / log triangles, divisions kept as divisions), and
 * the file is compiled with -ffp-contract=off, so on the reference's own
 * inputs the two codes agree to a few ulps.
 *
 * Twisted boundary conditions: the reference keeps copies of the boundary
 * links holding Omega U Omega^dag (lattice.h:236-1053, refreshed by
 * twist_boundary, nspt.cc:163-255).  This restatement applies the same
 * adjoint twist when a neighbour read crosses a twisted face: a forward wrap
 * in direction d reads Omega_d U Omega_d^dag (twist_d, nspt.cc:111-121), a
 * backward wrap reads Omega_d^dag U Omega_d (invtwist_d); for a read that
 * wraps backward in one direction and forward in another the backward twist
 * is applied first, as the reference's backward copy slabs hold
 * (lattice.h:733-790 + the justtwist pass, nspt.cc:221-253).  Twisted links
 * get flag = 1, as twist_* returns a default-constructed flag (VACUUM).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "nspt_oracle.h"
#include "fftw_shim/oracle_dft.h"

typedef struct {
  double re, im;
} cx;

#define SER(N) (1 + 9 * (N))

static const double D3 = 1.0 / 3.0; /* MyMath.h:42 */

struct oracle_ctx {
  int L[4];
  int N;
  int tw;
  long V;
  long sYZT, sZT, sT;
  cx *U, *F, *MM;
  /* on-the-fly update with twisted boundaries: the field as it was when the
   * reference's twisted copy sites were last refreshed (twist_boundary);
   * reads that cross a twisted face come from here.  NULL otherwise. */
  cx *snap;
  cx omega[4][9], omegadag[4][9];
  double *p2hat[4];
  double c1;          /* improved action: 0 = Wilson (Quenched.cc:311-322) */
  double last_w2[2 * (64 + 1)];  /* rectangle traces of the last sweep, /72V */
};

/* ---------------- complex and 3x3 primitives (MyMath.h) ---------------- */

static inline cx cmul(cx a, cx b) { /* Cplx::operator* MyMath.h:94 */
  cx r = {a.re * b.re - a.im * b.im, a.im * b.re + a.re * b.im};
  return r;
}
static inline cx cadd(cx a, cx b) {
  cx r = {a.re + b.re, a.im + b.im};
  return r;
}
static inline cx csub(cx a, cx b) {
  cx r = {a.re - b.re, a.im - b.im};
  return r;
}
static inline int cis0(cx a) { return a.re == 0.0 && a.im == 0.0; }

/* SU3::operator*(const SU3&), MyMath.h:791-849: each entry summed left to
 * right over l = 0,1,2 as re*re - im*im (+...) and re*im + im*re (+...). */
static void m_mul(cx *r, const cx *a, const cx *b) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      const cx *x = a + 3 * i;
      double re = x[0].re * b[j].re - x[0].im * b[j].im + x[1].re * b[3 + j].re -
                  x[1].im * b[3 + j].im + x[2].re * b[6 + j].re -
                  x[2].im * b[6 + j].im;
      double im = x[0].re * b[j].im + x[0].im * b[j].re + x[1].re * b[3 + j].im +
                  x[1].im * b[3 + j].re + x[2].re * b[6 + j].im +
                  x[2].im * b[6 + j].re;
      r[3 * i + j].re = re;
      r[3 * i + j].im = im;
    }
}
static void m_acc(cx *acc, const cx *x) { /* SU3 += */
  for (int e = 0; e < 9; e++) acc[e] = cadd(acc[e], x[e]);
}
static void m_dag(cx *r, const cx *a) { /* dag(SU3) MyMath.h:1064-1080 */
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      r[3 * i + j].re = a[3 * j + i].re;
      r[3 * i + j].im = -a[3 * j + i].im;
    }
}
static cx m_tr(const cx *a) { /* SU3::Tr MyMath.h:1001 */
  return cadd(cadd(a[0], a[4]), a[8]);
}

/* ---------------- series primitives (QCDpt.h, QCDpt.cc) ---------------- */
/* A series is SER(N) complex: s[0] = flag, s[1 + 9k + e] = order k+1. */

static void s_zero(cx *s, int N) { memset(s, 0, sizeof(cx) * SER(N)); }
static void s_copy(cx *d, const cx *s, int N) { memcpy(d, s, sizeof(cx) * SER(N)); }
static void s_acc(cx *a, const cx *b, int N) { /* ptSU3::operator+= QCDpt.cc:69 */
  for (int k = 1; k < SER(N); k++) a[k] = cadd(a[k], b[k]);
  a[0] = cadd(a[0], b[0]);
}
static void s_sub_acc(cx *a, const cx *b, int N) { /* operator-= QCDpt.cc:80 */
  for (int k = 1; k < SER(N); k++) a[k] = csub(a[k], b[k]);
  a[0] = csub(a[0], b[0]);
}
static void s_scale(cx *a, double x, int N) { /* operator*=(double) QCDpt.cc:162 */
  for (int k = 0; k < SER(N); k++) {
    a[k].re *= x;
    a[k].im *= x;
  }
}
static void s_div(cx *a, double x, int N) { /* operator/=(double) QCDpt.cc:171 */
  for (int k = 0; k < SER(N); k++) {
    a[k].re /= x;
    a[k].im /= x;
  }
}

/* Truncated Cauchy product B = A*C, ptSU3::operator* QCDpt.h:92-114. */
static void s_mul(cx *B, const cx *A, const cx *C, int N) {
  cx t[9];
  s_zero(B, N);
  for (int i = 0; i < N - 1; i++)
    for (int j = 0; j < N - 1 - i; j++) {
      m_mul(t, A + 1 + 9 * j, C + 1 + 9 * i);
      m_acc(B + 1 + 9 * (i + j + 1), t);
    }
  if (cis0(A[0]) && cis0(C[0])) {
    B[0].re = B[0].im = 0.0;
    return;
  }
  B[0] = cmul(A[0], C[0]);
  for (int i = 0; i < N; i++)
    for (int e = 0; e < 9; e++) {
      cx u = cadd(cmul(C[0], A[1 + 9 * i + e]), cmul(A[0], C[1 + 9 * i + e]));
      B[1 + 9 * i + e] = cadd(B[1 + 9 * i + e], u);
    }
}

/* dag(ptSU3), QCDpt.cc:185-194 */
static void s_dag(cx *B, const cx *A, int N) {
  for (int i = 0; i < N; i++) m_dag(B + 1 + 9 * i, A + 1 + 9 * i);
  B[0].re = A[0].re;
  B[0].im = -A[0].im;
}

/* ptSU3::reH, QCDpt.cc:197-209 */
static void s_reH(cx *A, int N) {
  cx d[9];
  for (int i = 0; i < N; i++) {
    cx *m = A + 1 + 9 * i;
    m_dag(d, m);
    for (int e = 0; e < 9; e++) {
      m[e] = csub(m[e], d[e]);
      m[e].re = .5 * m[e].re;
      m[e].im = .5 * m[e].im;
    }
    cx tr = m_tr(m);
    tr.re = tr.re * D3;
    tr.im = D3 * tr.im;
    m[0] = csub(m[0], tr);
    m[4] = csub(m[4], tr);
    m[8] = csub(m[8], tr);
  }
  A[0].re = A[0].im = 0.0;
}

/* ptSU3::Trless, QCDpt.cc:124-136 */
static void s_trless(cx *A, int N) {
  for (int i = 0; i < N; i++) {
    cx *m = A + 1 + 9 * i;
    cx t = m_tr(m);
    cx z = {D3 * t.re, D3 * t.im};
    m[0] = csub(m[0], z);
    m[4] = csub(m[4], z);
    m[8] = csub(m[8], z);
  }
  A[0].re = A[0].im = 0.0;
}

/* exp(const ptSU3&), QCDpt.h:200-220: res = sum_i A^i/i!, B_i = B_{i-1} A
 * pruned to orders >= i. Scratch: 2 series. */
static void s_exp(cx *res, const cx *A, int N, cx *B, cx *Bn) {
  cx t[9];
  s_copy(B, A, N);
  s_copy(res, A, N);
  for (int i = 2; i <= N; i++) {
    s_zero(Bn, N);
    for (int iA = 1; iA < N; iA++)
      for (int iB = i - 1; iB <= N - iA; iB++) {
        m_mul(t, B + 1 + 9 * (iB - 1), A + 1 + 9 * (iA - 1));
        m_acc(Bn + 1 + 9 * (iA + iB - 1), t);
      }
    double den = 1. / (double)i;
    for (int k = 0; k < SER(N); k++) {
      B[k].re = den * Bn[k].re;
      B[k].im = den * Bn[k].im;
    }
    s_acc(res, B, N);
  }
  res[0].re = 1.0;
  res[0].im = 0.0;
}

/* log(const ptSU3&), QCDpt.h:176-198: res = sum_i (-1)^(i+1) (U-1)^i / i. */
static void s_log(cx *res, const cx *U, int N, cx *B, cx *Bn) {
  cx t[9];
  s_copy(B, U, N);
  B[0].re = B[0].im = 0.0;
  s_copy(res, U, N);
  double segno = -1;
  for (int i = 2; i <= N; i++) {
    s_zero(Bn, N);
    for (int iU = 1; iU < N; iU++)
      for (int iB = i - 1; iB <= N - iU; iB++) {
        m_mul(t, B + 1 + 9 * (iB - 1), U + 1 + 9 * (iU - 1));
        m_acc(Bn + 1 + 9 * (iU + iB - 1), t);
      }
    memcpy(B + 1, Bn + 1, sizeof(cx) * 9 * (size_t)N);
    double aux = segno / (double)i;
    for (int k = 1; k < SER(N); k++) {
      cx v = {aux * B[k].re, aux * B[k].im};
      res[k] = cadd(res[k], v);
    }
    {
      cx v = {aux * B[0].re, aux * B[0].im};
      res[0] = cadd(res[0], v);
    }
    segno = -segno;
  }
  res[0].re = res[0].im = 0.0;
}

/* ---------------- lattice geometry (lattice.h) ---------------- */

/* GETINDEX, lattice.h:37: t (direction 3) fastest */
static inline long site_of(const oracle_ctx *c, const int *x) {
  return x[0] * c->sYZT + x[1] * c->sZT + x[2] * c->sT + x[3];
}
static inline void coords_of(const oracle_ctx *c, long s, int *x) {
  x[0] = (int)(s / c->sYZT);
  long r = s % c->sYZT;
  x[1] = (int)(r / c->sZT);
  r %= c->sZT;
  x[2] = (int)(r / c->sT);
  x[3] = (int)(r % c->sT);
}

static cx *link_ptr(cx *field, const oracle_ctx *c, long s, int mu) {
  return field + ((size_t)s * 4 + mu) * SER(c->N);
}

/* Fetch link U_mu at (possibly out-of-box by one step per direction)
 * coordinates y, applying the twists of the wrapped twisted directions. */
static void fetch_link(const oracle_ctx *c, const cx *field, const int *y,
                       int mu, cx *out) {
  int x[4], bwd[4], fwd[4];
  int N = c->N;
  for (int d = 0; d < 4; d++) {
    x[d] = y[d];
    fwd[d] = 0;
    bwd[d] = 0;
    if (x[d] < 0) {
      x[d] += c->L[d];
      bwd[d] = 1;
    } else if (x[d] >= c->L[d]) {
      x[d] -= c->L[d];
      fwd[d] = 1;
    }
  }
  int crosses = 0;
  for (int d = 0; d < 4; d++)
    if ((bwd[d] || fwd[d]) && ((c->tw >> d) & 1)) crosses = 1;
  /* the reference reads a twisted copy site there (lattice.h:236-300),
   * refreshed only by twist_boundary (nspt.cc:163-255) */
  const cx *base = crosses && c->snap ? c->snap : field;
  const cx *src = base + ((size_t)site_of(c, x) * 4 + mu) * SER(N);
  s_copy(out, src, N);
  int any = 0;
  cx t[9], u[9];
  for (int pass = 0; pass < 2; pass++)
    for (int d = 0; d < 4; d++) {
      int hit = pass == 0 ? bwd[d] : fwd[d];
      if (!hit || !((c->tw >> d) & 1)) continue;
      any = 1;
      const cx *l = pass == 0 ? c->omegadag[d] : c->omega[d];
      const cx *r = pass == 0 ? c->omega[d] : c->omegadag[d];
      for (int k = 0; k < N; k++) {
        m_mul(t, l, out + 1 + 9 * k);
        m_mul(u, t, r);
        memcpy(out + 1 + 9 * k, u, sizeof(u));
      }
    }
  if (any) {
    out[0].re = 1.0;
    out[0].im = 0.0;
  }
}

/* ---------------- context ---------------- */

oracle_ctx *oracle_create(const int L[4], int N, int twist_mask) {
  if (N < 1 || (twist_mask & 1) || (twist_mask & ~15)) return NULL;
  for (int d = 0; d < 4; d++)
    if (L[d] < 2) return NULL;
  oracle_ctx *c = (oracle_ctx *)calloc(1, sizeof(*c));
  memcpy(c->L, L, sizeof(int) * 4);
  c->N = N;
  c->tw = twist_mask;
  c->sT = L[3];
  c->sZT = (long)L[2] * L[3];
  c->sYZT = (long)L[1] * L[2] * L[3];
  c->V = (long)L[0] * c->sYZT;
  size_t n = (size_t)c->V * 4 * SER(N);
  c->U = (cx *)calloc(n, sizeof(cx));
  c->F = (cx *)calloc(n, sizeof(cx));
  c->snap = NULL;
  c->MM = (cx *)calloc(4 * (size_t)SER(N), sizeof(cx));
  /* twist matrices, twistmatrices.h:158-240 (y, z, t) */
  memset(c->omega, 0, sizeof(c->omega));
  for (int d = 0; d < 4; d++)
    for (int e = 0; e < 9; e += 4) c->omega[d][e].re = 1.0;
  cx *oy = c->omega[1];
  oy[0].re = cos(-2. * M_PI / 3.);
  oy[0].im = sin(-2. * M_PI / 3.);
  oy[8].re = cos(2. * M_PI / 3.);
  oy[8].im = sin(2. * M_PI / 3.);
  cx *oz = c->omega[2];
  memset(oz, 0, sizeof(cx) * 9);
  oz[1].re = 1;
  oz[5].re = 1;
  oz[6].re = 1;
  cx *ot = c->omega[3];
  memset(ot, 0, sizeof(cx) * 9);
  ot[1].re = cos(-2. * M_PI / 3.);
  ot[1].im = sin(-2. * M_PI / 3.);
  ot[5].re = 1;
  ot[6].re = cos(2. * M_PI / 3.);
  ot[6].im = sin(2. * M_PI / 3.);
  for (int d = 0; d < 4; d++) m_dag(c->omegadag[d], c->omega[d]);
  /* lattice momenta p2hat, lattice.h:1144-1169 (periodic) */
  for (int d = 0; d < 4; d++) {
    c->p2hat[d] = (double *)malloc(sizeof(double) * L[d]);
    for (int i = 0; i < L[d]; i++) {
      double p = 2 * M_PI * i / L[d];
      double h = sin(p * 0.5);
      h *= 4 * h;
      c->p2hat[d][i] = h;
    }
  }
  oracle_cold_start(c);
  return c;
}

void oracle_destroy(oracle_ctx *c) {
  if (!c) return;
  free(c->U);
  free(c->F);
  free(c->snap);
  free(c->MM);
  for (int d = 0; d < 4; d++) free(c->p2hat[d]);
  free(c);
}

double *oracle_links(oracle_ctx *c) { return (double *)c->U; }
long oracle_volume(oracle_ctx *c) { return c->V; }

/* cold start, Quenched.cc:596-603: flag = 1, all orders zero */
void oracle_cold_start(oracle_ctx *c) {
  size_t n = (size_t)c->V * 4;
  memset(c->U, 0, sizeof(cx) * n * SER(c->N));
  for (size_t l = 0; l < n; l++) c->U[l * SER(c->N)].re = 1.0;
}

/* ---------------- RNG (MyRand.cc, MyRand.h) ---------------- */

struct oracle_rng {
  uint64_t ring[55];
  int next[55];
  int n1, n2;
  int gen;
  double r, t;
};

static double rng_flat(oracle_rng *g) { /* Ranf, MyRand.h:81-91 */
  g->n1 = g->next[g->n1];
  g->n2 = g->next[g->n2];
  g->ring[g->n1] += g->ring[g->n2];
  /* Norm_Factor = 1/(double)ULONG_MAX = 2^-64 */
  return (double)g->ring[g->n1] * (1.0 / 18446744073709551616.0);
}

oracle_rng *oracle_rng_create(long seed) { /* MyRand::init, MyRand.cc:73-110 */
  oracle_rng *g = (oracle_rng *)calloc(1, sizeof(*g));
  for (int i = 0; i < 54; i++) g->next[i] = i + 1;
  g->next[54] = 0;
  uint64_t tmp = (uint64_t)(161803398L + seed); /* Seed, MyRand.cc:30 */
  g->ring[54] = tmp;
  uint64_t aux = 1;
  int j = 20;
  for (int i = 0; i < 54; i++, j += 21) {
    j %= 55;
    g->ring[j] = aux;
    aux += tmp;
    tmp = g->ring[j];
  }
  g->n1 = 0;
  g->n2 = 31;
  for (j = 0; j < 55 * 4; j++) rng_flat(g);
  g->gen = 0;
  return g;
}

void oracle_rng_destroy(oracle_rng *g) { free(g); }

/* generate_gauss, MyRand.cc:115-130 (sqrt(-log(1-u)), no factor 2) */
void oracle_rng_gauss(oracle_rng *g, double *out, long n) {
  const double MY_2pi = 6.28318530717959; /* MyRand.h:41 */
  for (long k = 0; k < n; k++) {
    if (g->gen == 0) {
      g->t = MY_2pi * rng_flat(g);
      g->r = sqrt(-log((1. - rng_flat(g))));
      out[k] = g->r * cos(g->t);
      g->gen = 1;
    } else {
      out[k] = g->r * sin(g->t);
      g->gen = 0;
    }
  }
}

/* SU3rand(MyRand&), MyMath.cc:256-292 */
void oracle_su3rand(const double *g, double *m18) {
  cx *P = (cx *)m18;
  memset(P, 0, sizeof(cx) * 9);
  P[1].im = g[0];
  P[3].im = g[0];
  P[1].re = g[1];
  P[3].re = -g[1];
  P[2].im = g[2];
  P[6].im = g[2];
  P[2].re = g[3];
  P[6].re = -g[3];
  P[5].im = g[4];
  P[7].im = g[4];
  P[5].re = g[5];
  P[7].re = -g[5];
  double gg = g[7] * sqrt(D3); /* sD3, MyMath.h:49 */
  P[0].im = gg + g[6];
  P[4].im = gg - g[6];
  P[8].im = -2. * gg;
}

/* ---------------- random start ---------------- */

void oracle_random_start(oracle_ctx *c, long seed, double sigma) {
  int N = c->N;
  oracle_rng *g = oracle_rng_create(seed);
  double *buf = (double *)malloc(sizeof(double) * 18 * N);
  for (long s = 0; s < c->V; s++)
    for (int mu = 0; mu < 4; mu++) {
      cx *u = link_ptr(c->U, c, s, mu);
      oracle_rng_gauss(g, buf, 18L * N);
      u[0].re = 1.0;
      u[0].im = 0.0;
      double f = 1.0;
      for (int k = 0; k < N; k++) {
        f *= sigma;
        for (int e = 0; e < 9; e++) {
          u[1 + 9 * k + e].re = f * buf[18 * k + 2 * e];
          u[1 + 9 * k + e].im = f * buf[18 * k + 2 * e + 1];
        }
      }
    }
  free(buf);
  oracle_rng_destroy(g);
  oracle_unitarise(c);
}

/* U = exp(reH(log U)) for every link, the rule the reference applies to a
   configuration loaded with fewer orders (QCDenvNODEpt_test.h:414-417) */
void oracle_unitarise(oracle_ctx *c) {
  int N = c->N;
  long nl = c->V * 4;
#pragma omp parallel
  {
    cx *W = (cx *)malloc(sizeof(cx) * SER(N) * 3);
    cx *B = W + SER(N), *Bn = W + 2 * SER(N);
#pragma omp for schedule(static)
    for (long l = 0; l < nl; l++) {
      cx *u = c->U + (size_t)l * SER(N);
      s_log(W, u, N, B, Bn);
      s_reH(W, N);
      s_exp(u, W, N, B, Bn);
    }
    free(W);
  }
}

/* ---------------- staple (QCDenvNODEpt_test.h:554-557) ---------------- */

/* S = U_nu(n+mu) dag(U_nu(n) U_mu(n+nu)) + dag(U_mu(n-nu) U_nu(n-nu+mu)) U_nu(n-nu)
 * scratch: 7 series */
static void staple(const oracle_ctx *c, const cx *field, const int *x, int mu,
                   int nu, cx *S, cx *scr) {
  int N = c->N, n = SER(N);
  cx *a = scr, *b = scr + n, *t1 = scr + 2 * n, *t2 = scr + 3 * n,
     *s1 = scr + 4 * n, *s2 = scr + 5 * n, *dg = scr + 6 * n;
  int y[4];
  /* upper: U_nu(n+mu) * dag(U_nu(n) * U_mu(n+nu)) */
  fetch_link(c, field, x, nu, a);
  memcpy(y, x, sizeof(y));
  y[nu]++;
  fetch_link(c, field, y, mu, b);
  s_mul(t1, a, b, N);
  s_dag(dg, t1, N);
  memcpy(y, x, sizeof(y));
  y[mu]++;
  fetch_link(c, field, y, nu, a);
  s_mul(s1, a, dg, N);
  /* lower: dag(U_mu(n-nu) * U_nu(n-nu+mu)) * U_nu(n-nu) */
  memcpy(y, x, sizeof(y));
  y[nu]--;
  fetch_link(c, field, y, mu, a);
  y[mu]++;
  fetch_link(c, field, y, nu, b);
  s_mul(t2, a, b, N);
  s_dag(dg, t2, N);
  memcpy(y, x, sizeof(y));
  y[nu]--;
  fetch_link(c, field, y, nu, a);
  s_mul(s2, dg, a, N);
  /* ptSU3::operator+ QCDpt.cc:48-56 */
  for (int k = 1; k < n; k++) S[k] = cadd(s1[k], s2[k]);
  S[0] = cadd(s1[0], s2[0]);
}

/* ptSU3::staple2x1 (QCDenvNODEpt_test.h:579-611), periodic: the six 2x1
 * rectangles through link (x, mu) in the plane (mu, nu), summed as the
 * reference sums them.  Scratch: 6 series. */
static void staple2x1(const oracle_ctx *c, const cx *field, const int *x, int mu, int nu,
                      cx *out, cx *scr) {
  int N = c->N, n = SER(N);
  cx *A = scr, *B = scr + n, *C = scr + 2 * n, *D = scr + 3 * n, *E = scr + 4 * n,
     *G = scr + 5 * n;
#define AT(i, j)                                                               \
  ({                                                                           \
    int y_[4];                                                                 \
    memcpy(y_, x, sizeof(y_));                                                 \
    y_[mu] = ((y_[mu] + (i)) % c->L[mu] + c->L[mu]) % c->L[mu];                \
    y_[nu] = ((y_[nu] + (j)) % c->L[nu] + c->L[nu]) % c->L[nu];                \
    site_of(c, y_);                                                            \
  })
#define LK(site, d) link_ptr((cx *)field, c, site, d)
  long x0 = site_of(c, x);
  long a = AT(1, 0), b = AT(1, 1), cc = AT(0, 1), d = AT(0, 2), e = AT(2, 0), f = AT(-1, 0),
       g = AT(-1, 1);
  /* U_nu(a) U_nu(b) dag(U_nu(x) U_nu(c) U_mu(d)) */
  s_mul(A, LK(a, nu), LK(b, nu), N);
  s_mul(B, LK(x0, nu), LK(cc, nu), N);
  s_mul(C, B, LK(d, mu), N);
  s_dag(D, C, N);
  s_mul(out, A, D, N);
  /* + U_mu(a) U_nu(e) dag(U_nu(x) U_mu(c) U_mu(b)) */
  s_mul(A, LK(a, mu), LK(e, nu), N);
  s_mul(B, LK(x0, nu), LK(cc, mu), N);
  s_mul(C, B, LK(b, mu), N);
  s_dag(D, C, N);
  s_mul(E, A, D, N);
  s_acc(out, E, N);
  /* + U_nu(a) dag(U_nu(f) U_mu(g) U_mu(c)) U_mu(f) */
  s_mul(B, LK(f, nu), LK(g, mu), N);
  s_mul(C, B, LK(cc, mu), N);
  s_dag(D, C, N);
  s_mul(A, LK(a, nu), D, N);
  s_mul(E, A, LK(f, mu), N);
  s_acc(out, E, N);
  long b2 = AT(1, -1), c2 = AT(0, -1), d2 = AT(0, -2), e2 = AT(1, -2), f2 = AT(2, -1),
       g2 = AT(-1, -1), h2 = AT(-1, 0);
  /* dag(U_mu(d) U_nu(e) U_nu(b)) U_nu(d) U_nu(c) */
  s_mul(B, LK(d2, mu), LK(e2, nu), N);
  s_mul(C, B, LK(b2, nu), N);
  s_dag(D, C, N);
  s_mul(A, D, LK(d2, nu), N);
  s_mul(G, A, LK(c2, nu), N);
  /* + U_mu(a) dag(U_mu(c) U_mu(b) U_nu(f)) U_nu(c) */
  s_mul(B, LK(c2, mu), LK(b2, mu), N);
  s_mul(C, B, LK(f2, nu), N);
  s_dag(D, C, N);
  s_mul(A, LK(a, mu), D, N);
  s_mul(E, A, LK(c2, nu), N);
  s_acc(G, E, N);
  /* + dag(U_mu(g) U_mu(c) U_nu(b)) U_nu(g) U_mu(h) */
  s_mul(B, LK(g2, mu), LK(c2, mu), N);
  s_mul(C, B, LK(b2, nu), N);
  s_dag(D, C, N);
  s_mul(A, D, LK(g2, nu), N);
  s_mul(E, A, LK(h2, mu), N);
  s_acc(G, E, N);
  s_acc(out, G, N);
#undef AT
#undef LK
}

/* ---------------- Langevin sweep (nspt.cc:258-600) ---------------- */

/* Per-link observables of a sweep, reduced in link order afterwards. */
typedef struct {
  cx *tr;      /* [nl][N+1] Tr(U W), nspt.cc:393 */
  double *nrm; /* [nl][N]   Tr(U_k U_k^dag), nspt.cc:398 */
  cx *tu;      /* [nl][N]   Tr U_k, nspt.cc:400 */
  cx *lg;      /* [nl][SER] log of the new link (zero modes), or NULL */
  cx *tr2;     /* [nl][N+1] Tr(U W2), improved actions, or NULL */
} sweep_obs;

/* One link of gauge_wilson (nspt.cc:362-439): the staples of (x, mu) from
 * the field c->U (twisted crossings from c->snap when set), the force
 * reH(U W) tau_g, the noise, and the new link exp(W1) U into out, which may
 * be the link itself (the on-the-fly update).  l: the link's index.
 * Scratch: 24 series. */
static void sweep_link(oracle_ctx *c, const int *x, int mu, long l, double tau_g, double stau,
                       const double *noise, cx *out, sweep_obs *ob, cx *scr) {
  const int N = c->N, n = SER(N);
  const int imp = c->c1 != 0.0;
  cx *W2 = scr + 14 * n, *S2 = scr + 15 * n, *P2 = scr + 16 * n, *rs = scr + 17 * n;
  cx *W = scr + 7 * n, *S = scr + 8 * n, *P = scr + 9 * n, *E = scr + 10 * n,
     *B = scr + 11 * n, *Bn = scr + 12 * n, *Fn = scr + 13 * n;
  cx t[9], d[9];
  const long s = site_of(c, x);
  const cx *u = link_ptr(c->U, c, s, mu);
  s_zero(W, N);
  if (imp) s_zero(W2, N);
  for (int nu = 0; nu < 4; nu++) {
    if (nu == mu) continue;
    staple(c, c->U, x, mu, nu, S, scr);
    s_acc(W, S, N);
    if (imp) {
      staple2x1(c, c->U, x, mu, nu, S2, rs);
      s_acc(W2, S2, N);
    }
  }
  s_mul(P, u, W, N);
  /* ptSU3::Tr QCDpt.cc:115-122 */
  cx *trl = ob->tr + (size_t)l * (N + 1);
  trl[0].re = 3. * P[0].re;
  trl[0].im = 3. * P[0].im;
  for (int k = 0; k < N; k++) {
    trl[k + 1] = m_tr(P + 1 + 9 * k);
    m_dag(d, u + 1 + 9 * k);
    m_mul(t, u + 1 + 9 * k, d);
    ob->nrm[(size_t)l * N + k] = m_tr(t).re;
    ob->tu[(size_t)l * N + k] = m_tr(u + 1 + 9 * k);
  }
  if (imp) { /* nspt.cc:294-303: W1 = c0 W1 + c1 (U W2) */
    s_mul(P2, u, W2, N);
    cx *t2l = ob->tr2 + (size_t)l * (N + 1);
    t2l[0].re = 3. * P2[0].re;
    t2l[0].im = 3. * P2[0].im;
    for (int k = 0; k < N; k++) t2l[k + 1] = m_tr(P2 + 1 + 9 * k);
    const double c0 = 1. - 8. * c->c1;
    for (int k = 0; k < n; k++) {
      cx a0 = {c0 * P[k].re, c0 * P[k].im}, b0 = {c->c1 * P2[k].re, c->c1 * P2[k].im};
      P[k] = cadd(a0, b0);
    }
  }
  s_reH(P, N);
  s_scale(P, tau_g, N);
  /* W1.ptU[0] -= stau*SU3rand(Rand) nspt.cc:423 */
  cx eta[9];
  oracle_su3rand(noise + (size_t)l * 8, (double *)eta);
  for (int e = 0; e < 9; e++) {
    cx v = {stau * eta[e].re, stau * eta[e].im};
    P[1 + e] = csub(P[1 + e], v);
  }
  s_exp(E, P, N, B, Bn);
  /* F[link] = exp(W1)*U[link] (nspt.cc:429), or U[link] on the fly (:427) */
  s_mul(Fn, E, u, N);
  s_copy(out, Fn, N);
  if (ob->lg) s_log(ob->lg + (size_t)l * n, out, N, B, Bn);
}

static void obs_alloc(const oracle_ctx *c, int zero_modes, sweep_obs *ob) {
  const int N = c->N;
  const long nl = c->V * 4;
  ob->tr = (cx *)calloc((size_t)nl * (N + 1), sizeof(cx));
  ob->nrm = (double *)calloc((size_t)nl * N, sizeof(double));
  ob->tu = (cx *)calloc((size_t)nl * N, sizeof(cx));
  ob->lg = zero_modes ? (cx *)calloc((size_t)nl * SER(N), sizeof(cx)) : NULL;
  ob->tr2 = c->c1 != 0.0 ? (cx *)calloc((size_t)nl * (N + 1), sizeof(cx)) : NULL;
}

/* The sweep's sums (w1, norm, trU, MM, w2) in link order and normalised as
 * nspt.cc:570-597 prints them; frees the per-link arrays. */
static void obs_reduce(oracle_ctx *c, sweep_obs *ob, double *plaq, double *norm, double *tru) {
  const int N = c->N, n = SER(N);
  const long nl = c->V * 4;
  cx *w1 = (cx *)calloc(N + 1, sizeof(cx));
  double *nm = (double *)calloc(N, sizeof(double));
  cx *tm = (cx *)calloc(4 * (size_t)N, sizeof(cx));
  for (int mu = 0; mu < 4; mu++) s_zero(c->MM + (size_t)mu * n, N);
  for (long l = 0; l < nl; l++) {
    int mu = (int)(l % 4);
    for (int k = 0; k <= N; k++) w1[k] = cadd(w1[k], ob->tr[(size_t)l * (N + 1) + k]);
    for (int k = 0; k < N; k++) {
      nm[k] += ob->nrm[(size_t)l * N + k];
      tm[mu * N + k] = cadd(tm[mu * N + k], ob->tu[(size_t)l * N + k]);
    }
    if (ob->lg) s_acc(c->MM + (size_t)mu * n, ob->lg + (size_t)l * n, N);
  }
  if (ob->tr2) {
    cx *w2 = (cx *)calloc(N + 1, sizeof(cx));
    for (long l = 0; l < nl; l++)
      for (int k = 0; k <= N; k++) w2[k] = cadd(w2[k], ob->tr2[(size_t)l * (N + 1) + k]);
    for (int k = 0; k <= N; k++) {
      c->last_w2[2 * k] = w2[k].re / (double)(72 * c->V);
      c->last_w2[2 * k + 1] = w2[k].im / (double)(72 * c->V);
    }
    free(w2);
  }
  if (plaq)
    for (int k = 0; k <= N; k++) {
      plaq[2 * k] = w1[k].re / (double)(72 * c->V);
      plaq[2 * k + 1] = w1[k].im / (double)(72 * c->V);
    }
  if (norm)
    for (int k = 0; k < N; k++) norm[k] = nm[k] / (double)(12 * c->V);
  if (tru)
    for (int mu = 0; mu < 4; mu++)
      for (int k = 0; k < N; k++) {
        tru[2 * (mu * N + k)] = tm[mu * N + k].re / (double)(3 * c->V);
        tru[2 * (mu * N + k) + 1] = tm[mu * N + k].im / (double)(3 * c->V);
      }
  free(w1);
  free(nm);
  free(tm);
  free(ob->tr);
  free(ob->nrm);
  free(ob->tu);
  free(ob->lg);
  free(ob->tr2);
}

/* gauge_wilson(Umu, Fmu) with UPDATE_ONTHEFLY off (the Jacobi update,
 * nspt.cc:428-430), then Umu = Fmu (nspt.cc:992).  QuenchedAllocate sets
 * stau = sqrt(dt), tau_g = -dt/6 (Quenched.cc:584-589). */
void oracle_sweep(oracle_ctx *c, double dt, const double *noise, double *plaq,
                  double *norm, double *tru, int zero_modes) {
  const long nl = c->V * 4;
  double stau = sqrt(dt);
  double tau_g = dt;
  tau_g /= -(2 * 3);
  sweep_obs ob;
  obs_alloc(c, zero_modes, &ob);
  free(c->snap); /* every read sees the field as it was: no stale copies */
  c->snap = NULL;
#pragma omp parallel
  {
    cx *scr = (cx *)malloc(sizeof(cx) * SER(c->N) * 24);
#pragma omp for schedule(static)
    for (long l = 0; l < nl; l++) {
      long s = l / 4;
      int mu = (int)(l % 4), x[4];
      coords_of(c, s, x);
      sweep_link(c, x, mu, l, tau_g, stau, noise, link_ptr(c->F, c, s, mu), &ob, scr);
    }
    free(scr);
  }
  obs_reduce(c, &ob, plaq, norm, tru);
  /* Umu = Fmu, nspt.cc:992 */
  cx *sw = c->U;
  c->U = c->F;
  c->F = sw;
}

/* The order in which the reference built with the OpenMP thread grid
 * grid = {ntt, ntx, nty, ntz} (choices.h:124-128, blocks set up at
 * Quenched.cc:518-531) visits the sites in gauge_wilson (nspt.cc:355-460)
 * and stochastic_gauge_fixing (nspt.cc:723-815): thread tid owns a block of
 * L_d / n_d sites per direction and walks it lexicographically; all threads
 * take a barrier after every iteration of the deepest split direction's
 * loop.  Threads between two barriers touch disjoint links (their sites are
 * >= 2 apart in a split direction), so running them one after another in
 * thread order gives the same field.  Fills order[V] with site indices in
 * that serial order; -1 for a grid the reference rejects. */
static int grid_order(const oracle_ctx *c, const int *grid, long *order) {
  int bs[4], dmax = -1;
  for (int d = 0; d < 4; d++) {
    if (grid[d] < 1 || c->L[d] % grid[d]) return -1;
    bs[d] = c->L[d] / grid[d];
    if (grid[d] > 1) {
      if (bs[d] < 2) return -1;
      dmax = d;
    }
  }
  const int nthr = grid[0] * grid[1] * grid[2] * grid[3];
  long steps = 1, seg = 1, m = 0;
  for (int d = 0; d < 4; d++) {
    if (d <= dmax)
      steps *= bs[d];
    else
      seg *= c->L[d];
  }
  for (long p = 0; p < steps; p++) {
    int rel[4] = {0, 0, 0, 0};
    long q = p;
    for (int d = dmax; d >= 0; d--) {
      rel[d] = (int)(q % bs[d]);
      q /= bs[d];
    }
    for (int tid = 0; tid < nthr; tid++) {
      int b[4];
      b[0] = tid / (grid[1] * grid[2] * grid[3]);
      b[1] = (tid / (grid[2] * grid[3])) % grid[1];
      b[2] = (tid / grid[3]) % grid[2];
      b[3] = tid % grid[3];
      for (long r = 0; r < seg; r++) {
        int x[4];
        long t = r;
        for (int d = 3; d >= 0; d--) {
          if (d <= dmax) {
            x[d] = bs[d] * b[d] + rel[d];
          } else {
            x[d] = (int)(t % c->L[d]);
            t /= c->L[d];
          }
        }
        order[m++] = site_of(c, x);
      }
    }
  }
  return 0;
}

/* gauge_wilson(Umu) with UPDATE_ONTHEFLY, the reference's default
 * (choices.h:61): every link updated in place, U = exp(W1) U (nspt.cc:427),
 * sites in the thread grid's order, mu = 0..3 inner, so that a link's
 * staples see the links updated before it.  With twisted boundaries a read
 * across a twisted face sees the reference's copy site, which holds the
 * field of the last twist_boundary (the start of the step): the oracle keeps
 * that field in c->snap until oracle_twist_boundary.  The log of each new
 * link goes to MM (nspt.cc:432-437). */
int oracle_sweep_onthefly(oracle_ctx *c, double dt, const double *noise, const int *grid,
                          double *plaq, double *norm, double *tru, int zero_modes) {
  const int N = c->N;
  long *order = (long *)malloc(sizeof(long) * c->V);
  if (grid_order(c, grid, order)) {
    free(order);
    return -1;
  }
  double stau = sqrt(dt);
  double tau_g = dt;
  tau_g /= -(2 * 3);
  const size_t bytes = sizeof(cx) * (size_t)c->V * 4 * SER(N);
  if (c->tw) {
    if (!c->snap) c->snap = (cx *)malloc(bytes);
    memcpy(c->snap, c->U, bytes);
  }
  sweep_obs ob;
  obs_alloc(c, zero_modes, &ob);
  cx *scr = (cx *)malloc(sizeof(cx) * SER(N) * 24);
  for (long i = 0; i < c->V; i++) {
    const long s = order[i];
    int x[4];
    coords_of(c, s, x);
    for (int mu = 0; mu < 4; mu++)
      sweep_link(c, x, mu, s * 4 + mu, tau_g, stau, noise, link_ptr(c->U, c, s, mu), &ob, scr);
  }
  free(scr);
  free(order);
  obs_reduce(c, &ob, plaq, norm, tru);
  return 0;
}

/* twist_boundary (nspt.cc:163-255): the reference's copy sites are
 * refreshed, so reads across a twisted face see the field again. */
void oracle_twist_boundary(oracle_ctx *c) {
  free(c->snap);
  c->snap = NULL;
}

/* zero_modes_subtraction, nspt.cc:605-654 */
void oracle_zero_modes(oracle_ctx *c) {
  int N = c->N, n = SER(N);
  double rVol = 1.0 / (double)c->V;
  for (int mu = 0; mu < 4; mu++) s_scale(c->MM + (size_t)mu * n, rVol, N);
  long nl = c->V * 4;
#pragma omp parallel
  {
    cx *W = (cx *)malloc(sizeof(cx) * n * 3);
    cx *B = W + n, *Bn = W + 2 * n;
#pragma omp for schedule(static)
    for (long l = 0; l < nl; l++) {
      int mu = (int)(l % 4);
      cx *u = c->U + (size_t)l * n;
      s_log(W, u, N, B, Bn);
      s_sub_acc(W, c->MM + (size_t)mu * n, N);
      s_reH(W, N);
      s_exp(u, W, N, B, Bn);
    }
    free(W);
  }
}

/* FAstochastic_gauge_fixing, nspt.cc:866-948 (periodic boundaries) */
void oracle_fa_gauge_fix(oracle_ctx *c, double alpha) {
  int N = c->N, n = SER(N);
  long V = c->V, nl = V * 4;
  cx *lg = (cx *)malloc(sizeof(cx) * (size_t)nl * n);
  cx *Wg = (cx *)calloc((size_t)V * n, sizeof(cx));
#pragma omp parallel
  {
    cx *B = (cx *)malloc(sizeof(cx) * n * 2), *Bn = B + n;
#pragma omp for schedule(static)
    for (long l = 0; l < nl; l++)
      s_log(lg + (size_t)l * n, c->U + (size_t)l * n, N, B, Bn);
    free(B);
  }
  /* Wg[x] = sum_mu log U_mu(x) - log U_mu(x-mu)  (nspt.cc:871-877) */
#pragma omp parallel
  {
    cx *T = (cx *)malloc(sizeof(cx) * n);
#pragma omp for schedule(static)
    for (long s = 0; s < V; s++) {
      int x[4];
      coords_of(c, s, x);
      cx *w = Wg + (size_t)s * n;
      s_zero(w, N);
      for (int mu = 0; mu < 4; mu++) {
        int y[4];
        memcpy(y, x, sizeof(y));
        y[mu] = (y[mu] - 1 + c->L[mu]) % c->L[mu];
        const cx *a = lg + ((size_t)s * 4 + mu) * n;
        const cx *b = lg + ((size_t)site_of(c, y) * 4 + mu) * n;
        for (int k = 0; k < n; k++) T[k] = csub(a[k], b[k]);
        s_acc(w, T, N);
      }
    }
    free(T);
  }
  free(lg);
  /* forward FFT over every component (Quenched.cc:827-832) */
  for (int m = 0; m < n; m++) oracle_dft_nd((double *)(Wg + m), 4, c->L, n, -1);
  s_scale(Wg, 0.0, N); /* Wgauge->W[0] *= 0.0 (PBC) nspt.cc:881-883 */
  for (long s = 1; s < V; s++) {
    int x[4];
    coords_of(c, s, x);
    double f = -(alpha / (c->p2hat[0][x[0]] + c->p2hat[1][x[1]] +
                          c->p2hat[2][x[2]] + c->p2hat[3][x[3]]));
    s_scale(Wg + (size_t)s * n, f, N);
  }
  for (int m = 0; m < n; m++) oracle_dft_nd((double *)(Wg + m), 4, c->L, n, +1);
#pragma omp parallel
  {
    cx *E = (cx *)malloc(sizeof(cx) * n * 3), *B = E + n, *Bn = E + 2 * n;
#pragma omp for schedule(static)
    for (long s = 0; s < V; s++) {
      cx *w = Wg + (size_t)s * n;
      s_div(w, (double)V, N);
      s_reH(w, N);
      s_exp(E, w, N, B, Bn);
      s_copy(w, E, N);
    }
    free(E);
  }
  /* U_mu(x) = Wg(x) U_mu(x) dag(Wg(x+mu)) (nspt.cc:912-916) */
#pragma omp parallel
  {
    cx *T = (cx *)malloc(sizeof(cx) * n * 2), *D = T + n;
#pragma omp for schedule(static)
    for (long l = 0; l < nl; l++) {
      long s = l / 4;
      int mu = (int)(l % 4), x[4];
      coords_of(c, s, x);
      x[mu] = (x[mu] + 1) % c->L[mu];
      cx *u = c->U + (size_t)l * n;
      s_mul(T, Wg + (size_t)s * n, u, N);
      s_dag(D, Wg + (size_t)site_of(c, x) * n, N);
      s_mul(u, T, D, N);
    }
    free(T);
  }
  free(Wg);
}

/* One site of stochastic_gauge_fixing (nspt.cc:665-720, OpenMP branch
 * nspt.cc:731-795): W = sum_mu U_mu(x) - U_mu(x-mu) (the backward link read
 * through the twisted copy when it crosses a twisted face), W -= W^dag,
 * Trless, then U_mu(x) <- exp(alpha W) U_mu(x) and U_mu(x-mu) <- U_mu(x-mu)
 * exp(-alpha W), where a backward link across a twisted face takes
 * twist_mu(exp(-alpha W)) = Omega W2 Omega^dag per order, flag VACUUM = 1
 * (nspt.cc:97-160). Scratch: 8 series. */
static void local_gf_site(oracle_ctx *c, const int *x, double alpha, cx *scr) {
  int N = c->N, n = SER(N);
  cx *W = scr, *T = scr + n, *D = scr + 2 * n, *A = scr + 3 * n, *E1 = scr + 4 * n,
     *E2 = scr + 5 * n, *B = scr + 6 * n, *Bn = scr + 7 * n;
  long s = site_of(c, x);
  s_zero(W, N);
  for (int mu = 0; mu < 4; mu++) {
    int y[4];
    memcpy(y, x, sizeof(y));
    y[mu] -= 1;
    const cx *a = link_ptr(c->U, c, s, mu);
    fetch_link(c, c->U, y, mu, D);
    for (int k = 0; k < n; k++) T[k] = csub(a[k], D[k]);
    s_acc(W, T, N);
  }
  s_dag(D, W, N);
  s_sub_acc(W, D, N);
  s_trless(W, N);
  for (int k = 0; k < n; k++) {
    A[k].re = alpha * W[k].re;
    A[k].im = alpha * W[k].im;
  }
  s_exp(E1, A, N, B, Bn);
  for (int k = 0; k < n; k++) {
    A[k].re = -alpha * W[k].re;
    A[k].im = -alpha * W[k].im;
  }
  s_exp(E2, A, N, B, Bn);
  for (int mu = 0; mu < 4; mu++) {
    cx *u = link_ptr(c->U, c, s, mu);
    s_mul(T, E1, u, N);
    s_copy(u, T, N);
    int y[4];
    memcpy(y, x, sizeof(y));
    const int wrap = y[mu] == 0;
    y[mu] = (y[mu] - 1 + c->L[mu]) % c->L[mu];
    cx *v = link_ptr(c->U, c, site_of(c, y), mu);
    const cx *w2 = E2;
    if (wrap && ((c->tw >> mu) & 1)) {
      cx t[9], q[9];
      for (int k = 0; k < N; k++) {
        m_mul(t, c->omega[mu], E2 + 1 + 9 * k);
        m_mul(q, t, c->omegadag[mu]);
        memcpy(D + 1 + 9 * k, q, sizeof(q));
      }
      D[0].re = 1.0;
      D[0].im = 0.0;
      w2 = D;
    }
    s_mul(T, v, w2, N);
    s_copy(v, T, N);
  }
}

/* stochastic_gauge_fixing, nspt.cc:660-862, in place, as the reference
 * built with the OpenMP thread grid grid = {ntt, ntx, nty, ntz}
 * (choices.h:124-128, blocks set up at Quenched.cc:518-531) runs it: thread
 * tid owns a block of L_d / n_d sites per direction and walks it
 * lexicographically; all threads take a barrier after every iteration of the
 * deepest split direction's loop (nspt.cc:796-815).  Threads between two
 * barriers touch disjoint links (their sites are >= 2 apart), so the result
 * is the sequential replay: barrier step by barrier step, thread by thread,
 * each thread's segment in order.  grid {1,1,1,1} is the plain lexicographic
 * sweep (nspt.cc:658-720).  Returns -1 if a block is not a whole number of
 * sites >= 2 in a split direction. */
int oracle_local_gauge_fix_grid(oracle_ctx *c, double alpha, const int *grid) {
  long *order = (long *)malloc(sizeof(long) * c->V);
  if (grid_order(c, grid, order)) {
    free(order);
    return -1;
  }
  cx *scr = (cx *)malloc(sizeof(cx) * SER(c->N) * 8);
  for (long i = 0; i < c->V; i++) {
    int x[4];
    coords_of(c, order[i], x);
    local_gf_site(c, x, alpha, scr);
  }
  free(scr);
  free(order);
  return 0;
}

/* stochastic_gauge_fixing with the reference's default grid {1,1,1,1}:
 * the sequential lexicographic sweep. */
void oracle_local_gauge_fix(oracle_ctx *c, double alpha) {
  const int one[4] = {1, 1, 1, 1};
  oracle_local_gauge_fix_grid(c, alpha, one);
}

/* ComputeLoops, nspt.cc:1148-1312 (periodic boundaries): per plane mu < nu
 * and site x the 1x2 (both orientations), 2x2, 2x4 (both) and 4x4 Wilson
 * loops as series, summed in the reference's order, then traced.  out holds
 * 4 x (N+1) complex traces, already normalised as the reference prints them
 * (loopNorm = 1/(3*2*3*V), with the extra 1/2 for 1x2 and 2x4): l21, l22,
 * l42, l44.  The reference prints the real parts of the even orders. */
void oracle_wilson_loops(oracle_ctx *c, double *out) {
  int N = c->N, n = SER(N);
  cx *scr = (cx *)malloc(sizeof(cx) * n * 24);
  cx *w22 = scr, *w21 = scr + n, *w42 = scr + 2 * n, *w44 = scr + 3 * n;
  cx *bl = scr + 4 * n, *ml = scr + 5 * n, *cd = scr + 6 * n, *ld = scr + 7 * n;
  cx *br = scr + 8 * n, *mr = scr + 9 * n, *tr = scr + 10 * n, *tl = scr + 11 * n;
  cx *lu = scr + 12 * n, *cu = scr + 13 * n, *ru = scr + 14 * n, *rd = scr + 15 * n;
  cx *t1 = scr + 16 * n, *t2 = scr + 17 * n, *t3 = scr + 18 * n, *t4 = scr + 19 * n;
  cx *t5 = scr + 20 * n, *t6 = scr + 21 * n;
  s_zero(w22, N);
  s_zero(w21, N);
  s_zero(w42, N);
  s_zero(w44, N);
#define LNK(site, d) link_ptr(c->U, c, site, d)
  for (int mu = 0; mu < 3; mu++)
    for (int nu = mu + 1; nu < 4; nu++)
      for (long x = 0; x < c->V; x++) {
        int X[4];
        coords_of(c, x, X);
        /* site at X + i mu + j nu (periodic) */
#define AT(i, j)                                                               \
  ({                                                                           \
    int y_[4];                                                                 \
    memcpy(y_, X, sizeof(y_));                                                 \
    y_[mu] = (y_[mu] + (i)) % c->L[mu];                                        \
    y_[nu] = (y_[nu] + (j)) % c->L[nu];                                        \
    site_of(c, y_);                                                            \
  })
        long a = AT(1, 0), b = AT(2, 0), cc = AT(2, 1), e = AT(0, 1), d = AT(1, 1);
        long f = AT(2, 2), g = AT(1, 2), h = AT(0, 2);
        s_mul(bl, LNK(x, mu), LNK(a, mu), N);
        s_mul(ml, LNK(h, mu), LNK(g, mu), N);
        s_mul(cd, LNK(b, nu), LNK(cc, nu), N);
        s_mul(ld, LNK(x, nu), LNK(e, nu), N);
        /* w22 += bl*cd*dag(ld*ml) */
        s_mul(t1, bl, cd, N);
        s_mul(t2, ld, ml, N);
        s_dag(t3, t2, N);
        s_mul(t4, t1, t3, N);
        s_acc(w22, t4, N);
        /* w21 += bl*U_nu(b)*dag(U_nu(x)*U_mu(e)*U_mu(d))
         *      + U_mu(x)*U_nu(a)*U_nu(d)*dag(ld*U_mu(h)) */
        s_mul(t1, bl, LNK(b, nu), N);
        s_mul(t2, LNK(x, nu), LNK(e, mu), N);
        s_mul(t3, t2, LNK(d, mu), N);
        s_dag(t2, t3, N);
        s_mul(t5, t1, t2, N);
        s_mul(t1, LNK(x, mu), LNK(a, nu), N);
        s_mul(t2, t1, LNK(d, nu), N);
        s_mul(t3, ld, LNK(h, mu), N);
        s_dag(t1, t3, N);
        s_mul(t6, t2, t1, N);
        s_acc(t5, t6, N);
        s_acc(w21, t5, N);
        long i = AT(0, 3), j = AT(2, 3), k = AT(2, 4), nn = AT(0, 4), l = AT(1, 4);
        long m = AT(3, 0), o = AT(4, 0), p = AT(4, 1), q = AT(4, 2), r = AT(3, 2);
        long ss = AT(4, 3), t = AT(3, 4);
        s_mul(br, LNK(b, mu), LNK(m, mu), N);
        s_mul(mr, LNK(f, mu), LNK(r, mu), N);
        s_mul(tr, LNK(k, mu), LNK(t, mu), N);
        s_mul(tl, LNK(nn, mu), LNK(l, mu), N);
        s_mul(lu, LNK(h, nu), LNK(i, nu), N);
        s_mul(cu, LNK(f, nu), LNK(j, nu), N);
        s_mul(ru, LNK(q, nu), LNK(ss, nu), N);
        s_mul(rd, LNK(o, nu), LNK(p, nu), N);
        /* w42 += bl*(br*rd*dag(ml*mr) + cd*cu*dag(lu*tl))*dag(ld) */
        s_mul(t1, br, rd, N);
        s_mul(t2, ml, mr, N);
        s_dag(t3, t2, N);
        s_mul(t5, t1, t3, N);
        s_mul(t1, cd, cu, N);
        s_mul(t2, lu, tl, N);
        s_dag(t3, t2, N);
        s_mul(t6, t1, t3, N);
        s_acc(t5, t6, N);
        s_mul(t1, bl, t5, N);
        s_dag(t2, ld, N);
        s_mul(t3, t1, t2, N);
        s_acc(w42, t3, N);
        /* w44 += bl*br*rd*ru*dag(ld*lu*tl*tr) */
        s_mul(t1, bl, br, N);
        s_mul(t2, t1, rd, N);
        s_mul(t1, t2, ru, N);
        s_mul(t2, ld, lu, N);
        s_mul(t3, t2, tl, N);
        s_mul(t2, t3, tr, N);
        s_dag(t3, t2, N);
        s_mul(t2, t1, t3, N);
        s_acc(w44, t2, N);
#undef AT
      }
#undef LNK
  const double norm = 1. / (3 * 2 * 3 * (double)c->V);
  const double fac[4] = {.5 * norm, norm, .5 * norm, norm};
  cx *ws[4] = {w21, w22, w42, w44};
  for (int q = 0; q < 4; q++) {
    double *o = out + (size_t)q * 2 * (N + 1);
    o[0] = 3. * ws[q][0].re * fac[q];
    o[1] = 3. * ws[q][0].im * fac[q];
    for (int k = 1; k <= N; k++) {
      cx tt = m_tr(ws[q] + 1 + 9 * (k - 1));
      o[2 * k] = tt.re * fac[q];
      o[2 * k + 1] = tt.im * fac[q];
    }
  }
  free(scr);
}

/* plaquette_measure, nspt.cc:1316-1406 (OpenMP variant) */
void oracle_plaquette(oracle_ctx *c, double *plaq) {
  int N = c->N, n = SER(N);
  long nl = c->V * 4;
  cx *tr = (cx *)calloc((size_t)nl * (N + 1), sizeof(cx));
#pragma omp parallel
  {
    cx *scr = (cx *)malloc(sizeof(cx) * n * 10);
    cx *W = scr + 7 * n, *S = scr + 8 * n, *P = scr + 9 * n;
#pragma omp for schedule(static)
    for (long l = 0; l < nl; l++) {
      long s = l / 4;
      int mu = (int)(l % 4), x[4];
      coords_of(c, s, x);
      s_zero(W, N);
      for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        staple(c, c->U, x, mu, nu, S, scr);
        s_acc(W, S, N);
      }
      s_mul(P, link_ptr(c->U, c, s, mu), W, N);
      cx *t = tr + (size_t)l * (N + 1);
      t[0].re = 3. * P[0].re;
      t[0].im = 3. * P[0].im;
      for (int k = 0; k < N; k++) t[k + 1] = m_tr(P + 1 + 9 * k);
    }
    free(scr);
  }
  for (int k = 0; k <= N; k++) {
    cx w = {0.0, 0.0};
    for (long l = 0; l < nl; l++) w = cadd(w, tr[(size_t)l * (N + 1) + k]);
    plaq[2 * k] = w.re / (double)(c->V * 72);
    plaq[2 * k + 1] = w.im / (double)(c->V * 72);
  }
  free(tr);
}

/* ---------------- single-series entry points for unit tests ---------------- */

void oracle_ser_mul(int N, const double *a, const double *b, double *out) {
  s_mul((cx *)out, (const cx *)a, (const cx *)b, N);
}
void oracle_ser_exp(int N, const double *a, double *out) {
  cx *s = (cx *)malloc(sizeof(cx) * SER(N) * 2);
  s_exp((cx *)out, (const cx *)a, N, s, s + SER(N));
  free(s);
}
void oracle_ser_log(int N, const double *a, double *out) {
  cx *s = (cx *)malloc(sizeof(cx) * SER(N) * 2);
  s_log((cx *)out, (const cx *)a, N, s, s + SER(N));
  free(s);
}
void oracle_ser_reH(int N, double *a) { s_reH((cx *)a, N); }
void oracle_ser_dag(int N, const double *a, double *out) {
  s_dag((cx *)out, (const cx *)a, N);
}

/* Improved gauge action (Quenched.cc:311-322): c1 = -1/12 (TLSYM), -0.331
 * (IWA), -1.4088 (DBW2), 0 (Wilson); c0 = 1 - 8 c1.  Periodic only. */
int oracle_set_action(oracle_ctx *c, double c1) {
  if (c1 != 0.0 && c->tw) return -1;
  if (c1 != 0.0 && c->N > 64) return -1;
  c->c1 = c1;
  return 0;
}

/* rectangle traces of the last sweep (w2 of nspt.cc:294-303), /72V */
void oracle_last_w2(oracle_ctx *c, double *out) {
  memcpy(out, c->last_w2, sizeof(double) * 2 * (c->N + 1));
}
