// Wilson loops of ComputeLoops (nspt.cc:1148-1312): 1x2 (both
// orientations), 2x2, 2x4 (both) and 4x4 loops in every plane mu < nu,
// summed over the lattice and traced, per order.  Periodic boundaries, as
// the reference computes them only there (__MANY_LOOP__ under PERIODIC_BC).
//
// One 9-lane group per (plane, site).  The reference closes each loop with a
// product by a daggered path, W += P Q^dag; only Tr W is printed, so the last
// product is replaced by Tr(P Q^dag) = sum over cells of P_ij conj(Q_ij),
// order by order.  Three slots per group (two paths and a staging slot) and
// the group's four trace accumulators; CTAs sum their groups, and a last
// kernel their rows, in a fixed order.
#pragma once

namespace nspt {

constexpr int LOOP_SLOTS = 3;

// acc[k] += Tr(X Y^dag)_k, k = 0..N (flags are multiples of the identity)
__device__ __forceinline__ void trace_dag_acc(const double2 *X, const double2 *Y, int N,
                                              const Lane &L, double2 *acc) {
  const double2 x0 = X[0], y0 = Y[0];
  for (int k = L.j; k <= N; k += GROUP) {
    double2 s;
    if (k == 0) {
      s = cscale(cmul(x0, cconj(y0)), 3.0);
    } else {
      const double2 trX = cadd(cadd(X[sidx(k, 0, 0)], X[sidx(k, 1, 1)]), X[sidx(k, 2, 2)]);
      const double2 trY = cadd(cadd(Y[sidx(k, 0, 0)], Y[sidx(k, 1, 1)]), Y[sidx(k, 2, 2)]);
      s = cadd(cmul(x0, cconj(trY)), cmul(trX, cconj(y0)));
      for (int i = 1; i < k; i++) {
        const double2 *xi = X + 1 + 9 * (i - 1), *yj = Y + 1 + 9 * (k - i - 1);
#pragma unroll
        for (int e = 0; e < 9; e++) {
          const double2 a = xi[e], b = yj[e];
          s.x = fma(a.x, b.x, s.x);
          s.x = fma(a.y, b.y, s.x);
          s.y = fma(a.y, b.x, s.y);
          s.y = fma(-a.x, b.y, s.y);
        }
      }
    }
    acc[k] = cadd(acc[k], s);
  }
  __syncwarp(L.mask);
}

// A path of the loops: a chain of forward links, link m in direction
// dir[m] at the site reached by the steps of the links before it.
struct LoopPath {
  int n;         // links
  int dir[8];    // 0: mu, 1: nu
};

struct LoopCtx {
  const double2 *U, *Uf;
  int N, mu, nu;
  int X[4];
  Geo geo;
};

// site X + i mu + j nu (periodic)
__device__ __forceinline__ int loop_site(const LoopCtx &q, int i, int j) {
  int y[4] = {q.X[0], q.X[1], q.X[2], q.X[3]};
  y[q.mu] = (y[q.mu] + i) % q.geo.L[q.mu];
  y[q.nu] = (y[q.nu] + j) % q.geo.L[q.nu];
  return y[0] * q.geo.s0 + y[1] * q.geo.s1 + y[2] * q.geo.s2 + y[3];
}

__device__ __forceinline__ void loop_stage(const LoopCtx &q, double2 *slot, int dir, int i, int j,
                                           const Lane &L) {
  Nb n;
  n.site = loop_site(q, i, j);
  n.fwd = n.bwd = 0;
  stage(slot, q.U, q.Uf, dir ? q.nu : q.mu, n, q.geo, q.N, L);
}

// A <- A S, in place
__device__ __noinline__ void loop_mul(double2 *A, const double2 *S, int N, const Lane &L) {
  const double2 a0 = A[0], b0 = S[0];
  const int c = L.c;
  product<MO, false>(LeftS{A}, a0, S, b0, N, L,
                     [&](int k, int r, double2 v) { A[sidx(k, r, c)] = v; });
  if (L.j == 0) A[0] = flag_mul(a0, b0);
  __syncwarp(L.mask);
}

// A <- path[from..n) applied to A (from = 0: A is formed from the first
// link); (i, j) is the site where link `from` starts, updated to the end
__device__ __forceinline__ void loop_chain(const LoopCtx &q, double2 *A, double2 *S,
                                           const LoopPath &p, int from, int &i, int &j,
                                           const Lane &L) {
  for (int m = from; m < p.n; m++) {
    loop_stage(q, m == 0 ? A : S, p.dir[m], i, j, L);
    if (m > 0) loop_mul(A, S, q.N, L);
    if (p.dir[m]) j++; else i++;
  }
}

// Per (plane, site), the loops of ComputeLoops as pairs of paths P, Q from
// x, traced as Tr(P Q^dag) (bl = mu mu from x, ld = nu nu from x, cd the
// two nu links after bl, and so on, as named in nspt.cc:1160-1270):
//   2x2        P = bl cd           Q = ld ml
//   2x4 up     P = bl cd cu        Q = ld lu tl
//   4x4        P = bl br rd ru     Q = ld lu tl tr
//   2x4 right  P = bl br rd        Q = ld ml mr
//   1x2        P = bl U_nu         Q = U_nu U_mu U_mu
//   1x2        P = U_mu U_nu U_nu  Q = ld U_mu
// Three slots per group: P and Q (paths, each extended in place link by
// link) and S (the staged link).  A path is extended when the next loop's
// path starts with it (bl cd -> bl cd cu, ld lu tl -> ld lu tl tr) and
// formed afresh otherwise: 40 products and 6 traces per (plane, site).
__global__ void __launch_bounds__(256, 1)
    k_loops(const double2 *U, const double2 *Uf, int N, int SS, Geo geo, double2 *partial) {
  extern __shared__ double2 sm[];
  Lane L;
  int g;
  const bool grouped = make_lane(L, g);
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int row = 4 * (N + 1);
  const size_t gsz = (size_t)LOOP_SLOTS * SS + row;
  double2 *base = sm + (size_t)(warp * LPW + g) * gsz;
  double2 *acc = base + (size_t)LOOP_SLOTS * SS;
  if (grouped) {
    double2 *P = base, *Q = base + SS, *S = base + 2 * SS;
    for (int e = L.j; e < row; e += GROUP) acc[e] = cz();
    __syncwarp(L.mask);
    double2 *a21 = acc, *a22 = acc + (N + 1), *a42 = acc + 2 * (N + 1), *a44 = acc + 3 * (N + 1);
    LoopCtx q;
    q.U = U;
    q.Uf = Uf;
    q.N = N;
    q.geo = geo;
    const LoopPath p22{4, {0, 0, 1, 1}}, q22{4, {1, 1, 0, 0}};
    const LoopPath p42u{6, {0, 0, 1, 1, 1, 1}}, q42u{6, {1, 1, 1, 1, 0, 0}};
    const LoopPath p44{8, {0, 0, 0, 0, 1, 1, 1, 1}}, q44{8, {1, 1, 1, 1, 0, 0, 0, 0}};
    const LoopPath p42r{6, {0, 0, 0, 0, 1, 1}}, q42r{6, {1, 1, 0, 0, 0, 0}};
    const LoopPath p21a{3, {0, 0, 1}}, q21a{3, {1, 0, 0}};
    const LoopPath p21b{3, {0, 1, 1}}, q21b{3, {1, 1, 0}};
    const long units = 6L * geo.V;
    const long stride = (long)gridDim.x * nw * LPW;
    for (long u = ((long)blockIdx.x * nw + warp) * LPW + g; u < units; u += stride) {
      const int pl = (int)(u / geo.V);
      const int x = (int)(u - (long)pl * geo.V);
      q.mu = pl < 3 ? 0 : (pl < 5 ? 1 : 2);
      q.nu = pl < 3 ? pl + 1 : (pl < 5 ? pl - 1 : 3);
      coords(geo, x, q.X);
      int pi = 0, pj = 0, qi = 0, qj = 0;
      // 2x2
      loop_chain(q, P, S, p22, 0, pi, pj, L);
      loop_chain(q, Q, S, q22, 0, qi, qj, L);
      trace_dag_acc(P, Q, N, L, a22);
      // 2x4 up: P = bl cd extended by cu
      loop_chain(q, P, S, p42u, 4, pi, pj, L);
      qi = qj = 0;
      loop_chain(q, Q, S, q42u, 0, qi, qj, L);
      trace_dag_acc(P, Q, N, L, a42);
      // 4x4: Q = ld lu tl extended by tr
      loop_chain(q, Q, S, q44, 6, qi, qj, L);
      pi = pj = 0;
      loop_chain(q, P, S, p44, 0, pi, pj, L);
      trace_dag_acc(P, Q, N, L, a44);
      // 2x4 right
      pi = pj = qi = qj = 0;
      loop_chain(q, P, S, p42r, 0, pi, pj, L);
      loop_chain(q, Q, S, q42r, 0, qi, qj, L);
      trace_dag_acc(P, Q, N, L, a42);
      // 1x2, both orientations
      pi = pj = qi = qj = 0;
      loop_chain(q, P, S, p21a, 0, pi, pj, L);
      loop_chain(q, Q, S, q21a, 0, qi, qj, L);
      trace_dag_acc(P, Q, N, L, a21);
      pi = pj = qi = qj = 0;
      loop_chain(q, P, S, p21b, 0, pi, pj, L);
      loop_chain(q, Q, S, q21b, 0, qi, qj, L);
      trace_dag_acc(P, Q, N, L, a21);
    }
  }
  __syncthreads();
  const int ngroups = nw * LPW;
  for (int e = threadIdx.x; e < row; e += blockDim.x) {
    double2 sum = cz();
    for (int gi = 0; gi < ngroups; gi++)
      sum = cadd(sum, sm[(size_t)gi * gsz + (size_t)LOOP_SLOTS * SS + e]);
    partial[(size_t)blockIdx.x * row + e] = sum;
  }
}

// out[e] = sum over rows of partial[row][e], rows in order
__global__ void k_rows_sum(const double2 *partial, int nrows, int width, double2 *out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < width; e += gridDim.x * blockDim.x) {
    double2 s = cz();
    for (int r = 0; r < nrows; r++) s = cadd(s, partial[(size_t)r * width + e]);
    out[e] = s;
  }
}

}  // namespace nspt
