// Wilson loops of ComputeLoops (nspt.cc:1148-1312): 1x2 (both
// orientations), 2x2, 2x4 (both) and 4x4 loops in every plane mu < nu,
// summed over the lattice and traced, per order.  Periodic boundaries, as
// the reference computes them only there (__MANY_LOOP__ under PERIODIC_BC).
//
// One 9-lane group per (plane, site).  The reference closes each loop with a
// product by a daggered path, W += P Q^dag; only Tr W is printed, so the last
// product is replaced by Tr(P Q^dag) = sum over cells of P_ij conj(Q_ij),
// order by order: 28 series products and 5 such traces per (plane, site).
// Nine slots per group (eight paths and a staging slot), the ring for the
// streamed left link, and the group's four trace accumulators.  CTAs sum
// their groups, and a last kernel their rows, in a fixed order.
#pragma once

namespace nspt {

constexpr int LOOP_SLOTS = 9;

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

// Loop paths, each one instance (the kernel calls them many times).
struct LoopCtx {
  const double2 *U, *Uf;
  double2 *STG, *ring;
  size_t V, plane;
  int N;
  Geo geo;
};

// out = U_d1(s1) U_d2(s2): the left link streamed, the right one staged
__device__ __noinline__ void loop_two(const LoopCtx &q, double2 *out, int d1, int s1, int d2,
                                      int s2, const Lane &L) {
  Nb n;
  n.site = s2;
  n.fwd = n.bwd = 0;
  stage(q.STG, q.U, q.Uf, d2, n, q.geo, q.N, L);
  const double2 a0 = __ldg(q.Uf + (size_t)d1 * q.V + s1), b0 = q.STG[0];
  const int c = L.c;
  product<MO, false>(LeftG{q.U + d1 * q.plane + s1, q.V, q.ring}, a0, q.STG, b0, q.N, L,
                     [&](int k, int r, double2 v) { out[sidx(k, r, c)] = v; });
  if (L.j == 0) out[0] = flag_mul(a0, b0);
  __syncwarp(L.mask);
}

// out = A B (slots)
__device__ __noinline__ void loop_mul(double2 *out, const double2 *A, const double2 *B, int N,
                                      const Lane &L) {
  const double2 a0 = A[0], b0 = B[0];
  const int c = L.c;
  product<MO, false>(LeftS{A}, a0, B, b0, N, L,
                     [&](int k, int r, double2 v) { out[sidx(k, r, c)] = v; });
  if (L.j == 0) out[0] = flag_mul(a0, b0);
  __syncwarp(L.mask);
}

// out = A U_d(s)
__device__ __noinline__ void loop_mul_link(const LoopCtx &q, double2 *out, const double2 *A, int d,
                                           int s, const Lane &L) {
  Nb n;
  n.site = s;
  n.fwd = n.bwd = 0;
  stage(q.STG, q.U, q.Uf, d, n, q.geo, q.N, L);
  loop_mul(out, A, q.STG, q.N, L);
}

__global__ void __launch_bounds__(256, 1)
    k_loops(const double2 *U, const double2 *Uf, int N, int SS, Geo geo, double2 *partial) {
  extern __shared__ double2 sm[];
  Lane L;
  int g;
  const bool grouped = make_lane(L, g);
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int row = 4 * (N + 1);
  const size_t gsz = (size_t)LOOP_SLOTS * SS + RING + row;
  double2 *base = sm + (size_t)(warp * LPW + g) * gsz;
  double2 *acc = base + (size_t)LOOP_SLOTS * SS + RING;
  if (grouped) {
    LoopCtx q;
    q.U = U;
    q.Uf = Uf;
    q.STG = base + (size_t)8 * SS;
    q.ring = q.STG + SS;
    q.V = (size_t)geo.V;
    q.plane = (size_t)9 * N * q.V;
    q.N = N;
    q.geo = geo;
    double2 *S0 = base, *S1 = base + SS, *S2 = base + 2 * SS, *S3 = base + 3 * SS;
    double2 *S4 = base + 4 * SS, *S5 = base + 5 * SS, *S6 = base + 6 * SS, *S7 = base + 7 * SS;
    for (int e = L.j; e < row; e += GROUP) acc[e] = cz();
    __syncwarp(L.mask);
    double2 *a21 = acc, *a22 = acc + (N + 1), *a42 = acc + 2 * (N + 1), *a44 = acc + 3 * (N + 1);
    const long units = 6L * geo.V;
    const long stride = (long)gridDim.x * nw * LPW;
    for (long u = ((long)blockIdx.x * nw + warp) * LPW + g; u < units; u += stride) {
      const int pl = (int)(u / geo.V);
      const int x = (int)(u - (long)pl * geo.V);
      const int mu = pl < 3 ? 0 : (pl < 5 ? 1 : 2);
      const int nu = pl < 3 ? pl + 1 : (pl < 5 ? pl - 1 : 3);
      int X[4];
      coords(geo, x, X);
      // site x + i mu + j nu
      auto at = [&](int i, int j) {
        int y[4] = {X[0], X[1], X[2], X[3]};
        y[mu] = (y[mu] + i) % geo.L[mu];
        y[nu] = (y[nu] + j) % geo.L[nu];
        return y[0] * geo.s0 + y[1] * geo.s1 + y[2] * geo.s2 + y[3];
      };
      loop_two(q, S0, mu, x, mu, at(1, 0), L);           // bl
      loop_two(q, S1, nu, x, nu, at(0, 1), L);           // ld
      // 2x2: bl cd (ld ml)^dag
      loop_two(q, S2, nu, at(2, 0), nu, at(2, 1), L);    // cd
      loop_mul(S3, S0, S2, N, L);                        // T1 = bl cd
      loop_two(q, S2, mu, at(0, 2), mu, at(1, 2), L);    // ml
      loop_mul(S4, S1, S2, N, L);                        // T2 = ld ml
      trace_dag_acc(S3, S4, N, L, a22);
      // 2x4, upper: bl cd cu (ld lu tl)^dag
      loop_two(q, S2, nu, at(2, 2), nu, at(2, 3), L);    // cu
      loop_mul(S5, S3, S2, N, L);
      loop_two(q, S2, nu, at(0, 2), nu, at(0, 3), L);    // lu
      loop_mul(S6, S1, S2, N, L);
      loop_two(q, S2, mu, at(0, 4), mu, at(1, 4), L);    // tl
      loop_mul(S7, S6, S2, N, L);                        // ld lu tl
      trace_dag_acc(S5, S7, N, L, a42);
      // 2x4, right: bl br rd (ld ml mr)^dag
      loop_two(q, S2, mu, at(2, 0), mu, at(3, 0), L);    // br
      loop_mul(S3, S0, S2, N, L);
      loop_two(q, S2, nu, at(4, 0), nu, at(4, 1), L);    // rd
      loop_mul(S5, S3, S2, N, L);                        // bl br rd
      loop_two(q, S2, mu, at(2, 2), mu, at(3, 2), L);    // mr
      loop_mul(S6, S4, S2, N, L);                        // T2 mr
      trace_dag_acc(S5, S6, N, L, a42);
      // 4x4: bl br rd ru (ld lu tl tr)^dag
      loop_two(q, S2, nu, at(4, 2), nu, at(4, 3), L);    // ru
      loop_mul(S3, S5, S2, N, L);
      loop_two(q, S2, mu, at(2, 4), mu, at(3, 4), L);    // tr
      loop_mul(S6, S7, S2, N, L);
      trace_dag_acc(S3, S6, N, L, a44);
      // 1x2, both orientations
      loop_mul_link(q, S3, S0, nu, at(2, 0), L);         // bl U_nu(b)
      loop_two(q, S2, nu, x, mu, at(0, 1), L);           // U_nu(x) U_mu(e)
      loop_mul_link(q, S5, S2, mu, at(1, 1), L);         // ... U_mu(d)
      trace_dag_acc(S3, S5, N, L, a21);
      loop_two(q, S2, mu, x, nu, at(1, 0), L);           // U_mu(x) U_nu(a)
      loop_mul_link(q, S3, S2, nu, at(1, 1), L);         // ... U_nu(d)
      loop_mul_link(q, S5, S1, mu, at(0, 2), L);         // ld U_mu(h)
      trace_dag_acc(S3, S5, N, L, a21);
    }
  }
  __syncthreads();
  const int ngroups = nw * LPW;
  for (int e = threadIdx.x; e < row; e += blockDim.x) {
    double2 sum = cz();
    for (int gi = 0; gi < ngroups; gi++)
      sum = cadd(sum, sm[(size_t)gi * gsz + (size_t)LOOP_SLOTS * SS + RING + e]);
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
