// series.cuh -- device arithmetic on truncated power series of 3x3 complex
// matrices (the reference's ptSU3, QCDpt.h:42-226), FP64.
//
// Shared-memory "slot" of one series, 1 + 9*N double2, COLUMN major inside
// each order:
//   slot[0]                     flag (order-0 coefficient times the identity)
//   slot[1 + 9*(k-1) + 3*c + r] order k, row r, column c        (k = 1..N)
// Global link planes (kernels.cuh) are row major: element (k, r, c) of link
// (mu, site) at  U[((mu*9N + 9(k-1) + 3r + c) * V + site].
//
// Work split of one series product C = A * B.  A "link group" of 9 lanes
// owns one series computation.  Lane (c, s), c, s in {0,1,2}, owns column c
// of the result orders k = s+1, s+4, s+7, ... (all orders of the column
// between the three lanes of that column).  Since C_k[:,c] = sum_i A_i
// B_{k-i}[:,c], the lane needs the whole left operand A and column c of the
// right operand B:
//   * every lane of the group walks the same i, so each left coefficient A_i
//     (9 complex) is one broadcast read for the group -- straight from the
//     global planes (L1/L2, prefetched one order ahead) or from a slot;
//   * each right column B_j[:,c] (3 complex, one 48-byte column of the slot)
//     feeds 9 complex FMAs.  A 128-bit shared load is served a quarter-warp
//     (8 lanes) at a time, and lane (c, s) of a group reads quad
//     (j + 3c + r + base) mod 8 of the 8 16-byte bank quads, the 9 lanes of
//     a group on 9 consecutive quads.  With the slot stride = 3 (mod 8)
//     quads, the group stride of a 3-slot kernel is = 1 (mod 8): the next
//     group continues the sequence, and every quarter-warp's 8 lanes land
//     on 8 distinct quads (4 wavefronts a load; with a slot stride = 1 the
//     quarters that straddle two groups take 5.2 on average).
// Accumulators of up to 3*MO orders per pass stay in registers; passes run
// from high to low order and every lane finishes reading a pass before any
// lane writes it, so a result may overwrite either operand in place.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace nspt {

__device__ __forceinline__ double2 cz() { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.y * b.x + a.x * b.y);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double x) {
  return make_double2(a.x * x, a.y * x);
}
__device__ __forceinline__ bool cis0(double2 a) { return a.x == 0.0 && a.y == 0.0; }
// acc += a * b  (4 FP64 FMAs)
__device__ __forceinline__ void cfma(double2 &acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// flag of a product: a0*b0, or an exact 0 when both are 0 (QCDpt.h:102-104)
__device__ __forceinline__ double2 flag_mul(double2 a0, double2 b0) {
  return (cis0(a0) && cis0(b0)) ? cz() : cmul(a0, b0);
}

// slot index of (order k, row r, column c)
__device__ __forceinline__ int sidx(int k, int r, int c) { return 1 + 9 * (k - 1) + 3 * c + r; }

// Twist matrices Omega_d and Omega_d^dag (twistmatrices.h:158-240).
__constant__ double2 c_om[4][9];
__constant__ double2 c_omd[4][9];

// 3x3 complex product r = a * b, row major (SU3::operator*, MyMath.h:791-849).
__device__ __forceinline__ void m3_mul(double2 *r, const double2 *a, const double2 *b) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int q = 0; q < 3; q++) {
      double2 t = cmul(a[3 * i], b[q]);
      t = cadd(t, cmul(a[3 * i + 1], b[3 + q]));
      t = cadd(t, cmul(a[3 * i + 2], b[6 + q]));
      r[3 * i + q] = t;
    }
}

// Omega U Omega^dag for every twisted face a read crossed: backward wraps
// first (Omega_d^dag U Omega_d), then forward wraps, as the reference's
// backward copy slabs hold them (lattice.h:733-790, nspt.cc:221-253).
// m is row major.
__device__ __forceinline__ void twist3(double2 *m, unsigned tb, unsigned tf) {
  double2 t[9];
#pragma unroll
  for (int d = 1; d < 4; d++)
    if ((tb >> d) & 1) {
      m3_mul(t, c_omd[d], m);
      m3_mul(m, t, c_om[d]);
    }
#pragma unroll
  for (int d = 1; d < 4; d++)
    if ((tf >> d) & 1) {
      m3_mul(t, c_om[d], m);
      m3_mul(m, t, c_omd[d]);
    }
}

// Identity of a lane inside its 9-lane link group.
struct Lane {
  int c;          // owned column
  int s;          // owned residue: orders k = s+1 (mod 3)
  int j;          // 3*c + s, 0..8
  unsigned mask;  // the group's lanes
};

__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Left operand in a slot (column major).
struct LeftS {
  const double2 *s;
  template <bool DAG>
  __device__ __forceinline__ void load(int k, double2 *a) const {
    const double2 *q = s + 1 + 9 * (k - 1);
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int l = 0; l < 3; l++) a[3 * r + l] = DAG ? cconj(q[3 * r + l]) : q[3 * l + r];
  }
  template <bool DAG>
  __device__ __forceinline__ void col(int k, int c, double2 *o) const {
#pragma unroll
    for (int r = 0; r < 3; r++) o[r] = DAG ? cconj(s[sidx(k, c, r)]) : s[sidx(k, r, c)];
  }
};

// C = op(A) * B, orders 1..M (truncated Cauchy product, ptSU3::operator*,
// QCDpt.h:92-114); op = dagger when DA.  a0 = flag of op(A), b0 = flag of B,
// supplied by the caller (the result's flag is the caller's business).
// emit(k, r, v) is called by the lane owning (k, column c) for r = 0..2.
// i0 > 1 skips left-operand orders below i0, for a caller whose left
// operand is exactly zero there (X^2 of a flag-0 series has no order 1).
template <int MO, bool DA, class Left, class Emit>
__device__ __forceinline__ void product(const Left &A, double2 a0, const double2 *B, double2 b0,
                                        int M, const Lane &L, Emit emit, int i0 = 1) {
  const int c = L.c;
  constexpr int PASS = 3 * MO;
  const int npass = (M + PASS - 1) / PASS;
  for (int ps = npass - 1; ps >= 0; --ps) {
    const int kb = ps * PASS;
    const int kend = min(kb + PASS, M);  // last order of the pass
    double2 acc[MO][3];
#pragma unroll
    for (int q = 0; q < MO; q++)
#pragma unroll
      for (int r = 0; r < 3; r++) acc[q][r] = cz();
    double2 a[9];
    for (int i = i0; i < kend; i++) {
      A.template load<DA>(i, a);
#pragma unroll
      for (int q = 0; q < MO; q++) {
        const int k = kb + L.s + 1 + 3 * q;
        if (k <= kend && k > i) {
          const double2 *bj = B + 1 + 9 * (k - i - 1) + 3 * c;
          const double2 b0_ = bj[0], b1 = bj[1], b2 = bj[2];
#pragma unroll
          for (int r = 0; r < 3; r++) {
            cfma(acc[q][r], a[3 * r], b0_);
            cfma(acc[q][r], a[3 * r + 1], b1);
            cfma(acc[q][r], a[3 * r + 2], b2);
          }
        }
      }
    }
    __syncwarp(L.mask);
    const bool fa = !cis0(a0), fb = !cis0(b0);
#pragma unroll
    for (int q = 0; q < MO; q++) {
      const int k = kb + L.s + 1 + 3 * q;
      if (k <= kend) {
        double2 ak[3];
        if (fb) A.template col<DA>(k, c, ak);
#pragma unroll
        for (int r = 0; r < 3; r++) {
          double2 v = acc[q][r];
          // b0*A_k + a0*B_k; a zero flag contributes an exact zero, so its
          // term is skipped (the operand may be unset there)
          if (fa || fb) {
            double2 u;
            if (!fa)
              u = cmul(b0, ak[r]);
            else if (!fb)
              u = cmul(a0, B[sidx(k, r, c)]);
            else
              u = cadd(cmul(b0, ak[r]), cmul(a0, B[sidx(k, r, c)]));
            v = cadd(v, u);
          }
          emit(k, r, v);
        }
      }
    }
    __syncwarp(L.mask);
  }
}

// ---------------- compensated float-float Cauchy product ----------------
//
// The same truncated product as product(), with every 3x3 multiply-add of
// the triangle in float-float arithmetic: a double x is split into
// hi = fl32(x 2^e) and lo = fl32(x 2^e - hi) (48 significant bits together);
// a product of two such numbers is formed with an exact FP32 product
// (p = xh yh, err = fma(xh, yh, -p)) plus the cross terms, and added to the
// accumulator by an error-free two-sum whose error is carried in the low
// word.  Order i of the left operand and order j of the right one are
// scaled by 2^(e i) and 2^(e j) before the split (exact), so that orders of
// very different size keep inside the FP32 exponent range; the order-k
// result is scaled back by 2^(-e k) when it is rejoined into FP64.  The flag
// terms, the output and everything around the products stay FP64.
struct ffc {
  float rh, rl, ih, il;  // re = rh + rl, im = ih + il
};

// 2^n as a double, exact for -1022 <= n <= 1023
__device__ __forceinline__ double pow2i(int n) { return __hiloint2double((1023 + n) << 20, 0); }

__device__ __forceinline__ ffc ff_split(double2 v, double scale) {
  const double x = v.x * scale, y = v.y * scale;
  const float xh = __double2float_rn(x), yh = __double2float_rn(y);
  return {xh, __double2float_rn(x - (double)xh), yh, __double2float_rn(y - (double)yh)};
}

// (ah, al) += (xh, xl) (yh, yl); rounding-explicit so nothing is contracted
__device__ __forceinline__ void ff_mac(float &ah, float &al, float xh, float xl, float yh,
                                       float yl) {
  const float p = __fmul_rn(xh, yh);
  float e = __fmaf_rn(xh, yh, -p);
  e = __fmaf_rn(xh, yl, e);
  e = __fmaf_rn(xl, yh, e);
  const float s = __fadd_rn(ah, p);
  const float b = __fsub_rn(s, ah);
  const float err = __fadd_rn(__fsub_rn(ah, __fsub_rn(s, b)), __fsub_rn(p, b));
  ah = s;
  al = __fadd_rn(al, __fadd_rn(err, e));
}

__device__ __forceinline__ void ff_cmac(ffc &acc, const ffc &a, const ffc &b) {
  ff_mac(acc.rh, acc.rl, a.rh, a.rl, b.rh, b.rl);
  ff_mac(acc.rh, acc.rl, -a.ih, -a.il, b.ih, b.il);
  ff_mac(acc.ih, acc.il, a.rh, a.rl, b.ih, b.il);
  ff_mac(acc.ih, acc.il, a.ih, a.il, b.rh, b.rl);
}

// product() with the triangle in float-float; e: per-order scale exponent,
// |e| * M <= 1022 (the caller clamps it).
template <int MO, bool DA, class Left, class Emit>
__device__ __forceinline__ void product_ff(const Left &A, double2 a0, const double2 *B, double2 b0,
                                           int M, const Lane &L, int e, Emit emit) {
  const int c = L.c;
  constexpr int PASS = 3 * MO;
  const int npass = (M + PASS - 1) / PASS;
  for (int ps = npass - 1; ps >= 0; --ps) {
    const int kb = ps * PASS;
    const int kend = min(kb + PASS, M);
    ffc acc[MO][3];
#pragma unroll
    for (int q = 0; q < MO; q++)
#pragma unroll
      for (int r = 0; r < 3; r++) acc[q][r] = {0.f, 0.f, 0.f, 0.f};
    double2 a[9];
    for (int i = 1; i < kend; i++) {
      A.template load<DA>(i, a);
      ffc af[9];
      const double sa = pow2i(e * i);
#pragma unroll
      for (int t = 0; t < 9; t++) af[t] = ff_split(a[t], sa);
#pragma unroll
      for (int q = 0; q < MO; q++) {
        const int k = kb + L.s + 1 + 3 * q;
        if (k <= kend && k > i) {
          const double2 *bj = B + 1 + 9 * (k - i - 1) + 3 * c;
          const double sb = pow2i(e * (k - i));
          const ffc b0_ = ff_split(bj[0], sb), b1 = ff_split(bj[1], sb), b2 = ff_split(bj[2], sb);
#pragma unroll
          for (int r = 0; r < 3; r++) {
            ff_cmac(acc[q][r], af[3 * r], b0_);
            ff_cmac(acc[q][r], af[3 * r + 1], b1);
            ff_cmac(acc[q][r], af[3 * r + 2], b2);
          }
        }
      }
    }
    __syncwarp(L.mask);
    const bool fa = !cis0(a0), fb = !cis0(b0);
#pragma unroll
    for (int q = 0; q < MO; q++) {
      const int k = kb + L.s + 1 + 3 * q;
      if (k <= kend) {
        double2 ak[3];
        if (fb) A.template col<DA>(k, c, ak);
        const double su = pow2i(-e * k);
#pragma unroll
        for (int r = 0; r < 3; r++) {
          const ffc &f = acc[q][r];
          double2 v = make_double2(((double)f.rh + (double)f.rl) * su,
                                   ((double)f.ih + (double)f.il) * su);
          if (fa || fb) {
            double2 u;
            if (!fa)
              u = cmul(b0, ak[r]);
            else if (!fb)
              u = cmul(a0, B[sidx(k, r, c)]);
            else
              u = cadd(cmul(b0, ak[r]), cmul(a0, B[sidx(k, r, c)]));
            v = cadd(v, u);
          }
          emit(k, r, v);
        }
      }
    }
    __syncwarp(L.mask);
  }
}

// Orders per lane and pass of the float-float product: its accumulators
// take as many registers as the FP64 ones, its split operands twice as many.
constexpr int MO_FF = 4;

// product() or product_ff(), chosen at compile time
template <bool FF, int MO, bool DA, class Left, class Emit>
__device__ __forceinline__ void cprod(const Left &A, double2 a0, const double2 *B, double2 b0,
                                      int M, const Lane &L, int e, Emit emit) {
  if constexpr (FF)
    product_ff<MO_FF, DA>(A, a0, B, b0, M, L, e, emit);
  else
    product<MO, DA>(A, a0, B, b0, M, L, emit);
}

// Polynomial p(X) = sum_{n<=N} coef(n) X^n of a series X with flag 0,
// truncated at order N, by Paterson-Stockmeyer with block 2.  Y = X^2 is
// formed once; then Horner in Y,
//   S_J = B_J,  S_j = Y S_{j+1} + B_j,  B_j = coef(2j) + coef(2j+1) X,
// with S_j needed only to order N - 2j (Y^j starts at order 2j).  X^n starts
// at order n, so this is the same truncated sum as Horner in X, with
// 1 + N/2 series products of sizes 2, 4, ..., N instead of N products of
// sizes 1..N (1354 instead of 2300 3x3 products at N = 24).  The last step
// goes to last(k, r, v) instead of S.  X, Y and S are slots.
template <int MO>
__device__ __forceinline__ void ser_square(const double2 *X, double2 *Y, int N, const Lane &L) {
  const int c = L.c;
  // Y = X X (order 1 comes out as an exact zero)
  product<MO, false>(LeftS{X}, cz(), X, cz(), N, L,
                     [&](int k, int r, double2 v) { Y[sidx(k, r, c)] = v; });
}

// The Horner part of ser_poly2, for a Y = X^2 already formed.
template <int MO, class Coef, class Last>
__device__ __forceinline__ void ser_horner2(const double2 *X, const double2 *Y, double2 *S, int N,
                                            const Lane &L, Coef coef, Last last) {
  const int c = L.c;
  const int J = N / 2;
  // S_J = coef(2J) + coef(2J+1) X to order N - 2J; higher orders zero (they
  // meet Y's zero order-1 coefficient and must be finite)
  {
    const double cx = coef(2 * J + 1);
    for (int k = L.s + 1; k <= N; k += 3) {
#pragma unroll
      for (int r = 0; r < 3; r++)
        S[sidx(k, r, c)] = k <= N - 2 * J ? cscale(X[sidx(k, r, c)], cx) : cz();
    }
    if (L.j == 0) S[0] = make_double2(coef(2 * J), 0.0);
    __syncwarp(L.mask);
  }
  if (J == 0) {  // N = 1: S_0 is the result
    for (int k = L.s + 1; k <= N; k += 3) {
#pragma unroll
      for (int r = 0; r < 3; r++) last(k, r, S[sidx(k, r, c)]);
    }
    __syncwarp(L.mask);
    return;
  }
  // Y = X^2 has no order 1 (X has flag 0): the products start at Y's order 2
  const LeftS Yl{Y};
  for (int j = J - 1; j >= 0; --j) {
    const int M = N - 2 * j;
    const double2 sf = S[0];
    const double cx = coef(2 * j + 1);
    if (j > 0) {
      product<MO, false>(
          Yl, cz(), S, sf, M, L,
          [&](int k, int r, double2 v) { S[sidx(k, r, c)] = cadd(v, cscale(X[sidx(k, r, c)], cx)); },
          2);
      if (L.j == 0) S[0] = make_double2(coef(2 * j), 0.0);
      __syncwarp(L.mask);
    } else {
      product<MO, false>(
          Yl, cz(), S, sf, M, L,
          [&](int k, int r, double2 v) { last(k, r, cadd(v, cscale(X[sidx(k, r, c)], cx))); }, 2);
    }
  }
}

template <int MO, class Coef, class Last>
__device__ __forceinline__ void ser_poly2(const double2 *X, double2 *Y, double2 *S, int N,
                                          const Lane &L, Coef coef, Last last) {
  ser_square<MO>(X, Y, N, L);
  ser_horner2<MO>(X, Y, S, N, L, coef, last);
}

__device__ __forceinline__ double inv_factorial(int n) {
  double f = 1.0;
  for (int m = 2; m <= n; m++) f *= (double)m;
  return 1.0 / f;
}

// R = exp(P) for P with flag 0 (exp(const ptSU3&), QCDpt.h:200-220):
// sum_{n<=N} P^n / n!, flag 1.  P, Y (scratch) and R are slots.
template <int MO>
__device__ __forceinline__ void ser_exp(const double2 *P, double2 *Y, double2 *R, int N,
                                        const Lane &L) {
  const int c = L.c;
  ser_poly2<MO>(P, Y, R, N, L, [](int n) { return inv_factorial(n); },
                [&](int k, int r, double2 v) { R[sidx(k, r, c)] = v; });
  if (L.j == 0) R[0] = make_double2(1.0, 0.0);
  __syncwarp(L.mask);
}

// log(U) for U with flag 1 (log(const ptSU3&), QCDpt.h:176-198): with
// X = U - 1, sum_{n<=N} (-1)^{n+1} X^n / n, flag 0.  U, Y and Sc are slots
// (Y, Sc scratch); emit(k, r, v) receives log_k[r][c].
template <int MO, class Emit>
__device__ __forceinline__ void ser_log(const double2 *U, double2 *Y, double2 *Sc, int N,
                                        const Lane &L, Emit emit) {
  ser_poly2<MO>(U, Y, Sc, N, L,
                [](int n) { return n == 0 ? 0.0 : ((n & 1) ? 1.0 : -1.0) / (double)n; }, emit);
}

// reH on a slot (ptSU3::reH, QCDpt.cc:197-209): per order (M - M^dag)/2
// minus a third of the trace times 1; flag 0.  The formula is the same for
// row- and column-major storage.  Lanes split the orders.
__device__ __forceinline__ void ser_reH(double2 *P, int N, const Lane &L) {
  const double D3 = 1.0 / 3.0;
  for (int k = 1 + L.j; k <= N; k += 9) {
    double2 *m = P + 1 + 9 * (k - 1);
    double2 a[9];
#pragma unroll
    for (int e = 0; e < 9; e++) a[e] = m[e];
    double2 b[9];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int q = 0; q < 3; q++) {
        double2 d = csub(a[3 * r + q], cconj(a[3 * q + r]));
        b[3 * r + q] = make_double2(.5 * d.x, .5 * d.y);
      }
    double2 tr = cadd(cadd(b[0], b[4]), b[8]);
    tr = make_double2(tr.x * D3, D3 * tr.y);
    b[0] = csub(b[0], tr);
    b[4] = csub(b[4], tr);
    b[8] = csub(b[8], tr);
#pragma unroll
    for (int e = 0; e < 9; e++) m[e] = b[e];
  }
  if (L.j == 0) P[0] = cz();
}

}  // namespace nspt
