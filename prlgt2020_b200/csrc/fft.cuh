// fft.cuh -- the 4-D FFT of Fourier-accelerated gauge fixing (the reference
// calls FFTW for it: Quenched.cc:801-838, nspt.cc:879-897): 9N complex
// planes of V sites, one 1-D transform per line along each direction,
// unnormalised, exp(-2 pi i k x / n) forward (FFTW_FORWARD) and
// exp(+2 pi i k x / n) backward.
//
// One line (n points) is transformed in registers by a mixed-radix
// decimation-in-frequency FFT whose plan (radix 4, 2, 3 or 5 at each level,
// the largest first) is fixed at compile time: every element index, every
// butterfly and every twiddle position is a constant, so the line lives in
// registers.  A DIF leaves X[k] at the position whose mixed-radix digits are
// those of k reversed; dif_index() gives k for a position, and since it is a
// compile-time constant the reordering costs no instruction.  Twiddles
// w_n^t = exp(-2 pi i t / n) come from a per-direction table of the
// context's extents (computed on the host), conjugated for the backward
// transform.
//
// Passes and memory:
//   * direction t (stride 1): the lines of a CTA are one contiguous chunk,
//     staged through shared memory (coalesced in and out, each thread then
//     reads its own line at a padded pitch); the first forward pass computes
//     its input, the divergence sum_mu [log U_mu(x) - log U_mu(x - mu)]
//     (nspt.cc:871-877), on the fly instead of reading a stored field;
//   * directions z, y: one thread per line, consecutive threads on
//     consecutive sites, so every load and store is coalesced;
//   * direction x: the last forward and the first backward transform in one
//     kernel, with the momentum-space factor -alpha / p^2 (zero at p = 0,
//     nspt.cc:881-894) applied between them.
// Seven passes over the 9N planes instead of ten (divergence, four forward
// passes, the scaling, four backward passes).
#pragma once
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace nspt {

// ---------------- compile-time plan ----------------
__host__ __device__ constexpr int fft_radix(int L) {
  return L % 4 == 0 ? 4 : L % 2 == 0 ? 2 : L % 3 == 0 ? 3 : L % 5 == 0 ? 5 : L;
}
__host__ __device__ constexpr bool fft_plannable(int L) {
  while (L > 1) {
    const int r = fft_radix(L);
    if (r > 5) return false;
    L /= r;
  }
  return true;
}
// frequency index held at position p after the DIF of n points
__host__ __device__ constexpr int dif_index(int n, int p) {
  int k = 0, mul = 1, L = n;
  while (L > 1) {
    const int r = fft_radix(L), m = L / r;
    k += (p / m) * mul;
    p %= m;
    mul *= r;
    L = m;
  }
  return k;
}

// multiply by i*s (s = +1 or -1)
__device__ __forceinline__ double2 fft_mul_is(double2 a, double s) {
  return make_double2(-s * a.y, s * a.x);
}

// r-point DFT of x[0..r) in place, X_k = sum_q x_q exp(s 2 pi i k q / r)
template <int r>
__device__ __forceinline__ void fft_small(double2 (&x)[r], double s) {
  if constexpr (r == 2) {
    const double2 a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
  } else if constexpr (r == 4) {
    const double2 t0 = cadd(x[0], x[2]), t1 = csub(x[0], x[2]);
    const double2 t2 = cadd(x[1], x[3]), t3 = fft_mul_is(csub(x[1], x[3]), s);
    x[0] = cadd(t0, t2);
    x[2] = csub(t0, t2);
    x[1] = cadd(t1, t3);
    x[3] = csub(t1, t3);
  } else if constexpr (r == 3) {
    const double h = 0.86602540378443864676;  // sqrt(3) / 2
    const double2 a = x[0], t1 = cadd(x[1], x[2]);
    const double2 t2 = make_double2(a.x - 0.5 * t1.x, a.y - 0.5 * t1.y);
    const double2 t3 = fft_mul_is(cscale(csub(x[1], x[2]), h), s);
    x[0] = cadd(a, t1);
    x[1] = cadd(t2, t3);
    x[2] = csub(t2, t3);
  } else if constexpr (r == 5) {
    // cos(2 pi / 5), cos(4 pi / 5), sin(2 pi / 5), sin(4 pi / 5)
    const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
    const double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
    const double2 a = x[0];
    const double2 t1 = cadd(x[1], x[4]), t2 = cadd(x[2], x[3]);
    const double2 t3 = csub(x[1], x[4]), t4 = csub(x[2], x[3]);
    const double2 u1 = make_double2(a.x + c1 * t1.x + c2 * t2.x, a.y + c1 * t1.y + c2 * t2.y);
    const double2 u2 = make_double2(a.x + c2 * t1.x + c1 * t2.x, a.y + c2 * t1.y + c1 * t2.y);
    const double2 v1 = fft_mul_is(make_double2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y), s);
    const double2 v2 = fft_mul_is(make_double2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y), s);
    x[0] = cadd(a, cadd(t1, t2));
    x[1] = cadd(u1, v1);
    x[4] = csub(u1, v1);
    x[2] = cadd(u2, v2);
    x[3] = csub(u2, v2);
  }
}

// w_n^t for the transform's sign (table: exp(-2 pi i t / n))
__device__ __forceinline__ double2 fft_tw(const double2 *tw, int t, bool inv) {
  const double2 w = __ldg(tw + t);
  return inv ? make_double2(w.x, -w.y) : w;
}

// DIF on the block v[O .. O+L) of an n-point line
template <int n, int L, int O>
struct FftDif {
  static __device__ __forceinline__ void run(double2 (&v)[n], const double2 *tw, bool inv) {
    if constexpr (L > 1) {
      constexpr int r = fft_radix(L), m = L / r;
      const double s = inv ? 1.0 : -1.0;
#pragma unroll
      for (int j = 0; j < m; j++) {
        double2 x[r];
#pragma unroll
        for (int q = 0; q < r; q++) x[q] = v[O + j + q * m];
        fft_small<r>(x, s);
#pragma unroll
        for (int q = 1; q < r; q++)
          if (j * q) x[q] = cmul(x[q], fft_tw(tw, ((j * q) * (n / L)) % n, inv));
#pragma unroll
        for (int q = 0; q < r; q++) v[O + j + q * m] = x[q];
      }
      Sub<r, m, 0>::run(v, tw, inv);
    }
  }
  template <int r, int m, int q>
  struct Sub {
    static __device__ __forceinline__ void run(double2 (&v)[n], const double2 *tw, bool inv) {
      if constexpr (q < r) {
        FftDif<n, m, O + q * m>::run(v, tw, inv);
        Sub<r, m, q + 1>::run(v, tw, inv);
      }
    }
  };
};

// o[dif_index(n, p)] = v[p] for every p, the indices as template constants
template <int n, int p>
struct FftReorder {
  static constexpr int k = dif_index(n, p);
  static __device__ __forceinline__ void run(double2 (&o)[n], const double2 (&v)[n]) {
    if constexpr (p < n) {
      o[k] = v[p];
      FftReorder<n, p + 1>::run(o, v);
    }
  }
};

// v (natural order) -> its DFT (natural order)
template <int n>
__device__ __forceinline__ void fft_line(double2 (&v)[n], const double2 *tw, bool inv) {
  FftDif<n, n, 0>::run(v, tw, inv);
  double2 o[n];
  FftReorder<n, 0>::run(o, v);
#pragma unroll
  for (int k = 0; k < n; k++) v[k] = o[k];
}

// ---------------- passes ----------------

// Direction with site stride st > 1 (x, y, z): one thread per line, lines
// numbered (plane, outer, inner) with inner in [0, st) fastest.
template <int n>
__global__ void __launch_bounds__(128) k_fft_strided(double2 *data, long nlines, int st, size_t V,
                                                     const double2 *tw, int inv) {
  const long id = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (id >= nlines) return;
  const long per_plane = (long)V / n;
  const long p = id / per_plane, rem = id - p * per_plane;
  const long outer = rem / st, inner = rem - outer * st;
  double2 *b = data + (size_t)p * V + (size_t)outer * n * st + inner;
  double2 v[n];
#pragma unroll
  for (int i = 0; i < n; i++) v[i] = b[(size_t)i * st];
  fft_line<n>(v, tw, inv != 0);
#pragma unroll
  for (int i = 0; i < n; i++) b[(size_t)i * st] = v[i];
}

// Direction t (stride 1): the CTA's T lines are the contiguous elements
// [g0 n, (g0 + T) n) of the planes, staged through shared memory at pitch
// n | 1 (odd, so that the 8 lanes of a quarter-warp reading their lines'
// element k hit distinct 16-byte bank groups).  DIV: the input is the
// divergence of the per-link logs Lg (planes mu*9N + e), not data.
template <int n, bool DIV>
__global__ void __launch_bounds__(128) k_fft_t(double2 *data, const double2 *__restrict__ Lg,
                                               long nlines, int N9, Geo geo, const double2 *tw,
                                               int inv) {
  constexpr int T = 128, PITCH = n | 1;
  extern __shared__ double2 sh[];
  const long g0 = (long)blockIdx.x * T;
  const int lines = (int)min((long)T, nlines - g0);
  const size_t e0 = (size_t)g0 * n;
  const size_t V = (size_t)geo.V;
  for (int x = threadIdx.x; x < lines * n; x += T) {
    const size_t E = e0 + x;
    double2 val;
    if constexpr (DIV) {
      const size_t e = E / V;
      const int site = (int)(E - e * V);
      int c[4];
      coords(geo, site, c);
      val = cz();
#pragma unroll
      for (int mu = 0; mu < 4; mu++) {
        const Nb b = neighbour(geo, c, mu, -1, 0, 0);
        const double2 *pl = Lg + ((size_t)mu * N9 + e) * V;
        val = cadd(val, csub(__ldg(pl + site), __ldg(pl + b.site)));
      }
    } else {
      val = data[E];
    }
    sh[(x / n) * PITCH + (x % n)] = val;
  }
  __syncthreads();
  if (threadIdx.x < lines) {
    double2 v[n];
    double2 *row = sh + threadIdx.x * PITCH;
#pragma unroll
    for (int i = 0; i < n; i++) v[i] = row[i];
    fft_line<n>(v, tw, inv != 0);
#pragma unroll
    for (int i = 0; i < n; i++) row[i] = v[i];
  }
  __syncthreads();
  for (int x = threadIdx.x; x < lines * n; x += T) data[e0 + x] = sh[(x / n) * PITCH + (x % n)];
}

// Direction x (stride V / L0): forward transform, times -alpha / p^2 of the
// element's momentum (zero at p = 0; p2: p2hat[4][128], lattice.h:1144-1169),
// backward transform, in one pass.
template <int n>
__global__ void __launch_bounds__(128) k_fft_x_scale(double2 *data, long nlines, Geo geo,
                                                     const double2 *tw, double alpha,
                                                     const double *__restrict__ p2) {
  const long id = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (id >= nlines) return;
  const size_t V = (size_t)geo.V;
  const long st = (long)V / n;
  const long p = id / st, inner = id - p * st;
  double2 *b = data + (size_t)p * V + inner;
  int c[4];
  coords(geo, (int)inner, c);
  const double q1 = __ldg(p2 + 128 + c[1]), q2 = __ldg(p2 + 256 + c[2]), q3 = __ldg(p2 + 384 + c[3]);
  const bool zero_rest = c[1] == 0 && c[2] == 0 && c[3] == 0;
  double2 v[n];
#pragma unroll
  for (int i = 0; i < n; i++) v[i] = b[(size_t)i * st];
  fft_line<n>(v, tw, false);
#pragma unroll
  for (int k = 0; k < n; k++) {
    const double f = (zero_rest && k == 0) ? 0.0 : -(alpha / (__ldg(p2 + k) + q1 + q2 + q3));
    v[k] = cscale(v[k], f);
  }
  fft_line<n>(v, tw, true);
#pragma unroll
  for (int i = 0; i < n; i++) b[(size_t)i * st] = v[i];
}

}  // namespace nspt
