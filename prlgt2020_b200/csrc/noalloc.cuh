// Allocation-free static plaquette of a caller-owned device field.
//
// Same quantity as nspt_plaquette_measure (plaquette_measure, OpenMP
// branch, nspt.cc:1362-1404: sum over links of Tr(U_mu(x) * staples) / 72V
// per order) computed without a context.  The field is read where the caller
// keeps it -- the reference's AoS layout (ptGluon_fld, QCDenvNODEpt_test.h:
// 331-338) in device memory -- and the only scratch is a fixed, file-scope
// device array: one row of per-order partial sums per CTA plus one result
// row.  Nothing is allocated, on the device or the host.
//
// Scratch contents: every call writes each partial row it later reads and
// the result row before reading them, so nothing in the array has to start
// at zero and stale contents from an earlier call are never used.  Two calls
// that overlap on one device (different host threads or streams) share the
// array and race; callers serialise them.
#pragma once

#include <mutex>

namespace nspt {

constexpr int NOALLOC_BLOCKS = 1024;               // partial rows (max CTAs per call)
constexpr int NOALLOC_ROW = NSPT_MAX_ORDER + 1;    // orders 0..NSPT_MAX_ORDER
constexpr int NOALLOC_MAX_DEVICES = 64;
// (NOALLOC_BLOCKS + 1) rows of NOALLOC_ROW complex doubles: 803,600 bytes
static __device__ __align__(256) double2 g_noalloc_scratch[(NOALLOC_BLOCKS + 1) * NOALLOC_ROW];

struct AosField {
  const double2 *p;  // V * 4 series of 1 + 9A complex doubles (site, mu)
  int A;             // allocORD of the caller's layout (>= N)
  int N;
  int SS;
  Geo g;
};

// Copy link (mu, n.site) of an AoS field into a column-major slot (DAG:
// its dagger), applying the twists of the faces the read crossed; a twisted
// link gets flag 1 (nspt.cc:115-121).
__device__ __forceinline__ void stage_aos(double2 *slot, const AosField &f, int mu, Nb n,
                                          const Lane &L, bool dag = false) {
  const double2 *src = f.p + ((size_t)n.site * 4 + mu) * (1 + 9 * (size_t)f.A);
  const unsigned tb = n.bwd & f.g.twist, tf = n.fwd & f.g.twist;
  if (!(tb | tf)) {
    const int r = L.j / 3, c = L.j - 3 * (L.j / 3);
    const int off = dag ? 3 * r + c : 3 * c + r;
    for (int k = 1; k <= f.N; k++) {
      const double2 v = __ldg(src + 1 + 9 * (k - 1) + L.j);
      slot[1 + 9 * (k - 1) + off] = dag ? cconj(v) : v;
    }
    if (L.j == 0) {
      const double2 fl = __ldg(src);
      slot[0] = dag ? cconj(fl) : fl;
    }
  } else {
    for (int k = 1 + L.j; k <= f.N; k += GROUP) {
      double2 m[9];
#pragma unroll
      for (int e = 0; e < 9; e++) m[e] = __ldg(src + 1 + 9 * (k - 1) + e);
      twist3(m, tb, tf);
      double2 *p = slot + 1 + 9 * (k - 1);
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) p[dag ? 3 * r + c : 3 * c + r] = dag ? cconj(m[3 * r + c]) : m[3 * r + c];
    }
    if (L.j == 0) slot[0] = make_double2(1.0, 0.0);
  }
  __syncwarp(L.mask);
}

// Per-CTA partial sums of Tr(U_mu(x) * staples) per order.  Groups walk the
// links grid-stride; each lane keeps the orders k = 1 + j (mod 9) it owns in
// registers; the CTA sums its groups in a fixed order into partial[blockIdx].
constexpr int NOALLOC_PER_LANE = (NSPT_MAX_ORDER + GROUP - 1) / GROUP;

__global__ void __launch_bounds__(256, 1) k_plaq_noalloc(AosField f, double2 *partial) {
  extern __shared__ double2 sm[];
  Lane L;
  int g;
  const bool grouped = make_lane(L, g);
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int N = f.N, SS = f.SS;
  double2 acc[NOALLOC_PER_LANE];
#pragma unroll
  for (int q = 0; q < NOALLOC_PER_LANE; q++) acc[q] = cz();
  double2 acc0 = cz();
  if (grouped) {
    const int c = L.c;
    double2 *W = sm + (size_t)(warp * LPW + g) * (3 * SS), *T = W + SS, *Y = T + SS;
    const long nl = 4L * f.g.V;
    const long stride = (long)gridDim.x * nw * LPW;
    for (long link = ((long)blockIdx.x * nw + warp) * LPW + g; link < nl; link += stride) {
      const int mu = (int)(link / f.g.V);
      const int site = (int)(link - (long)mu * f.g.V);
      int x[4];
      coords(f.g, site, x);
      Nb self;
      self.site = site;
      self.fwd = self.bwd = 0;
      double2 wflag = cz();
      bool first = true;
      for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        // upper staple, as the dagger of U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag
        // (QCDenvNODEpt_test.h:555), accumulated transposed and conjugated
        {
          stage_aos(T, f, nu, self, L);
          stage_aos(Y, f, mu, neighbour(f.g, x, nu, 1), L);
          const double2 t0 = T[0], y0 = Y[0];
          product<MO, false>(LeftS{T}, t0, Y, y0, N, L,
                             [&](int k, int r, double2 v) { T[sidx(k, r, c)] = v; });
          if (L.j == 0) T[0] = flag_mul(t0, y0);
          __syncwarp(L.mask);
          stage_aos(Y, f, nu, neighbour(f.g, x, mu, 1), L, true);
          const double2 a0 = T[0], b0 = Y[0];
          const bool f0 = first;
          product<MO, false>(LeftS{T}, a0, Y, b0, N, L, [&](int k, int r, double2 v) {
            double2 &w = W[sidx(k, c, r)];
            w = f0 ? cconj(v) : cadd(w, cconj(v));
          });
          const double2 fl = cconj(flag_mul(a0, b0));
          wflag = first ? fl : cadd(wflag, fl);
          first = false;
          __syncwarp(L.mask);
        }
        // lower staple [U_mu(x-nu) U_nu(x-nu+mu)]^dag U_nu(x-nu) (QCDenvNODEpt_test.h:556)
        {
          const Nb d = neighbour(f.g, x, nu, -1);
          stage_aos(Y, f, nu, neighbour(f.g, x, nu, -1, mu, 1), L);
          stage_aos(T, f, mu, d, L);
          const double2 a0 = T[0], y0 = Y[0];
          product<MO, false>(LeftS{T}, a0, Y, y0, N, L,
                             [&](int k, int r, double2 v) { T[sidx(k, r, c)] = v; });
          if (L.j == 0) T[0] = flag_mul(a0, y0);
          __syncwarp(L.mask);
          stage_aos(Y, f, nu, d, L);
          const double2 ta = cconj(T[0]);
          product<MO, true>(LeftS{T}, ta, Y, Y[0], N, L, [&](int k, int r, double2 v) {
            double2 &w = W[sidx(k, r, c)];
            w = cadd(w, v);
          });
          wflag = cadd(wflag, flag_mul(ta, Y[0]));
          __syncwarp(L.mask);
        }
      }
      if (L.j == 0) W[0] = wflag;
      // Tr(U_mu(x) * staples) per order (ptSU3::Tr, QCDpt.cc:115-122)
      stage_aos(Y, f, mu, self, L);
      const double2 pflag = flag_mul(Y[0], wflag);
      product<MO, false>(LeftS{Y}, Y[0], W, wflag, N, L,
                         [&](int k, int r, double2 v) { T[sidx(k, r, c)] = v; });
      __syncwarp(L.mask);
      if (L.j == 0) acc0 = cadd(acc0, make_double2(3. * pflag.x, 3. * pflag.y));
#pragma unroll
      for (int q = 0; q < NOALLOC_PER_LANE; q++) {
        const int k = 1 + L.j + GROUP * q;
        if (k <= N)
          acc[q] = cadd(acc[q], cadd(cadd(T[sidx(k, 0, 0)], T[sidx(k, 1, 1)]), T[sidx(k, 2, 2)]));
      }
      __syncwarp(L.mask);
    }
  }
  // CTA reduction in a fixed order over the groups (the slots are free now)
  __syncthreads();
  const int ngroups = nw * LPW;
  double2 *red = sm;  // [ngroups][N + 1]
  if (grouped) {
    double2 *row = red + (size_t)(warp * LPW + g) * (N + 1);
    if (L.j == 0) row[0] = acc0;
#pragma unroll
    for (int q = 0; q < NOALLOC_PER_LANE; q++) {
      const int k = 1 + L.j + GROUP * q;
      if (k <= N) row[k] = acc[q];
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k <= N; k += blockDim.x) {
    double2 s = cz();
    for (int gi = 0; gi < ngroups; gi++) s = cadd(s, red[(size_t)gi * (N + 1) + k]);
    partial[(size_t)blockIdx.x * NOALLOC_ROW + k] = s;
  }
}

// Sum the CTAs' partial rows in block order into the result row.
__global__ void k_plaq_noalloc_sum(const double2 *partial, int nblocks, int N, double2 *out) {
  for (int k = threadIdx.x; k <= N; k += blockDim.x) {
    double2 s = cz();
    for (int b = 0; b < nblocks; b++) s = cadd(s, partial[(size_t)b * NOALLOC_ROW + k]);
    out[k] = s;
  }
}

}  // namespace nspt

namespace {

// Per-device set-up, done once with that device current: the scratch
// array's address, the launch limits and the twist matrices.  It is kept
// until the process exits; a cudaDeviceReset after the first call reloads
// the module and leaves these values stale, which the header documents as
// unsupported.
struct NoallocDevice {
  bool ready;
  double2 *scratch;
  int nsm;
  int smem_optin;
};
NoallocDevice g_noalloc_dev[nspt::NOALLOC_MAX_DEVICES];
std::mutex g_noalloc_mu;

int noalloc_setup(int dev, NoallocDevice **out) {
  using namespace nspt;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoallocDevice &d = g_noalloc_dev[dev];
  if (!d.ready) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return NSPT_ERR_CUDA;
    if (!p || (reinterpret_cast<uintptr_t>(p) & 255u)) return NSPT_ERR_CUDA;
    if (cudaDeviceGetAttribute(&d.nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return NSPT_ERR_CUDA;
    if (cudaDeviceGetAttribute(&d.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
        cudaSuccess)
      return NSPT_ERR_CUDA;
    if (cudaFuncSetAttribute(k_plaq_noalloc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             d.smem_optin) != cudaSuccess)
      return NSPT_ERR_CUDA;
    // twist matrices (twistmatrices.h:158-240), the values nspt_create uploads
    double2 om[4][9], omd[4][9];
    for (int a = 0; a < 4; a++)
      for (int e = 0; e < 9; e++) om[a][e] = make_double2(0.0, 0.0);
    for (int a = 0; a < 2; a++)
      for (int e = 0; e < 9; e += 4) om[a][e] = make_double2(1.0, 0.0);
    om[1][0] = make_double2(cos(-2. * M_PI / 3.), sin(-2. * M_PI / 3.));
    om[1][8] = make_double2(cos(2. * M_PI / 3.), sin(2. * M_PI / 3.));
    om[2][1] = om[2][5] = om[2][6] = make_double2(1.0, 0.0);
    om[3][1] = make_double2(cos(-2. * M_PI / 3.), sin(-2. * M_PI / 3.));
    om[3][5] = make_double2(1.0, 0.0);
    om[3][6] = make_double2(cos(2. * M_PI / 3.), sin(2. * M_PI / 3.));
    for (int a = 0; a < 4; a++)
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
          omd[a][3 * i + j] = make_double2(om[a][3 * j + i].x, -om[a][3 * j + i].y);
    if (cudaMemcpyToSymbol(c_om, om, sizeof(om)) != cudaSuccess) return NSPT_ERR_CUDA;
    if (cudaMemcpyToSymbol(c_omd, omd, sizeof(omd)) != cudaSuccess) return NSPT_ERR_CUDA;
    d.scratch = static_cast<double2 *>(p);
    d.ready = true;
  }
  *out = &d;
  return NSPT_OK;
}

}  // namespace

extern "C" int nspt_plaquette_measure_noalloc(const void *links_dev, int allocORD, const int L[4],
                                              int N, unsigned flags, double *plaq, void *stream) {
  using namespace nspt;
  if (!links_dev || !L || !plaq) return NSPT_ERR_ARG;
  if (N < 1 || N > NSPT_MAX_ORDER) return NSPT_ERR_ORDER;  // beyond the scratch rows
  if (allocORD < N) return NSPT_ERR_ARG;
  if (flags & ~(NSPT_TWIST_Y | NSPT_TWIST_Z | NSPT_TWIST_T)) return NSPT_ERR_ARG;
  if (reinterpret_cast<uintptr_t>(links_dev) & 15u) return NSPT_ERR_ARG;
  long V = 1;
  for (int d = 0; d < 4; d++) {
    if (L[d] < 1) return NSPT_ERR_ARG;
    V *= L[d];
  }
  if (V > (1L << 29)) return NSPT_ERR_ARG;  // 4V links index an int site range
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return NSPT_ERR_NODEVICE;
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return NSPT_ERR_ARG;
  NoallocDevice *d = nullptr;
  int rc = noalloc_setup(dev, &d);
  if (rc) return rc;

  AosField f;
  f.p = static_cast<const double2 *>(links_dev);
  f.A = allocORD;
  f.N = N;
  f.SS = 1 + 9 * N;
  while (f.SS % 8 != 3) f.SS++;  // bank quads: see series.cuh
  Geo &g = f.g;
  for (int k = 0; k < 4; k++) g.L[k] = L[k];
  g.s2 = L[3];
  g.s1 = L[2] * g.s2;
  g.s0 = L[1] * g.s1;
  g.V = (int)V;
  g.t0 = g.t1 = 1;
  g.t2 = L[2];
  g.twist = 0;
  if (flags & NSPT_TWIST_Y) g.twist |= 2u;
  if (flags & NSPT_TWIST_Z) g.twist |= 4u;
  if (flags & NSPT_TWIST_T) g.twist |= 8u;

  // 3 slots per group; as many warps (<= 8) as shared memory allows
  const size_t per_warp = (size_t)LPW * 3 * f.SS * sizeof(double2);
  const int warps = (int)std::min<size_t>(8, (size_t)d->smem_optin / per_warp);
  if (warps < 1) return NSPT_ERR_ORDER;
  const size_t smem = std::max((size_t)warps * per_warp,
                               (size_t)warps * LPW * (N + 1) * sizeof(double2));
  if (smem > (size_t)d->smem_optin) return NSPT_ERR_ORDER;
  const long groups = 4 * V;
  const long per_cta = (long)warps * LPW;
  const long want = (groups + per_cta - 1) / per_cta;
  const int blocks = (int)std::min<long>(want, NOALLOC_BLOCKS);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double2 *partial = d->scratch;
  double2 *result = d->scratch + (size_t)NOALLOC_BLOCKS * NOALLOC_ROW;
  k_plaq_noalloc<<<blocks, 32 * warps, smem, st>>>(f, partial);
  if (cudaGetLastError() != cudaSuccess) return NSPT_ERR_CUDA;
  k_plaq_noalloc_sum<<<1, 64, 0, st>>>(partial, blocks, N, result);
  if (cudaGetLastError() != cudaSuccess) return NSPT_ERR_CUDA;
  if (cudaMemcpyAsync(plaq, result, (size_t)(N + 1) * sizeof(double2), cudaMemcpyDeviceToHost,
                      st) != cudaSuccess)
    return NSPT_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return NSPT_ERR_CUDA;
  for (int k = 0; k <= N; k++) {  // nspt.cc:1398-1404
    plaq[2 * k] /= (double)(V * 72);
    plaq[2 * k + 1] /= (double)(V * 72);
  }
  return NSPT_OK;
}
