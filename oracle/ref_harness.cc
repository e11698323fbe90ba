/*
 * TEST INFRASTRUCTURE (oracle).  Driver for the reference's own NSPT code.
 *
 * This file is project-written.  It is compiled together with the UNMODIFIED
 * reference translation units (nspt.cc, QCDpt.cc, MyMath.cc, MyRand.cc,
 * MyQCD.cc, ranlxd/ranlxd.cc) by oracle/ref.mk, with a choices.h derived from
 * the reference's choices.h (allocORD = PTORD, Jacobi update, boundary
 * conditions and OpenMP thread grid set per build variant).  It replaces the
 * reference's `main` (Quenched.cc:760-873) and defines the globals that
 * nspt.cc:37-94 declares extern (the reference defines them in
 * Quenched.cc:42-81).
 *
 * What it does mirrors Quenched.cc: initialise the lattice and the field
 * (cold start as Quenched.cc:596-603, or a configuration file in the
 * reference's binary format as Quenched.cc:605-630), set tau_g / stau as
 * QuenchedAllocate (Quenched.cc:584-589), seed MyRand as Quenched.cc:296-299,
 * then call NsptEvolve (nspt.cc:953-1039) once per step.  The reference's
 * per-step output files (plaquette, norm, trU; nspt.cc:570-597) are opened
 * with 17 significant digits so that parity checks can read them.
 *
 * Extra options, none of which changes the reference's arithmetic:
 *   --noise FILE   replay second MyRands with the same seeds and dump the
 *                  8 Gaussians SU3rand draws per link (MyMath.cc:256-292),
 *                  by link (site lexicographic, mu inner) -- one record of
 *                  V*4*8 doubles per step.  Thread tid of an OpenMP build
 *                  draws from Rand[tid] for the sites of its block, in the
 *                  block's lexicographic order with mu inner (nspt.cc:
 *                  355-440); with one thread that is the lattice's order;
 *   --twist-init   refresh the twisted copy sites once after a file start
 *                  (Quenched.cc does not; the copies would otherwise hold the
 *                  identity for the first step);
 *   --lower LO     the --start file holds LO <= allocORD orders: load it with
 *                  the reference's ptGluon_fld::loadlowerorder
 *                  (QCDenvNODEpt_test.h:376-426) after a cold start;
 *   --project      apply the reference's unitarisation U = exp(reH(log U))
 *                  (QCDenvNODEpt_test.h:414-417) to every link of a file start
 *                  before the run;
 *   --time         print the wall time of the NsptEvolve calls, and each
 *                  step's own time;
 *   --sweep-only   each step is the Jacobi sweep part of NsptEvolve alone:
 *                  the per-step observables zeroed (nspt.cc:965-980),
 *                  gauge_wilson(Umu, Fmu), Umu = Fmu and, with twisted
 *                  boundaries, twist_boundary(Umu) (nspt.cc:989-995) -- no
 *                  zero modes and no gauge fixing.  This is the CPU side of
 *                  the benchmark's timed sweep.
 *
 * Usage:
 *   ref_harness --L l0 l1 l2 l3 --steps S --dt DT --alpha A --seed SEED
 *               --start cold|FILE --out PREFIX [--noise FILE] [--twist-init]
 *               [--project] [--time] [--sweep-only] [--lower LO]
 */
#include "nspt.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <fftw3.h>

/* Globals nspt.cc expects (declared extern at nspt.cc:37-94). */
Cplx *w, *w1, *w2;
double *norm, *norm1;
Cplx **trU;
int ratio = 0;
ptSUX *U;
#ifndef UPDATE_ONTHEFLY
ptSUX *F;
#endif
nspt_params_t nspt_pars;
act_params_t act_pars;
thread_params_t thr_pars[NTHR];
MyRand Rand[NTHR];
std::ofstream plaqfile, normfile, logfile, trufile;
#ifdef __WILLOOP_2x2__
std::ofstream loop2x2;
#endif
#ifdef __MANY_LOOP__
std::ofstream loop_nxm;
#endif

extern ptSUX_fld *Wgauge;
extern fftw_plan *planFA;

static void usage() {
  fprintf(stderr,
          "ref_harness --L l0 l1 l2 l3 --steps S --dt DT --alpha A --seed S "
          "--start cold|FILE --out PREFIX [--noise FILE] [--twist-init] "
          "[--project] [--time] [--sweep-only] [--lower LO] [--loops FILE] [--wl2x2 FILE]\n");
  exit(2);
}

int main(int argc, char **argv) {
  int sz[4] = {4, 4, 4, 4};
  int steps = 1;
  double dt = 0.01, alpha = 0.0;
  long seed = 12345;
  std::string start = "cold", out = "ref", noise_path, loops_path, wl2x2_path;
  bool twist_init = false, project = false, timing = false, sweep_only = false;
  int lower = 0;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    if (a == "--L" && i + 4 < argc) {
      for (int d = 0; d < 4; d++) sz[d] = atoi(argv[++i]);
    } else if (a == "--steps" && i + 1 < argc) {
      steps = atoi(argv[++i]);
    } else if (a == "--dt" && i + 1 < argc) {
      dt = atof(argv[++i]);
    } else if (a == "--alpha" && i + 1 < argc) {
      alpha = atof(argv[++i]);
    } else if (a == "--seed" && i + 1 < argc) {
      seed = atol(argv[++i]);
    } else if (a == "--start" && i + 1 < argc) {
      start = argv[++i];
    } else if (a == "--out" && i + 1 < argc) {
      out = argv[++i];
    } else if (a == "--noise" && i + 1 < argc) {
      noise_path = argv[++i];
    } else if (a == "--twist-init") {
      twist_init = true;
    } else if (a == "--project") {
      project = true;
    } else if (a == "--time") {
      timing = true;
    } else if (a == "--sweep-only") {
      sweep_only = true;
    } else if (a == "--lower" && i + 1 < argc) {
      lower = atoi(argv[++i]);
    } else if (a == "--loops" && i + 1 < argc) {
      loops_path = argv[++i];
    } else if (a == "--wl2x2" && i + 1 < argc) {
      wl2x2_path = argv[++i];
    } else {
      usage();
    }
  }

  PTORD = allocORD;
  w = new Cplx[allocORD + 1];
  w1 = new Cplx[allocORD + 1];
  w2 = new Cplx[allocORD + 1];
  norm = new double[allocORD];
  norm1 = new double[allocORD];
  trU = new Cplx *[dim];
  for (int i = 0; i < dim; i++) trU[i] = new Cplx[allocORD];

  act_pars.sz = new int[dim];
  for (int d = 0; d < 4; d++) act_pars.sz[d] = sz[d];
  act_pars.iVol = sz[0] * sz[1] * sz[2] * sz[3];
  act_pars.rVol = 1.0 / (double)act_pars.iVol;
  act_pars.tau_g = dt;
  act_pars.alpha = alpha;
  /* improved action parameters, Quenched.cc:311-322 */
#if GAUGE_ACTION == WIL
  act_pars.c1 = 0.0;
#elif GAUGE_ACTION == TLSYM
  act_pars.c1 = -1.0 / 12.0;
#elif GAUGE_ACTION == IWA
  act_pars.c1 = -0.331;
#elif GAUGE_ACTION == DBW2
  act_pars.c1 = -1.4088;
#endif
  act_pars.c0 = 1. - 8. * act_pars.c1;
  act_pars.stau = sqrt(act_pars.tau_g);
  act_pars.tau_g /= -(2 * NC);
  nspt_pars.Beat = 1;
  nspt_pars.Sweep = steps;

  /* OpenMP block partition, as Quenched.cc:518-544 */
  for (int tid = 0; tid < NTHR; tid++) {
    thr_pars[tid].xi = new int[dim];
    thr_pars[tid].xf = new int[dim];
    thr_pars[tid].xi[0] = (sz[0] / ntt) * (tid / (ntx * nty * ntz));
    thr_pars[tid].xi[1] = (sz[1] / ntx) * ((tid / (nty * ntz)) % ntx);
    thr_pars[tid].xi[2] = (sz[2] / nty) * ((tid / (ntz)) % nty);
    thr_pars[tid].xi[3] = (sz[3] / ntz) * (tid % ntz);
    for (int d = 0; d < 4; d++) {
      int nt = d == 0 ? ntt : d == 1 ? ntx : d == 2 ? nty : ntz;
      thr_pars[tid].xf[d] = thr_pars[tid].xi[d] + sz[d] / nt;
    }
    Rand[tid].init(seed + tid);
  }

  std::string plaqn = out + ".plaq", normn = out + ".nor", trun = out + ".tru";
  plaqfile.open(plaqn.c_str());
  normfile.open(normn.c_str());
  trufile.open(trun.c_str());
  plaqfile.precision(17);
  normfile.precision(17);
  trufile.precision(17);
  plaqfile << std::scientific;
  normfile << std::scientific;
  trufile << std::scientific;
#ifdef __MANY_LOOP__
  /* ComputeLoops' stream (nspt.cc:1283-1306): the loops of the final field */
  loop_nxm.open(loops_path.empty() ? "/dev/null" : loops_path.c_str());
  loop_nxm.precision(17);
  loop_nxm << std::scientific;
#else
  if (!loops_path.empty()) {
    fprintf(stderr, "ref_harness: --loops needs a periodic build\n");
    return 2;
  }
#endif

#ifdef __WILLOOP_2x2__
  /* WL2x2's stream (nspt.cc:1064-1140): the 2x2 loops of the final field */
  loop2x2.open(wl2x2_path.empty() ? "/dev/null" : wl2x2_path.c_str());
  loop2x2.precision(17);
  loop2x2 << std::scientific;
#else
  if (!wl2x2_path.empty()) {
    fprintf(stderr, "ref_harness: --wl2x2 needs a periodic build\n");
    return 2;
  }
#endif

  latt LL(act_pars.sz);
  LL.p_init();
  ptSUXGluon_fld Umu(&LL);
#ifndef UPDATE_ONTHEFLY
  ptSUXGluon_fld Fmu(&LL);
#endif
  ptSUX_fld WFA(&LL);
  Wgauge = &WFA;
  planFA = new fftw_plan[2];
  planFA[0] = fftw_plan_many_dft(dim, LL.Sz, NC * NC * PTORD + 1,
                                 (fftw_complex *)WFA.W, NULL,
                                 NC * NC * allocORD + 1, 1,
                                 (fftw_complex *)WFA.W, NULL,
                                 NC * NC * allocORD + 1, 1, FFTW_FORWARD,
                                 FFTW_ESTIMATE);
  planFA[1] = fftw_plan_many_dft(dim, LL.Sz, NC * NC * PTORD + 1,
                                 (fftw_complex *)WFA.W, NULL,
                                 NC * NC * allocORD + 1, 1,
                                 (fftw_complex *)WFA.W, NULL,
                                 NC * NC * allocORD + 1, 1, FFTW_BACKWARD,
                                 FFTW_ESTIMATE);

  if (start == "cold") {
    for (int i = 0; i < LL.TSize; i++)
      for (int mu = 0; mu < dim; mu++) Umu.W[i].U[mu].id();
  } else if (lower > 0) {
    for (int i = 0; i < LL.TSize; i++)
      for (int mu = 0; mu < dim; mu++) Umu.W[i].U[mu].id();
    std::vector<Cplx> plq(allocORD + 1);
    if (Umu.loadlowerorder(start.c_str(), lower, plq.data())) {
      fprintf(stderr, "ref_harness: loadlowerorder %s failed\n", start.c_str());
      return 1;
    }
  } else {
    if (Umu.load(start.c_str(), w1)) {
      fprintf(stderr, "ref_harness: cannot load %s\n", start.c_str());
      return 1;
    }
    if (project) {
      for (int x = 0; x < LL.Size; x++)
        for (int mu = 0; mu < dim; mu++) {
          ptSU3 myapp = log(Umu.W[x].U[mu]);
          myapp = myapp.reH();
          Umu.W[x].U[mu] = exp(myapp);
        }
    }
#ifdef TWISTED_BC
    if (twist_init) twist_boundary(Umu);
#else
    (void)twist_init;
#endif
  }
  U = Umu.handle();
#ifndef UPDATE_ONTHEFLY
  F = Fmu.handle();
#endif

  FILE *fnoise = NULL;
  std::vector<MyRand> replay(NTHR);
  if (!noise_path.empty()) {
    fnoise = fopen(noise_path.c_str(), "wb");
    for (int tid = 0; tid < NTHR; tid++) replay[tid].init(seed + tid);
  }

  /* initial static plaquette (nspt.cc:1316-1406) */
  plaquette_measure(Umu, act_pars);
  {
    std::string p0 = out + ".plaq0";
    FILE *f = fopen(p0.c_str(), "w");
    for (int i = 0; i <= PTORD; i++) fprintf(f, "%.17e %.17e\n", w[i].re, w[i].im);
    fclose(f);
  }

  double secs = 0.0;
  std::vector<double> step_secs;
  for (int s = 0; s < steps; s++) {
    if (fnoise) {
      /* the draws of gauge_wilson: each thread's stream over its block */
      size_t n = (size_t)act_pars.iVol * dim * 8;
      double *buf = new double[n];
      for (int tid = 0; tid < NTHR; tid++)
        for (int y0 = thr_pars[tid].xi[0]; y0 < thr_pars[tid].xf[0]; y0++)
          for (int y1 = thr_pars[tid].xi[1]; y1 < thr_pars[tid].xf[1]; y1++)
            for (int y2 = thr_pars[tid].xi[2]; y2 < thr_pars[tid].xf[2]; y2++)
              for (int y3 = thr_pars[tid].xi[3]; y3 < thr_pars[tid].xf[3]; y3++) {
                const size_t site =
                    y3 + (size_t)sz[3] * (y2 + (size_t)sz[2] * (y1 + (size_t)sz[1] * y0));
                for (int k = 0; k < dim * 8; k++)
                  buf[site * dim * 8 + k] = replay[tid].generate_gauss();
              }
      fwrite(buf, sizeof(double), n, fnoise);
      delete[] buf;
    }
    auto t0 = std::chrono::steady_clock::now();
#ifdef UPDATE_ONTHEFLY
    NsptEvolve(Umu);
#else
    if (sweep_only) {
      /* the sweep part of NsptEvolve, nspt.cc:965-995 */
      for (int i1 = 0; i1 < PTORD; i1++) {
        w1[i1] = 0.0;
        norm[i1] = 0.0;
        for (int mu = 0; mu < dim; mu++) trU[mu][i1] = 0.0;
      }
      w1[PTORD] = 0.0;
      gauge_wilson(Umu, Fmu);
      Umu = Fmu;
#ifdef TWISTED_BC
      twist_boundary(Umu);
#endif
    } else {
      NsptEvolve(Umu, Fmu);
    }
#endif
    auto t1 = std::chrono::steady_clock::now();
    const double dts = std::chrono::duration<double>(t1 - t0).count();
    step_secs.push_back(dts);
    secs += dts;
  }
  if (fnoise) fclose(fnoise);

  plaquette_measure(Umu, act_pars);
#ifdef __MANY_LOOP__
  if (!loops_path.empty()) ComputeLoops(Umu);
#endif
#ifdef __WILLOOP_2x2__
  if (!wl2x2_path.empty()) WL2x2(Umu);
  loop2x2.close();
#endif
  std::string conf = out + ".dat";
  std::vector<char> name(conf.begin(), conf.end());
  name.push_back('\0');
  Umu.save(name.data(), w);
  if (timing) {
    printf("steps %d seconds %.6f seconds_per_sweep %.6f threads %d\n", steps,
           secs, secs / (steps > 0 ? steps : 1), NTHR);
    printf("step_seconds");
    for (double t : step_secs) printf(" %.6f", t);
    printf("\n");
  }
  plaqfile.close();
  normfile.close();
  trufile.close();
  return 0;
}
