// nspt_quenched -- the reference's quenched NSPT program (Quenched.cc) on
// the B200 engine.
//
// The same inputs and outputs as the reference's executable:
//   * Quench.cfg in the working directory, read key by key in the
//     reference's order (Quenched.cc:158-172): "taglia L0 L1 L2 L3", SWEEP,
//     BEAT, tau_g, alpha, init_status, plaq_out, last_conf, PTORD, seed;
//   * the same command-line overrides (-l -s -b -r -g -a -t -p -c -d -n -h,
//     Quenched.cc:182-236; -a sets alpha = -value as there);
//   * damocle.dag, re-read after every BEAT steps for SWEEP, BEAT, tau_g,
//     alpha, save_config and kill_run (AggiornaParametri, Quenched.cc:662-713);
//   * output files named as the reference names them (Quenched.cc:376-407):
//     the plaquette series <plaq_out>_SU3_wil_nf0_<L>_a<alpha>_tg<tau>_o<N>.txt
//     (appended, 30 digits), .nor, .trU, .log, and the final configuration
//     <last_conf>SU3_wil_nf0_..._o<N> in the reference's binary format
//     (checkpoints add _<k>.dat), one line per order per step as
//     gauge_wilson writes them (nspt.cc:570-597);
//   * beside every saved configuration a noise-state sidecar <name>.rng (no
//     reference counterpart), read back on a hot start when present, so a run
//     resumed from a checkpoint continues the same noise stream.
// The reference fixes some choices at compile time (choices.h); here they are
// options: -T <dirs> twisted boundaries in y/z/t (TWISTED_BC, _TWIST_*),
// -F Fourier-accelerated gauge fixing (__FA_GAUGE_FIXING__, periodic only),
// -G ntt,ntx,nty,ntz the thread grid whose order the local gauge fixing
// reproduces (choices.h:124-128; default: the finest the reference accepts),
// -Z 0|1 zero-mode subtraction (default: on with periodic boundaries, as
// REMOVE_GLUON_ZEROMOM), -A tlsym|iwa|dbw2 an improved gauge action
// (GAUGE_ACTION; file names and the plaquette file's extra two columns of
// rectangle traces follow Quenched.cc:327-348 and nspt.cc:586-597), -P
// device Philox noise instead of the reference's rand55 stream, -O the
// reference's default on-the-fly update (UPDATE_ONTHEFLY: links updated in
// place in the thread grid's order); without -O the Jacobi update.  -M
// draws the noise as an OpenMP build of the reference does: one rand55
// stream per thread of the -G grid, seeded from the `seed` lines of
// Quench.cfg (one per thread) or by -r through srand/rand; a hot start
// reseeds them, as the reference keeps no noise state.
// With periodic boundaries the Wilson loops of ComputeLoops (__MANY_LOOP__,
// the reference's periodic default) go to <plaq_out>_nxm_SU3_wil_..._o<N>.txt
// after every BEAT steps and at the end (nspt.cc:1283-1306); with -W also
// the 2x2 loops of WL2x2 (__WILLOOP_2x2__, periodic only) go to
// <plaq_out>2x2_SU3_wil_..._o<N>.txt at the same points (Quenched.cc:389-393,
// 658-660, 737-739; nspt.cc:1118-1124).
#include <getopt.h>
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "../../include/nspt_b200.h"
#include "rand55.h"

namespace {

struct Params {
  int L[4] = {0, 0, 0, 0};
  int sweep = 0, beat = 0, init = 0, N = 0;
  double tau_g = 0.0, alpha = 0.0;
  long seed = 0;
  std::string plaqn, confn, damon = "damocle.dag";
  unsigned twist = 0;
  bool fa = false, philox = false, wl2x2 = false, otf = false;
  bool thread_noise = false;  // -M: one rand55 stream per thread of the -G grid
  std::vector<long> seeds;    // every `seed` line of Quench.cfg (one per thread)
  bool seed_given = false;    // -r
  int zm = -1;  // -1: as the boundary conditions imply
  int grid[4] = {0, 0, 0, 0};
  unsigned action = 0;  // NSPT_ACTION_* or 0 (Wilson)
};

// get_val (Quenched.cc:97-114): the next word must be `key`, then a value.
bool get_word(FILE *fp, const char *key, char *val, size_t n) {
  char w[128];
  if (fscanf(fp, "%127s", w) != 1 || strcmp(w, key) != 0) {
    fprintf(stderr, "Error reading input file: expected %s\n", key);
    return false;
  }
  char fmt[16];
  snprintf(fmt, sizeof(fmt), "%%%zus", n - 1);
  if (fscanf(fp, fmt, val) != 1) {
    fprintf(stderr, "Error reading input file at %s\n", key);
    return false;
  }
  return true;
}
bool get_int(FILE *fp, const char *key, int *v) {
  char s[128];
  if (!get_word(fp, key, s, sizeof(s))) return false;
  *v = atoi(s);
  return true;
}
bool get_double(FILE *fp, const char *key, double *v) {
  char s[128];
  if (!get_word(fp, key, s, sizeof(s))) return false;
  *v = atof(s);
  return true;
}

bool read_cfg(Params &p) {
  FILE *fp = fopen("Quench.cfg", "r");
  if (!fp) {
    fprintf(stderr, "Errore: impossibile leggere il file di configurazione.\n");
    return false;
  }
  bool ok = fscanf(fp, " taglia %d %d %d %d", &p.L[0], &p.L[1], &p.L[2], &p.L[3]) == 4;
  char s[128];
  ok = ok && get_int(fp, "SWEEP", &p.sweep) && get_int(fp, "BEAT", &p.beat) &&
       get_double(fp, "tau_g", &p.tau_g) && get_double(fp, "alpha", &p.alpha) &&
       get_int(fp, "init_status", &p.init);
  if (ok && (ok = get_word(fp, "plaq_out", s, sizeof(s)))) p.plaqn = s;
  if (ok && (ok = get_word(fp, "last_conf", s, sizeof(s)))) p.confn = s;
  ok = ok && get_int(fp, "PTORD", &p.N);
  if (ok && (ok = get_word(fp, "seed", s, sizeof(s)))) p.seed = atol(s);
  if (ok) {
    // the reference reads one `seed` line per OpenMP thread (Quenched.cc:171-174)
    p.seeds.push_back(p.seed);
    char w[128], v[128];
    while (fscanf(fp, "%127s %127s", w, v) == 2 && strcmp(w, "seed") == 0)
      p.seeds.push_back(atol(v));
  }
  fclose(fp);
  if (!ok) fprintf(stderr, "Errore: Quench.cfg non valido.\n");
  return ok;
}

void usage() {
  printf("\n"
         "-l\t\ttaglia (reticolo t==x==y==z)\n"
         "-s\t\tnumero iterazioni (SWEEP)\n"
         "-b\t\titerazioni tra letture damocle (BEAT)\n"
         "-r\t\tseed generatore random\n"
         "-g\t\ttau gluoni\n"
         "-a\t\talpha\n"
         "-t\t\tstato iniziale: 1)da configurazione; 0)freddo\n"
         "-p\t\tnome file placchetta\n"
         "-c\t\tnome configurazione salvata\n"
         "-d\t\tnome file damocle\n"
         "-n\t\tordine pt\n"
         "-T dirs\t\ttwisted boundaries in the directions dirs (y, z, t)\n"
         "-F\t\tFourier-accelerated gauge fixing (periodic boundaries)\n"
         "-G a,b,c,d\tthread grid (ntt,ntx,nty,ntz) of the local gauge fixing\n"
         "-Z 0|1\t\tzero-mode subtraction off/on\n"
         "-A action\timproved gauge action: tlsym, iwa or dbw2\n"
         "-P\t\tdevice Philox noise instead of the reference's generator\n"
         "-O\t\ton-the-fly update (UPDATE_ONTHEFLY) in the thread grid's order\n"
         "-M\t\tone noise stream per thread of the -G grid (an OpenMP build)\n"
         "-W\t\t2x2 Wilson loops file (WL2x2, periodic boundaries)\n\n");
}

// Noise-state sidecar <configuration>.rng, written beside every saved
// configuration: the device generator's seed and counter and the host
// rand55 state.  The reference keeps no noise state (a hot start reseeds,
// Quenched.cc:612-637); with the sidecar a run split at a checkpoint draws
// the same noise as one that ran through.  A hot start without a sidecar
// reseeds from Quench.cfg, as the reference does.
int write_rng_sidecar(const std::string &path, nspt_ctx *ctx, const Rand55 &rng) {
  uint64_t seed = 0, counter = 0;
  const int rc = nspt_get_seed(ctx, &seed, &counter);
  if (rc) return rc;
  FILE *f = fopen(path.c_str(), "w");
  if (!f) return NSPT_ERR_IO;
  fprintf(f, "nspt_rng 1\nphilox %llu %llu\n", (unsigned long long)seed,
          (unsigned long long)counter);
  rng.save(f);
  return fclose(f) == 0 ? NSPT_OK : NSPT_ERR_IO;
}

int read_rng_sidecar(const std::string &path, nspt_ctx *ctx, Rand55 &rng) {
  FILE *f = fopen(path.c_str(), "r");
  if (!f) return NSPT_OK;  // none: fresh seed, as the reference
  int version = 0;
  unsigned long long seed = 0, counter = 0;
  const bool ok = fscanf(f, " nspt_rng %d philox %llu %llu", &version, &seed, &counter) == 3 &&
                  version == 1 && rng.load(f);
  fclose(f);
  if (!ok) {
    fprintf(stderr, "nspt_quenched: unreadable noise state %s\n", path.c_str());
    return NSPT_ERR_IO;
  }
  return nspt_seed(ctx, seed, counter);
}

// AggiornaParametri's damocle.dag read (Quenched.cc:677-685)
bool read_damocle(const std::string &path, int &sweep, int &beat, double &tau_g, double &alpha,
                  int &save, int &kill) {
  FILE *df = fopen(path.c_str(), "r");
  if (!df) {
    fprintf(stderr, "Errore, impossibile trovare file damocle.\n");
    return false;
  }
  const bool ok = get_int(df, "SWEEP", &sweep) && get_int(df, "BEAT", &beat) &&
                  get_double(df, "tau_g", &tau_g) && get_double(df, "alpha", &alpha) &&
                  get_int(df, "save_config", &save) && get_int(df, "kill_run", &kill);
  fclose(df);
  return ok;
}

std::string stem(const Params &p, const char *type) {
  char buf[256];
  snprintf(buf, sizeof(buf), "%s_nf0_%dx%dx%dx%d_a%2.2f_tg%3.3f_o%d", type, p.L[0], p.L[1], p.L[2],
           p.L[3], std::fabs(p.alpha), p.tau_g, p.N);
  return buf;
}

void stamp(FILE *log, const char *what) {
  time_t t = time(nullptr);
  fprintf(log, "%s\t\t%s\n", what, ctime(&t));
}

int fail(nspt_ctx *ctx, int rc, const char *where) {
  fprintf(stderr, "nspt_quenched: %s: %s (%s)\n", where, nspt_error_string(rc),
          ctx ? nspt_last_error(ctx) : "");
  return 2;
}

}  // namespace

int main(int argc, char **argv) {
  Params p;
  for (int i = 1; i < argc; i++)
    if (!strcmp(argv[i], "-h")) {
      usage();
      return 0;
    }
  if (!read_cfg(p)) return 1;
  int opt;
  while ((opt = getopt(argc, argv, "l:s:b:d:r:g:a:t:p:c:n:hT:FG:Z:PA:WOM")) != -1) {
    switch (opt) {
      case 'l': p.L[0] = p.L[1] = p.L[2] = p.L[3] = atoi(optarg); break;
      case 's': p.sweep = atoi(optarg); break;
      case 'b': p.beat = atoi(optarg); break;
      case 'r':
        p.seed = atol(optarg);
        p.seed_given = true;
        break;
      case 'n': p.N = atoi(optarg); break;
      case 'g': p.tau_g = atof(optarg); break;
      case 'a': p.alpha = -atof(optarg); break;
      case 't': p.init = atoi(optarg); break;
      case 'p': p.plaqn = optarg; break;
      case 'c': p.confn = optarg; break;
      case 'd': p.damon = optarg; break;
      case 'T':
        for (const char *c = optarg; *c; c++) {
          if (*c == 'y') p.twist |= NSPT_TWIST_Y;
          else if (*c == 'z') p.twist |= NSPT_TWIST_Z;
          else if (*c == 't') p.twist |= NSPT_TWIST_T;
          else {
            fprintf(stderr, "nspt_quenched: -T takes y, z and t\n");
            return 1;
          }
        }
        break;
      case 'F': p.fa = true; break;
      case 'G':
        if (sscanf(optarg, "%d,%d,%d,%d", &p.grid[0], &p.grid[1], &p.grid[2], &p.grid[3]) != 4) {
          fprintf(stderr, "nspt_quenched: -G takes ntt,ntx,nty,ntz\n");
          return 1;
        }
        break;
      case 'Z': p.zm = atoi(optarg); break;
      case 'P': p.philox = true; break;
      case 'W': p.wl2x2 = true; break;
      case 'O': p.otf = true; break;
      case 'M': p.thread_noise = true; break;
      case 'A':
        if (!strcmp(optarg, "tlsym")) p.action = NSPT_ACTION_TLSYM;
        else if (!strcmp(optarg, "iwa")) p.action = NSPT_ACTION_IWA;
        else if (!strcmp(optarg, "dbw2")) p.action = NSPT_ACTION_DBW2;
        else {
          fprintf(stderr, "nspt_quenched: -A takes tlsym, iwa or dbw2\n");
          return 1;
        }
        break;
      default: usage(); return 1;
    }
  }
  {
    FILE *df = fopen(p.damon.c_str(), "r");
    if (!df) {
      fprintf(stderr, "Errore, impossibile trovare file damocle.\n");
      return 1;
    }
    fclose(df);
  }
  if (p.beat < 1 || p.N < 1) {
    fprintf(stderr, "nspt_quenched: BEAT and PTORD must be positive\n");
    return 1;
  }
  const bool periodic = p.twist == 0;
  const bool zm = p.zm < 0 ? periodic : p.zm != 0;
  unsigned flags = p.twist | (zm ? NSPT_ZEROMODE : 0u) | (p.fa ? NSPT_GF_FA : NSPT_GF_LOCAL) |
                   p.action | (p.otf ? NSPT_UPDATE_ONTHEFLY : 0u);

  // file names (Quenched.cc:376-407)
  const char *type = p.action == NSPT_ACTION_TLSYM  ? "SU3_tls"
                     : p.action == NSPT_ACTION_IWA  ? "SU3_iwa"
                     : p.action == NSPT_ACTION_DBW2 ? "SU3_dbw"
                                                    : "SU3_wil";
  const std::string plaq_name = p.plaqn + "_" + stem(p, type) + ".txt";
  const std::string conf_name = p.confn + stem(p, type);
  const std::string log_name = stem(p, type) + ".log";
  const std::string norm_name = stem(p, type) + ".nor";
  const std::string tru_name = stem(p, type) + ".trU";
  FILE *plaqf = fopen(plaq_name.c_str(), "a");
  const std::string loops_name = p.plaqn + "_nxm_" + stem(p, type) + ".txt";
  FILE *loopf = periodic ? fopen(loops_name.c_str(), "a") : nullptr;
  if (periodic && !loopf) {
    fprintf(stderr, "nspt_quenched: cannot open %s\n", loops_name.c_str());
    return 1;
  }
  const std::string wl_name = p.plaqn + "2x2_" + stem(p, type) + ".txt";
  if (p.wl2x2 && !periodic) {
    fprintf(stderr, "nspt_quenched: -W (WL2x2) needs periodic boundaries\n");
    return 1;
  }
  FILE *wlf = p.wl2x2 ? fopen(wl_name.c_str(), "a") : nullptr;
  if (p.wl2x2 && !wlf) {
    fprintf(stderr, "nspt_quenched: cannot open %s\n", wl_name.c_str());
    return 1;
  }
  FILE *normf = fopen(norm_name.c_str(), "w");
  FILE *truf = fopen(tru_name.c_str(), "w");
  FILE *logf = fopen(log_name.c_str(), "w");
  if (!plaqf || !normf || !truf || !logf) {
    fprintf(stderr, "nspt_quenched: cannot open the output files\n");
    return 1;
  }
  fprintf(logf, "Gauge group\t\tSU3\n\tgauge field update %s\"on the fly\"\n",
          p.otf ? "" : "not ");
  fprintf(logf, "Gauge field boundary conditions\t\t%s\n", periodic ? "PERIODIC" : "TWISTED");
  fprintf(logf,
          "Taglia\t\t%d %d %d %d\nSweep\t\t%d\nBeat\t\t%d\nTau_g\t\t%g\nAlpha\t\t%g\n"
          "Init status\t%d\nOrdine\t\t%d\n\nPlacchetta\t%s\nConfigurazione\t%s\nDamocle\t\t%s\n"
          "Norma\t\t%s\nTr(U)\t\t%s\n\n",
          p.L[0], p.L[1], p.L[2], p.L[3], p.sweep, p.beat, p.tau_g, p.alpha, p.init, p.N,
          plaq_name.c_str(), conf_name.c_str(), p.damon.c_str(), norm_name.c_str(),
          tru_name.c_str());

  nspt_ctx *ctx = nullptr;
  int rc = nspt_create(p.L, p.N, flags, p.alpha, &ctx);
  if (rc) return fail(nullptr, rc, "nspt_create");
  if (p.grid[0] && (rc = nspt_set_gf_grid(ctx, p.grid))) return fail(ctx, rc, "thread grid");
  const int N = p.N;
  std::vector<double> plaq(2 * (N + 1)), w(2 * (N + 1)), norm(N), tru(8 * N);
  std::vector<double> loops(8 * (N + 1)), w2(2 * (N + 1));
  // ComputeLoops' line: per loop (1x2, 2x2, 2x4, 4x4) the even orders
  auto write_loops = [&]() -> int {
    if (!loopf) return NSPT_OK;
    const int r = nspt_wilson_loops(ctx, loops.data());
    if (r) return r;
    for (int q = 0; q < 4; q++)
      for (int k = 0; k <= N; k += 2) fprintf(loopf, "%.30e\t", loops[2 * (q * (N + 1) + k)]);
    fprintf(loopf, "\n");
    fflush(loopf);
    return NSPT_OK;
  };
  // WL2x2's line: Re Tr of orders 2, 4, ... <= N (its ptU[1], ptU[3], ...)
  std::vector<double> wl(2 * (N + 1));
  auto write_wl2x2 = [&]() -> int {
    if (!wlf) return NSPT_OK;
    const int r = nspt_wl2x2(ctx, wl.data());
    if (r) return r;
    for (int k = 2; k <= N; k += 2) fprintf(wlf, "%.30e\t", wl[2 * k]);
    fprintf(wlf, "\n");
    fflush(wlf);
    return NSPT_OK;
  };
  if (p.init) {  // hot start from the saved configuration (Quenched.cc:612-637)
    if ((rc = nspt_load_config(ctx, conf_name.c_str(), N, w.data())))
      return fail(ctx, rc, "Errore nella lettura della configurazione");
    if ((rc = nspt_plaquette_measure(ctx, plaq.data()))) return fail(ctx, rc, "plaquette");
    bool same = true;  // plaquette_check (nspt.cc:1042-1052)
    for (int k = 0; k <= N; k++)
      if (std::hypot(plaq[2 * k] - w[2 * k], plaq[2 * k + 1] - w[2 * k + 1]) > 1e-7) same = false;
    if (!same) printf("La misura della placchetta non corrisponde.\n");
    printf("\nMisura della placchetta:\n");
    for (int k = 0; k <= N; k++) printf("%e %e\n", plaq[2 * k], plaq[2 * k + 1]);
  }
  Rand55 rng(p.seed);
  if (p.philox && (rc = nspt_seed(ctx, (uint64_t)p.seed, 0))) return fail(ctx, rc, "seed");
  if (p.init && (rc = read_rng_sidecar(conf_name + ".rng", ctx, rng)))
    return fail(ctx, rc, "noise state");
  std::vector<double> eta;
  if (!p.philox) eta.resize((size_t)p.L[0] * p.L[1] * p.L[2] * p.L[3] * 32);
  // -M: the noise of an OpenMP build.  Thread tid draws from its own rand55
  // seeded with the tid-th `seed` line (Quenched.cc:171-174, 296-299), or
  // with rand() after srand(-r) (Quenched.cc:199-205); it draws the 8
  // Gaussians of every link of its block (Quenched.cc:518-531), sites in the
  // block's lexicographic order and mu inner (nspt.cc:355-440).
  std::vector<Rand55> trng;
  std::vector<std::vector<long>> tsites;
  if (p.thread_noise && !p.philox) {
    if (!p.grid[0]) {
      fprintf(stderr, "nspt_quenched: -M needs the build's thread grid (-G)\n");
      return 1;
    }
    const int nthr = p.grid[0] * p.grid[1] * p.grid[2] * p.grid[3];
    std::vector<long> sd(nthr);
    if (p.seed_given) {
      srand((unsigned)p.seed);
      for (int t = 0; t < nthr; t++) sd[t] = rand();
    } else {
      if ((int)p.seeds.size() < nthr) {
        fprintf(stderr, "Error reading input file at seed\n");
        return 1;
      }
      for (int t = 0; t < nthr; t++) sd[t] = p.seeds[t];
    }
    int bs[4];
    for (int d = 0; d < 4; d++) bs[d] = p.L[d] / p.grid[d];
    for (int t = 0; t < nthr; t++) {
      trng.emplace_back(sd[t]);
      const int b[4] = {t / (p.grid[1] * p.grid[2] * p.grid[3]),
                        (t / (p.grid[2] * p.grid[3])) % p.grid[1], (t / p.grid[3]) % p.grid[2],
                        t % p.grid[3]};
      std::vector<long> st;
      for (int x0 = b[0] * bs[0]; x0 < (b[0] + 1) * bs[0]; x0++)
        for (int x1 = b[1] * bs[1]; x1 < (b[1] + 1) * bs[1]; x1++)
          for (int x2 = b[2] * bs[2]; x2 < (b[2] + 1) * bs[2]; x2++)
            for (int x3 = b[3] * bs[3]; x3 < (b[3] + 1) * bs[3]; x3++)
              st.push_back(((long)(x0 * p.L[1] + x1) * p.L[2] + x2) * p.L[3] + x3);
      tsites.push_back(st);
    }
  }
  stamp(logf, "Inizio run");

  int t1 = 0, done = 0, config_counter = 0;
  while (t1 < p.sweep) {
    t1 += p.beat;
    for (int t2 = 0; t2 < p.beat; t2++) {  // NsptEvolve (nspt.cc:963-1036)
      if (!p.philox) {
        if (trng.empty()) {
          rng.fill(eta.data(), (long)eta.size());
        } else {
          for (size_t t = 0; t < trng.size(); t++)
            for (long site : tsites[t]) trng[t].fill(eta.data() + site * 32, 32);
        }
        if ((rc = nspt_set_noise(ctx, eta.data()))) return fail(ctx, rc, "noise");
      }
      if ((rc = nspt_gauge_wilson(ctx, p.tau_g))) return fail(ctx, rc, "gauge_wilson");
      if ((rc = nspt_observables(ctx, plaq.data(), norm.data(), tru.data())))
        return fail(ctx, rc, "observables");
      if (p.action && (rc = nspt_rect_observables(ctx, w2.data())))
        return fail(ctx, rc, "observables");
      auto plaq_line = [&](int k) {  // nspt.cc:576-597
        if (p.action)
          fprintf(plaqf, "%.30e\t%.30e\t%.30e\t%.30e\n", plaq[2 * k], plaq[2 * k + 1], w2[2 * k],
                  w2[2 * k + 1]);
        else
          fprintf(plaqf, "%.30e\t%.30e\n", plaq[2 * k], plaq[2 * k + 1]);
      };
      for (int k = 0; k < N; k++) {
        plaq_line(k);
        fprintf(normf, "%g\n", norm[k]);
        for (int mu = 0; mu < 4; mu++)
          fprintf(truf, "%g\t%g\t", tru[2 * (mu * N + k)], tru[2 * (mu * N + k) + 1]);
        fprintf(truf, "\n");
      }
      plaq_line(N);
      if (zm && (rc = nspt_zero_modes_subtraction(ctx))) return fail(ctx, rc, "zero modes");
      if (p.fa)
        rc = nspt_fa_gauge_fixing(ctx, p.alpha);
      else
        rc = nspt_local_gauge_fixing(ctx, p.alpha);
      if (rc) return fail(ctx, rc, "gauge fixing");
      if ((rc = nspt_twist_boundary(ctx))) return fail(ctx, rc, "twist_boundary");
      done++;
    }
    fflush(plaqf);
    fflush(normf);
    fflush(truf);
    // AggiornaParametri (Quenched.cc:656-713)
    if ((rc = write_wl2x2())) return fail(ctx, rc, "WL2x2");
    if ((rc = write_loops())) return fail(ctx, rc, "ComputeLoops");
    fprintf(logf, "______________________________________\n\n");
    stamp(logf, "Damocle Update");
    fprintf(logf, "# Iterazioni\t\t%d\n", done);
    int save = 0, kill = 0;
    if (!read_damocle(p.damon, p.sweep, p.beat, p.tau_g, p.alpha, save, kill)) return 1;
    fprintf(logf, "Tau_g\t\t\t%g\n\n", p.tau_g);
    fflush(logf);
    if (p.beat < 1) {
      fprintf(stderr, "nspt_quenched: BEAT must be positive\n");
      return 1;
    }
    if (save == 1) {
      const std::string name = conf_name + "_" + std::to_string(++config_counter) + ".dat";
      if ((rc = nspt_save_config(ctx, name.c_str(), N))) return fail(ctx, rc, "checkpoint");
      if ((rc = write_rng_sidecar(name + ".rng", ctx, rng))) return fail(ctx, rc, "checkpoint");
    }
    if (kill == 1) p.sweep = 0;
  }
  // NsptFinalize (Quenched.cc:718-757)
  fprintf(logf, "__________________________________\n");
  stamp(logf, "Termine simulazione");
  fprintf(logf, "# Iterazioni\t\t%d\n", t1);
  if ((rc = nspt_plaquette_measure(ctx, plaq.data()))) return fail(ctx, rc, "plaquette");
  printf("Misura della placchetta:\n");
  for (int k = 0; k <= N; k++) printf("%e\t%e\n", plaq[2 * k], plaq[2 * k + 1]);
  if ((rc = write_wl2x2())) return fail(ctx, rc, "WL2x2");
  if (wlf) fclose(wlf);
  if ((rc = write_loops())) return fail(ctx, rc, "ComputeLoops");
  if (loopf) fclose(loopf);
  if ((rc = nspt_save_config(ctx, conf_name.c_str(), N))) return fail(ctx, rc, "save");
  if ((rc = write_rng_sidecar(conf_name + ".rng", ctx, rng))) return fail(ctx, rc, "save");
  fclose(plaqf);
  fclose(normf);
  fclose(truf);
  fclose(logf);
  nspt_destroy(ctx);
  return 0;
}
