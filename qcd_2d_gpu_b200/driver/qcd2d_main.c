/*
 * qcd2d — drop-in for the reference's program (kernel.cu:49-268) on the
 * B200 library: the same knobs, now command-line flags with kernel.cu's
 * #define values as defaults, the same run loop (thermalisation,
 * measurements every N_cor sweeps, periodic re-projection, partial saves) and
 * the same output files and prints.
 *
 *   qcd2d [--algo hb|metro] [--dt 96] [--dx 96] [--dy 4] [--beta 20]
 *         [--boundary 0|1|2] [--readconf 0|1|2] [--init 0|1] [--sconf 0|1]
 *         [--save 0|1] [--N 50000] [--N-term 20000] [--N-block 20]
 *         [--Nblock-term 10] [--Nsave 5] [--N-cor 1] [--epsilon 0.1]
 *         [--upd 1] [--W 80] [--seed S] [--nsave 1] [--nconfr 1] [--nconfs 1]
 *         [--outdir DIR]
 *   extensions: [--precision fp64|fp32] [--n-or K] [--renorm-every K]
 *               [--schedule auto|phases|wavefront] [--report]
 *               [--rng-state 1: save the generator state next to the Config_
 *                files and resume from it, so a restart continues the chain]
 *
 * With --precision fp64 (the default) the update arithmetic and the random
 * draws are the reference's, so for the same seed the files match a run of
 * the reference (heat-bath: the same link field bit for bit).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "qcd2d.h"
#include "refio.h"

typedef struct {
  int algo, d_t, d_x, d_y, boundary, readconf, init, sconf, save;
  double beta, epsilon;
  int N, N_term, N_block, Nblock_term, Nsave, N_cor, upd, W;
  long long seed;
  int have_seed;
  char nsave[16], nconfr[16], nconfs[16];
  const char* outdir;
  int precision, n_or, renorm_every, schedule, report, rng_state;
} knobs;

static void defaults(knobs* k) {  // kernel.cu:11-46
  memset(k, 0, sizeof(*k));
  k->algo = QCD_ALGO_HEATBATH;
  k->d_y = 4;
  k->d_x = 96;
  k->d_t = 96;
  k->beta = 20;
  k->boundary = 2;
  k->readconf = 0;
  k->init = 0;
  k->sconf = 0;
  k->save = 0;
  k->N = 50000;
  k->N_term = 20000;
  k->N_block = 20;
  k->Nblock_term = 10;
  k->Nsave = 5;
  k->N_cor = 1;
  k->epsilon = 0.1;
  k->upd = 1;
  k->W = 80;
  strcpy(k->nsave, "1");
  strcpy(k->nconfr, "1");
  strcpy(k->nconfs, "1");
  k->outdir = "";
  k->precision = QCD_PREC_FP64;
  k->schedule = QCD_SCHED_AUTO;
}

static int usage(void) {
  fprintf(stderr,
          "usage: qcd2d [--algo hb|metro] [--dt N] [--dx N] [--dy N] [--beta B] [--boundary 0|1|2]\n"
          "             [--readconf 0|1|2] [--init 0|1] [--sconf 0|1] [--save 0|1] [--N N] [--N-term N]\n"
          "             [--N-block N] [--Nblock-term N] [--Nsave N] [--N-cor N] [--epsilon E] [--upd N]\n"
          "             [--W N] [--seed S] [--nsave S] [--nconfr S] [--nconfs S] [--outdir DIR]\n"
          "             [--precision fp64|fp32] [--n-or K] [--renorm-every K]\n"
          "             [--schedule auto|phases|wavefront] [--report] [--rng-state 0|1]\n");
  return 2;
}

static int parse(int argc, char** argv, knobs* k) {
  for (int i = 1; i < argc; i++) {
    const char* a = argv[i];
    if (!strcmp(a, "--report")) {
      k->report = 1;
      continue;
    }
    if (i + 1 >= argc) return usage();
    const char* v = argv[++i];
#define INT_OPT(name, field) \
  else if (!strcmp(a, name)) k->field = atoi(v);
    if (!strcmp(a, "--algo")) {
      if (!strcmp(v, "hb")) k->algo = QCD_ALGO_HEATBATH;
      else if (!strcmp(v, "metro")) k->algo = QCD_ALGO_METROPOLIS;
      else return usage();
    }
    INT_OPT("--dt", d_t)
    INT_OPT("--dx", d_x)
    INT_OPT("--dy", d_y)
    INT_OPT("--boundary", boundary)
    INT_OPT("--readconf", readconf)
    INT_OPT("--init", init)
    INT_OPT("--sconf", sconf)
    INT_OPT("--save", save)
    INT_OPT("--N", N)
    INT_OPT("--N-term", N_term)
    INT_OPT("--N-block", N_block)
    INT_OPT("--Nblock-term", Nblock_term)
    INT_OPT("--Nsave", Nsave)
    INT_OPT("--N-cor", N_cor)
    INT_OPT("--upd", upd)
    INT_OPT("--W", W)
    INT_OPT("--n-or", n_or)
    INT_OPT("--renorm-every", renorm_every)
    INT_OPT("--rng-state", rng_state)
    else if (!strcmp(a, "--beta")) k->beta = atof(v);
    else if (!strcmp(a, "--epsilon")) k->epsilon = atof(v);
    else if (!strcmp(a, "--seed")) {
      k->seed = atoll(v);
      k->have_seed = 1;
    } else if (!strcmp(a, "--nsave")) snprintf(k->nsave, sizeof(k->nsave), "%s", v);
    else if (!strcmp(a, "--nconfr")) snprintf(k->nconfr, sizeof(k->nconfr), "%s", v);
    else if (!strcmp(a, "--nconfs")) snprintf(k->nconfs, sizeof(k->nconfs), "%s", v);
    else if (!strcmp(a, "--outdir")) k->outdir = v;
    else if (!strcmp(a, "--precision")) {
      if (!strcmp(v, "fp64")) k->precision = QCD_PREC_FP64;
      else if (!strcmp(v, "fp32")) k->precision = QCD_PREC_FP32;
      else return usage();
    } else if (!strcmp(a, "--schedule")) {
      if (!strcmp(v, "auto")) k->schedule = QCD_SCHED_AUTO;
      else if (!strcmp(v, "phases")) k->schedule = QCD_SCHED_PHASES;
      else if (!strcmp(v, "wavefront")) k->schedule = QCD_SCHED_WAVEFRONT;
      else return usage();
    } else return usage();
#undef INT_OPT
  }
  if (k->N < 1 || k->N_cor < 1 || k->N_term < 0 || k->Nsave < 1 || k->W < 1 || k->N_block < 1 ||
      k->Nblock_term < 1 || k->upd < 1 || k->boundary < 0 || k->boundary > 2 || k->readconf < 0 ||
      k->readconf > 2)
    return usage();
  return 0;
}

/* Config_<...>_rng.bin: the qcd_rng_words u32 generator words (qcd_store_rng) */
static void rng_path(char* out, size_t cap, const char* dir, const refio_lattice* l, const char* bound,
                     const char* n) {
  snprintf(out, cap, "%s%sConfig_%d_%d_%d_B_%.2lf_%s_%s_rng.bin", dir, dir[0] ? "/" : "", l->t, l->x, l->y,
           (double)l->beta, bound, n);
}

#define CHECK(call)                                                                       \
  do {                                                                                    \
    int rc_ = (call);                                                                     \
    if (rc_ != QCD_OK) {                                                                  \
      fprintf(stderr, "%s failed: %s (%s)\n", #call, qcd_status_string(rc_),             \
              h ? qcd_last_error(h) : "");                                                \
      exit(1);                                                                            \
    }                                                                                     \
  } while (0)

int main(int argc, char** argv) {
  knobs k;
  defaults(&k);
  int prc = parse(argc, argv, &k);
  if (prc) return prc;
  qcd_lattice* h = NULL;

  refio_lattice l = {k.d_y, k.d_x, k.d_t, k.d_y * k.d_x * k.d_t, 3, (float)k.beta, (float)k.epsilon, k.upd};
  printf("N %d Lt %d L %d Ly %d V %d Dim %d DimRep %d Dimtot %d \n", k.N, l.t, l.x, l.y, l.V, l.d, 4, 12);
  if (l.t % 2 || l.x % 2 || l.y % 2) {  // kernel.cu:61-64
    printf("Lt, Lx and Ly must be even\n");
    return 1;
  }
  int nthreads = 256;  // kernel.cu:66-70, printed for fidelity (the library sizes its own grids)
  while ((l.V / 2) % nthreads != 0) nthreads--;
  printf("nblocks %d nthreads %d\n", 2 * ((l.V / 2) / nthreads), nthreads);
  if (k.algo == QCD_ALGO_METROPOLIS) printf("METROPOLIS UPDATES epsilon %.2f hits %d\n", (double)l.epsilon, l.updates);
  if (k.algo == QCD_ALGO_HEATBATH) printf("HEAT-BATH UPDATES\n");
  const int hits = k.algo == QCD_ALGO_METROPOLIS ? l.updates : 1;

  const char* bound = k.boundary == 0 ? "per" : k.boundary == 1 ? "pcc" : "pmc";
  const size_t nphi = (size_t)l.V * 12;
  double* phi = (double*)malloc(nphi * sizeof(double));
  int* accepth = (int*)malloc((size_t)l.V * sizeof(int));
  double* en = (double*)malloc((size_t)k.N * sizeof(double));
  double* en2 = (double*)malloc((size_t)k.N * sizeof(double));
  double* autoc = (double*)malloc((size_t)k.W * sizeof(double));
  double* autoc2 = (double*)malloc((size_t)k.W * sizeof(double));
  if (!phi || !accepth || !en || !en2 || !autoc || !autoc2) {
    fprintf(stderr, "out of host memory\n");
    return 1;
  }
  int Nterms = 0, inits = k.init;
  // a configuration to resume from is read (and checked) before the GPU is touched
  if (k.readconf != 0 && refio_read_conf(k.outdir, phi, &l, &Nterms, &inits, bound, k.nconfr)) return 1;

  qcd_params p;
  qcd_params_default(&p, k.d_t, k.d_x, k.d_y);
  p.beta = (float)k.beta;
  p.epsilon = (float)k.epsilon;
  p.upd = k.upd;
  p.algo = k.algo;
  p.boundary = k.boundary;
  p.precision = k.precision;
  p.n_or = k.n_or;
  p.renorm_every = k.renorm_every;
  // setup_kernel(devStates, time(NULL)) takes an int seed (kernel.cu:79)
  p.seed = (unsigned long long)(long long)(int)(k.have_seed ? k.seed : (long long)time(NULL));
  CHECK(qcd_create(&p, &h));
  CHECK(qcd_set_schedule(h, k.schedule));

  if (k.boundary == 0) printf("PERIODIC BOUNDARY CONDITIONS\n\n");
  else if (k.boundary == 1) printf("PERFECT COLOUR CONDUCTOR BOUNDARY CONDITIONS\n\n");
  else printf("PERFECT MAGNETIC CONDUCTOR BOUNDARY CONDITIONS\n\n");
  if (k.readconf == 0) {
    if (k.init == 0) CHECK(qcd_init_hot(h));
    else CHECK(qcd_init_cold(h));
  } else {
    CHECK(qcd_load_config(h, phi));
    if (k.rng_state) {  // resume the generator chain saved with the configuration
      char rp[1024];
      rng_path(rp, sizeof(rp), k.outdir, &l, bound, k.nconfr);
      const size_t nw = (size_t)qcd_rng_words(h);
      unsigned int* w = (unsigned int*)malloc(nw * sizeof(unsigned int));
      FILE* f = fopen(rp, "rb");
      if (!w || !f || fread(w, sizeof(unsigned int), nw, f) != nw) {
        printf("Error reading %s\n", rp);
        exit(1);
      }
      fclose(f);
      CHECK(qcd_load_rng(h, w));
      free(w);
    }
  }
  CHECK(qcd_store_config(h, phi));
  refio_print_det(phi, &l);

  CHECK(qcd_accept_reset(h));
  CHECK(qcd_series_reserve(h, k.N));
  const int block_size_t = k.N_term / k.Nblock_term, block_size = k.N / k.N_block, block_s_size = k.N / k.Nsave;
  long t_ini = (long)time(NULL), t_n = t_ini, t_ini_mc, t_fin;
  double energy[2], energy2[2], saccept;

  if (k.readconf < 2) {  // thermalisation, kernel.cu:161-187
    for (int i = 1; i < k.N_term + 1; i++) {
      if (i % 100 == 0) CHECK(qcd_normalize(h));
      CHECK(qcd_sweep(h, 1));
      if (block_size_t > 0 && i % block_size_t == 0) {
        long now = (long)time(NULL);
        printf("%lf Time %d Left(min)%lf\n", (double)i / (k.N_term), (int)(now - t_n),
               (double)(now - t_ini) * (k.N_term - i) / i / 60);
        fflush(stdout);
        t_n = (long)time(NULL);
      }
    }
    CHECK(qcd_normalize(h));
    Nterms = k.N_term + Nterms;
    if (k.sconf == 0) {
      CHECK(qcd_store_config(h, phi));
      if (refio_save_conf(k.outdir, phi, &l, Nterms, inits, bound, k.nconfs)) exit(1);
      if (k.rng_state) {
        char rp[1024];
        rng_path(rp, sizeof(rp), k.outdir, &l, bound, k.nconfs);
        const size_t nw = (size_t)qcd_rng_words(h);
        unsigned int* w = (unsigned int*)malloc(nw * sizeof(unsigned int));
        if (!w) exit(1);
        CHECK(qcd_store_rng(h, w));
        FILE* f = fopen(rp, "wb");
        if (!f || fwrite(w, sizeof(unsigned int), nw, f) != nw) {
          printf("Error creating the file");
          exit(1);
        }
        fclose(f);
        free(w);
      }
    }
  }
  CHECK(qcd_store_config(h, phi));
  refio_print_det(phi, &l);
  CHECK(qcd_accept_reset(h));
  t_ini_mc = (long)time(NULL);
  t_n = t_ini_mc;
  for (int i = 1; i < k.N + 1; i++) {  // measurements, kernel.cu:192-236
    CHECK(qcd_sweep(h, k.N_cor));
    if (i % 100 == 0) CHECK(qcd_normalize(h));
    CHECK(qcd_measure_into_series(h, i - 1));
    if (block_size > 0 && i % block_size == 0) {
      long now = (long)time(NULL);
      printf("%lf Time %d Left(min)%lf\n", (double)i / k.N, (int)(now - t_n),
             (double)(now - t_ini_mc) * (k.N - i) / i / 60);
      t_n = (long)time(NULL);
      fflush(stdout);
    }
    if (block_s_size > 0 && i % block_s_size == 0) {
      CHECK(qcd_series_read(h, en, en2, i));
      printf("Energy ");
      refio_mean_variance(en, i, energy, 1);
      refio_autocorrelation(en, i, k.W, energy[0], energy[1], autoc);
      printf("Plaquette ");
      refio_mean_variance(en2, i, energy2, 1);
      refio_autocorrelation(en2, i, k.W, energy2[0], energy2[1], autoc2);
      fflush(stdout);
      if (k.save == 0) {
        CHECK(qcd_accept_counts(h, accepth));
        saccept = refio_mean_lattice_int(accepth, i * k.N_cor * l.d * hits, &l, 0);
        if (k.boundary == 1) saccept = saccept / ((double)(l.y - 1) / l.y + 1 / (double)l.y / 3);
        if (refio_save_energy(k.outdir, energy[0], energy[1], Nterms, k.N, k.N_cor, saccept, &l, bound, k.nsave) ||
            refio_save_energy_av(k.outdir, energy[0], energy[1], energy2[0], energy2[1], Nterms, k.N, k.N_cor,
                                 saccept, &l, bound, k.nsave) ||
            refio_save_autocorrelation(k.outdir, autoc, k.W, i, k.N_cor, Nterms, &l, bound, k.nsave, 0) ||
            refio_save_autocorrelation(k.outdir, autoc2, k.W, i, k.N_cor, Nterms, &l, bound, k.nsave, 1) ||
            refio_save_en_seq(k.outdir, en2, en, Nterms, i, k.N_cor, 1, &l, bound, k.nsave))
          exit(1);
      }
    }
  }
  t_fin = (long)time(NULL);
  printf("Time %d\n", (int)(t_fin - t_ini));

  CHECK(qcd_series_read(h, en, en2, k.N));
  CHECK(qcd_accept_counts(h, accepth));
  saccept = refio_mean_lattice_int(accepth, k.N * k.N_cor * l.d * hits, &l, 1);
  if (k.boundary == 1) saccept = saccept / ((double)(l.y - 1) / l.y + 1 / (double)l.y / 3);
  printf("accept %lf\n\n", saccept);
  printf("Energy ");
  refio_mean_variance(en, k.N, energy, 1);
  refio_autocorrelation(en, k.N, k.W, energy[0], energy[1], autoc);
  printf("Plaquette ");
  refio_mean_variance(en2, k.N, energy2, 1);
  refio_autocorrelation(en2, k.N, k.W, energy2[0], energy2[1], autoc2);
  if (k.save == 0) {
    if (refio_save_energy(k.outdir, energy[0], energy[1], Nterms, k.N, k.N_cor, saccept, &l, bound, k.nsave) ||
        refio_save_energy_av(k.outdir, energy[0], energy[1], energy2[0], energy2[1], Nterms, k.N, k.N_cor, saccept,
                             &l, bound, k.nsave) ||
        refio_save_en_seq(k.outdir, en2, en, Nterms, k.N, k.N_cor, 1, &l, bound, k.nsave) ||
        refio_save_autocorrelation(k.outdir, autoc, k.W, k.N, k.N_cor, Nterms, &l, bound, k.nsave, 0) ||
        refio_save_autocorrelation(k.outdir, autoc2, k.W, k.N, k.N_cor, Nterms, &l, bound, k.nsave, 1))
      exit(1);
  }
  if (k.report) {  // binned errors and tau_int, which the reference leaves to post-processing
    const double* s[2] = {en, en2};
    const char* name[2] = {"Energy", "Plaquette"};
    for (int j = 0; j < 2; j++) {
      double tau = 0, dtau = 0, bm = 0, be = 0;
      int w = 0;
      qcd_stats_tau_int(s[j], k.N, 6.0, &tau, &w, &dtau);
      int bin = (int)ceil(4 * tau) > 1 ? (int)ceil(4 * tau) : 1;
      if (k.N / bin < 2) bin = k.N / 2 > 0 ? k.N / 2 : 1;
      qcd_stats_binned(s[j], k.N, bin, &bm, &be);
      printf("report %s mean %.12f binned_error %.3e (bin %d) tau_int %.3f +- %.3f (W %d)\n", name[j], bm, be, bin,
             tau, dtau, w);
    }
  }
  qcd_destroy(h);
  free(phi);
  free(accepth);
  free(en);
  free(en2);
  free(autoc);
  free(autoc2);
  return 0;
}
