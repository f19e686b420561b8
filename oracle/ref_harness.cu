// Test-infrastructure harness around the REFERENCE's own CUDA kernels.
//
// This file is part of the oracle, not of the product.  It compiles the
// reference's headers where they lie (functions/su2.h, lattice_setup.h,
// mc_updates.h, mc_updates_pcc.h, mc_updates_pmc.h, observables.h of
// fezquerro/QCD_2d_GPU) through `-I <reference>/functions`; nothing of the
// reference is copied.  The recipe in oracle/Makefile writes the binary to
// oracle/_ref/ only.  It is the reference side of three checks:
//
//   tape   dump, per MRG32k3a stream `curand_init(seed, id, 0)`
//          (lattice_setup.h:15-21), the first K draws in both the float and
//          the double flavour, with the CUDA float transcendental values the
//          reference's heat-bath applies to a single draw (mc_updates.h:47-55).
//          The CPU restatement replays this tape instead of re-deriving cuRAND.
//   run    drive the reference's sweep kernels (mc_up_per/pcc/pmc,
//          mc_updates.h:467-475, mc_updates_pcc.h:216-224,
//          mc_updates_pmc.h:249-257) exactly as kernel.cu:162-208 does, and
//          dump the link field (reference AoS layout), the per-sweep energy
//          and plaquette of en_av (observables.h:99-141) and the accept array.
//   bench  time the reference's sweep with CUDA events (the reference arm of
//          the benchmark).
//
// kernel.cu's knobs are #defines without guards, so the harness cannot
// reuse its main(); it re-creates only the launch geometry (kernel.cu:66-70)
// and the call order (kernel.cu:79-208).  Both update algorithms are built
// into one binary by including the headers into two namespaces, because
// link_update selects the algorithm with `#if ALGO==HEATBATH`
// (mc_updates.h:119-128).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <time.h>
#include <algorithm>
#include <vector>
#include <string>
#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <curand.h>

#define METROPOLIS 0
#define HEATBATH 1

namespace ref_hb {
#define ALGO HEATBATH
#include "su2.h"
#include "lattice_setup.h"
#include "mc_updates.h"
#include "mc_updates_pcc.h"
#include "mc_updates_pmc.h"
#include "observables.h"
#include "statistics.h"
#include "output.h"
#undef ALGO
}  // namespace ref_hb

namespace ref_metro {
#define ALGO METROPOLIS
#include "su2.h"
#include "lattice_setup.h"
#include "mc_updates.h"
#include "mc_updates_pcc.h"
#include "mc_updates_pmc.h"
#include "observables.h"
#include "statistics.h"
#include "output.h"
#undef ALGO
}  // namespace ref_metro

#define CK(x)                                                                   \
  do {                                                                          \
    cudaError_t e_ = (x);                                                       \
    if (e_ != cudaSuccess) {                                                    \
      fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_),      \
              __FILE__, __LINE__);                                              \
      exit(3);                                                                  \
    }                                                                           \
  } while (0)

// ---------------------------------------------------------------- tape ----
// One record per draw; the float view and the double view of draw k come from
// two copies of the same state, and `same_step` says whether both calls left
// the generator in the same position (checked, never assumed).
struct TapeRec {
  double ud;        // curand_uniform_double
  float uf;         // curand_uniform
  float log_uf;     // logf(uf)                      (mc_updates.h:49)
  float cospi_2uf;  // cospif(2*uf)                  (mc_updates.h:48)
  float sc_sin;     // sincospif(2*uf) sine part     (mc_updates.h:55)
  float sc_cos;     // sincospif(2*uf) cosine part
  unsigned int same_step;
};

__global__ void tape_kernel(unsigned long long seed, long long first, int n_streams,
                            int n_draws, TapeRec* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_streams) return;
  curandStateMRG32k3a_t st;
  curand_init(seed, (unsigned long long)(first + i), 0, &st);
  for (int k = 0; k < n_draws; k++) {
    curandStateMRG32k3a_t cp = st;
    float f = curand_uniform(&cp);
    double d = curand_uniform_double(&st);
    unsigned int same = 1;
    for (int j = 0; j < 3; j++)
      same &= (cp.s1[j] == st.s1[j]) & (cp.s2[j] == st.s2[j]);
    TapeRec r;
    r.ud = d;
    r.uf = f;
    r.log_uf = logf(f);
    r.cospi_2uf = cospif(2 * f);
    float s, c;
    sincospif(2 * f, &s, &c);
    r.sc_sin = s;
    r.sc_cos = c;
    r.same_step = same;
    out[(size_t)i * n_draws + k] = r;
  }
}

// ---------------------------------------------------------------- args ----
struct Args {
  std::string mode = "run";
  int lt = 4, lx = 4, ly = 4;
  double beta = 6.0, eps = 0.2;
  int upd = 1;
  int algo = HEATBATH;  // 0 metropolis, 1 heat-bath, 2 over-relaxation (periodic only)
  int bc = 0;
  int hot = 0;
  long long seed = 1234;
  int sweeps = 10;
  int warmup = 3;
  std::vector<int> dumps;  // sweep counts after which the field is dumped
  int phase_dumps = 0;     // also dump after each of the 6 phases of sweep 1
  int measure = 1;
  std::string out = "ref";
  long long first = 0;
  int n_streams = 0, n_draws = 0;
  // knobs of kernel.cu's main (mode "main")
  int readconf = 0, sconf = 0, save = 0, N = 100, N_term = 10, N_block = 20, Nblock_term = 10, Nsave = 5,
      N_cor = 1, W = 10;
  std::string nsave = "1", nconfr = "1", nconfs = "1";
  std::string list;  // mode "batch": one replica per line "lt lx ly beta bc hot seed"
};

static void usage() {
  fprintf(stderr,
          "ref_harness tape|run|bench [--lt N --lx N --ly N --beta B --eps E "
          "--upd U --algo hb|metro|or --bc 0|1|2 --hot 0|1 --seed S --sweeps K "
          "--warmup W --dumps a,b,c --phase-dumps 0|1 --measure 0|1 --out PREFIX "
          "--first F --streams N --draws D] [main: --readconf --sconf --save --N --N-term --N-block "
          "--Nblock-term --Nsave --N-cor --W --nsave --nconfr --nconfs]\n");
  exit(2);
}

static Args parse(int argc, char** argv) {
  Args a;
  if (argc < 2) usage();
  a.mode = argv[1];
  for (int i = 2; i < argc; i++) {
    std::string k = argv[i];
    if (i + 1 >= argc) usage();
    const char* v = argv[++i];
    if (k == "--lt") a.lt = atoi(v);
    else if (k == "--lx") a.lx = atoi(v);
    else if (k == "--ly") a.ly = atoi(v);
    else if (k == "--beta") a.beta = atof(v);
    else if (k == "--eps") a.eps = atof(v);
    else if (k == "--upd") a.upd = atoi(v);
    else if (k == "--algo") {
      std::string s = v;
      a.algo = s == "hb" ? HEATBATH : s == "metro" ? METROPOLIS : s == "or" ? 2 : -1;
      if (a.algo < 0) usage();
    } else if (k == "--bc") a.bc = atoi(v);
    else if (k == "--hot") a.hot = atoi(v);
    else if (k == "--seed") a.seed = atoll(v);
    else if (k == "--sweeps") a.sweeps = atoi(v);
    else if (k == "--warmup") a.warmup = atoi(v);
    else if (k == "--dumps") {
      std::string s = v;
      size_t p = 0;
      while (p < s.size()) {
        size_t q = s.find(',', p);
        if (q == std::string::npos) q = s.size();
        a.dumps.push_back(atoi(s.substr(p, q - p).c_str()));
        p = q + 1;
      }
    } else if (k == "--phase-dumps") a.phase_dumps = atoi(v);
    else if (k == "--measure") a.measure = atoi(v);
    else if (k == "--out") a.out = v;
    else if (k == "--first") a.first = atoll(v);
    else if (k == "--streams") a.n_streams = atoi(v);
    else if (k == "--draws") a.n_draws = atoi(v);
    else if (k == "--readconf") a.readconf = atoi(v);
    else if (k == "--sconf") a.sconf = atoi(v);
    else if (k == "--save") a.save = atoi(v);
    else if (k == "--N") a.N = atoi(v);
    else if (k == "--N-term") a.N_term = atoi(v);
    else if (k == "--N-block") a.N_block = atoi(v);
    else if (k == "--Nblock-term") a.Nblock_term = atoi(v);
    else if (k == "--Nsave") a.Nsave = atoi(v);
    else if (k == "--N-cor") a.N_cor = atoi(v);
    else if (k == "--W") a.W = atoi(v);
    else if (k == "--nsave") a.nsave = v;
    else if (k == "--nconfr") a.nconfr = v;
    else if (k == "--nconfs") a.nconfs = v;
    else if (k == "--list") a.list = v;
    else usage();
  }
  return a;
}

static void write_file(const std::string& name, const void* p, size_t bytes) {
  FILE* f = fopen(name.c_str(), "wb");
  if (!f) {
    fprintf(stderr, "cannot write %s\n", name.c_str());
    exit(4);
  }
  if (fwrite(p, 1, bytes, f) != bytes) {
    fprintf(stderr, "short write %s\n", name.c_str());
    exit(4);
  }
  fclose(f);
}

// ---------------------------------------------------------------- run -----
// The reference's types and kernels are identical in both namespaces except
// for link_update; the macro instantiates one driver per namespace.
#define DEFINE_DRIVER(NS)                                                               \
  static void NS##_phase(int k, int bc, int upd_flag, int nb, int nt, double* phi,      \
                         curandStateMRG32k3a_t* st, int* acc, NS::lattice l2) {         \
    /* call order of mc_up_per/pcc/pmc (mc_updates.h:467-475,                        */ \
    /* mc_updates_pcc.h:216-224, mc_updates_pmc.h:249-257)                          */ \
    switch (k) {                                                                        \
      case 0: NS::MC_update_even_y<<<nb, nt>>>(phi, st, acc, l2, upd_flag); break;      \
      case 1: NS::MC_update_odd_y<<<nb, nt>>>(phi, st, acc, l2, upd_flag); break;       \
      case 2:                                                                           \
        if (bc == 0) NS::MC_update_even_x<<<nb, nt>>>(phi, st, acc, l2, upd_flag);      \
        else if (bc == 1) NS::MC_update_even_x_pcc<<<nb, nt>>>(phi, st, acc, l2);       \
        else NS::MC_update_even_x_pmc<<<nb, nt>>>(phi, st, acc, l2);                    \
        break;                                                                          \
      case 3:                                                                           \
        if (bc == 0) NS::MC_update_odd_x<<<nb, nt>>>(phi, st, acc, l2, upd_flag);       \
        else if (bc == 1) NS::MC_update_odd_x_pcc<<<nb, nt>>>(phi, st, acc, l2);        \
        else NS::MC_update_odd_x_pmc<<<nb, nt>>>(phi, st, acc, l2);                     \
        break;                                                                          \
      case 4:                                                                           \
        if (bc == 0) NS::MC_update_even_t<<<nb, nt>>>(phi, st, acc, l2, upd_flag);      \
        else if (bc == 1) NS::MC_update_even_t_pcc<<<nb, nt>>>(phi, st, acc, l2);       \
        else NS::MC_update_even_t_pmc<<<nb, nt>>>(phi, st, acc, l2);                    \
        break;                                                                          \
      case 5:                                                                           \
        if (bc == 0) NS::MC_update_odd_t<<<nb, nt>>>(phi, st, acc, l2, upd_flag);       \
        else if (bc == 1) NS::MC_update_odd_t_pcc<<<nb, nt>>>(phi, st, acc, l2);        \
        else NS::MC_update_odd_t_pmc<<<nb, nt>>>(phi, st, acc, l2);                     \
        break;                                                                          \
    }                                                                                   \
  }                                                                                     \
  static void NS##_sweep(int bc, int upd_flag, int nblocks, int nt, double* phi,        \
                         curandStateMRG32k3a_t* st, int* acc, NS::lattice l2) {         \
    if (bc == 0) NS::mc_up_per(nt, nblocks, phi, l2, acc, st, upd_flag);                \
    else if (bc == 1) NS::mc_up_pcc(nt, nblocks, phi, l2, acc, st);                     \
    else NS::mc_up_pmc(nt, nblocks, phi, l2, acc, st);                                  \
  }                                                                                     \
  static int NS##_main(const Args& a) {                                                 \
    /* lattice structs as kernel.cu:58-59 */                                            \
    NS::lattice l = {a.ly, a.lx, a.lt, a.ly * a.lx * a.lt, 3, 4, 12, (float)a.beta,     \
                     (float)a.eps, a.upd};                                              \
    NS::lattice l2 = {l.y / 2, l.x, l.t, l.V / 2, 3, 4, 12, l.beta, l.epsilon, a.upd};  \
    if (l.t % 2 || l.x % 2 || l.y % 2) {                                                \
      fprintf(stderr, "Lt, Lx and Ly must be even\n");                                  \
      return 1;                                                                         \
    }                                                                                   \
    if (a.algo == 2 && a.bc != 0) {                                                     \
      fprintf(stderr, "the reference has over-relaxation for periodic BC only\n");      \
      return 1;                                                                         \
    }                                                                                   \
    int nthreads = 256; /* kernel.cu:66-70 */                                           \
    while (l2.V % nthreads != 0) nthreads--;                                            \
    int nblocks = 2 * (l2.V / nthreads);                                                \
    int upd_flag = a.algo == 2 ? 1 : 0;                                                 \
    curandStateMRG32k3a_t* st;                                                          \
    CK(cudaMalloc((void**)&st, (size_t)l2.V * sizeof(curandStateMRG32k3a_t)));          \
    NS::setup_kernel<<<nblocks / 2, nthreads>>>(st, (int)a.seed);                       \
    size_t nphi = (size_t)l.V * l.dt;                                                   \
    std::vector<double> phi(nphi);                                                      \
    double* phid;                                                                       \
    CK(cudaMalloc(&phid, nphi * sizeof(double)));                                       \
    if (a.hot) {                                                                        \
      if (a.bc == 1) NS::rand_init2_pcc<<<nblocks / 2, nthreads>>>(phid, st, l2);       \
      else NS::rand_init2<<<nblocks / 2, nthreads>>>(phid, st, l2);                     \
    } else {                                                                            \
      NS::id_init2<<<nblocks / 2, nthreads>>>(phid, l2);                                \
    }                                                                                   \
    int* acc;                                                                           \
    CK(cudaMalloc(&acc, (size_t)l.V * sizeof(int)));                                    \
    CK(cudaMemset(acc, 0, (size_t)l.V * sizeof(int)));                                  \
    double *end, *end2;                                                                 \
    int nmeas = a.sweeps > 0 ? a.sweeps : 1;                                            \
    CK(cudaMalloc(&end, nmeas * sizeof(double)));                                       \
    CK(cudaMalloc(&end2, nmeas * sizeof(double)));                                      \
    CK(cudaMemset(end, 0, nmeas * sizeof(double)));                                     \
    CK(cudaMemset(end2, 0, nmeas * sizeof(double)));                                    \
    CK(cudaDeviceSynchronize());                                                        \
    if (a.mode == "bench") {                                                            \
      for (int i = 0; i < a.warmup; i++)                                                \
        NS##_sweep(a.bc, upd_flag, nblocks, nthreads, phid, st, acc, l2);               \
      cudaEvent_t e0, e1;                                                               \
      CK(cudaEventCreate(&e0));                                                         \
      CK(cudaEventCreate(&e1));                                                         \
      CK(cudaDeviceSynchronize());                                                      \
      CK(cudaEventRecord(e0));                                                          \
      for (int i = 0; i < a.sweeps; i++)                                                \
        NS##_sweep(a.bc, upd_flag, nblocks, nthreads, phid, st, acc, l2);               \
      CK(cudaEventRecord(e1));                                                          \
      CK(cudaEventSynchronize(e1));                                                     \
      CK(cudaGetLastError());                                                           \
      float ms = 0;                                                                     \
      CK(cudaEventElapsedTime(&ms, e0, e1));                                            \
      /* one en_av measurement timed alone (observables.h:99-141) */                    \
      cudaEvent_t m0, m1;                                                               \
      CK(cudaEventCreate(&m0));                                                         \
      CK(cudaEventCreate(&m1));                                                         \
      CK(cudaEventRecord(m0));                                                          \
      if (a.bc == 2) NS::en_av<1><<<nblocks, nthreads>>>(phid, end, end2, l2);          \
      else NS::en_av<0><<<nblocks, nthreads>>>(phid, end, end2, l2);                    \
      CK(cudaEventRecord(m1));                                                          \
      CK(cudaEventSynchronize(m1));                                                     \
      float mms = 0;                                                                    \
      CK(cudaEventElapsedTime(&mms, m0, m1));                                           \
      double ups = 3.0 * l.V * a.sweeps / (ms * 1e-3);                                  \
      printf("{\"ms_total\": %.6f, \"ms_per_sweep\": %.6f, \"ms_measure\": %.6f, "      \
             "\"link_updates_per_s\": %.6e, \"V\": %d, \"sweeps\": %d, "               \
             "\"nthreads\": %d, \"nblocks\": %d}\n",                                    \
             ms, ms / a.sweeps, mms, ups, l.V, a.sweeps, nthreads, nblocks);            \
      return 0;                                                                         \
    }                                                                                   \
    std::vector<double> E(nmeas, 0.0), P(nmeas, 0.0);                                   \
    for (int d : a.dumps)                                                               \
      if (d == 0) {                                                                     \
        CK(cudaMemcpy(phi.data(), phid, nphi * 8, cudaMemcpyDeviceToHost));             \
        write_file(a.out + "_field_0.bin", phi.data(), nphi * 8);                       \
      }                                                                                 \
    for (int i = 1; i <= a.sweeps; i++) {                                               \
      if (i == 1 && a.phase_dumps) {                                                    \
        for (int k = 0; k < 6; k++) {                                                   \
          NS##_phase(k, a.bc, upd_flag, nblocks / 2, nthreads, phid, st, acc, l2);      \
          CK(cudaDeviceSynchronize());                                                  \
          CK(cudaMemcpy(phi.data(), phid, nphi * 8, cudaMemcpyDeviceToHost));           \
          write_file(a.out + "_phase_" + std::to_string(k + 1) + ".bin", phi.data(),     \
                     nphi * 8);                                                         \
        }                                                                               \
      } else {                                                                          \
        NS##_sweep(a.bc, upd_flag, nblocks, nthreads, phid, st, acc, l2);               \
      }                                                                                 \
      if (a.measure) {                                                                  \
        if (a.bc == 2) NS::en_av<1><<<nblocks, nthreads>>>(phid, end + i - 1, end2 + i - 1, l2); \
        else NS::en_av<0><<<nblocks, nthreads>>>(phid, end + i - 1, end2 + i - 1, l2);  \
      }                                                                                 \
      for (int d : a.dumps)                                                             \
        if (d == i) {                                                                   \
          CK(cudaMemcpy(phi.data(), phid, nphi * 8, cudaMemcpyDeviceToHost));           \
          write_file(a.out + "_field_" + std::to_string(i) + ".bin", phi.data(),        \
                     nphi * 8);                                                         \
        }                                                                               \
    }                                                                                   \
    CK(cudaDeviceSynchronize());                                                        \
    CK(cudaGetLastError());                                                             \
    if (a.measure) {                                                                    \
      CK(cudaMemcpy(E.data(), end, nmeas * 8, cudaMemcpyDeviceToHost));                 \
      CK(cudaMemcpy(P.data(), end2, nmeas * 8, cudaMemcpyDeviceToHost));                \
      std::vector<double> EP(2 * (size_t)a.sweeps);                                     \
      for (int i = 0; i < a.sweeps; i++) {                                              \
        EP[2 * i] = E[i];                                                               \
        EP[2 * i + 1] = P[i];                                                           \
      }                                                                                 \
      write_file(a.out + "_obs.bin", EP.data(), EP.size() * 8);                         \
    }                                                                                   \
    std::vector<int> acch(l.V);                                                         \
    CK(cudaMemcpy(acch.data(), acc, (size_t)l.V * 4, cudaMemcpyDeviceToHost));          \
    write_file(a.out + "_accept.bin", acch.data(), (size_t)l.V * 4);                    \
    printf("{\"ok\": 1, \"V\": %d, \"sweeps\": %d, \"E_last\": %.17g, \"P_last\": %.17g}\n", \
           l.V, a.sweeps, a.sweeps ? E[a.sweeps - 1] : 0.0, a.sweeps ? P[a.sweeps - 1] : 0.0); \
    cudaFree(st); cudaFree(phid); cudaFree(acc); cudaFree(end); cudaFree(end2);         \
    return 0;                                                                           \
  }

DEFINE_DRIVER(ref_hb)
DEFINE_DRIVER(ref_metro)

// kernel.cu:49-268 with the knobs at run time: the same calls, in the same
// order, to the reference's own functions (setup, starts, mc_up_*, normalize,
// en_av, mean_variance, autocorrelation, mean_lattice, save_*, read_conf,
// save_conf, print_det); output files land in the working directory.
#define DEFINE_MAIN(NS)                                                                      \
  static int NS##_kernel_main(const Args& a) {                                               \
    char nsave[16], nconfr[16], nconfs[16];                                                   \
    snprintf(nsave, sizeof nsave, "%s", a.nsave.c_str());                                     \
    snprintf(nconfr, sizeof nconfr, "%s", a.nconfr.c_str());                                  \
    snprintf(nconfs, sizeof nconfs, "%s", a.nconfs.c_str());                                  \
    int Nterms = 0, inits;                                                                    \
    NS::lattice l = {a.ly, a.lx, a.lt, a.ly * a.lx * a.lt, 3, 4, 12, (float)a.beta,           \
                     (float)a.eps, a.upd};                                                    \
    NS::lattice l2 = {l.y / 2, l.x, l.t, l.V / 2, 3, 4, 12, l.beta, l.epsilon, a.upd};        \
    printf("N %d Lt %d L %d Ly %d V %d Dim %d DimRep %d Dimtot %d \n", a.N, l.t, l.x, l.y,    \
           l.V, l.d, l.dg, l.dt);                                                             \
    if (l.t % 2 || l.x % 2 || l.y % 2) {                                                      \
      printf("Lt, Lx and Ly must be even\n");                                                 \
      return 1;                                                                               \
    }                                                                                         \
    int nblocks, nthreads = 256;                                                              \
    while (l2.V % nthreads != 0) nthreads--;                                                  \
    nblocks = 2 * (l2.V / nthreads);                                                          \
    printf("nblocks %d nthreads %d\n", nblocks, nthreads);                                    \
    if (a.algo == METROPOLIS)                                                                 \
      printf("METROPOLIS UPDATES epsilon %.2f hits %d\n", l.epsilon, l.updates);              \
    if (a.algo == HEATBATH) printf("HEAT-BATH UPDATES\n");                                    \
    int hits = (a.algo == METROPOLIS) ? l.updates : 1;                                        \
    curandStateMRG32k3a_t* devStates;                                                         \
    CK(cudaMalloc((void**)&devStates, l2.V * sizeof(curandStateMRG32k3a_t)));                 \
    NS::setup_kernel<<<nblocks / 2, nthreads>>>(devStates, (int)a.seed);                      \
    double *phi = (double*)malloc(l.V * l.dt * sizeof(double)), *phid;                        \
    CK(cudaMalloc(&phid, l.V * l.dt * sizeof(double)));                                       \
    char bound[12];                                                                           \
    snprintf(bound, sizeof bound, "%s", a.bc == 0 ? "per" : a.bc == 1 ? "pcc" : "pmc");       \
    if (a.bc == 0) printf("PERIODIC BOUNDARY CONDITIONS\n\n");                                \
    else if (a.bc == 1) printf("PERFECT COLOUR CONDUCTOR BOUNDARY CONDITIONS\n\n");           \
    else printf("PERFECT MAGNETIC CONDUCTOR BOUNDARY CONDITIONS\n\n");                         \
    if (a.readconf == 0) {                                                                    \
      inits = a.hot ? 0 : 1;                                                                  \
      if (a.hot) {                                                                            \
        if (a.bc == 1) NS::rand_init2_pcc<<<nblocks / 2, nthreads>>>(phid, devStates, l2);    \
        else NS::rand_init2<<<nblocks / 2, nthreads>>>(phid, devStates, l2);                  \
      } else {                                                                                \
        NS::id_init2<<<nblocks / 2, nthreads>>>(phid, l2);                                    \
      }                                                                                       \
    } else {                                                                                  \
      NS::read_conf(phi, l, &Nterms, &inits, bound, nconfr);                                  \
      CK(cudaMemcpy(phid, phi, l.V * l.dt * sizeof(double), cudaMemcpyHostToDevice));         \
    }                                                                                         \
    CK(cudaMemcpy(phi, phid, l.V * l.dt * sizeof(double), cudaMemcpyDeviceToHost));           \
    NS::print_det(phi, l);                                                                    \
    int *accept, *accepth = (int*)malloc(l.V * sizeof(int));                                  \
    CK(cudaMalloc(&accept, l.V * sizeof(int)));                                               \
    CK(cudaMemset(accept, 0, l.V * sizeof(int)));                                             \
    double *end, *en = (double*)malloc(a.N * sizeof(double));                                 \
    CK(cudaMalloc(&end, a.N * sizeof(double)));                                               \
    CK(cudaMemset(end, 0, a.N * sizeof(double)));                                             \
    double *end2, *en2 = (double*)malloc(a.N * sizeof(double));                               \
    CK(cudaMalloc(&end2, a.N * sizeof(double)));                                              \
    CK(cudaMemset(end2, 0, a.N * sizeof(double)));                                            \
    int i, j;                                                                                 \
    int t_ini, t_ini_mc, t_fin, t_n, block_size_t = a.N_term / a.Nblock_term,                 \
        block_size = a.N / a.N_block, block_s_size = a.N / a.Nsave;                           \
    t_ini = time(NULL);                                                                       \
    t_n = time(NULL);                                                                         \
    double energy[2], energy2[2];                                                             \
    std::vector<double> autoc(a.W), autoc2(a.W);                                              \
    double saccept;                                                                           \
    if (a.readconf < 2) {                                                                     \
      for (i = 1; i < a.N_term + 1; i++) {                                                    \
        if (i % 100 == 0) NS::normalize<<<nblocks, nthreads>>>(phid, l);                      \
        NS##_sweep(a.bc, 0, nblocks, nthreads, phid, devStates, accept, l2);                  \
        if (block_size_t > 0 && i % block_size_t == 0) {                                      \
          printf("%lf Time %d Left(min)%lf\n", (double)i / (a.N_term), (int)(time(NULL) - t_n), \
                 (double)(time(NULL) - t_ini) * (a.N_term - i) / i / 60);                     \
          fflush(stdout);                                                                     \
          t_n = time(NULL);                                                                   \
        }                                                                                     \
      }                                                                                       \
      NS::normalize<<<nblocks, nthreads>>>(phid, l);                                          \
      Nterms = a.N_term + Nterms;                                                             \
      if (a.sconf == 0) {                                                                     \
        CK(cudaMemcpy(phi, phid, l.V * l.dt * sizeof(double), cudaMemcpyDeviceToHost));       \
        NS::save_conf(phi, l, Nterms, inits, bound, nconfs);                                  \
      }                                                                                       \
    }                                                                                         \
    CK(cudaMemcpy(phi, phid, l.V * l.dt * sizeof(double), cudaMemcpyDeviceToHost));           \
    NS::print_det(phi, l);                                                                    \
    CK(cudaMemset(accept, 0, l.V * sizeof(int)));                                             \
    t_ini_mc = time(NULL);                                                                    \
    t_n = time(NULL);                                                                         \
    for (i = 1; i < a.N + 1; i++) {                                                           \
      for (j = 0; j < a.N_cor; j++) NS##_sweep(a.bc, 0, nblocks, nthreads, phid, devStates, accept, l2); \
      if (i % 100 == 0) NS::normalize<<<nblocks, nthreads>>>(phid, l);                        \
      if (a.bc == 2) NS::en_av<1><<<nblocks, nthreads>>>(phid, end + i - 1, end2 + i - 1, l2); \
      else NS::en_av<0><<<nblocks, nthreads>>>(phid, end + i - 1, end2 + i - 1, l2);          \
      if (block_size > 0 && i % block_size == 0) {                                            \
        printf("%lf Time %d Left(min)%lf\n", (double)i / a.N, (int)(time(NULL) - t_n),       \
               (double)(time(NULL) - t_ini_mc) * (a.N - i) / i / 60);                         \
        t_n = time(NULL);                                                                     \
        fflush(stdout);                                                                       \
      }                                                                                       \
      if (block_s_size > 0 && i % block_s_size == 0) {                                        \
        CK(cudaMemcpy(en, end, i * sizeof(double), cudaMemcpyDeviceToHost));                  \
        CK(cudaMemcpy(en2, end2, i * sizeof(double), cudaMemcpyDeviceToHost));                \
        printf("Energy ");                                                                    \
        NS::mean_variance(en, i, energy, true);                                               \
        NS::autocorrelation(en, i, a.W, energy[0], energy[1], autoc.data());                  \
        printf("Plaquette ");                                                                 \
        NS::mean_variance(en2, i, energy2, true);                                             \
        NS::autocorrelation(en2, i, a.W, energy2[0], energy2[1], autoc2.data());              \
        fflush(stdout);                                                                       \
        if (a.save == 0) {                                                                    \
          saccept = NS::mean_lattice(accept, accepth, i * a.N_cor * l.d * hits, l, false);    \
          if (a.bc == 1) saccept = saccept / ((double)(l.y - 1) / l.y + 1 / (double)l.y / 3); \
          NS::save_energy(energy[0], energy[1], Nterms, a.N, a.N_cor, saccept, l, bound, nsave); \
          NS::save_energy_av(energy[0], energy[1], energy2[0], energy2[1], Nterms, a.N, a.N_cor, \
                             saccept, l, bound, nsave);                                       \
          NS::save_autocorrelation(autoc.data(), a.W, i, a.N_cor, Nterms, l, bound, nsave);   \
          NS::save_autocorrelation_av(autoc2.data(), a.W, i, a.N_cor, Nterms, l, bound, nsave); \
          NS::save_en_seq(en2, en, Nterms, i, a.N_cor, 1, l, bound, nsave);                   \
        }                                                                                     \
      }                                                                                       \
    }                                                                                         \
    t_fin = time(NULL);                                                                       \
    printf("Time %d\n", t_fin - t_ini);                                                       \
    CK(cudaMemcpy(en, end, a.N * sizeof(double), cudaMemcpyDeviceToHost));                    \
    CK(cudaMemcpy(en2, end2, a.N * sizeof(double), cudaMemcpyDeviceToHost));                  \
    saccept = NS::mean_lattice(accept, accepth, a.N * a.N_cor * l.d * hits, l, true);         \
    if (a.bc == 1) saccept = saccept / ((double)(l.y - 1) / l.y + 1 / (double)l.y / 3);       \
    printf("accept %lf\n\n", saccept);                                                        \
    printf("Energy ");                                                                        \
    NS::mean_variance(en, a.N, energy, true);                                                 \
    NS::autocorrelation(en, a.N, a.W, energy[0], energy[1], autoc.data());                    \
    printf("Plaquette ");                                                                     \
    NS::mean_variance(en2, a.N, energy2, true);                                               \
    NS::autocorrelation(en2, a.N, a.W, energy2[0], energy2[1], autoc2.data());                \
    if (a.save == 0) {                                                                        \
      NS::save_energy(energy[0], energy[1], Nterms, a.N, a.N_cor, saccept, l, bound, nsave);  \
      NS::save_energy_av(energy[0], energy[1], energy2[0], energy2[1], Nterms, a.N, a.N_cor,  \
                         saccept, l, bound, nsave);                                           \
      NS::save_en_seq(en2, en, Nterms, a.N, a.N_cor, 1, l, bound, nsave);                     \
      NS::save_autocorrelation(autoc.data(), a.W, a.N, a.N_cor, Nterms, l, bound, nsave);     \
      NS::save_autocorrelation_av(autoc2.data(), a.W, a.N, a.N_cor, Nterms, l, bound, nsave); \
    }                                                                                         \
    CK(cudaGetLastError());                                                                   \
    free(phi); free(accepth); cudaFree(phid); cudaFree(accept); cudaFree(devStates);          \
    free(en); free(en2); cudaFree(end); cudaFree(end2);                                       \
    return 0;                                                                                 \
  }

DEFINE_MAIN(ref_hb)
DEFINE_MAIN(ref_metro)



// Mode "batch": the replicas of a list run one after the other, each exactly
// as one run of the reference program would run it (setup_kernel, start,
// `sweeps` x (mc_up_* + en_av)), timed on the device from the first replica's
// setup to the last replica's last measurement (allocation excluded).
static int batch_main(const Args& a) {
  FILE* f = fopen(a.list.c_str(), "r");
  if (!f) {
    fprintf(stderr, "cannot read %s\n", a.list.c_str());
    return 2;
  }
  struct Rep { int lt, lx, ly, bc, hot; double beta; long long seed; };
  std::vector<Rep> reps;
  Rep r;
  while (fscanf(f, "%d %d %d %lf %d %d %lld", &r.lt, &r.lx, &r.ly, &r.beta, &r.bc, &r.hot, &r.seed) == 7)
    reps.push_back(r);
  fclose(f);
  size_t max_v = 0;
  for (const Rep& x : reps) max_v = std::max(max_v, (size_t)x.lt * x.lx * x.ly);
  curandStateMRG32k3a_t* st;
  double *phid, *end, *end2;
  int* acc;
  CK(cudaMalloc((void**)&st, max_v / 2 * sizeof(curandStateMRG32k3a_t)));
  CK(cudaMalloc(&phid, max_v * 12 * sizeof(double)));
  CK(cudaMalloc(&acc, max_v * sizeof(int)));
  CK(cudaMalloc(&end, a.sweeps * sizeof(double)));
  CK(cudaMalloc(&end2, a.sweeps * sizeof(double)));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  double sites = 0;
  CK(cudaDeviceSynchronize());
  CK(cudaEventRecord(e0));
  for (const Rep& x : reps) {
    ref_hb::lattice l2 = {x.ly / 2, x.lx, x.lt, x.lt * x.lx * x.ly / 2, 3, 4, 12, (float)x.beta, (float)a.eps, a.upd};
    int nthreads = 256;  // kernel.cu:66-70
    while (l2.V % nthreads != 0) nthreads--;
    int nblocks = 2 * (l2.V / nthreads);
    ref_hb::setup_kernel<<<nblocks / 2, nthreads>>>(st, (int)x.seed);
    if (x.hot) {
      if (x.bc == 1) ref_hb::rand_init2_pcc<<<nblocks / 2, nthreads>>>(phid, st, l2);
      else ref_hb::rand_init2<<<nblocks / 2, nthreads>>>(phid, st, l2);
    } else {
      ref_hb::id_init2<<<nblocks / 2, nthreads>>>(phid, l2);
    }
    CK(cudaMemsetAsync(end, 0, a.sweeps * sizeof(double)));
    CK(cudaMemsetAsync(end2, 0, a.sweeps * sizeof(double)));
    for (int i = 0; i < a.sweeps; i++) {
      ref_hb_sweep(x.bc, 0, nblocks, nthreads, phid, st, acc, l2);
      if (x.bc == 2) ref_hb::en_av<1><<<nblocks, nthreads>>>(phid, end + i, end2 + i, l2);
      else ref_hb::en_av<0><<<nblocks, nthreads>>>(phid, end + i, end2 + i, l2);
    }
    sites += 2.0 * l2.V;
  }
  CK(cudaEventRecord(e1));
  CK(cudaEventSynchronize(e1));
  CK(cudaGetLastError());
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  printf("{\"ms_total\": %.6f, \"replicas\": %zu, \"sweeps\": %d, \"sites\": %.0f, \"replicas_per_s\": %.6e, "
         "\"link_updates_per_s\": %.6e}\n",
         ms, reps.size(), a.sweeps, sites, reps.size() / (ms * 1e-3), 3.0 * sites * a.sweeps / (ms * 1e-3));
  return 0;
}

int main(int argc, char** argv) {
  Args a = parse(argc, argv);
  if (a.mode == "tape") {
    if (a.n_streams <= 0 || a.n_draws <= 0) usage();
    TapeRec* d;
    size_t n = (size_t)a.n_streams * a.n_draws;
    CK(cudaMalloc(&d, n * sizeof(TapeRec)));
    tape_kernel<<<(a.n_streams + 127) / 128, 128>>>((unsigned long long)a.seed, a.first,
                                                    a.n_streams, a.n_draws, d);
    CK(cudaGetLastError());
    std::vector<TapeRec> h(n);
    CK(cudaMemcpy(h.data(), d, n * sizeof(TapeRec), cudaMemcpyDeviceToHost));
    size_t bad = 0;
    for (size_t i = 0; i < n; i++) bad += h[i].same_step ? 0 : 1;
    write_file(a.out + "_tape.bin", h.data(), n * sizeof(TapeRec));
    printf("{\"ok\": 1, \"records\": %zu, \"record_bytes\": %zu, \"steps_differ\": %zu}\n", n,
           sizeof(TapeRec), bad);
    cudaFree(d);
    return 0;
  }
  if (a.mode == "batch") return batch_main(a);
  if (a.mode == "main") return a.algo == METROPOLIS ? ref_metro_kernel_main(a) : ref_hb_kernel_main(a);
  if (a.mode != "run" && a.mode != "bench") usage();
  // over-relaxation (update==1) and heat-bath share the HEATBATH namespace: the
  // `update` flag bypasses link_update (mc_updates.h:178-181).
  if (a.algo == METROPOLIS) return ref_metro_main(a);
  return ref_hb_main(a);
}
