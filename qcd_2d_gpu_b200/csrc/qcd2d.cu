// Host side of the C ABI declared in include/qcd2d.h.
//
// A qcd_lattice owns its device buffers and one CUDA stream.  Every CUDA call
// is checked; failures come back as qcd_status codes with a message in
// qcd_last_error (the reference checks none, kernel.cu:77-151).
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <mutex>
#include <new>
#include <vector>
#include "kernels.cuh"
#include "paired.cuh"
#include "pairs.h"
#include "qcd2d.h"
#include "wave.cuh"

using namespace qcd;

struct qcd_lattice {
  qcd_params p;
  Geo g;
  long long V;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  // link store
  double2* lo = nullptr;
  double2* hi = nullptr;
  float4* q32 = nullptr;     // FP32 store holding the current links
  float4* q32alt = nullptr;  // second FP32 store: the fused-pair schedule writes each pass's new links here
  size_t link_bytes = 0;
  // FP32 store in site pairs (paired.cuh): FP32 lattices with Lt % 4 == 0 under
  // the per-phase schedule; gh is the half geometry whose t-slices are its rows
  bool paired = false;
  bool pair_ok = true;  // qcd_set_pair_layout: pairs allowed
  Geo gh;
  // MRG32k3a streams, 6 u32 planes, and the jump matrices that seed them
  uint32_t* rng = nullptr;
  uint32_t* mrg_jumps = nullptr;
  // Metropolis accept counters (V ints) and analytic unit counts for HB/OR
  int* accept = nullptr;
  long long unit_passes = 0;  // HB/OR passes since the last reset
  // reductions
  double2* partials = nullptr;
  unsigned int* counter = nullptr;
  double* result = nullptr;      // 2 doubles on the device
  double* result_host = nullptr; // pinned
  int* err = nullptr;            // device error word
  // measurement series
  double* series = nullptr;
  int series_cap = 0;
  // conversion staging for host configs
  double* aos_stage = nullptr;
  long long sweeps_done = 0;
  // drawing phases run so far (6 per heat-bath or Metropolis pass), on the
  // device: the counter of the FP32 Philox draws, part of the generator
  // checkpoint
  unsigned long long* draw_dev = nullptr;
  unsigned long long draw_key = 0;  // key of the FP32 draws: the seed, or the one a checkpoint restored
  // wavefront scheduler
  int sched = QCD_SCHED_AUTO;
  unsigned int* wave_done = nullptr;   // Lt arrival counters
  unsigned int* wave_queue = nullptr;  // ticket counter
  int* wave_abort = nullptr;
  int wave_grid = 0;                   // persistent CTAs (all SMs x occupancy)
  int wave_chain = 0;                  // passes chained per launch (0: not planned yet)
  int wave_chunk = 256;                // sites per wavefront task
  int wave_fronts = 1;                 // ring fronts (arcs of Lt / fronts slices)
  unsigned int* wave_tasks[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // per chain length
  int wave_tasks_chunk[5] = {0, 0, 0, 0, 0};
  int wave_tasks_fronts[5] = {0, 0, 0, 0, 0};
  int sms = 0;       // multiprocessors of the device (fused pairs)
  // fused pairs: the two FP32 stores and their tensor maps (pair_buf[0] is
  // the store allocated at create; q32 / q32alt point at one each)
  float4* pair_buf[2] = {nullptr, nullptr};
  PairMaps pair_maps[2];
  int pair_seg = 0;  // fused pairs: streamed slices per CTA (0: automatic)
  char msg[512] = {0};
};

namespace {

int fail(qcd_lattice* h, int code, const char* fmt, ...) {
  if (h) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(h->msg, sizeof(h->msg), fmt, ap);
    va_end(ap);
  }
  return code;
}

#define CUDA_OR_FAIL(h, call)                                                                 \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) {                                                                  \
      if (e_ == cudaErrorMemoryAllocation) {                                                  \
        cudaGetLastError();                                                                   \
        return fail(h, QCD_ERR_NOMEM, "%s: %s", #call, cudaGetErrorString(e_));               \
      }                                                                                       \
      return fail(h, QCD_ERR_CUDA, "%s (%s:%d): %s", #call, __FILE__, __LINE__,               \
                  cudaGetErrorString(e_));                                                    \
    }                                                                                         \
  } while (0)

#define LAUNCH_CHECK(h) CUDA_OR_FAIL(h, cudaGetLastError())

inline unsigned int nblocks(long long n) { return (unsigned int)((n + kBlock - 1) / kBlock); }

Links64 links64(const qcd_lattice* h) { return Links64{h->lo, h->hi, h->g.vh}; }
Links32 links32(const qcd_lattice* h) { return Links32{h->q32, h->g.vh}; }
Pair32 pair32(const qcd_lattice* h) { return Pair32{h->q32, h->g.vh / 2}; }
bool pairable(const qcd_lattice* h) { return h->p.precision == QCD_PREC_FP32 && h->g.lt % 4 == 0; }
RngStore rngs(const qcd_lattice* h) { return RngStore{h->rng, h->g.vh}; }

// ------------------------------------------------------------ dispatch --
typedef void (*Phase64Fn)(Links64, RngStore, Geo, PhaseArgs);
typedef void (*Phase32Fn)(Links32, RngStore, Geo, PhaseArgs);

template <int MU, int PAR, int BC>
Phase64Fn pick64(int kind) {
  switch (kind) {
    case KIND_METRO: return phase64<MU, PAR, BC, KIND_METRO>;
    case KIND_HB: return phase64<MU, PAR, BC, KIND_HB>;
    default: return phase64<MU, PAR, BC, KIND_OR>;
  }
}
template <int MU, int PAR, int BC>
Phase32Fn pick32(int kind) {
  switch (kind) {
    case KIND_METRO: return phase32<MU, PAR, BC, KIND_METRO>;
    case KIND_HB: return phase32<MU, PAR, BC, KIND_HB>;
    default: return phase32<MU, PAR, BC, KIND_OR>;
  }
}
template <int MU, int PAR>
Phase64Fn pick64_bc(int bc, int kind) {
  return bc == BC_PER ? pick64<MU, PAR, BC_PER>(kind)
         : bc == BC_PCC ? pick64<MU, PAR, BC_PCC>(kind)
                        : pick64<MU, PAR, BC_PMC>(kind);
}
template <int MU, int PAR>
Phase32Fn pick32_bc(int bc, int kind) {
  return bc == BC_PER ? pick32<MU, PAR, BC_PER>(kind)
         : bc == BC_PCC ? pick32<MU, PAR, BC_PCC>(kind)
                        : pick32<MU, PAR, BC_PMC>(kind);
}

// phase k of a sweep: k = 2*mu + parity, mu = y, x, t (mc_updates.h:468-473)
Phase64Fn phase_fn64(int k, int bc, int kind) {
  switch (k) {
    case 0: return pick64_bc<DIR_Y, 0>(bc, kind);
    case 1: return pick64_bc<DIR_Y, 1>(bc, kind);
    case 2: return pick64_bc<DIR_X, 0>(bc, kind);
    case 3: return pick64_bc<DIR_X, 1>(bc, kind);
    case 4: return pick64_bc<DIR_T, 0>(bc, kind);
    default: return pick64_bc<DIR_T, 1>(bc, kind);
  }
}
Phase32Fn phase_fn32(int k, int bc, int kind) {
  switch (k) {
    case 0: return pick32_bc<DIR_Y, 0>(bc, kind);
    case 1: return pick32_bc<DIR_Y, 1>(bc, kind);
    case 2: return pick32_bc<DIR_X, 0>(bc, kind);
    case 3: return pick32_bc<DIR_X, 1>(bc, kind);
    case 4: return pick32_bc<DIR_T, 0>(bc, kind);
    default: return pick32_bc<DIR_T, 1>(bc, kind);
  }
}

typedef void (*Phase32pFn)(Pair32, Geo, PhaseArgs);
template <int MU, int PAR, int BC>
Phase32pFn pick32p(int kind) {
  switch (kind) {
    case KIND_METRO: return phase32p<MU, PAR, BC, KIND_METRO>;
    case KIND_HB: return phase32p<MU, PAR, BC, KIND_HB>;
    default: return phase32p<MU, PAR, BC, KIND_OR>;
  }
}
template <int MU, int PAR>
Phase32pFn pick32p_bc(int bc, int kind) {
  return bc == BC_PER ? pick32p<MU, PAR, BC_PER>(kind)
         : bc == BC_PCC ? pick32p<MU, PAR, BC_PCC>(kind)
                        : pick32p<MU, PAR, BC_PMC>(kind);
}
Phase32pFn phase_fn32p(int k, int bc, int kind) {
  switch (k) {
    case 0: return pick32p_bc<DIR_Y, 0>(bc, kind);
    case 1: return pick32p_bc<DIR_Y, 1>(bc, kind);
    case 2: return pick32p_bc<DIR_X, 0>(bc, kind);
    case 3: return pick32p_bc<DIR_X, 1>(bc, kind);
    case 4: return pick32p_bc<DIR_T, 0>(bc, kind);
    default: return pick32p_bc<DIR_T, 1>(bc, kind);
  }
}

// one pass over the six phases with one update kind; with `renorm` (FP32
// only) every link is re-projected as it is stored
int pass(qcd_lattice* h, int kind, int renorm = 0) {
  PhaseArgs a{h->p.beta, h->p.epsilon, h->p.upd, h->err, h->accept, renorm, h->draw_key, h->draw_dev, 0, 0, philox_keys(h->draw_key)};
  const dim3 grid(nblocks(h->g.slice), (unsigned int)h->g.lt);
  const dim3 grid_p(nblocks(h->gh.slice), (unsigned int)h->gh.lt);
  for (int k = 0; k < 6; k++) {
    a.phase_off = (unsigned int)k;
    if (h->paired)
      phase_fn32p(k, h->p.boundary, kind)<<<grid_p, kBlock, 0, h->stream>>>(pair32(h), h->gh, a);
    else if (h->p.precision == QCD_PREC_FP64)
      phase_fn64(k, h->p.boundary, kind)<<<grid, kBlock, 0, h->stream>>>(links64(h), rngs(h), h->g, a);
    else
      phase_fn32(k, h->p.boundary, kind)<<<grid, kBlock, 0, h->stream>>>(links32(h), rngs(h), h->g, a);
    LAUNCH_CHECK(h);
  }
  if (kind != KIND_METRO) h->unit_passes++;
  if (kind != KIND_OR) {
    advance_counter<<<1, 1, 0, h->stream>>>(h->draw_dev, 6ull);
    LAUNCH_CHECK(h);
  }
  return QCD_OK;
}

// ------------------------------------------------------------ wavefront --
// Link classes are (direction, parity); a phase of type (mu, p) writes class
// (mu, p) of its own slice and reads the classes below at slice offsets
// -1, 0, +1 (the staple sites of mc_updates.h:158-176 and its siblings; the
// PMC masks only remove reads, so this superset is safe for every boundary).
struct ClassRef {
  int dir, par, off;
};

int read_set(int mu, int p, ClassRef* r) {
  int k = 0;
  const int q = 1 - p;
  if (mu != DIR_T) {
    const int nu = 1 - mu;  // the other spatial direction
    const ClassRef v[] = {{nu, p, 0}, {nu, q, 0}, {mu, q, 0}, {mu, q, 1}, {mu, q, -1},
                          {DIR_T, q, 0}, {DIR_T, p, 0}, {DIR_T, p, -1}, {DIR_T, q, -1}, {mu, p, 0}};
    for (const ClassRef& c : v) r[k++] = c;
  } else {
    for (int nu = DIR_Y; nu <= DIR_X; nu++) {
      const ClassRef v[] = {{nu, q, 1}, {nu, p, 0}, {nu, p, 1}, {nu, q, 0}};
      for (const ClassRef& c : v) r[k++] = c;
    }
    r[k++] = ClassRef{DIR_T, q, 0};
    r[k++] = ClassRef{DIR_T, p, 0};
  }
  return k;
}

bool reads(int mu, int p, int dir, int par, int off) {
  ClassRef r[16];
  const int k = read_set(mu, p, r);
  for (int i = 0; i < k; i++)
    if (r[i].dir == dir && r[i].par == par && r[i].off == off) return true;
  return false;
}

// must phase m at slice t+o finish before phase n at slice t?
bool conflict(int mu_m, int p_m, int mu_n, int p_n, int o) {
  return reads(mu_n, p_n, mu_m, p_m, o) ||   // n reads what m wrote
         reads(mu_m, p_m, mu_n, p_n, -o) ||  // m reads what n overwrites
         (mu_m == mu_n && p_m == p_n && o == 0);
}

// Seam s_n and start T_n of each phase: the seam advances (by one slice) only
// where a dependency on slice t-1 needs it, and T_n is the earliest start that
// keeps every conflicting task of an earlier phase at a strictly earlier time
// step for every t of the ring: T_n - T_m >= (s_n - s_m) + o + 1.
int plan_wave(const int* mu, const int* par, int P, short need[3][kMaxWavePhases], int* seam, int* start) {
  if (P < 1 || P > kMaxWavePhases) return QCD_ERR_INVALID;
  for (int n = 0; n < P; n++) {
    for (int o = -1; o <= 1; o++) {
      int best = -1;
      for (int m = 0; m < n; m++)
        if (conflict(mu[m], par[m], mu[n], par[n], o)) best = m;
      need[o + 1][n] = (short)best;
    }
  }
  seam[0] = 0;
  start[0] = 0;
  for (int n = 1; n < P; n++) {
    seam[n] = seam[n - 1];
    for (int m = 0; m < n; m++)
      if (conflict(mu[m], par[m], mu[n], par[n], -1) && seam[n] - seam[m] < 1) seam[n] = seam[m] + 1;
    int lo = start[n - 1] + 1;
    for (int m = 0; m < n; m++)
      for (int o = -1; o <= 1; o++)
        if (conflict(mu[m], par[m], mu[n], par[n], o)) {
          const int d = seam[n] - seam[m];
          if (d + o < 0) return QCD_ERR_INVALID;  // cannot happen with the seam rule above
          lo = lo > start[m] + d + o + 1 ? lo : start[m] + d + o + 1;
        }
    start[n] = lo;
  }
  return QCD_OK;
}

struct PassSpec {
  int kind;    // KIND_HB / KIND_METRO / KIND_OR
  int renorm;  // FP32: re-project each link as this pass stores it
};

constexpr unsigned int kWaveSpin = 1u << 22;  // ~1 s of polling per wait

// slices kept live by a chain of `passes` passes (the L2 working set)
int wave_window(int passes) {
  int mu[kMaxWavePhases], par[kMaxWavePhases], seam[kMaxWavePhases], start[kMaxWavePhases];
  short need[3][kMaxWavePhases];
  const int P = 6 * passes;
  for (int n = 0; n < P; n++) {
    mu[n] = (n % 6) / 2;
    par[n] = n % 2;
  }
  plan_wave(mu, par, P, need, seam, start);
  return (start[P - 1] - seam[P - 1]) - (start[0] - seam[0]) + 3;
}

template <class L, int BC, int SK>
void* wave_fn() {
  return (void*)wave<L, BC, SK>;
}

void* pick_wave(int prec, int bc, int sk) {
  if (prec == QCD_PREC_FP64) {
    if (sk == KIND_HB)
      return bc == 0 ? wave_fn<Links64T<true>, 0, KIND_HB>() : bc == 1 ? wave_fn<Links64T<true>, 1, KIND_HB>()
                                                                    : wave_fn<Links64T<true>, 2, KIND_HB>();
    return bc == 0 ? wave_fn<Links64T<true>, 0, KIND_METRO>() : bc == 1 ? wave_fn<Links64T<true>, 1, KIND_METRO>()
                                                                       : wave_fn<Links64T<true>, 2, KIND_METRO>();
  }
  if (sk == KIND_HB)
    return bc == 0 ? wave_fn<Links32T<true>, 0, KIND_HB>() : bc == 1 ? wave_fn<Links32T<true>, 1, KIND_HB>()
                                                                  : wave_fn<Links32T<true>, 2, KIND_HB>();
  return bc == 0 ? wave_fn<Links32T<true>, 0, KIND_METRO>() : bc == 1 ? wave_fn<Links32T<true>, 1, KIND_METRO>()
                                                                     : wave_fn<Links32T<true>, 2, KIND_METRO>();
}

int wave_setup(qcd_lattice* h) {
  if (h->wave_chain) return QCD_OK;
  if (!h->wave_done) CUDA_OR_FAIL(h, cudaMalloc(&h->wave_done, (size_t)h->g.lt * sizeof(unsigned int)));
  if (!h->wave_queue) CUDA_OR_FAIL(h, cudaMalloc(&h->wave_queue, sizeof(unsigned int)));
  if (!h->wave_abort) CUDA_OR_FAIL(h, cudaMalloc(&h->wave_abort, sizeof(int)));
  int dev = 0, sms = 0, per_sm = 0;
  CUDA_OR_FAIL(h, cudaGetDevice(&dev));
  CUDA_OR_FAIL(h, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int sk = h->p.algo == QCD_ALGO_HEATBATH ? KIND_HB : KIND_METRO;
  CUDA_OR_FAIL(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pick_wave(h->p.precision, h->p.boundary, sk),
                                                                 kBlock, 0));
  h->wave_grid = sms * (per_sm > 0 ? per_sm : 1);
  // chain as many passes per launch as keep the live slices within ~64 MB of L2
  const double slice_bytes =
      (double)h->g.slice * (6.0 * (h->p.precision == QCD_PREC_FP64 ? 32.0 : 16.0) + 24.0);
  int chain = 1;
  while (chain < kMaxWavePhases / 6 && wave_window(chain + 1) * slice_bytes <= 64.0 * 1024 * 1024) chain++;
  h->wave_chain = chain;
  return QCD_OK;
}

// Ticket order of a chain of np passes: tasks sorted by time step, then by
// phase, arc and chunk.  With K fronts the ring of Lt slices is cut into K
// arcs of L' = Lt/K slices that advance together:
//     tau(n, t) = T_n + ((t - s_n) mod L').
// The conditions on (s_n, T_n) only involve slice offsets -1..+1 modulo the
// period, so a plan valid for a ring of L' >= 2 slices is valid for every arc
// at once; K fronts give K times the ready tasks and K times the live slices.
int wave_task_table(qcd_lattice* h, int np, const WaveSched& S, int fronts, const unsigned int** out) {
  if (h->wave_tasks[np] && h->wave_tasks_chunk[np] == S.chunk_sites && h->wave_tasks_fronts[np] == fronts) {
    *out = h->wave_tasks[np];
    return QCD_OK;
  }
  const int lt = S.lt, arc = S.lt / fronts;
  unsigned int* host = (unsigned int*)malloc((size_t)S.n_tasks * sizeof(unsigned int));
  if (!host) return fail(h, QCD_ERR_NOMEM, "wavefront task table");
  size_t k = 0;
  const int steps = S.start[S.P - 1] + arc;
  for (int tau = 0; tau < steps; tau++)
    for (int n = 0; n < S.P; n++) {
      if (tau < S.start[n] || tau >= S.start[n] + arc) continue;
      const int u = (S.seam[n] + (tau - S.start[n])) % arc;
      for (int a = 0; a < fronts; a++)
        for (int c = 0; c < S.chunks; c++) host[k++] = wave_pack(n, c, a * arc + u);
    }
  (void)lt;
  cudaError_t e = cudaSuccess;
  if (k != S.n_tasks) {
    free(host);
    return fail(h, QCD_ERR_INVALID, "wavefront task table has %zu of %u tasks", k, S.n_tasks);
  }
  if (h->wave_tasks[np]) cudaFree(h->wave_tasks[np]);
  h->wave_tasks[np] = nullptr;
  e = cudaMalloc(&h->wave_tasks[np], (size_t)S.n_tasks * sizeof(unsigned int));
  if (e == cudaSuccess)
    e = cudaMemcpy(h->wave_tasks[np], host, (size_t)S.n_tasks * sizeof(unsigned int), cudaMemcpyHostToDevice);
  free(host);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(h, QCD_ERR_CUDA, "wavefront task table: %s", cudaGetErrorString(e));
  }
  h->wave_tasks_chunk[np] = S.chunk_sites;
  h->wave_tasks_fronts[np] = fronts;
  *out = h->wave_tasks[np];
  return QCD_OK;
}

int launch_wave(qcd_lattice* h, const PassSpec* ps, int np, int stall_test = 0,
                unsigned int spin = kWaveSpin) {
  int rc = wave_setup(h);
  if (rc) return rc;
  WaveSched S;
  memset(&S, 0, sizeof(S));
  int mu[kMaxWavePhases], par[kMaxWavePhases];
  S.P = 6 * np;
  if (np < 1 || S.P > kMaxWavePhases) return fail(h, QCD_ERR_INVALID, "wavefront program of %d passes", np);
  for (int n = 0; n < S.P; n++) {
    mu[n] = (n % 6) / 2;
    par[n] = n % 2;
    S.mu[n] = (signed char)mu[n];
    S.par[n] = (signed char)par[n];
    S.kind[n] = (signed char)ps[n / 6].kind;
    S.renorm[n] = (signed char)ps[n / 6].renorm;
  }
  for (int n = 0, d = 0; n < S.P; n++) {  // drawing phases numbered in program order
    S.draw[n] = (unsigned char)d;
    if (S.kind[n] != KIND_OR) d++;
  }
  rc = plan_wave(mu, par, S.P, S.need, S.seam, S.start);
  if (rc) return fail(h, rc, "wavefront plan failed");
  S.lt = h->g.lt;
  S.chunk_sites = h->g.slice < h->wave_chunk ? h->g.slice : h->wave_chunk;
  S.chunks = (h->g.slice + S.chunk_sites - 1) / S.chunk_sites;
  S.n_tasks = (unsigned int)S.P * (unsigned int)S.lt * (unsigned int)S.chunks;
  S.n_steps = S.start[S.P - 1] + S.lt;
  if (S.chunks > 4096 || h->g.lt >= 32768)
    return fail(h, QCD_ERR_UNSUPPORTED, "wavefront task words hold at most 4096 chunks and 32767 slices");
  const unsigned int* tasks = nullptr;
  const int fronts = (h->wave_fronts >= 1 && h->g.lt % h->wave_fronts == 0 && h->g.lt / h->wave_fronts >= 2)
                         ? h->wave_fronts
                         : 1;
  rc = wave_task_table(h, np, S, fronts, &tasks);
  if (rc) return rc;
  WaveCtl c{h->wave_done, h->wave_queue, h->wave_abort, tasks, spin, stall_test};
  CUDA_OR_FAIL(h, cudaMemsetAsync(h->wave_done, 0, (size_t)h->g.lt * sizeof(unsigned int), h->stream));
  CUDA_OR_FAIL(h, cudaMemsetAsync(h->wave_queue, 0, sizeof(unsigned int), h->stream));
  CUDA_OR_FAIL(h, cudaMemsetAsync(h->wave_abort, 0, sizeof(int), h->stream));
  PhaseArgs a{h->p.beta, h->p.epsilon, h->p.upd, h->err, h->accept, 0, h->draw_key, h->draw_dev, 0, 0, philox_keys(h->draw_key)};
  const int sk = h->p.algo == QCD_ALGO_HEATBATH ? KIND_HB : KIND_METRO;
  const int bc = h->p.boundary;
  const unsigned int grid = (unsigned int)h->wave_grid;
  RngStoreT<true> R{h->rng, h->g.vh};
  if (h->p.precision == QCD_PREC_FP64) {
    Links64T<true> L{h->lo, h->hi, h->g.vh};
    if (sk == KIND_HB) {
      if (bc == 0) wave<Links64T<true>, 0, KIND_HB><<<grid, kBlock, 0, h->stream>>>(L, R, h->g, a, S, c);
      else if (bc == 1) wave<Links64T<true>, 1, KIND_HB><<<grid, kBlock, 0, h->stream>>>(L, R, h->g, a, S, c);
      else wave<Links64T<true>, 2, KIND_HB><<<grid, kBlock, 0, h->stream>>>(L, R, h->g, a, S, c);
    } else {
      if (bc == 0) wave<Links64T<true>, 0, KIND_METRO><<<grid, kBlock, 0, h->stream>>>(L, R, h->g, a, S, c);
      else if (bc == 1) wave<Links64T<true>, 1, KIND_METRO><<<grid, kBlock, 0, h->stream>>>(L, R, h->g, a, S, c);
      else wave<Links64T<true>, 2, KIND_METRO><<<grid, kBlock, 0, h->stream>>>(L, R, h->g, a, S, c);
    }
  } else {
    Links32T<true> L{h->q32, h->g.vh};
    if (sk == KIND_HB) {
      if (bc == 0) wave<Links32T<true>, 0, KIND_HB><<<grid, kBlock, 0, h->stream>>>(L, R, h->g, a, S, c);
      else if (bc == 1) wave<Links32T<true>, 1, KIND_HB><<<grid, kBlock, 0, h->stream>>>(L, R, h->g, a, S, c);
      else wave<Links32T<true>, 2, KIND_HB><<<grid, kBlock, 0, h->stream>>>(L, R, h->g, a, S, c);
    } else {
      if (bc == 0) wave<Links32T<true>, 0, KIND_METRO><<<grid, kBlock, 0, h->stream>>>(L, R, h->g, a, S, c);
      else if (bc == 1) wave<Links32T<true>, 1, KIND_METRO><<<grid, kBlock, 0, h->stream>>>(L, R, h->g, a, S, c);
      else wave<Links32T<true>, 2, KIND_METRO><<<grid, kBlock, 0, h->stream>>>(L, R, h->g, a, S, c);
    }
  }
  LAUNCH_CHECK(h);
  unsigned long long drawn = 0;
  for (int i = 0; i < np; i++) {
    if (ps[i].kind != KIND_METRO) h->unit_passes++;
    if (ps[i].kind != KIND_OR) drawn += 6;
  }
  if (drawn) {
    advance_counter<<<1, 1, 0, h->stream>>>(h->draw_dev, drawn);
    LAUNCH_CHECK(h);
  }
  return QCD_OK;
}

bool use_wave(const qcd_lattice* h) {
  // automatic never picks the wavefront: per-phase launches measured faster
  // on B200 at every size tried; the wavefront is selected explicitly
  return h->sched == QCD_SCHED_WAVEFRONT;
}

bool use_pairs(const qcd_lattice* h) { return h->sched == QCD_SCHED_PAIRS && h->p.precision == QCD_PREC_FP32; }

// The second store and the device facts the fused pairs need (allocated
// when the schedule is chosen, never inside a pass, so that passes can be
// captured in a CUDA graph).
int pairs_setup(qcd_lattice* h) {
  if (!h->q32alt) {
    CUDA_OR_FAIL(h, cudaMalloc(&h->q32alt, h->link_bytes));
    h->pair_buf[0] = h->q32;
    h->pair_buf[1] = h->q32alt;
    for (int b = 0; b < 2; b++) {
      cudaError_t e = pair_encode_maps(h->pair_buf[b], h->g, &h->pair_maps[b]);
      if (e != cudaSuccess) {
        cudaFree(h->q32alt);
        h->q32alt = nullptr;
        return fail(h, QCD_ERR_UNSUPPORTED, "fused pairs: tensor maps of the link store: %s", cudaGetErrorString(e));
      }
    }
  }
  if (!h->sms) {
    int dev = 0;
    CUDA_OR_FAIL(h, cudaGetDevice(&dev));
    CUDA_OR_FAIL(h, cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, dev));
  }
  return QCD_OK;
}

// One pass as three fused pairs (y, x, t), reading the current store and
// writing the other one, which then becomes current.
int pass_pairs(qcd_lattice* h, int kind, int renorm) {
  if (!h->q32alt || !h->sms) return fail(h, QCD_ERR_INVALID, "fused pairs used before their setup");
  PhaseArgs a{h->p.beta, h->p.epsilon, h->p.upd, h->err, h->accept, renorm, h->draw_key, h->draw_dev, 0, 0, philox_keys(h->draw_key)};
  const PairMaps& mc = h->pair_maps[h->q32 == h->pair_buf[0] ? 0 : 1];
  const PairMaps& ma = h->pair_maps[h->q32 == h->pair_buf[0] ? 1 : 0];
  CUDA_OR_FAIL(h, pair_pass32(h->q32, h->q32alt, mc, ma, h->g, h->p.boundary, kind, a, h->pair_seg, h->sms, h->stream));
  float4* t = h->q32;
  h->q32 = h->q32alt;
  h->q32alt = t;
  if (kind != KIND_METRO) h->unit_passes++;
  if (kind != KIND_OR) {
    advance_counter<<<1, 1, 0, h->stream>>>(h->draw_dev, 6ull);
    LAUNCH_CHECK(h);
  }
  return QCD_OK;
}

int run_passes(qcd_lattice* h, const PassSpec* ps, int np);

int check_device_error(qcd_lattice* h) {
  int e = 0;
  CUDA_OR_FAIL(h, cudaMemcpyAsync(&h->result_host[2], h->err, sizeof(int), cudaMemcpyDeviceToHost,
                                  h->stream));
  CUDA_OR_FAIL(h, cudaStreamSynchronize(h->stream));
  memcpy(&e, &h->result_host[2], sizeof(int));
  if (e & DEVERR_TIMEOUT) {
    CUDA_OR_FAIL(h, cudaMemsetAsync(h->err, 0, sizeof(int), h->stream));
    CUDA_OR_FAIL(h, cudaStreamSynchronize(h->stream));
    return fail(h, QCD_ERR_TIMEOUT, "a bounded device wait ran out (a wavefront task waiting for a neighbour slice, "
                                     "or a fused-pair CTA waiting for its staged links)");
  }
  if (e & DEVERR_HB_LOOP)
    return fail(h, QCD_ERR_NONUNITARY,
                "heat-bath rejection loop exceeded %d tries (staple sum zero or not finite)",
                QCD_HB_MAX_TRIES);
  return QCD_OK;
}

int reduce_result(qcd_lattice* h, double* a, double* b) {
  CUDA_OR_FAIL(h, cudaMemcpyAsync(h->result_host, h->result, 2 * sizeof(double),
                                  cudaMemcpyDeviceToHost, h->stream));
  int rc = check_device_error(h);  // synchronises the stream
  if (rc) return rc;
  if (a) *a = h->result_host[0];
  if (b) *b = h->result_host[1];
  return QCD_OK;
}

int launch_measure(qcd_lattice* h, double* out_dev) {
  const unsigned int nb = measure_blocks(h->g.vh);
  const bool pmc = h->p.boundary == QCD_BC_PMC;
  if (h->p.precision == QCD_PREC_FP64) {
    if (pmc)
      measure<Links64, 1><<<nb, kBlock, 0, h->stream>>>(links64(h), h->g, h->partials, h->counter, out_dev);
    else
      measure<Links64, 0><<<nb, kBlock, 0, h->stream>>>(links64(h), h->g, h->partials, h->counter, out_dev);
  } else if (h->paired) {
    if (pmc)
      measure_p<1><<<nb, kBlock, 0, h->stream>>>(pair32(h), h->gh, h->partials, h->counter, out_dev);
    else
      measure_p<0><<<nb, kBlock, 0, h->stream>>>(pair32(h), h->gh, h->partials, h->counter, out_dev);
  } else {
    if (pmc)
      measure<Links32, 1><<<nb, kBlock, 0, h->stream>>>(links32(h), h->g, h->partials, h->counter, out_dev);
    else
      measure<Links32, 0><<<nb, kBlock, 0, h->stream>>>(links32(h), h->g, h->partials, h->counter, out_dev);
  }
  LAUNCH_CHECK(h);
  return QCD_OK;
}

int run_passes(qcd_lattice* h, const PassSpec* ps, int np) {
  if (np == 0) return QCD_OK;
  if (use_pairs(h)) {
    for (int i = 0; i < np; i++) {
      int rc = pass_pairs(h, ps[i].kind, ps[i].renorm);
      if (rc) return rc;
    }
    return QCD_OK;
  }
  if (use_wave(h)) {
    int rc = wave_setup(h);
    if (rc) return rc;
    for (int i = 0; i < np; i += h->wave_chain) {
      const int k = np - i < h->wave_chain ? np - i : h->wave_chain;
      rc = launch_wave(h, ps + i, k);
      if (rc) return rc;
    }
    return QCD_OK;
  }
  for (int i = 0; i < np; i++) {
    int rc = pass(h, ps[i].kind, ps[i].renorm);
    if (rc) return rc;
  }
  return QCD_OK;
}

// The MRG32k3a streams, seeded curand_init(seed, id, 0) on first use: at
// create for FP64 lattices, at the first hot start or generator checkpoint
// for FP32 ones (whose sweep draws from the counter-based stream).  Seeding
// late gives the same words as seeding at create.
int ensure_rng(qcd_lattice* h) {
  if (h->rng) return QCD_OK;
  if (!h->mrg_jumps) {
    CUDA_OR_FAIL(h, cudaMalloc(&h->mrg_jumps, kMrgJumpWords * sizeof(uint32_t)));
    CUDA_OR_FAIL(h, cudaMemcpyAsync(h->mrg_jumps, mrg_jump_host(), kMrgJumpWords * sizeof(uint32_t),
                                    cudaMemcpyHostToDevice, h->stream));
  }
  CUDA_OR_FAIL(h, cudaMalloc(&h->rng, 6 * (size_t)h->g.vh * sizeof(uint32_t)));
  rng_setup<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(rngs(h), h->p.seed, h->g.vh, h->mrg_jumps);
  LAUNCH_CHECK(h);
  return QCD_OK;
}

void release(qcd_lattice* h) {
  cudaFree(h->lo);
  cudaFree(h->hi);
  cudaFree(h->q32);
  cudaFree(h->q32alt);
  cudaFree(h->rng);
  cudaFree(h->mrg_jumps);
  cudaFree(h->accept);
  cudaFree(h->partials);
  cudaFree(h->counter);
  cudaFree(h->result);
  cudaFree(h->err);
  cudaFree(h->draw_dev);
  cudaFree(h->series);
  cudaFree(h->aos_stage);
  cudaFree(h->wave_done);
  cudaFree(h->wave_queue);
  cudaFree(h->wave_abort);
  for (int i = 0; i < 5; i++) cudaFree(h->wave_tasks[i]);
  if (h->result_host) cudaFreeHost(h->result_host);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
}

}  // namespace

// =================================================================== ABI ==
extern "C" {

void qcd_params_default(qcd_params* p, int lt, int lx, int ly) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->lt = lt;
  p->lx = lx;
  p->ly = ly;
  p->beta = 20.0f;    // kernel.cu:27
  p->epsilon = 0.1f;  // kernel.cu:43
  p->upd = 1;         // kernel.cu:44
  p->algo = QCD_ALGO_HEATBATH;
  p->boundary = QCD_BC_PERIODIC;
  p->precision = QCD_PREC_FP64;
  p->n_or = 0;
  p->renorm_every = 0;
  p->seed = 1234ull;
}

const char* qcd_status_string(int s) {
  switch (s) {
    case QCD_OK: return "ok";
    case QCD_ERR_INVALID: return "invalid argument";
    case QCD_ERR_CUDA: return "CUDA error";
    case QCD_ERR_NOMEM: return "out of device memory";
    case QCD_ERR_NONUNITARY: return "links not unitary";
    case QCD_ERR_TIMEOUT: return "device wait timed out";
    case QCD_ERR_IO: return "configuration I/O error";
    case QCD_ERR_UNSUPPORTED: return "unsupported combination";
    default: return "unknown status";
  }
}

const char* qcd_last_error(const qcd_lattice* h) { return h ? h->msg : "null handle"; }

int qcd_create(const qcd_params* p, qcd_lattice** out) {
  if (!p || !out) return QCD_ERR_INVALID;
  *out = nullptr;
  if (p->lt < 2 || p->lx < 2 || p->ly < 2 || (p->lt & 1) || (p->lx & 1) || (p->ly & 1))
    return QCD_ERR_INVALID;  // kernel.cu:61-64: every extent even
  if (p->algo != QCD_ALGO_METROPOLIS && p->algo != QCD_ALGO_HEATBATH) return QCD_ERR_INVALID;
  if (p->boundary < 0 || p->boundary > 2) return QCD_ERR_INVALID;
  if (p->precision != QCD_PREC_FP64 && p->precision != QCD_PREC_FP32) return QCD_ERR_INVALID;
  if (!(p->beta > 0.f) || p->upd < 0 || p->n_or < 0 || p->renorm_every < 0) return QCD_ERR_INVALID;
  if (p->algo == QCD_ALGO_METROPOLIS && !(p->epsilon > 0.f && p->epsilon < 1.f)) return QCD_ERR_INVALID;
  if (0.5 * (double)p->lt * (double)p->lx * (double)p->ly >= (double)((1ll << 31) / 6))
    return QCD_ERR_INVALID;  // 32-bit plane indices (checked in double: the product can overflow)
  long long V = (long long)p->lt * p->lx * p->ly;

  qcd_lattice* h = new (std::nothrow) qcd_lattice();
  if (!h) return QCD_ERR_NOMEM;
  h->p = *p;
  h->V = V;
  h->g = make_geo(p->lt, p->lx, p->ly);
  h->gh = make_geo(p->lt / 2, p->lx, p->ly);
  h->paired = pairable(h);  // the store is written in pairs from the first start or load on
  h->draw_key = p->seed;
  const size_t vh = (size_t)h->g.vh;
  int rc = QCD_OK;
  auto step = [&](cudaError_t e, const char* what) {
    if (rc == QCD_OK && e != cudaSuccess) {
      rc = e == cudaErrorMemoryAllocation ? QCD_ERR_NOMEM : QCD_ERR_CUDA;
      cudaGetLastError();
      snprintf(h->msg, sizeof(h->msg), "%s: %s", what, cudaGetErrorString(e));
    }
  };
  step(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking), "cudaStreamCreate");
  h->stream = h->own_stream;
  if (p->precision == QCD_PREC_FP64) {
    h->link_bytes = 6 * vh * sizeof(double2) * 2;
    if (rc == QCD_OK) step(cudaMalloc(&h->lo, 6 * vh * sizeof(double2)), "cudaMalloc(links)");
    if (rc == QCD_OK) step(cudaMalloc(&h->hi, 6 * vh * sizeof(double2)), "cudaMalloc(links)");
  } else {
    h->link_bytes = 6 * vh * sizeof(float4);
    if (rc == QCD_OK) step(cudaMalloc(&h->q32, 6 * vh * sizeof(float4)), "cudaMalloc(links)");
  }
  if (rc == QCD_OK && p->algo == QCD_ALGO_METROPOLIS) {
    step(cudaMalloc(&h->accept, 2 * vh * sizeof(int)), "cudaMalloc(accept)");
    if (rc == QCD_OK) step(cudaMemsetAsync(h->accept, 0, 2 * vh * sizeof(int), h->stream), "memset");
  }
  const size_t nb = nblocks(h->g.vh);  // one partial per CTA of the largest reduction launch
  if (rc == QCD_OK) step(cudaMalloc(&h->partials, nb * sizeof(double2)), "cudaMalloc(partials)");
  if (rc == QCD_OK) step(cudaMalloc(&h->counter, sizeof(unsigned int)), "cudaMalloc(counter)");
  if (rc == QCD_OK) step(cudaMalloc(&h->result, 2 * sizeof(double)), "cudaMalloc(result)");
  if (rc == QCD_OK) step(cudaMalloc(&h->err, sizeof(int)), "cudaMalloc(err)");
  if (rc == QCD_OK) step(cudaMalloc(&h->draw_dev, sizeof(unsigned long long)), "cudaMalloc(draw counter)");
  if (rc == QCD_OK) step(cudaMemsetAsync(h->draw_dev, 0, sizeof(unsigned long long), h->stream), "memset");
  if (rc == QCD_OK) step(cudaMallocHost(&h->result_host, 4 * sizeof(double)), "cudaMallocHost");
  if (rc == QCD_OK) step(cudaMemsetAsync(h->counter, 0, sizeof(unsigned int), h->stream), "memset");
  if (rc == QCD_OK) step(cudaMemsetAsync(h->err, 0, sizeof(int), h->stream), "memset");
  // the FP64 sweep draws from the stored MRG32k3a streams at every update; an
  // FP32 lattice needs them only for a hot start or a generator checkpoint,
  // so it seeds them on first use
  if (rc == QCD_OK && p->precision == QCD_PREC_FP64) rc = ensure_rng(h);
  if (rc == QCD_OK) step(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  if (rc != QCD_OK) {
    fprintf(stderr, "qcd_create: %s\n", h->msg);
    release(h);
    delete h;
    return rc;
  }
  *out = h;
  return QCD_OK;
}

int qcd_destroy(qcd_lattice* h) {
  if (!h) return QCD_ERR_INVALID;
  if (h->stream) cudaStreamSynchronize(h->stream);
  release(h);
  delete h;
  return QCD_OK;
}

int qcd_set_stream(qcd_lattice* h, void* stream) {
  if (!h) return QCD_ERR_INVALID;
  CUDA_OR_FAIL(h, cudaStreamSynchronize(h->stream));
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  return QCD_OK;
}

void* qcd_get_stream(qcd_lattice* h) { return h ? (void*)h->stream : nullptr; }

int qcd_init_cold(qcd_lattice* h) {
  if (!h) return QCD_ERR_INVALID;
  if (h->p.precision == QCD_PREC_FP64)
    init_cold<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(links64(h), h->g.vh);
  else if (h->paired)
    init_cold<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(pair32(h), h->g.vh);
  else
    init_cold<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(links32(h), h->g.vh);
  LAUNCH_CHECK(h);
  return QCD_OK;
}

int qcd_init_hot(qcd_lattice* h) {
  if (!h) return QCD_ERR_INVALID;
  int rc = ensure_rng(h);
  if (rc) return rc;
  const int pcc = h->p.boundary == QCD_BC_PCC;
  if (h->p.precision == QCD_PREC_FP64)
    init_hot<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(links64(h), rngs(h), h->g, pcc);
  else if (h->paired)
    init_hot<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(pair32(h), rngs(h), h->g, pcc);
  else
    init_hot<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(links32(h), rngs(h), h->g, pcc);
  LAUNCH_CHECK(h);
  return QCD_OK;
}

static int ensure_stage(qcd_lattice* h) {
  if (!h->aos_stage) CUDA_OR_FAIL(h, cudaMalloc(&h->aos_stage, (size_t)h->V * 12 * sizeof(double)));
  return QCD_OK;
}

int qcd_load_config_device(qcd_lattice* h, const double* aos_dev) {
  if (!h || !aos_dev) return QCD_ERR_INVALID;
  if (h->p.precision == QCD_PREC_FP64)
    aos_to_soa64<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(aos_dev, links64(h), h->g.vh);
  else if (h->paired)
    aos_to_pair32<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(aos_dev, pair32(h), h->g.vh);
  else
    aos_to_soa32<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(aos_dev, links32(h), h->g.vh);
  LAUNCH_CHECK(h);
  return QCD_OK;
}

int qcd_store_config_device(qcd_lattice* h, double* aos_dev) {
  if (!h || !aos_dev) return QCD_ERR_INVALID;
  if (h->p.precision == QCD_PREC_FP64)
    soa_to_aos64<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(links64(h), aos_dev, h->g.vh);
  else if (h->paired)
    pair32_to_aos<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(pair32(h), aos_dev, h->g.vh);
  else
    soa_to_aos32<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(links32(h), aos_dev, h->g.vh);
  LAUNCH_CHECK(h);
  return QCD_OK;
}

int qcd_load_config(qcd_lattice* h, const double* aos_host) {
  if (!h || !aos_host) return QCD_ERR_INVALID;
  int rc = ensure_stage(h);
  if (rc) return rc;
  CUDA_OR_FAIL(h, cudaMemcpyAsync(h->aos_stage, aos_host, (size_t)h->V * 12 * sizeof(double),
                                  cudaMemcpyHostToDevice, h->stream));
  rc = qcd_load_config_device(h, h->aos_stage);
  if (rc) return rc;
  CUDA_OR_FAIL(h, cudaStreamSynchronize(h->stream));  // host buffer may be reused on return
  return QCD_OK;
}

int qcd_store_config(qcd_lattice* h, double* aos_host) {
  if (!h || !aos_host) return QCD_ERR_INVALID;
  int rc = ensure_stage(h);
  if (rc) return rc;
  rc = qcd_store_config_device(h, h->aos_stage);
  if (rc) return rc;
  CUDA_OR_FAIL(h, cudaMemcpyAsync(aos_host, h->aos_stage, (size_t)h->V * 12 * sizeof(double),
                                  cudaMemcpyDeviceToHost, h->stream));
  return check_device_error(h);
}

int qcd_normalize(qcd_lattice* h) {
  if (!h) return QCD_ERR_INVALID;
  if (h->p.precision == QCD_PREC_FP64)
    normalize64<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(links64(h), h->g.vh);
  else if (h->paired)
    normalize32p<<<nblocks(h->gh.vh), kBlock, 0, h->stream>>>(pair32(h));
  else
    normalize32<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(links32(h), h->g.vh);
  LAUNCH_CHECK(h);
  return QCD_OK;
}

int qcd_sweep(qcd_lattice* h, int n) {
  if (!h || n < 0) return QCD_ERR_INVALID;
  const int kind = h->p.algo == QCD_ALGO_HEATBATH ? KIND_HB : KIND_METRO;
  PassSpec buf[64];
  int np = 0;
  for (int i = 0; i < n; i++) {
    const bool renorm = h->p.renorm_every > 0 && (h->sweeps_done + 1) % h->p.renorm_every == 0;
    // FP32: the re-projection rides on the sweep's last pass, each link being
    // re-projected at its last update (no extra read of the store); FP64
    // keeps the reference's separate normalize after the sweep
    const bool fused = renorm && h->p.precision == QCD_PREC_FP32;
    if (np + 1 + h->p.n_or > 64) {
      int rc = run_passes(h, buf, np);
      if (rc) return rc;
      np = 0;
    }
    buf[np++] = PassSpec{kind, fused && h->p.n_or == 0};
    for (int r = 0; r < h->p.n_or; r++) buf[np++] = PassSpec{KIND_OR, fused && r == h->p.n_or - 1};
    h->sweeps_done++;
    if (renorm && !fused) {
      int rc = run_passes(h, buf, np);
      np = 0;
      if (rc == QCD_OK) rc = qcd_normalize(h);
      if (rc) return rc;
    }
  }
  return run_passes(h, buf, np);
}

int qcd_overrelax(qcd_lattice* h, int n) {
  if (!h || n < 0) return QCD_ERR_INVALID;
  PassSpec buf[64];
  while (n > 0) {
    const int k = n < 64 ? n : 64;
    for (int i = 0; i < k; i++) buf[i] = PassSpec{KIND_OR, 0};
    int rc = run_passes(h, buf, k);
    if (rc) return rc;
    n -= k;
  }
  return QCD_OK;
}

// The FP32 store rewritten in the other layout (site pairs <-> one float4
// plane per class) through a scratch store; the links keep their values.
int set_paired(qcd_lattice* h, bool paired) {
  if (h->paired == paired) return QCD_OK;
  if (paired && !pairable(h)) return fail(h, QCD_ERR_INVALID, "site pairs need an FP32 lattice with Lt %% 4 == 0");
  float4* tmp = nullptr;
  CUDA_OR_FAIL(h, cudaMalloc(&tmp, h->link_bytes));
  cudaError_t e = cudaSuccess;
  if (paired) {
    e = cudaMemcpyAsync(tmp, h->q32, h->link_bytes, cudaMemcpyDeviceToDevice, h->stream);
    if (e == cudaSuccess) plain_to_pair32<<<nblocks(h->gh.vh), kBlock, 0, h->stream>>>(tmp, pair32(h));
  } else {
    pair32_to_plain<<<nblocks(h->gh.vh), kBlock, 0, h->stream>>>(pair32(h), tmp);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->q32, tmp, h->link_bytes, cudaMemcpyDeviceToDevice, h->stream);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) return fail(h, QCD_ERR_CUDA, "changing the FP32 store layout: %s", cudaGetErrorString(e));
  h->paired = paired;
  return QCD_OK;
}

int qcd_set_schedule(qcd_lattice* h, int mode) {
  if (!h || mode < QCD_SCHED_AUTO || mode > QCD_SCHED_PAIRS) return QCD_ERR_INVALID;
  if (mode == QCD_SCHED_PAIRS) {
    if (h->p.precision != QCD_PREC_FP32)
      return fail(h, QCD_ERR_UNSUPPORTED, "fused pairs are an FP32 schedule (FP64 keeps the reference's kernels)");
    int rc = pairs_setup(h);
    if (rc) return rc;
  }
  // the per-phase schedule runs FP32 lattices with Lt % 4 == 0 on the paired
  // store; the wavefront and the fused pairs read one float4 plane per class
  if (h->p.precision == QCD_PREC_FP32) {
    int rc = set_paired(h, pairable(h) && h->pair_ok && (mode == QCD_SCHED_AUTO || mode == QCD_SCHED_PHASES));
    if (rc) return rc;
  }
  h->sched = mode;
  return QCD_OK;
}

int qcd_set_pair_layout(qcd_lattice* h, int on) {
  if (!h || on < 0 || on > 1) return QCD_ERR_INVALID;
  h->pair_ok = on != 0;
  if (h->p.precision != QCD_PREC_FP32) return QCD_OK;
  return set_paired(h, pairable(h) && h->pair_ok && (h->sched == QCD_SCHED_AUTO || h->sched == QCD_SCHED_PHASES));
}

int qcd_get_pair_layout(const qcd_lattice* h) {
  if (!h) return QCD_ERR_INVALID;
  return h->paired ? 1 : 0;
}

int qcd_get_schedule(const qcd_lattice* h) {
  if (!h) return QCD_ERR_INVALID;
  return use_pairs(h) ? QCD_SCHED_PAIRS : use_wave(h) ? QCD_SCHED_WAVEFRONT : QCD_SCHED_PHASES;
}

int qcd_set_pair_tuning(qcd_lattice* h, int slices_per_cta) {
  if (!h || slices_per_cta < 0) return QCD_ERR_INVALID;
  h->pair_seg = slices_per_cta;
  return QCD_OK;
}

int qcd_set_wave_tuning(qcd_lattice* h, int chunk_sites, int passes_per_launch, int fronts) {
  if (!h || chunk_sites < 0 || passes_per_launch < 0 || passes_per_launch > kMaxWavePhases / 6 || fronts < 0)
    return QCD_ERR_INVALID;
  if (fronts && (h->g.lt % fronts || h->g.lt / fronts < 2))
    return fail(h, QCD_ERR_INVALID, "fronts must divide Lt = %d into arcs of >= 2 slices", h->g.lt);
  int rc = wave_setup(h);
  if (rc) return rc;
  if (chunk_sites) h->wave_chunk = (chunk_sites + kBlock - 1) / kBlock * kBlock;
  if (passes_per_launch) h->wave_chain = passes_per_launch;
  if (fronts) h->wave_fronts = fronts;
  return QCD_OK;
}

// ------------------------------------------------------------- autotune --
namespace {

struct TuneKey {
  int lt, lx, ly, prec, algo, bc, n_or;
  bool operator==(const TuneKey& o) const {
    return lt == o.lt && lx == o.lx && ly == o.ly && prec == o.prec && algo == o.algo && bc == o.bc && n_or == o.n_or;
  }
};
struct TuneChoice {
  TuneKey key;
  qcd_tuning t;
};
std::mutex g_tune_mu;
std::vector<TuneChoice> g_tune_cache;

int apply_tuning(qcd_lattice* h, const qcd_tuning& t) {
  int rc = qcd_set_schedule(h, t.schedule);
  if (rc == QCD_OK && t.schedule == QCD_SCHED_WAVEFRONT)
    rc = qcd_set_wave_tuning(h, t.chunk_sites, t.passes_per_launch, t.fronts);
  if (rc == QCD_OK && t.schedule == QCD_SCHED_PAIRS) rc = qcd_set_pair_tuning(h, t.chunk_sites);
  return rc;
}

}  // namespace

int qcd_autotune(qcd_lattice* h, int sweeps_per_trial, qcd_tuning* chosen) {
  if (!h || sweeps_per_trial < 0) return QCD_ERR_INVALID;
  const TuneKey key{h->p.lt, h->p.lx, h->p.ly, h->p.precision, h->p.algo, h->p.boundary, h->p.n_or};
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    for (const TuneChoice& c : g_tune_cache)
      if (c.key == key) {
        if (chosen) *chosen = c.t;
        return apply_tuning(h, c.t);
      }
  }
  if (sweeps_per_trial == 0) sweeps_per_trial = 2;
  // candidates: per-phase launches, and the wavefront with the task sizes,
  // fronts and chain lengths whose live slices fit in L2
  std::vector<qcd_tuning> cand;
  cand.push_back(qcd_tuning{QCD_SCHED_PHASES, 0, 0, 0, 0.0});
  // FP32: the fused pairs with the automatic segment and two fixed ones
  if (h->p.precision == QCD_PREC_FP32)
    for (int seg : {0, 32, 64}) cand.push_back(qcd_tuning{QCD_SCHED_PAIRS, seg, 0, 0, 0.0});
  int rc = wave_setup(h);
  if (rc) return rc;
  const double slice_bytes = (double)h->g.slice * (6.0 * (h->p.precision == QCD_PREC_FP64 ? 32.0 : 16.0) + 24.0);
  const int max_chain = h->wave_chain;
  for (int chunk : {256, 512, 1024})
    for (int fronts : {1, 2, 4, 8, 16, 32})
      for (int passes : {1, max_chain}) {
        if (h->g.lt % fronts || h->g.lt / fronts < 2) continue;
        if (passes != 1 && passes == max_chain && max_chain == 1) continue;
        if (fronts > 1 && fronts * wave_window(passes) * slice_bytes > 100.0 * 1024 * 1024) continue;
        cand.push_back(qcd_tuning{QCD_SCHED_WAVEFRONT, chunk, passes, fronts, 0.0});
      }
  // the trials advance the lattice: save links, streams and counters, restore after
  const size_t rng_bytes = 6 * (size_t)h->g.vh * sizeof(uint32_t);
  // the backups are freed on every way out of this function (a failed
  // allocation or copy returns early)
  struct Backups {
    void *links = nullptr, *links2 = nullptr, *rng = nullptr, *acc = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~Backups() {
      cudaFree(links);
      cudaFree(links2);
      cudaFree(rng);
      cudaFree(acc);
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
    }
  } bk;
  void *&links_save = bk.links, *&links2_save = bk.links2, *&rng_save = bk.rng, *&acc_save = bk.acc;
  const size_t lb = h->p.precision == QCD_PREC_FP64 ? h->link_bytes / 2 : h->link_bytes;
  // (the fused pairs swap the FP32 stores: the restore goes to whichever is current then)
  void* lp = h->p.precision == QCD_PREC_FP64 ? (void*)h->lo : (void*)h->q32;
  CUDA_OR_FAIL(h, cudaMalloc(&links_save, lb));
  if (h->p.precision == QCD_PREC_FP64) CUDA_OR_FAIL(h, cudaMalloc(&links2_save, lb));
  if (h->rng) CUDA_OR_FAIL(h, cudaMalloc(&rng_save, rng_bytes));
  if (h->accept) CUDA_OR_FAIL(h, cudaMalloc(&acc_save, (size_t)h->V * sizeof(int)));
  CUDA_OR_FAIL(h, cudaMemcpyAsync(links_save, lp, lb, cudaMemcpyDeviceToDevice, h->stream));
  if (links2_save) CUDA_OR_FAIL(h, cudaMemcpyAsync(links2_save, h->hi, lb, cudaMemcpyDeviceToDevice, h->stream));
  if (rng_save) CUDA_OR_FAIL(h, cudaMemcpyAsync(rng_save, h->rng, rng_bytes, cudaMemcpyDeviceToDevice, h->stream));
  if (acc_save)
    CUDA_OR_FAIL(h, cudaMemcpyAsync(acc_save, h->accept, (size_t)h->V * sizeof(int), cudaMemcpyDeviceToDevice, h->stream));
  const long long passes_save = h->unit_passes, sweeps_save = h->sweeps_done;
  unsigned long long draws_save = 0;
  CUDA_OR_FAIL(h, cudaMemcpyAsync(&draws_save, h->draw_dev, sizeof(draws_save), cudaMemcpyDeviceToHost, h->stream));
  CUDA_OR_FAIL(h, cudaStreamSynchronize(h->stream));
  const int sched_save = h->sched, chunk_save = h->wave_chunk, chain_save = h->wave_chain, fronts_save = h->wave_fronts,
            pseg_save = h->pair_seg;
  const bool paired_save = h->paired;  // the saved links are in this layout
  cudaEvent_t &e0 = bk.e0, &e1 = bk.e1;
  CUDA_OR_FAIL(h, cudaEventCreate(&e0));
  CUDA_OR_FAIL(h, cudaEventCreate(&e1));
  int best = 0;
  for (size_t i = 0; i < cand.size() && rc == QCD_OK; i++) {
    rc = apply_tuning(h, cand[i]);
    if (rc == QCD_OK) rc = qcd_sweep(h, 1);  // warm-up (task tables, first launches)
    if (rc == QCD_OK) rc = cudaEventRecord(e0, h->stream) == cudaSuccess ? QCD_OK : QCD_ERR_CUDA;
    if (rc == QCD_OK) rc = qcd_sweep(h, sweeps_per_trial);
    if (rc == QCD_OK) rc = cudaEventRecord(e1, h->stream) == cudaSuccess ? QCD_OK : QCD_ERR_CUDA;
    if (rc == QCD_OK) rc = check_device_error(h);
    float ms = 0;
    if (rc == QCD_OK) rc = cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess ? QCD_OK : QCD_ERR_CUDA;
    cand[i].ms_per_sweep = ms / sweeps_per_trial;
    if (rc == QCD_OK && cand[i].ms_per_sweep < cand[best].ms_per_sweep) best = (int)i;
  }
  // restore the lattice as it was
  lp = h->p.precision == QCD_PREC_FP64 ? (void*)h->lo : (void*)h->q32;
  cudaMemcpyAsync(lp, links_save, lb, cudaMemcpyDeviceToDevice, h->stream);
  if (links2_save) cudaMemcpyAsync(h->hi, links2_save, lb, cudaMemcpyDeviceToDevice, h->stream);
  if (rng_save) cudaMemcpyAsync(h->rng, rng_save, rng_bytes, cudaMemcpyDeviceToDevice, h->stream);
  if (acc_save) cudaMemcpyAsync(h->accept, acc_save, (size_t)h->V * sizeof(int), cudaMemcpyDeviceToDevice, h->stream);
  cudaStreamSynchronize(h->stream);
  cudaMemcpyAsync(h->draw_dev, &draws_save, sizeof(draws_save), cudaMemcpyHostToDevice, h->stream);
  cudaStreamSynchronize(h->stream);
  h->unit_passes = passes_save;
  h->sweeps_done = sweeps_save;
  h->sched = sched_save;
  h->paired = paired_save;
  h->wave_chunk = chunk_save;
  h->wave_chain = chain_save;
  h->wave_fronts = fronts_save;
  h->pair_seg = pseg_save;
  if (rc) return rc;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache.push_back(TuneChoice{key, cand[best]});
  }
  if (chosen) *chosen = cand[best];
  return apply_tuning(h, cand[best]);
}

int qcd_wave_plan(const int* mu, const int* par, int n_phases, int* seam, int* start, int* need) {
  if (!mu || !par || !seam || !start || !need || n_phases < 1 || n_phases > kMaxWavePhases)
    return QCD_ERR_INVALID;
  short nd[3][kMaxWavePhases];
  int rc = plan_wave(mu, par, n_phases, nd, seam, start);
  if (rc) return rc;
  for (int o = 0; o < 3; o++)
    for (int n = 0; n < n_phases; n++) need[o * n_phases + n] = nd[o][n];
  return QCD_OK;
}

int qcd_wave_selftest_timeout(qcd_lattice* h) {
  if (!h) return QCD_ERR_INVALID;
  PassSpec p{KIND_OR, 0};
  int rc = launch_wave(h, &p, 1, /*stall_test=*/1, /*spin=*/4096);
  if (rc) return rc;
  h->unit_passes--;  // the pass did not complete
  return check_device_error(h);
}

int qcd_measure(qcd_lattice* h, double* energy, double* plaquette) {
  if (!h) return QCD_ERR_INVALID;
  int rc = launch_measure(h, h->result);
  if (rc) return rc;
  return reduce_result(h, energy, plaquette);
}

int qcd_series_reserve(qcd_lattice* h, int capacity) {
  if (!h || capacity < 0) return QCD_ERR_INVALID;
  CUDA_OR_FAIL(h, cudaStreamSynchronize(h->stream));
  cudaFree(h->series);
  h->series = nullptr;
  h->series_cap = 0;
  if (capacity == 0) return QCD_OK;
  CUDA_OR_FAIL(h, cudaMalloc(&h->series, (size_t)capacity * 2 * sizeof(double)));
  CUDA_OR_FAIL(h, cudaMemsetAsync(h->series, 0, (size_t)capacity * 2 * sizeof(double), h->stream));
  h->series_cap = capacity;
  return QCD_OK;
}

int qcd_measure_into_series(qcd_lattice* h, int index) {
  if (!h || index < 0 || index >= h->series_cap)
    return fail(h, QCD_ERR_INVALID, "series index %d outside capacity %d", index, h ? h->series_cap : 0);
  return launch_measure(h, h->series + 2 * (size_t)index);
}

int qcd_series_read(qcd_lattice* h, double* energy, double* plaquette, int n) {
  if (!h || n < 0 || n > h->series_cap) return QCD_ERR_INVALID;
  if (n == 0) return check_device_error(h);
  double* tmp = (double*)malloc((size_t)n * 2 * sizeof(double));
  if (!tmp) return QCD_ERR_NOMEM;
  cudaError_t e = cudaMemcpyAsync(tmp, h->series, (size_t)n * 2 * sizeof(double),
                                  cudaMemcpyDeviceToHost, h->stream);
  if (e != cudaSuccess) {
    free(tmp);
    return fail(h, QCD_ERR_CUDA, "series copy: %s", cudaGetErrorString(e));
  }
  int rc = check_device_error(h);
  if (rc == QCD_OK)
    for (int i = 0; i < n; i++) {
      if (energy) energy[i] = tmp[2 * i];
      if (plaquette) plaquette[i] = tmp[2 * i + 1];
    }
  free(tmp);
  return rc;
}

int qcd_accept_counts(qcd_lattice* h, int* out) {
  if (!h || !out) return QCD_ERR_INVALID;
  const long long V = h->V;
  const int vh = h->g.vh;
  if (h->accept) {
    CUDA_OR_FAIL(h, cudaMemcpyAsync(out, h->accept, (size_t)V * sizeof(int), cudaMemcpyDeviceToHost,
                                    h->stream));
    int rc = check_device_error(h);
    if (rc) return rc;
  } else {
    memset(out, 0, (size_t)V * sizeof(int));
  }
  // heat-bath and over-relaxation: 1 per link update (mc_updates.h:63,114); PCC
  // skips the x and t links on the plane y = 0 (mc_updates_pcc.h:29)
  if (h->unit_passes) {
    const int lyh = h->g.lyh, lx = h->g.lx;
    for (int p = 0; p < 2; p++)
      for (int id = 0; id < vh; id++) {
        int yq = id % lyh, r = id / lyh, x = r % lx, t = r / lx;
        int q = ((t + x) & 1) ^ p;
        int links = (h->p.boundary == QCD_BC_PCC && yq == 0 && q == 0) ? 1 : 3;
        out[(size_t)p * vh + id] += (int)(links * h->unit_passes);
      }
  }
  return QCD_OK;
}

int qcd_accept_reset(qcd_lattice* h) {
  if (!h) return QCD_ERR_INVALID;
  if (h->accept) CUDA_OR_FAIL(h, cudaMemsetAsync(h->accept, 0, (size_t)h->V * sizeof(int), h->stream));
  h->unit_passes = 0;
  return QCD_OK;
}

int qcd_check_unitarity(qcd_lattice* h, double tol, double* mean_det) {
  if (!h || !(tol >= 0)) return QCD_ERR_INVALID;
  const unsigned int nb = nblocks(h->g.vh);
  if (h->p.precision == QCD_PREC_FP64)
    unitarity<<<nb, kBlock, 0, h->stream>>>(links64(h), h->g.vh, tol, h->partials, h->counter, h->result);
  else if (h->paired)
    unitarity_p<<<nblocks(h->gh.vh), kBlock, 0, h->stream>>>(pair32(h), tol, h->partials, h->counter, h->result);
  else
    unitarity<<<nb, kBlock, 0, h->stream>>>(links32(h), h->g.vh, tol, h->partials, h->counter, h->result);
  LAUNCH_CHECK(h);
  double sum = 0, bad = 0;
  int rc = reduce_result(h, &sum, &bad);
  if (rc) return rc;
  if (mean_det) *mean_det = sum / (3.0 * (double)h->V);
  if (bad > 0)
    return fail(h, QCD_ERR_NONUNITARY, "%.0f of %lld links have |det-1| > %g or are not finite", bad,
                3 * h->V, tol);
  return QCD_OK;
}

// The generator checkpoint: the six u32 words of each of the V/2 MRG32k3a
// streams, plane by plane (word j of stream id at [j * V/2 + id]), then the
// drawing-phase counter and the key of the FP32 Philox draws (low word
// first).  The reference keeps no generator state across runs (a restart
// re-seeds, kernel.cu:79); saving it next to the configuration makes a
// resumed run continue the exact same chain.
long long qcd_rng_words(const qcd_lattice* h) { return h ? 6 * (long long)h->g.vh + 4 : 0; }

int qcd_store_rng(qcd_lattice* h, uint32_t* host_out) {
  if (!h || !host_out) return QCD_ERR_INVALID;
  int rc0 = ensure_rng(h);
  if (rc0) return rc0;
  const size_t n = 6 * (size_t)h->g.vh;
  CUDA_OR_FAIL(h, cudaMemcpyAsync(host_out, h->rng, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  unsigned long long* c = reinterpret_cast<unsigned long long*>(&h->result_host[3]);
  CUDA_OR_FAIL(h, cudaMemcpyAsync(c, h->draw_dev, sizeof(*c), cudaMemcpyDeviceToHost, h->stream));
  int rc = check_device_error(h);  // synchronises the stream
  host_out[n] = (uint32_t)*c;
  host_out[n + 1] = (uint32_t)(*c >> 32);
  host_out[n + 2] = (uint32_t)h->draw_key;
  host_out[n + 3] = (uint32_t)(h->draw_key >> 32);
  return rc;
}

int qcd_load_rng(qcd_lattice* h, const uint32_t* host_in) {
  if (!h || !host_in) return QCD_ERR_INVALID;
  int rc0 = ensure_rng(h);
  if (rc0) return rc0;
  const size_t n = 6 * (size_t)h->g.vh;
  const unsigned long long c = (unsigned long long)host_in[n] | ((unsigned long long)host_in[n + 1] << 32);
  CUDA_OR_FAIL(h, cudaMemcpyAsync(h->rng, host_in, n * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
  CUDA_OR_FAIL(h, cudaMemcpyAsync(h->draw_dev, &c, sizeof(c), cudaMemcpyHostToDevice, h->stream));
  CUDA_OR_FAIL(h, cudaStreamSynchronize(h->stream));
  h->draw_key = (unsigned long long)host_in[n + 2] | ((unsigned long long)host_in[n + 3] << 32);
  return QCD_OK;
}

void qcd_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  Philox4x32::block(ctr, key, out);
}

long long qcd_volume(const qcd_lattice* h) { return h ? h->V : 0; }

int qcd_get_params(const qcd_lattice* h, qcd_params* out) {
  if (!h || !out) return QCD_ERR_INVALID;
  *out = h->p;
  return QCD_OK;
}

int qcd_link_store(const qcd_lattice* h, void** dev_ptr, size_t* bytes) {
  if (!h) return QCD_ERR_INVALID;
  if (dev_ptr) *dev_ptr = h->p.precision == QCD_PREC_FP64 ? (void*)h->lo : (void*)h->q32;
  if (bytes) *bytes = h->link_bytes;
  return QCD_OK;
}

int qcd_rng_tape(unsigned long long seed, long long first, int n_streams, int n_draws,
                 qcd_tape_record* host_out) {
  static_assert(sizeof(qcd_tape_record) == sizeof(TapeRec), "tape record layout");
  if (n_streams <= 0 || n_draws <= 0 || first < 0 || !host_out) return QCD_ERR_INVALID;
  size_t n = (size_t)n_streams * n_draws;
  TapeRec* d = nullptr;
  if (cudaMalloc(&d, n * sizeof(TapeRec)) != cudaSuccess) {
    cudaGetLastError();
    return QCD_ERR_NOMEM;
  }
  rng_tape<<<nblocks(n_streams), kBlock>>>(seed, first, n_streams, n_draws, d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(host_out, d, n * sizeof(TapeRec), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e == cudaSuccess ? QCD_OK : QCD_ERR_CUDA;
}

}  // extern "C"

// ======================================================== no allocation ==
// Measurement of a caller-held configuration that allocates nothing: the
// reduction scratch (one partial sum per CTA and the arrival counter) is the
// file-scope array below instead of cudaMalloc'd memory.  A program that has
// sized its lattice to fill the GPU, or whose device memory belongs to the
// pooling allocator of its host framework, or whose sweep loop cannot take
// the implicit device synchronisation of cudaMalloc/cudaFree, can still
// measure.  The kernel is measure<> (same per-site arithmetic, CTA size and
// summation order as qcd_measure) reading the reference's AoS FP64 layout.
namespace qcd {

struct LinksAoS {
  const double* phi;  // V*12 doubles: site (p*Vh + id), link d, component c
  int vh;
  __device__ __forceinline__ Quat<double> ld(int d, int p, int id) const {
    const double* s = phi + ((size_t)p * vh + id) * 12 + d * 4;
    double2 a = __ldg(reinterpret_cast<const double2*>(s));
    double2 b = __ldg(reinterpret_cast<const double2*>(s + 2));
    return Quat<double>{a.x, a.y, b.x, b.y};
  }
};
template <>
__device__ __forceinline__ Quat<double> ld64<LinksAoS>(const LinksAoS& links, int d, int p, int id) {
  return links.ld(d, p, id);
}

}  // namespace qcd

// partial sums of at most QCD_NOALLOC_MAX_BLOCKS CTAs, then the arrival counter
static_assert(kMeasureMaxBlocks <= QCD_NOALLOC_MAX_BLOCKS,
              "a measurement may launch more CTAs than the no-allocation scratch has partial sums");
static_assert((long long)QCD_NOALLOC_MAX_HALF_SITES * 6 < (1ll << 31), "32-bit plane indices");
static constexpr size_t kNoAllocCounterOffset = (size_t)QCD_NOALLOC_MAX_BLOCKS * sizeof(double2);
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocCounterOffset + 256];

namespace {
// Host code may not use g_noalloc_scratch itself (on the host it names a
// stand-in, not device memory): look up its device address on the current
// device at every call.  The lookup allocates nothing and is cheap once the
// module is loaded; not caching it keeps the address right after a
// cudaDeviceReset or under another context on the same device.
int noalloc_scratch(void** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    int dev = -1;
    cudaGetDevice(&dev);
    cudaGetLastError();
    fprintf(stderr, "qcd_measure_aos_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
            cudaGetErrorString(e));
    return QCD_ERR_CUDA;
  }
  *out = p;
  return QCD_OK;
}
}  // namespace

extern "C" int qcd_measure_aos_noalloc(const double* phi_dev, int lt, int lx, int ly, int boundary,
                                       double* out_dev, void* stream) {
  if (!phi_dev || !out_dev) return QCD_ERR_INVALID;
  if (lt < 2 || lx < 2 || ly < 2 || (lt & 1) || (lx & 1) || (ly & 1)) return QCD_ERR_INVALID;
  if (boundary < 0 || boundary > 2) return QCD_ERR_INVALID;
  if (((uintptr_t)phi_dev & 15) || ((uintptr_t)out_dev & 7)) return QCD_ERR_INVALID;
  // in double first: the product of three ints can overflow 64 bits
  if (0.5 * (double)lt * (double)lx * (double)ly > (double)QCD_NOALLOC_MAX_HALF_SITES) {
    fprintf(stderr,
            "qcd_measure_aos_noalloc: %dx%dx%d has V/2 = %.0f sites, above the %d that 32-bit site "
            "indices address\n",
            lt, lx, ly, 0.5 * (double)lt * (double)lx * (double)ly, QCD_NOALLOC_MAX_HALF_SITES);
    return QCD_ERR_UNSUPPORTED;
  }
  const long long vh = (long long)lt * lx * ly / 2;
  if (measure_blocks(vh) > QCD_NOALLOC_MAX_BLOCKS) return QCD_ERR_UNSUPPORTED;  // excluded by the static_assert
  void* base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc) return rc;
  double2* partials = reinterpret_cast<double2*>(base);
  unsigned int* counter = reinterpret_cast<unsigned int*>(static_cast<char*>(base) + kNoAllocCounterOffset);
  cudaStream_t s = (cudaStream_t)stream;
  // the array keeps whatever the previous call left: the arrival counter must start at zero
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), s);
  if (e == cudaSuccess) {
    Geo g = make_geo(lt, lx, ly);
    LinksAoS L{phi_dev, (int)vh};
    const unsigned int grid = measure_blocks(vh);  // the same grid, so the same sums, as qcd_measure
    if (boundary == QCD_BC_PMC)
      measure<LinksAoS, 1><<<grid, kBlock, 0, s>>>(L, g, partials, counter, out_dev);
    else
      measure<LinksAoS, 0><<<grid, kBlock, 0, s>>>(L, g, partials, counter, out_dev);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    fprintf(stderr, "qcd_measure_aos_noalloc: %s\n", cudaGetErrorString(e));
    return QCD_ERR_CUDA;
  }
  return QCD_OK;
}
