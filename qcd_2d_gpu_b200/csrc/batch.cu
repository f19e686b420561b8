// Batched replicas: many independent lattices of different size, coupling
// and boundary condition advanced together.
//
// All replicas live in one link store and one MRG32k3a store (each
// replica's planes contiguous, offsets in a device replica table; the FP32
// sweep draws from Philox counters instead, as a single lattice does).  One launch per
// checkerboard phase covers every replica: CTA c belongs to the replica whose
// [cta_begin, cta_begin + ceil(V/2 / 256)) range holds c, so a sweep of the
// whole batch is 6 launches (plus passes of over-relaxation) instead of
// 6 x n_replicas, and a measurement is one launch writing every replica's
// (energy, plaquette) into a device series at a device-side cursor.  The
// sweep + measurement is captured once as a CUDA graph and replayed.  The
// per-link code is the single-lattice code (site32 / site64), so replica r
// reproduces a single lattice with the same seed and stream offset.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <new>
#include <utility>
#include <vector>

#include "qcd2d.h"
#include "sites.cuh"

using namespace qcd;

namespace {

struct Replica {
  Geo g;
  float beta;
  int bc;
  int hot;
  long long link_off;  // float4 units (FP32) or double2 units per lo/hi plane (FP64)
  long long rng_off;   // u32 words
  long long site_off;  // accept counters
  int cta_begin;       // first CTA of this replica in a batched launch
  int mcta_begin;      // first CTA of this replica in a batched measurement (measure_blocks per replica)
  unsigned long long seed;
  long long stream_off;
};

struct BatchView {
  const Replica* rep;
  const int* cta_rep;  // replica of every CTA of a batched launch
  const int* mcta_rep; // replica of every CTA of a batched measurement
  int n;               // replicas the launch covers
  int cta0, mcta0;     // first CTA of the launch in the batch's CTA tables (a group's offset)
  float4* q32;
  double2* lo;
  double2* hi;
  uint32_t* rng;
};

// a launch's CTA in the batch's CTA table, and its replica
__device__ __forceinline__ int batch_cta(const BatchView& B) { return (int)blockIdx.x + B.cta0; }
__device__ __forceinline__ int replica_of(const BatchView& B, int cta) { return __ldg(B.cta_rep + cta); }

struct BatchArgs {
  float eps;
  int upd;
  int* err;
  int* accept;
  int renorm;
  const unsigned long long* phase_ptr;  // drawing phases run so far (device word)
  unsigned int phase_off;               // this phase's offset from it
};

template <int MU, int PAR, int KIND, bool FP64>
__global__ void __launch_bounds__(kBlock, 6) batch_phase(BatchView B, BatchArgs a) {
  const int cta = batch_cta(B);
  const int r = replica_of(B, cta);
  const Replica& R = B.rep[r];
  const int id = (cta - R.cta_begin) * kBlock + threadIdx.x;
  if (id >= R.g.vh) return;
  const Nbr n = make_nbr_fast(R.g, id, PAR);
  // FP32 draws: the replica's seed as key, its stream offset added to the
  // site index, the batch-wide drawing-phase counter (as for one lattice)
  PhaseArgs pa{R.beta, a.eps, a.upd, a.err, a.accept ? a.accept + R.site_off : nullptr, a.renorm,
               R.seed, a.phase_ptr, a.phase_off, (unsigned int)R.stream_off, philox_keys(R.seed)};
  RngStore RS{B.rng + R.rng_off, R.g.vh};
  if (FP64) {
    Links64 L{B.lo + R.link_off, B.hi + R.link_off, R.g.vh};
    switch (R.bc) {
      case BC_PER: site64<MU, PAR, BC_PER, KIND, false>(L, RS, R.g, pa, n); break;
      case BC_PCC: site64<MU, PAR, BC_PCC, KIND, false>(L, RS, R.g, pa, n); break;
      default: site64<MU, PAR, BC_PMC, KIND, false>(L, RS, R.g, pa, n); break;
    }
  } else {
    Links32 L{B.q32 + R.link_off, R.g.vh};
    switch (R.bc) {
      case BC_PER: site32<MU, PAR, BC_PER, KIND, false>(L, RS, R.g, pa, n, a.renorm); break;
      case BC_PCC: site32<MU, PAR, BC_PCC, KIND, false>(L, RS, R.g, pa, n, a.renorm); break;
      default: site32<MU, PAR, BC_PMC, KIND, false>(L, RS, R.g, pa, n, a.renorm); break;
    }
  }
}

// curand_init(seed_r, stream_off_r + id, 0) per site of every replica (one
// curand_init per CTA and a jump per thread, as rng_setup), then the
// replica's start (rand_init2 / rand_init2_pcc / id_init2 semantics)
template <bool FP64>
__global__ void __launch_bounds__(kBlock) batch_setup(BatchView B, const uint32_t* __restrict__ jumps) {
  const int cta = batch_cta(B);
  const int r = replica_of(B, cta);
  const Replica& R = B.rep[r];
  const int id0 = (cta - R.cta_begin) * kBlock;
  __shared__ unsigned int base[6];
  if (threadIdx.x == 0) mrg_cta_base(base, jumps, R.seed, (unsigned long long)(R.stream_off + id0));
  __syncthreads();
  const int id = id0 + threadIdx.x;
  if (id >= R.g.vh) return;
  curandStateMRG32k3a_t st;
  mrg_jump_from(base, jumps, threadIdx.x, &st);
  for (int p = 0; p < 2; p++) {
    const Nbr n = make_nbr(R.g, id, p);
    const bool frozen = R.bc == BC_PCC && at_y0(R.g, n);
    for (int d = 0; d < 3; d++) {
      Quat<double> u = q_one<double>();
      if (R.hot && !(d != DIR_Y && frozen)) {
        u.w = curand_uniform_double(&st) - 0.5;
        u.x = curand_uniform_double(&st) - 0.5;
        u.y = curand_uniform_double(&st) - 0.5;
        u.z = curand_uniform_double(&st) - 0.5;
        u = q_normalize(u);
      }
      if (FP64) {
        Links64 L{B.lo + R.link_off, B.hi + R.link_off, R.g.vh};
        L.st(d, p, id, u);
      } else {
        Links32 L{B.q32 + R.link_off, R.g.vh};
        L.st(d, p, id, Quat<float>{(float)u.w, (float)u.x, (float)u.y, (float)u.z});
      }
    }
  }
  RngStore RS{B.rng + R.rng_off, R.g.vh};
  RS.store(id, &st);
}

template <bool FP64>
__global__ void __launch_bounds__(kBlock) batch_normalize(BatchView B) {
  const int cta = batch_cta(B);
  const int r = replica_of(B, cta);
  const Replica& R = B.rep[r];
  const int id = (cta - R.cta_begin) * kBlock + threadIdx.x;
  if (id >= R.g.vh) return;
  for (int p = 0; p < 2; p++)
    for (int d = 0; d < 3; d++) {
      if (FP64) {
        Links64 L{B.lo + R.link_off, B.hi + R.link_off, R.g.vh};
        L.st(d, p, id, q_normalize(L.ld_own(d, p, id)));
      } else {
        Links32 L{B.q32 + R.link_off, R.g.vh};
        L.st(d, p, id, renorm_fast(L.ld_own(d, p, id)));
      }
    }
}

// energy / plaquette of every replica (en_av semantics, observables.h:99-141)
// into series[r * cap + *cursor]; per-replica fixed-order sums as in measure<>
// Energy and plaquette of every replica into series[r * cap + k], k the
// device cursor.  Each replica's CTAs cover it as a single-lattice
// measurement does (measure_blocks CTAs striding over its sites) and its last
// CTA adds their partials in the same order, so every replica's numbers are
// those of the same lattice measured alone, bit for bit.
template <bool FP64>
__global__ void __launch_bounds__(kBlock) batch_measure(BatchView B, double2* partials, unsigned int* rep_count,
                                                        unsigned int* all_count, int* cursor, double2* series,
                                                        int cap) {
  const int mcta = (int)blockIdx.x + B.mcta0;  // CTA in the batch's measurement table
  const int r = __ldg(B.mcta_rep + mcta);
  const Replica& R = B.rep[r];
  const int nblk = (int)measure_blocks(R.g.vh);
  const int k = *(volatile int*)cursor;  // advanced only by the last CTA below
  double e = 0, pl = 0;
  if (FP64) {
    Links64 L{B.lo + R.link_off, B.hi + R.link_off, R.g.vh};
    if (R.bc == BC_PMC)
      measure_sites<Links64, true>(L, R.g, mcta - R.mcta_begin, nblk, e, pl);
    else
      measure_sites<Links64, false>(L, R.g, mcta - R.mcta_begin, nblk, e, pl);
  } else {
    Links32 L{B.q32 + R.link_off, R.g.vh};
    if (R.bc == BC_PMC)
      measure_sites<Links32, true>(L, R.g, mcta - R.mcta_begin, nblk, e, pl);
    else
      measure_sites<Links32, false>(L, R.g, mcta - R.mcta_begin, nblk, e, pl);
  }
  double se, sp;
  block_sum2(e, pl * (1.0 / 3.0), &se, &sp);
  __shared__ bool last_rep;
  if (threadIdx.x == 0) {
    partials[mcta] = make_double2(se, sp);
    __threadfence();
    last_rep = atomicAdd(rep_count + r, 1u) == (unsigned int)nblk - 1;
  }
  __syncthreads();
  if (last_rep) {
    __threadfence();
    double a = 0, b = 0;
    for (int i = threadIdx.x; i < nblk; i += kBlock) {
      double2 v = __ldcg(partials + R.mcta_begin + i);
      a += v.x;
      b += v.y;
    }
    __syncthreads();
    double sa, sb;
    block_sum2(a, b, &sa, &sb);
    if (threadIdx.x == 0) {
      const double scale = 1.0 / (2.0 * (double)R.g.vh);
      if (k < cap) series[(size_t)r * cap + k] = make_double2(sa * scale, sb * scale);
      rep_count[r] = 0u;
      // the last replica of the launch to finish (every CTA done) moves the
      // cursor of the launch's replicas: one atomic per replica, not per CTA
      __threadfence();
      const bool last_all = atomicAdd(all_count, 1u) == (unsigned int)B.n - 1;
      if (last_all) {
        *all_count = 0u;
        *cursor = k + 1;
      }
    }
  }
}

typedef void (*BatchPhaseFn)(BatchView, BatchArgs);

template <int MU, int PAR, bool FP64>
BatchPhaseFn pick_kind(int kind) {
  return kind == KIND_HB ? batch_phase<MU, PAR, KIND_HB, FP64>
         : kind == KIND_METRO ? batch_phase<MU, PAR, KIND_METRO, FP64>
                              : batch_phase<MU, PAR, KIND_OR, FP64>;
}

template <bool FP64>
BatchPhaseFn batch_phase_fn(int k, int kind) {
  switch (k) {
    case 0: return pick_kind<DIR_Y, 0, FP64>(kind);
    case 1: return pick_kind<DIR_Y, 1, FP64>(kind);
    case 2: return pick_kind<DIR_X, 0, FP64>(kind);
    case 3: return pick_kind<DIR_X, 1, FP64>(kind);
    case 4: return pick_kind<DIR_T, 0, FP64>(kind);
    default: return pick_kind<DIR_T, 1, FP64>(kind);
  }
}

}  // namespace

// A group: a run of consecutive replicas swept together.  Replicas are
// independent, so a group can go through all the sweeps of a run while its
// links stay in L2 before the next group starts (each group with its own
// drawing-phase counter and measurement cursor, so every replica draws and
// records exactly what it would in one group of everything).
// default grouping (the autotuner's choice for 96 mixed replicas, C4): groups
// of up to 32 MB of links, well inside the 126 MB L2, two at a time
constexpr long long kBatchGroupBytes = 32ll << 20;
constexpr int kBatchLanes = 2;

struct BatchGroup {
  int r0, r1;         // replicas [r0, r1)
  int cta0, ctas;     // its CTAs in the phase launches' table
  int mcta0, mctas;   // its CTAs in the measurement's table
  cudaGraphExec_t graph = nullptr;  // one measurement interval of this group
};

struct qcd_batch {
  std::vector<Replica> rep;
  qcd_params common;
  int n = 0;
  long long sites = 0;
  int ctas = 0;
  cudaStream_t own = nullptr, stream = nullptr;
  Replica* rep_dev = nullptr;
  int* cta_rep = nullptr;
  int* mcta_rep = nullptr;
  int mctas = 0;
  float4* q32 = nullptr;
  double2* lo = nullptr;
  double2* hi = nullptr;
  uint32_t* rng = nullptr;
  uint32_t* mrg_jumps = nullptr;  // jump matrices that seed the streams (mrg_jump_table)
  // per group (n entries, groups use the first ones): drawing phases run so
  // far (FP32 draws), arrival counter and cursor of the measurement
  unsigned long long* draw_dev = nullptr;
  unsigned int* all_count = nullptr;
  int* cursor = nullptr;
  int* accept = nullptr;
  int* err = nullptr;
  double2* partials = nullptr;
  unsigned int* rep_count = nullptr;
  double2* series = nullptr;
  int cap = 0;
  long long sweeps_done = 0;
  std::vector<BatchGroup> groups;
  long long group_bytes = 0;  // target link bytes per group (0: one group)
  // lanes: streams that run groups concurrently (group g on lane g mod lanes),
  // forked from and joined back into `stream` by events
  static constexpr int kMaxLanes = 4;
  int lanes = kBatchLanes;
  cudaStream_t lane[kMaxLanes] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t fork_ev = nullptr, join_ev[kMaxLanes] = {nullptr, nullptr, nullptr, nullptr};
  int graph_every = 0;
  char msg[512] = {0};
};

namespace {

int bfail(qcd_batch* b, int code, const char* fmt, ...) {
  if (b) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(b->msg, sizeof(b->msg), fmt, ap);
    va_end(ap);
  }
  return code;
}

#define BCUDA(b, call)                                                                              \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess) {                                                                        \
      cudaGetLastError();                                                                           \
      return bfail(b, e_ == cudaErrorMemoryAllocation ? QCD_ERR_NOMEM : QCD_ERR_CUDA, "%s: %s", #call, \
                   cudaGetErrorString(e_));                                                         \
    }                                                                                               \
  } while (0)

// every replica (setup, whole-batch launches)
BatchView view(const qcd_batch* b) {
  return BatchView{b->rep_dev, b->cta_rep, b->mcta_rep, b->n, 0, 0, b->q32, b->lo, b->hi, b->rng};
}
// the replicas of one group
BatchView view(const qcd_batch* b, const BatchGroup& g) {
  return BatchView{b->rep_dev, b->cta_rep, b->mcta_rep, g.r1 - g.r0, g.cta0, g.mcta0, b->q32, b->lo, b->hi, b->rng};
}

bool fp64(const qcd_batch* b) { return b->common.precision == QCD_PREC_FP64; }

long long link_bytes_of(const qcd_batch* b, int r) {
  return 6ll * b->rep[r].g.vh * (fp64(b) ? 32 : 16);
}

void drop_graphs(qcd_batch* b) {
  for (BatchGroup& g : b->groups)
    if (g.graph) {
      cudaGraphExecDestroy(g.graph);
      g.graph = nullptr;
    }
}

// consecutive replicas up to `bytes` of links per group (at least one
// replica each); 0 puts every replica in one group
void form_groups(qcd_batch* b, long long bytes) {
  drop_graphs(b);
  b->groups.clear();
  b->group_bytes = bytes;
  int r = 0;
  while (r < b->n) {
    BatchGroup g;
    g.r0 = r;
    long long acc = 0;
    do {
      acc += link_bytes_of(b, r);
      r++;
    } while (r < b->n && (bytes <= 0 || acc + link_bytes_of(b, r) <= bytes));
    g.r1 = r;
    g.cta0 = b->rep[g.r0].cta_begin;
    g.ctas = (g.r1 < b->n ? b->rep[g.r1].cta_begin : b->ctas) - g.cta0;
    g.mcta0 = b->rep[g.r0].mcta_begin;
    g.mctas = (g.r1 < b->n ? b->rep[g.r1].mcta_begin : b->mctas) - g.mcta0;
    b->groups.push_back(g);
  }
}

// All groups hold the same counter and cursor between runs: give every
// group slot the values of slot 0 (after the groups were formed anew).
__global__ void spread_group_state(unsigned long long* draw, int* cursor, unsigned int* all_count, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    draw[i] = draw[0];
    cursor[i] = cursor[0];
    all_count[i] = 0u;
  }
}

int batch_pass(qcd_batch* b, int gi, int kind, int renorm) {
  const BatchGroup& g = b->groups[gi];
  BatchArgs a{b->common.epsilon, b->common.upd, b->err, b->accept, renorm, b->draw_dev + gi, 0};
  for (int k = 0; k < 6; k++) {
    a.phase_off = (unsigned int)k;
    if (fp64(b))
      batch_phase_fn<true>(k, kind)<<<g.ctas, kBlock, 0, b->stream>>>(view(b, g), a);
    else
      batch_phase_fn<false>(k, kind)<<<g.ctas, kBlock, 0, b->stream>>>(view(b, g), a);
    BCUDA(b, cudaGetLastError());
  }
  if (kind != KIND_OR) {
    advance_counter<<<1, 1, 0, b->stream>>>(b->draw_dev + gi, 6ull);
    BCUDA(b, cudaGetLastError());
  }
  return QCD_OK;
}

// one sweep of a group's replicas (+ n_or over-relaxation passes; FP32 links
// are re-projected at their last update when `renorm`, FP64 by a normalize launch)
int batch_sweep(qcd_batch* b, int gi, bool renorm) {
  const int kind = b->common.algo == QCD_ALGO_HEATBATH ? KIND_HB : KIND_METRO;
  const bool fused = renorm && !fp64(b);
  int rc = batch_pass(b, gi, kind, fused && b->common.n_or == 0);
  for (int r = 0; rc == QCD_OK && r < b->common.n_or; r++) rc = batch_pass(b, gi, KIND_OR, fused && r == b->common.n_or - 1);
  if (rc) return rc;
  if (renorm && !fused) {
    const BatchGroup& g = b->groups[gi];
    if (fp64(b))
      batch_normalize<true><<<g.ctas, kBlock, 0, b->stream>>>(view(b, g));
    else
      batch_normalize<false><<<g.ctas, kBlock, 0, b->stream>>>(view(b, g));
    BCUDA(b, cudaGetLastError());
  }
  return QCD_OK;
}

int batch_measure_launch(qcd_batch* b, int gi) {
  const BatchGroup& g = b->groups[gi];
  if (fp64(b))
    batch_measure<true><<<g.mctas, kBlock, 0, b->stream>>>(view(b, g), b->partials, b->rep_count, b->all_count + gi,
                                                           b->cursor + gi, b->series, b->cap);
  else
    batch_measure<false><<<g.mctas, kBlock, 0, b->stream>>>(view(b, g), b->partials, b->rep_count,
                                                            b->all_count + gi, b->cursor + gi, b->series, b->cap);
  BCUDA(b, cudaGetLastError());
  return QCD_OK;
}

bool renorm_due(const qcd_batch* b, long long sweep_index) {
  return b->common.renorm_every > 0 && (sweep_index + 1) % b->common.renorm_every == 0;
}

void release(qcd_batch* b) {
  drop_graphs(b);
  cudaFree(b->rep_dev);
  cudaFree(b->cta_rep);
  cudaFree(b->mcta_rep);
  cudaFree(b->q32);
  cudaFree(b->lo);
  cudaFree(b->hi);
  cudaFree(b->rng);
  cudaFree(b->mrg_jumps);
  cudaFree(b->accept);
  cudaFree(b->err);
  cudaFree(b->draw_dev);
  cudaFree(b->partials);
  cudaFree(b->rep_count);
  cudaFree(b->all_count);
  cudaFree(b->cursor);
  cudaFree(b->series);
  for (int k = 0; k < qcd_batch::kMaxLanes; k++) {
    if (b->lane[k]) cudaStreamDestroy(b->lane[k]);
    if (b->join_ev[k]) cudaEventDestroy(b->join_ev[k]);
  }
  if (b->fork_ev) cudaEventDestroy(b->fork_ev);
  if (b->own) cudaStreamDestroy(b->own);
}

}  // namespace

extern "C" {

int qcd_batch_create(const qcd_replica* r, int n, const qcd_params* common, qcd_batch** out) {
  if (!r || n < 1 || !common || !out) return QCD_ERR_INVALID;
  *out = nullptr;
  if (common->algo != QCD_ALGO_HEATBATH && common->algo != QCD_ALGO_METROPOLIS) return QCD_ERR_INVALID;
  if (common->precision != QCD_PREC_FP64 && common->precision != QCD_PREC_FP32) return QCD_ERR_INVALID;
  if (common->n_or < 0 || common->renorm_every < 0 || common->upd < 0) return QCD_ERR_INVALID;
  if (common->algo == QCD_ALGO_METROPOLIS && !(common->epsilon > 0.f && common->epsilon < 1.f)) return QCD_ERR_INVALID;
  qcd_batch* b = new (std::nothrow) qcd_batch();
  if (!b) return QCD_ERR_NOMEM;
  b->common = *common;
  b->n = n;
  long long link_off = 0, rng_off = 0, site_off = 0;
  int cta = 0, mcta = 0;
  for (int i = 0; i < n; i++) {
    const qcd_replica& x = r[i];
    if (x.lt < 2 || x.lx < 2 || x.ly < 2 || (x.lt & 1) || (x.lx & 1) || (x.ly & 1) || !(x.beta > 0.f) ||
        x.boundary < 0 || x.boundary > 2 || x.stream_offset < 0 ||
        x.stream_offset > kMrgMaxStreams - (long long)x.lt * x.lx * x.ly / 2) {
      delete b;
      return QCD_ERR_INVALID;
    }
    const long long V = (long long)x.lt * x.lx * x.ly;
    if (V / 2 >= (1ll << 31) / 6) {
      delete b;
      return QCD_ERR_INVALID;
    }
    Replica R;
    R.g = make_geo(x.lt, x.lx, x.ly);
    R.beta = x.beta;
    R.bc = x.boundary;
    R.hot = x.hot;
    R.link_off = link_off;
    R.rng_off = rng_off;
    R.site_off = site_off;
    R.cta_begin = cta;
    R.mcta_begin = mcta;
    R.seed = x.seed;
    R.stream_off = x.stream_offset;
    b->rep.push_back(R);
    link_off += 6 * (V / 2);
    rng_off += 6 * (V / 2);
    site_off += V;
    cta += (int)((V / 2 + kBlock - 1) / kBlock);
    mcta += (int)measure_blocks(V / 2);
  }
  b->sites = site_off;
  b->ctas = cta;
  b->mctas = mcta;
  int rc = QCD_OK;
  auto step = [&](cudaError_t e, const char* what) {
    if (rc == QCD_OK && e != cudaSuccess) {
      rc = e == cudaErrorMemoryAllocation ? QCD_ERR_NOMEM : QCD_ERR_CUDA;
      cudaGetLastError();
      snprintf(b->msg, sizeof(b->msg), "%s: %s", what, cudaGetErrorString(e));
    }
  };
  step(cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking), "cudaStreamCreate");
  b->stream = b->own;
  for (int k = 0; k < qcd_batch::kMaxLanes; k++) {
    if (rc == QCD_OK) step(cudaStreamCreateWithFlags(&b->lane[k], cudaStreamNonBlocking), "cudaStreamCreate(lane)");
    if (rc == QCD_OK) step(cudaEventCreateWithFlags(&b->join_ev[k], cudaEventDisableTiming), "cudaEventCreate");
  }
  if (rc == QCD_OK) step(cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming), "cudaEventCreate");
  if (rc == QCD_OK) step(cudaMalloc(&b->rep_dev, n * sizeof(Replica)), "cudaMalloc(replicas)");
  if (rc == QCD_OK)
    step(cudaMemcpy(b->rep_dev, b->rep.data(), n * sizeof(Replica), cudaMemcpyHostToDevice), "replica table");
  if (rc == QCD_OK) {
    std::vector<int> owner((size_t)cta);
    for (int i = 0; i < n; i++) {
      const int end = i + 1 < n ? b->rep[i + 1].cta_begin : cta;
      for (int c = b->rep[i].cta_begin; c < end; c++) owner[c] = i;
    }
    step(cudaMalloc(&b->cta_rep, (size_t)cta * sizeof(int)), "cudaMalloc(cta table)");
    if (rc == QCD_OK)
      step(cudaMemcpy(b->cta_rep, owner.data(), (size_t)cta * sizeof(int), cudaMemcpyHostToDevice), "cta table");
    std::vector<int> mowner((size_t)mcta);
    for (int i = 0; i < n; i++) {
      const int end = i + 1 < n ? b->rep[i + 1].mcta_begin : mcta;
      for (int c = b->rep[i].mcta_begin; c < end; c++) mowner[c] = i;
    }
    if (rc == QCD_OK) step(cudaMalloc(&b->mcta_rep, (size_t)mcta * sizeof(int)), "cudaMalloc(cta table)");
    if (rc == QCD_OK)
      step(cudaMemcpy(b->mcta_rep, mowner.data(), (size_t)mcta * sizeof(int), cudaMemcpyHostToDevice),
           "cta table");
  }
  if (common->precision == QCD_PREC_FP64) {
    if (rc == QCD_OK) step(cudaMalloc(&b->lo, link_off * sizeof(double2)), "cudaMalloc(links)");
    if (rc == QCD_OK) step(cudaMalloc(&b->hi, link_off * sizeof(double2)), "cudaMalloc(links)");
  } else if (rc == QCD_OK) {
    step(cudaMalloc(&b->q32, link_off * sizeof(float4)), "cudaMalloc(links)");
  }
  if (rc == QCD_OK) step(cudaMalloc(&b->rng, rng_off * sizeof(uint32_t)), "cudaMalloc(rng)");
  if (rc == QCD_OK) step(cudaMalloc(&b->mrg_jumps, kMrgJumpWords * sizeof(uint32_t)), "cudaMalloc(jumps)");
  if (rc == QCD_OK)
    step(cudaMemcpy(b->mrg_jumps, mrg_jump_host(), kMrgJumpWords * sizeof(uint32_t), cudaMemcpyHostToDevice),
         "jump table");
  if (rc == QCD_OK && common->algo == QCD_ALGO_METROPOLIS) {
    step(cudaMalloc(&b->accept, site_off * sizeof(int)), "cudaMalloc(accept)");
    if (rc == QCD_OK) step(cudaMemsetAsync(b->accept, 0, site_off * sizeof(int), b->stream), "memset");
  }
  if (rc == QCD_OK) step(cudaMalloc(&b->err, sizeof(int)), "cudaMalloc(err)");
  if (rc == QCD_OK) step(cudaMalloc(&b->draw_dev, n * sizeof(unsigned long long)), "cudaMalloc(draw counters)");
  if (rc == QCD_OK) step(cudaMemsetAsync(b->draw_dev, 0, n * sizeof(unsigned long long), b->stream), "memset");
  if (rc == QCD_OK)
    step(cudaMalloc(&b->partials, (size_t)(mcta > cta ? mcta : cta) * sizeof(double2)), "cudaMalloc(partials)");
  if (rc == QCD_OK) step(cudaMalloc(&b->rep_count, n * sizeof(unsigned int)), "cudaMalloc(counters)");
  if (rc == QCD_OK) step(cudaMalloc(&b->all_count, n * sizeof(unsigned int)), "cudaMalloc(counters)");
  if (rc == QCD_OK) step(cudaMalloc(&b->cursor, n * sizeof(int)), "cudaMalloc(cursor)");
  if (rc == QCD_OK) step(cudaMemsetAsync(b->err, 0, sizeof(int), b->stream), "memset");
  if (rc == QCD_OK) step(cudaMemsetAsync(b->rep_count, 0, n * sizeof(unsigned int), b->stream), "memset");
  if (rc == QCD_OK) step(cudaMemsetAsync(b->all_count, 0, n * sizeof(unsigned int), b->stream), "memset");
  if (rc == QCD_OK) step(cudaMemsetAsync(b->cursor, 0, n * sizeof(int), b->stream), "memset");
  if (rc == QCD_OK) step(cudaStreamSynchronize(b->stream), "cudaStreamSynchronize");
  if (rc != QCD_OK) {
    fprintf(stderr, "qcd_batch_create: %s\n", b->msg);
    release(b);
    delete b;
    return rc;
  }
  form_groups(b, kBatchGroupBytes);
  *out = b;
  return QCD_OK;
}

int qcd_batch_destroy(qcd_batch* b) {
  if (!b) return QCD_ERR_INVALID;
  if (b->stream) cudaStreamSynchronize(b->stream);
  release(b);
  delete b;
  return QCD_OK;
}

int qcd_batch_set_stream(qcd_batch* b, void* stream) {
  if (!b) return QCD_ERR_INVALID;
  BCUDA(b, cudaStreamSynchronize(b->stream));
  b->stream = stream ? (cudaStream_t)stream : b->own;
  drop_graphs(b);
  return QCD_OK;
}

int qcd_batch_init(qcd_batch* b) {
  if (!b) return QCD_ERR_INVALID;
  if (fp64(b))
    batch_setup<true><<<b->ctas, kBlock, 0, b->stream>>>(view(b), b->mrg_jumps);
  else
    batch_setup<false><<<b->ctas, kBlock, 0, b->stream>>>(view(b), b->mrg_jumps);
  BCUDA(b, cudaGetLastError());
  BCUDA(b, cudaMemsetAsync(b->cursor, 0, b->n * sizeof(int), b->stream));
  // a fresh start: the streams are re-seeded above, the counter of the FP32
  // draws starts again at 0 (as for a newly created lattice)
  BCUDA(b, cudaMemsetAsync(b->draw_dev, 0, b->n * sizeof(unsigned long long), b->stream));
  b->sweeps_done = 0;
  return QCD_OK;
}

int qcd_batch_reserve(qcd_batch* b, int capacity) {
  if (!b || capacity < 0) return QCD_ERR_INVALID;
  BCUDA(b, cudaStreamSynchronize(b->stream));
  cudaFree(b->series);
  b->series = nullptr;
  b->cap = 0;
  drop_graphs(b);  // the graphs hold the old series pointer
  if (capacity) {
    BCUDA(b, cudaMalloc(&b->series, (size_t)capacity * b->n * sizeof(double2)));
    BCUDA(b, cudaMemsetAsync(b->series, 0, (size_t)capacity * b->n * sizeof(double2), b->stream));
  }
  BCUDA(b, cudaMemsetAsync(b->cursor, 0, b->n * sizeof(int), b->stream));
  b->cap = capacity;
  return QCD_OK;
}

int qcd_batch_run(qcd_batch* b, int sweeps, int measure_every, int use_graph) {
  if (!b || sweeps < 0 || measure_every < 0) return QCD_ERR_INVALID;
  if (measure_every > 0 && b->cap == 0) return bfail(b, QCD_ERR_INVALID, "reserve a series before measuring");
  int rc = QCD_OK;
  // a graph of one measurement interval per group; its re-projection pattern
  // must not vary between replays, so it is used when renorm_every divides
  // the interval
  const int every = measure_every > 0 ? measure_every : 1;
  const bool graphable = use_graph && measure_every > 0 &&
                         (b->common.renorm_every == 0 || every % b->common.renorm_every == 0) &&
                         b->sweeps_done % every == 0 &&
                         (b->common.renorm_every == 0 || b->sweeps_done % b->common.renorm_every == 0);
  if (graphable && b->graph_every != every) {
    drop_graphs(b);
    b->graph_every = every;
  }
  // every group goes through all the sweeps before the next one starts on
  // its lane; with several lanes the groups of different lanes run at the
  // same time (one group's measurement next to another group's phases)
  const int lanes = b->lanes < (int)b->groups.size() ? b->lanes : (int)b->groups.size();
  cudaStream_t main = b->stream;
  if (lanes > 1) {
    BCUDA(b, cudaEventRecord(b->fork_ev, main));
    for (int k = 0; k < lanes; k++) BCUDA(b, cudaStreamWaitEvent(b->lane[k], b->fork_ev, 0));
  }
  for (int gi = 0; gi < (int)b->groups.size() && rc == QCD_OK; gi++) {
    BatchGroup& G = b->groups[gi];
    b->stream = lanes > 1 ? b->lane[gi % lanes] : main;  // the launch helpers use b->stream
    long long swept = b->sweeps_done;
    int done = 0;
    if (graphable && sweeps >= every) {
      if (!G.graph) {
        cudaGraph_t g;
        cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) {
          rc = bfail(b, QCD_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
          break;
        }
        for (int s = 0; rc == QCD_OK && s < every; s++) rc = batch_sweep(b, gi, renorm_due(b, s));
        if (rc == QCD_OK) rc = batch_measure_launch(b, gi);
        e = cudaStreamEndCapture(b->stream, &g);
        if (rc) {
          if (e == cudaSuccess) cudaGraphDestroy(g);
          break;
        }
        if (e == cudaSuccess) {
          e = cudaGraphInstantiate(&G.graph, g, 0);
          cudaGraphDestroy(g);
        }
        if (e != cudaSuccess) {
          rc = bfail(b, QCD_ERR_CUDA, "graph: %s", cudaGetErrorString(e));
          break;
        }
      }
      for (; done + every <= sweeps && rc == QCD_OK; done += every) {
        if (cudaGraphLaunch(G.graph, b->stream) != cudaSuccess) rc = bfail(b, QCD_ERR_CUDA, "graph launch");
        swept += every;
      }
    }
    for (; done < sweeps && rc == QCD_OK; done++) {
      rc = batch_sweep(b, gi, renorm_due(b, swept));
      swept++;
      if (rc == QCD_OK && measure_every > 0 && swept % measure_every == 0) rc = batch_measure_launch(b, gi);
    }
  }
  b->stream = main;
  if (lanes > 1) {
    for (int k = 0; k < lanes; k++) {
      cudaEventRecord(b->join_ev[k], b->lane[k]);
      cudaStreamWaitEvent(main, b->join_ev[k], 0);
    }
  }
  if (rc) return rc;
  b->sweeps_done += sweeps;
  return QCD_OK;
}

int qcd_batch_set_lanes(qcd_batch* b, int lanes) {
  if (!b || lanes < 1 || lanes > qcd_batch::kMaxLanes) return QCD_ERR_INVALID;
  b->lanes = lanes;
  return QCD_OK;
}

int qcd_batch_set_groups(qcd_batch* b, long long bytes_per_group) {
  if (!b || bytes_per_group < 0) return QCD_ERR_INVALID;
  BCUDA(b, cudaStreamSynchronize(b->stream));
  form_groups(b, bytes_per_group);
  // the new groups start from the common counter and cursor of the old ones
  spread_group_state<<<(b->n + 255) / 256, 256, 0, b->stream>>>(b->draw_dev, b->cursor, b->all_count, b->n);
  BCUDA(b, cudaGetLastError());
  return QCD_OK;
}

int qcd_batch_groups(const qcd_batch* b) { return b ? (int)b->groups.size() : QCD_ERR_INVALID; }

int qcd_batch_autotune(qcd_batch* b, int sweeps_per_trial, long long* bytes_out, int* lanes_out, double* ms_out) {
  if (!b || sweeps_per_trial < 0) return QCD_ERR_INVALID;
  if (sweeps_per_trial == 0) sweeps_per_trial = 20;
  BCUDA(b, cudaStreamSynchronize(b->stream));
  // the trials advance the batch: save links, streams, counters, cursors and
  // series, restore them afterwards
  struct Saved {
    void *l0 = nullptr, *l1 = nullptr, *rng = nullptr, *acc = nullptr, *draw = nullptr, *cur = nullptr,
         *ser = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~Saved() {
      cudaFree(l0);
      cudaFree(l1);
      cudaFree(rng);
      cudaFree(acc);
      cudaFree(draw);
      cudaFree(cur);
      cudaFree(ser);
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
    }
  } sv;
  long long links = 0;
  for (int r = 0; r < b->n; r++) links += link_bytes_of(b, r);
  const size_t lb = fp64(b) ? (size_t)links / 2 : (size_t)links;  // per store (FP64: lo and hi)
  const size_t rngb = (size_t)(b->sites / 2) * 6 * sizeof(uint32_t);
  const size_t serb = (size_t)b->cap * b->n * sizeof(double2);
  void* L0 = fp64(b) ? (void*)b->lo : (void*)b->q32;
  BCUDA(b, cudaMalloc(&sv.l0, lb));
  BCUDA(b, cudaMemcpyAsync(sv.l0, L0, lb, cudaMemcpyDeviceToDevice, b->stream));
  if (fp64(b)) {
    BCUDA(b, cudaMalloc(&sv.l1, lb));
    BCUDA(b, cudaMemcpyAsync(sv.l1, b->hi, lb, cudaMemcpyDeviceToDevice, b->stream));
    BCUDA(b, cudaMalloc(&sv.rng, rngb));
    BCUDA(b, cudaMemcpyAsync(sv.rng, b->rng, rngb, cudaMemcpyDeviceToDevice, b->stream));
  }
  if (b->accept) {
    BCUDA(b, cudaMalloc(&sv.acc, (size_t)b->sites * sizeof(int)));
    BCUDA(b, cudaMemcpyAsync(sv.acc, b->accept, (size_t)b->sites * sizeof(int), cudaMemcpyDeviceToDevice, b->stream));
  }
  BCUDA(b, cudaMalloc(&sv.draw, b->n * sizeof(unsigned long long)));
  BCUDA(b, cudaMemcpyAsync(sv.draw, b->draw_dev, b->n * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, b->stream));
  BCUDA(b, cudaMalloc(&sv.cur, b->n * sizeof(int)));
  BCUDA(b, cudaMemcpyAsync(sv.cur, b->cursor, b->n * sizeof(int), cudaMemcpyDeviceToDevice, b->stream));
  if (serb) {
    BCUDA(b, cudaMalloc(&sv.ser, serb));
    BCUDA(b, cudaMemcpyAsync(sv.ser, b->series, serb, cudaMemcpyDeviceToDevice, b->stream));
  }
  BCUDA(b, cudaEventCreate(&sv.e0));
  BCUDA(b, cudaEventCreate(&sv.e1));
  const long long swept = b->sweeps_done, bytes_save = b->group_bytes;
  const int lanes_save = b->lanes;
  // candidates (bytes per group, lanes): one group of everything; the batch
  // cut in two halves side by side; L2-sized groups one after the other or
  // two to four at a time
  struct Cand {
    long long bytes;
    int lanes;
  };
  const long long T = links;
  const Cand cand[] = {{0, 1},          {T / 2 + 1, 2},  {128ll << 20, 1}, {64ll << 20, 1},  {32ll << 20, 1},
                       {64ll << 20, 2}, {48ll << 20, 2}, {32ll << 20, 2},  {24ll << 20, 2},  {16ll << 20, 2},
                       {32ll << 20, 3}, {32ll << 20, 4}, {16ll << 20, 3},  {16ll << 20, 4}};
  const int measure = b->cap > 0 ? 1 : 0;
  long long best = bytes_save;
  int best_lanes = lanes_save;
  double best_ms = 1e300;
  int rc = QCD_OK;
  std::vector<std::pair<int, int>> seen;  // (groups, lanes) already timed
  for (const Cand& c : cand) {
    rc = qcd_batch_set_groups(b, c.bytes);
    if (rc) break;
    const int ng = (int)b->groups.size(), nl = c.lanes < ng ? c.lanes : ng;
    bool dup = false;
    for (auto& p : seen) dup |= p.first == ng && p.second == nl;
    if (dup) continue;
    seen.push_back({ng, nl});
    b->lanes = nl;
    rc = qcd_batch_run(b, 1, measure, measure);  // builds the graphs
    if (rc) break;
    if (cudaEventRecord(sv.e0, b->stream) != cudaSuccess) {
      rc = bfail(b, QCD_ERR_CUDA, "autotune: event record");
      break;
    }
    rc = qcd_batch_run(b, sweeps_per_trial, measure, measure);
    if (rc) break;
    if (cudaEventRecord(sv.e1, b->stream) != cudaSuccess || cudaEventSynchronize(sv.e1) != cudaSuccess) {
      rc = bfail(b, QCD_ERR_CUDA, "autotune: event wait");
      break;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, sv.e0, sv.e1);
    if (ms < best_ms) {
      best_ms = ms;
      best = c.bytes;
      best_lanes = nl;
    }
  }
  // restore the batch as it was
  cudaMemcpyAsync(L0, sv.l0, lb, cudaMemcpyDeviceToDevice, b->stream);
  if (fp64(b)) {
    cudaMemcpyAsync(b->hi, sv.l1, lb, cudaMemcpyDeviceToDevice, b->stream);
    cudaMemcpyAsync(b->rng, sv.rng, rngb, cudaMemcpyDeviceToDevice, b->stream);
  }
  if (sv.acc) cudaMemcpyAsync(b->accept, sv.acc, (size_t)b->sites * sizeof(int), cudaMemcpyDeviceToDevice, b->stream);
  cudaMemcpyAsync(b->draw_dev, sv.draw, b->n * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, b->stream);
  cudaMemcpyAsync(b->cursor, sv.cur, b->n * sizeof(int), cudaMemcpyDeviceToDevice, b->stream);
  cudaMemsetAsync(b->all_count, 0, b->n * sizeof(unsigned int), b->stream);
  if (serb) cudaMemcpyAsync(b->series, sv.ser, serb, cudaMemcpyDeviceToDevice, b->stream);
  cudaStreamSynchronize(b->stream);
  b->sweeps_done = swept;
  if (rc) {
    form_groups(b, bytes_save);
    b->lanes = lanes_save;
    return rc;
  }
  form_groups(b, best);
  b->lanes = best_lanes;
  if (bytes_out) *bytes_out = best;
  if (lanes_out) *lanes_out = best_lanes;
  if (ms_out) *ms_out = best_ms / sweeps_per_trial;
  BCUDA(b, cudaGetLastError());
  return QCD_OK;
}

int qcd_batch_synchronize(qcd_batch* b) {
  if (!b) return QCD_ERR_INVALID;
  int e = 0;
  BCUDA(b, cudaMemcpyAsync(&e, b->err, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  BCUDA(b, cudaStreamSynchronize(b->stream));
  if (e & DEVERR_HB_LOOP)
    return bfail(b, QCD_ERR_NONUNITARY, "heat-bath rejection loop exceeded %d tries", QCD_HB_MAX_TRIES);
  return QCD_OK;
}

int qcd_batch_measured(qcd_batch* b) {
  if (!b) return QCD_ERR_INVALID;
  int k = 0;
  BCUDA(b, cudaMemcpyAsync(&k, b->cursor, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  BCUDA(b, cudaStreamSynchronize(b->stream));
  return k;
}

int qcd_batch_series(qcd_batch* b, int replica, double* energy, double* plaquette, int n) {
  if (!b || replica < 0 || replica >= b->n || n < 0 || n > b->cap) return QCD_ERR_INVALID;
  int rc = qcd_batch_synchronize(b);
  if (rc) return rc;
  if (n == 0) return QCD_OK;
  std::vector<double2> tmp(n);
  BCUDA(b, cudaMemcpy(tmp.data(), b->series + (size_t)replica * b->cap, n * sizeof(double2), cudaMemcpyDeviceToHost));
  for (int i = 0; i < n; i++) {
    if (energy) energy[i] = tmp[i].x;
    if (plaquette) plaquette[i] = tmp[i].y;
  }
  return QCD_OK;
}

int qcd_batch_store_config(qcd_batch* b, int replica, double* aos_host) {
  if (!b || !aos_host || replica < 0 || replica >= b->n) return QCD_ERR_INVALID;
  int rc = qcd_batch_synchronize(b);
  if (rc) return rc;
  const Replica& R = b->rep[replica];
  const size_t vh = (size_t)R.g.vh;
  // SoA planes -> the reference's AoS layout, on the host
  if (fp64(b)) {
    std::vector<double2> lo(6 * vh), hi(6 * vh);
    BCUDA(b, cudaMemcpy(lo.data(), b->lo + R.link_off, 6 * vh * sizeof(double2), cudaMemcpyDeviceToHost));
    BCUDA(b, cudaMemcpy(hi.data(), b->hi + R.link_off, 6 * vh * sizeof(double2), cudaMemcpyDeviceToHost));
    for (int p = 0; p < 2; p++)
      for (size_t id = 0; id < vh; id++)
        for (int d = 0; d < 3; d++) {
          const size_t i = (size_t)(d * 2 + p) * vh + id;
          double* s = aos_host + ((size_t)p * vh + id) * 12 + d * 4;
          s[0] = lo[i].x;
          s[1] = lo[i].y;
          s[2] = hi[i].x;
          s[3] = hi[i].y;
        }
  } else {
    std::vector<float4> q(6 * vh);
    BCUDA(b, cudaMemcpy(q.data(), b->q32 + R.link_off, 6 * vh * sizeof(float4), cudaMemcpyDeviceToHost));
    for (int p = 0; p < 2; p++)
      for (size_t id = 0; id < vh; id++)
        for (int d = 0; d < 3; d++) {
          const float4 u = q[(size_t)(d * 2 + p) * vh + id];
          double* s = aos_host + ((size_t)p * vh + id) * 12 + d * 4;
          s[0] = u.x;
          s[1] = u.y;
          s[2] = u.z;
          s[3] = u.w;
        }
  }
  return QCD_OK;
}

long long qcd_batch_sites(const qcd_batch* b) { return b ? b->sites : 0; }

const char* qcd_batch_last_error(const qcd_batch* b) { return b ? b->msg : "null batch"; }

}  // extern "C"
