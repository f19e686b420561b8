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
#include <mutex>
#include <new>
#include "kernels.cuh"
#include "qcd2d.h"

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
  float4* q32 = nullptr;
  size_t link_bytes = 0;
  // MRG32k3a streams, 6 u32 planes
  uint32_t* rng = nullptr;
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

// one pass over the six phases with one update kind; with `renorm` (FP32
// only) every link is re-projected as it is stored
int pass(qcd_lattice* h, int kind, int renorm = 0) {
  PhaseArgs a{h->p.beta, h->p.epsilon, h->p.upd, h->err, h->accept, renorm};
  const dim3 grid(nblocks(h->g.slice), (unsigned int)h->g.lt);
  for (int k = 0; k < 6; k++) {
    if (h->p.precision == QCD_PREC_FP64)
      phase_fn64(k, h->p.boundary, kind)<<<grid, kBlock, 0, h->stream>>>(links64(h), rngs(h), h->g, a);
    else
      phase_fn32(k, h->p.boundary, kind)<<<grid, kBlock, 0, h->stream>>>(links32(h), rngs(h), h->g, a);
    LAUNCH_CHECK(h);
  }
  if (kind != KIND_METRO) h->unit_passes++;
  return QCD_OK;
}

int check_device_error(qcd_lattice* h) {
  int e = 0;
  CUDA_OR_FAIL(h, cudaMemcpyAsync(&h->result_host[2], h->err, sizeof(int), cudaMemcpyDeviceToHost,
                                  h->stream));
  CUDA_OR_FAIL(h, cudaStreamSynchronize(h->stream));
  memcpy(&e, &h->result_host[2], sizeof(int));
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
  const unsigned int nb = nblocks(h->g.vh);
  const bool pmc = h->p.boundary == QCD_BC_PMC;
  if (h->p.precision == QCD_PREC_FP64) {
    if (pmc)
      measure<Links64, 1><<<nb, kBlock, 0, h->stream>>>(links64(h), h->g, h->partials, h->counter, out_dev);
    else
      measure<Links64, 0><<<nb, kBlock, 0, h->stream>>>(links64(h), h->g, h->partials, h->counter, out_dev);
  } else {
    if (pmc)
      measure<Links32, 1><<<nb, kBlock, 0, h->stream>>>(links32(h), h->g, h->partials, h->counter, out_dev);
    else
      measure<Links32, 0><<<nb, kBlock, 0, h->stream>>>(links32(h), h->g, h->partials, h->counter, out_dev);
  }
  LAUNCH_CHECK(h);
  return QCD_OK;
}

void release(qcd_lattice* h) {
  cudaFree(h->lo);
  cudaFree(h->hi);
  cudaFree(h->q32);
  cudaFree(h->rng);
  cudaFree(h->accept);
  cudaFree(h->partials);
  cudaFree(h->counter);
  cudaFree(h->result);
  cudaFree(h->err);
  cudaFree(h->series);
  cudaFree(h->aos_stage);
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
  long long V = (long long)p->lt * p->lx * p->ly;
  if (V / 2 >= (1ll << 31) / 6) return QCD_ERR_INVALID;  // 32-bit plane indices

  qcd_lattice* h = new (std::nothrow) qcd_lattice();
  if (!h) return QCD_ERR_NOMEM;
  h->p = *p;
  h->V = V;
  h->g = make_geo(p->lt, p->lx, p->ly);
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
  if (rc == QCD_OK) step(cudaMalloc(&h->rng, 6 * vh * sizeof(uint32_t)), "cudaMalloc(rng)");
  if (rc == QCD_OK && p->algo == QCD_ALGO_METROPOLIS) {
    step(cudaMalloc(&h->accept, 2 * vh * sizeof(int)), "cudaMalloc(accept)");
    if (rc == QCD_OK) step(cudaMemsetAsync(h->accept, 0, 2 * vh * sizeof(int), h->stream), "memset");
  }
  const size_t nb = nblocks(h->g.vh);
  if (rc == QCD_OK) step(cudaMalloc(&h->partials, nb * sizeof(double2)), "cudaMalloc(partials)");
  if (rc == QCD_OK) step(cudaMalloc(&h->counter, sizeof(unsigned int)), "cudaMalloc(counter)");
  if (rc == QCD_OK) step(cudaMalloc(&h->result, 2 * sizeof(double)), "cudaMalloc(result)");
  if (rc == QCD_OK) step(cudaMalloc(&h->err, sizeof(int)), "cudaMalloc(err)");
  if (rc == QCD_OK) step(cudaMallocHost(&h->result_host, 4 * sizeof(double)), "cudaMallocHost");
  if (rc == QCD_OK) step(cudaMemsetAsync(h->counter, 0, sizeof(unsigned int), h->stream), "memset");
  if (rc == QCD_OK) step(cudaMemsetAsync(h->err, 0, sizeof(int), h->stream), "memset");
  if (rc == QCD_OK) {
    rng_setup<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(rngs(h), p->seed, h->g.vh);
    step(cudaGetLastError(), "rng_setup");
  }
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
  else
    init_cold<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(links32(h), h->g.vh);
  LAUNCH_CHECK(h);
  return QCD_OK;
}

int qcd_init_hot(qcd_lattice* h) {
  if (!h) return QCD_ERR_INVALID;
  const int pcc = h->p.boundary == QCD_BC_PCC;
  if (h->p.precision == QCD_PREC_FP64)
    init_hot<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(links64(h), rngs(h), h->g, pcc);
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
  else
    aos_to_soa32<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(aos_dev, links32(h), h->g.vh);
  LAUNCH_CHECK(h);
  return QCD_OK;
}

int qcd_store_config_device(qcd_lattice* h, double* aos_dev) {
  if (!h || !aos_dev) return QCD_ERR_INVALID;
  if (h->p.precision == QCD_PREC_FP64)
    soa_to_aos64<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(links64(h), aos_dev, h->g.vh);
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
  else
    normalize32<<<nblocks(h->g.vh), kBlock, 0, h->stream>>>(links32(h), h->g.vh);
  LAUNCH_CHECK(h);
  return QCD_OK;
}

int qcd_sweep(qcd_lattice* h, int n) {
  if (!h || n < 0) return QCD_ERR_INVALID;
  const int kind = h->p.algo == QCD_ALGO_HEATBATH ? KIND_HB : KIND_METRO;
  for (int i = 0; i < n; i++) {
    const bool renorm = h->p.renorm_every > 0 && (h->sweeps_done + 1) % h->p.renorm_every == 0;
    // FP32: the re-projection rides on the sweep's last pass, each link being
    // re-projected at its last update (no extra read of the store); FP64
    // keeps the reference's separate normalize after the sweep
    const bool fused = renorm && h->p.precision == QCD_PREC_FP32;
    int rc = pass(h, kind, fused && h->p.n_or == 0);
    for (int r = 0; rc == QCD_OK && r < h->p.n_or; r++) rc = pass(h, KIND_OR, fused && r == h->p.n_or - 1);
    if (rc) return rc;
    h->sweeps_done++;
    if (renorm && !fused) {
      rc = qcd_normalize(h);
      if (rc) return rc;
    }
  }
  return QCD_OK;
}

int qcd_overrelax(qcd_lattice* h, int n) {
  if (!h || n < 0) return QCD_ERR_INVALID;
  for (int i = 0; i < n; i++) {
    int rc = pass(h, KIND_OR);
    if (rc) return rc;
  }
  return QCD_OK;
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
static constexpr size_t kNoAllocCounterOffset = (size_t)QCD_NOALLOC_MAX_BLOCKS * sizeof(double2);
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocCounterOffset + 256];

namespace {
std::mutex g_noalloc_mu;
void* g_noalloc_addr[256];  // device address of g_noalloc_scratch, per device ordinal

// Host code may not use g_noalloc_scratch itself (on the host it names a
// stand-in, not device memory): look up its device address once per device,
// with that device current.
int noalloc_scratch(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 256) {
    cudaGetLastError();
    return QCD_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      fprintf(stderr, "qcd_measure_aos_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
              cudaGetErrorString(e));
      return QCD_ERR_CUDA;
    }
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return QCD_OK;
}
}  // namespace

extern "C" int qcd_measure_aos_noalloc(const double* phi_dev, int lt, int lx, int ly, int boundary,
                                       double* out_dev, void* stream) {
  if (!phi_dev || !out_dev) return QCD_ERR_INVALID;
  if (lt < 2 || lx < 2 || ly < 2 || (lt & 1) || (lx & 1) || (ly & 1)) return QCD_ERR_INVALID;
  if (boundary < 0 || boundary > 2) return QCD_ERR_INVALID;
  if (((uintptr_t)phi_dev & 15) || ((uintptr_t)out_dev & 7)) return QCD_ERR_INVALID;
  const long long vh = (long long)lt * lx * ly / 2;
  const long long nb = (vh + kBlock - 1) / kBlock;
  if (vh > QCD_NOALLOC_MAX_HALF_SITES || nb > QCD_NOALLOC_MAX_BLOCKS) {
    fprintf(stderr,
            "qcd_measure_aos_noalloc: %dx%dx%d has V/2 = %lld sites, above the %d that its fixed "
            "scratch holds; use qcd_measure on a handle instead\n",
            lt, lx, ly, vh, QCD_NOALLOC_MAX_HALF_SITES);
    return QCD_ERR_UNSUPPORTED;
  }
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
    if (boundary == QCD_BC_PMC)
      measure<LinksAoS, 1><<<(unsigned int)nb, kBlock, 0, s>>>(L, g, partials, counter, out_dev);
    else
      measure<LinksAoS, 0><<<(unsigned int)nb, kBlock, 0, s>>>(L, g, partials, counter, out_dev);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    fprintf(stderr, "qcd_measure_aos_noalloc: %s\n", cudaGetErrorString(e));
    return QCD_ERR_CUDA;
  }
  return QCD_OK;
}
