// Temporal blocking of the sweep: one persistent launch carries every t-slice
// through a program of up to kMaxWavePhases checkerboard phases while the
// slice and its neighbours are resident in L2, instead of streaming the whole
// link store through HBM once per phase.
//
// Work unit ("task") = one chunk of chunk_sites sites of one t-slice for one
// phase of the program.  Phase n visits the slices in ring order starting at
// its seam s_n, one slice per time step from its start time T_n:
//     tau(n, t) = T_n + ((t - s_n) mod Lt).
// Tasks are handed out by an atomic ticket counter in (tau, n) order; the host
// chooses (s_n, T_n) so that every task another task depends on has a smaller
// tau (a dependency is any pair of phases at slices t+o, t, o in {-1,0,+1},
// where one writes a link class the other reads or writes).  Each slice has
// one arrival counter: phases complete at a slice in program order, so
// "phase m finished at slice t" is "counter[t] >= (m+1) * chunks".  A task
// therefore waits on at most three counters (t-1, t, t+1) before it starts.
// A CTA only waits for tickets drawn before its own, by CTAs that are already
// running, so the scheme needs no co-residency and cannot deadlock; every
// wait is still bounded and reports QCD_ERR_TIMEOUT instead of spinning.
//
// The per-link arithmetic is the per-phase kernels' (site64 / site32), with
// loads and stores at L2 (.cg), so results are identical bit for bit.
#pragma once
#include "kernels.cuh"

namespace qcd {

constexpr int kMaxWavePhases = 24;

// device error word bit for a wait that ran out

struct WaveSched {
  int P;                 // phases in the program
  int lt;                // t-slices
  int chunks;            // tasks per (phase, slice)
  int chunk_sites;       // sites per task
  unsigned int n_tasks;  // P * lt * chunks
  int n_steps;           // T_{P-1} + lt
  signed char mu[kMaxWavePhases], par[kMaxWavePhases], kind[kMaxWavePhases], renorm[kMaxWavePhases];
  short need[3][kMaxWavePhases];  // latest earlier phase waited for at t-1, t, t+1 (-1: none)
  int seam[kMaxWavePhases], start[kMaxWavePhases];
  unsigned char draw[kMaxWavePhases];  // drawing-phase offset from the launch's counter (FP32 draws)
};

struct WaveCtl {
  unsigned int* done;          // lt arrival counters, zero at launch
  unsigned int* queue;         // ticket counter, zero at launch
  int* abort;                  // set when a wait gave up; every CTA then stops
  const unsigned int* tasks;   // ticket -> packed (phase, chunk, slice), built on the host
  unsigned int spin_limit;
  int stall_test;              // self-test: ticket 0 waits for a count that is never reached
};

// packed task word: phase in bits 0-4, chunk in bits 5-16, slice in bits 17-31
__host__ __device__ __forceinline__ unsigned int wave_pack(int n, int chunk, int t) {
  return (unsigned int)n | ((unsigned int)chunk << 5) | ((unsigned int)t << 17);
}

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// number of tasks whose time step is before tau
__device__ __forceinline__ long long wave_tasks_before(const WaveSched& S, int tau) {
  long long c = 0;
  for (int n = 0; n < S.P; n++) {
    int d = tau - S.start[n];
    c += d <= 0 ? 0 : (d >= S.lt ? S.lt : d);
  }
  return c * S.chunks;
}

#define QCD_WAVE_CASE64(MU, PAR)                                                           \
  case MU * 2 + PAR:                                                                        \
    if (kind == KIND_OR)                                                                    \
      site64<MU, PAR, BC, KIND_OR, true>(L, R, g, a, make_nbr_slice(g, s, t, PAR));        \
    else                                                                                    \
      site64<MU, PAR, BC, SK, true>(L, R, g, a, make_nbr_slice(g, s, t, PAR));             \
    break;

#define QCD_WAVE_CASE32(MU, PAR)                                                           \
  case MU * 2 + PAR:                                                                        \
    if (kind == KIND_OR)                                                                    \
      site32<MU, PAR, BC, KIND_OR, true>(L, R, g, a, make_nbr_slice(g, s, t, PAR), rn);    \
    else                                                                                    \
      site32<MU, PAR, BC, SK, true>(L, R, g, a, make_nbr_slice(g, s, t, PAR), rn);         \
    break;

template <int BC, int SK>
__device__ __forceinline__ void wave_site(const Links64T<true>& L, const RngStoreT<true>& R, const Geo& g,
                                          const PhaseArgs& a, int type, int kind, int rn, int s, int t) {
  switch (type) {
    QCD_WAVE_CASE64(DIR_Y, 0)
    QCD_WAVE_CASE64(DIR_Y, 1)
    QCD_WAVE_CASE64(DIR_X, 0)
    QCD_WAVE_CASE64(DIR_X, 1)
    QCD_WAVE_CASE64(DIR_T, 0)
    QCD_WAVE_CASE64(DIR_T, 1)
  }
}

template <int BC, int SK>
__device__ __forceinline__ void wave_site(const Links32T<true>& L, const RngStoreT<true>& R, const Geo& g,
                                          const PhaseArgs& a, int type, int kind, int rn, int s, int t) {
  switch (type) {
    QCD_WAVE_CASE32(DIR_Y, 0)
    QCD_WAVE_CASE32(DIR_Y, 1)
    QCD_WAVE_CASE32(DIR_X, 0)
    QCD_WAVE_CASE32(DIR_X, 1)
    QCD_WAVE_CASE32(DIR_T, 0)
    QCD_WAVE_CASE32(DIR_T, 1)
  }
}

// LinksT: Links64T<true> or Links32T<true>; BC: boundary; SK: the sweep's
// update kind (heat-bath or Metropolis); over-relaxation phases are KIND_OR.
template <class LinksT, int BC, int SK>
__global__ void __launch_bounds__(kBlock, 5) wave(LinksT L, RngStoreT<true> R, Geo g, PhaseArgs a,
                                                  WaveSched S, WaveCtl c) {
  __shared__ int sh_ok, sh_n, sh_t, sh_chunk;
  // Thread 0 keeps one ticket in hand: the atomic for the next ticket is
  // issued before the CTA computes the current task, so its latency hides
  // behind the work.  A CTA never waits while holding an unstarted ticket
  // that others need: the current task's waits are over before the next
  // ticket is drawn, so the current task finishes and the next one starts.
  unsigned int tk = 0;
  if (threadIdx.x == 0) tk = atomicAdd(c.queue, 1u);
  for (;;) {
    if (threadIdx.x == 0) {
      int ok = 0, n = 0, t = 0, chunk = 0;
      if (tk < S.n_tasks && !*(volatile int*)c.abort) {
        const unsigned int w = __ldg(c.tasks + tk);
        n = (int)(w & 31u);
        chunk = (int)((w >> 5) & 4095u);
        t = (int)(w >> 17);
        ok = 1;
        if (c.stall_test && tk == 0) {
          // self-test of the bounded wait: a count that no task produces
          unsigned int it = 0;
          while ((int)(ld_acquire_u32(c.done + t) - 0x40000000u) < 0) {
            if (*(volatile int*)c.abort || ++it > c.spin_limit) {
              atomicExch(c.abort, 1);
              atomicOr(a.err, DEVERR_TIMEOUT);
              ok = 0;
              break;
            }
            __nanosleep(128);
          }
        }
        for (int o = -1; o <= 1 && ok; o++) {
          const int m = S.need[o + 1][n];
          if (m < 0) continue;
          int ts = t + o;
          ts = ts < 0 ? ts + S.lt : (ts >= S.lt ? ts - S.lt : ts);
          const unsigned int target = (unsigned int)(m + 1) * (unsigned int)S.chunks;
          unsigned int it = 0;
          while ((int)(ld_acquire_u32(c.done + ts) - target) < 0) {
            if (*(volatile int*)c.abort || ++it > c.spin_limit) {
              atomicExch(c.abort, 1);
              atomicOr(a.err, DEVERR_TIMEOUT);
              ok = 0;
              break;
            }
            if (it > 32) __nanosleep(64);
          }
        }
        if (ok) tk = atomicAdd(c.queue, 1u);  // next ticket, in flight during the work
      }
      sh_ok = ok;
      sh_n = n;
      sh_t = t;
      sh_chunk = chunk;
    }
    __syncthreads();
    if (!sh_ok) break;
    const int n = sh_n, t = sh_t;
    const int type = S.mu[n] * 2 + S.par[n], kind = S.kind[n], rn = S.renorm[n];
    const int s0 = sh_chunk * S.chunk_sites;
    const int s1 = min(s0 + S.chunk_sites, g.slice);
    PhaseArgs an = a;
    an.phase_off = S.draw[n];
    for (int s = s0 + (int)threadIdx.x; s < s1; s += kBlock) wave_site<BC, SK>(L, R, g, an, type, kind, rn, s, t);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(c.done + t, 1u);
    }
  }
}

}  // namespace qcd
