// Device kernels of the sweep, the starts, re-projection, measurement and the
// layout conversions.  Launch geometry: one thread per sublattice site,
// 256 threads per CTA, ragged tail masked (the reference instead requires the
// CTA size to divide V/2, kernel.cu:66-70).
#pragma once
#include <curand_kernel.h>
#include "lattice.cuh"
#include "rng.cuh"
#include "su2.cuh"
#include "updates.cuh"
#include "sites.cuh"

namespace qcd {

// ------------------------------------------------------------ one phase --
// Launch grid (ceil(slice / kBlock), Lt): blockIdx.y is the t-slice.
template <int MU, int PAR, int BC, int KIND>
__global__ void __launch_bounds__(kBlock) phase64(Links64 L, RngStore R, Geo g, PhaseArgs a) {
  const int s = blockIdx.x * kBlock + threadIdx.x;
  if (s >= g.slice) return;
  site64<MU, PAR, BC, KIND, false>(L, R, g, a, make_nbr_slice(g, s, blockIdx.y, PAR));
}

template <int MU, int PAR, int BC, int KIND>
__global__ void __launch_bounds__(kBlock) phase32(Links32 L, RngStore R, Geo g, PhaseArgs a) {
  const int s = blockIdx.x * kBlock + threadIdx.x;
  if (s >= g.slice) return;
  site32<MU, PAR, BC, KIND, false>(L, R, g, a, make_nbr_slice(g, s, blockIdx.y, PAR), a.renorm);
}

// ------------------------------------------------------------ RNG setup --
// curand_init(seed, id, 0) per half-lattice site (lattice_setup.h:15-21),
// by jumps from curand_init(seed, 0, 0) (mrg_cta_base, mrg_jump_from;
// `jumps` holds mrg_jump_table).
static_assert(kBlock == kMrgJumps, "one jump matrix per thread of a CTA");
__global__ void __launch_bounds__(kBlock) rng_setup(RngStore R, unsigned long long seed, int vh,
                                                    const uint32_t* __restrict__ jumps) {
  __shared__ unsigned int base[6];
  const int id0 = blockIdx.x * kBlock;
  if (threadIdx.x == 0) mrg_cta_base(base, jumps, seed, (unsigned long long)id0);
  __syncthreads();
  const int id = id0 + threadIdx.x;
  if (id >= vh) return;
  curandStateMRG32k3a_t st;
  mrg_jump_from(base, jumps, threadIdx.x, &st);
  R.store(id, &st);
}

// ------------------------------------------------------------ starts -----
__device__ __forceinline__ void put(const Links64& L, int d, int p, int id, const Quat<double>& u) {
  L.st(d, p, id, u);
}
__device__ __forceinline__ void put(const Links32& L, int d, int p, int id, const Quat<double>& u) {
  L.st(d, p, id, Quat<float>{(float)u.w, (float)u.x, (float)u.y, (float)u.z});
}

// Cold start (id_init2, lattice_setup.h:38-51).
template <class L>
__global__ void __launch_bounds__(kBlock) init_cold(L links, int vh) {
  const int id = blockIdx.x * kBlock + threadIdx.x;
  if (id >= vh) return;
  for (int p = 0; p < 2; p++)
    for (int d = 0; d < 3; d++) put(links, d, p, id, q_one<double>());
}

// uniform cube (-0.5, 0.5]^4, normalised (su2_rand, su2.h:29-34)
__device__ __forceinline__ Quat<double> random_link(curandStateMRG32k3a_t* st) {
  Quat<double> a;
  a.w = curand_uniform_double(st) - 0.5;
  a.x = curand_uniform_double(st) - 0.5;
  a.y = curand_uniform_double(st) - 0.5;
  a.z = curand_uniform_double(st) - 0.5;
  return q_normalize(a);
}

// Hot start (rand_init2 lattice_setup.h:24-37; rand_init2_pcc :52-81): stream id
// fills even y, x, t then odd y, x, t; with PCC the x and t links at y = 0 are
// the identity and consume no draws.

template <class L>
__global__ void __launch_bounds__(kBlock) init_hot(L links, RngStore R, Geo g, int pcc) {
  const int id = blockIdx.x * kBlock + threadIdx.x;
  if (id >= g.vh) return;
  curandStateMRG32k3a_t st;
  R.load(id, &st);
  for (int p = 0; p < 2; p++) {
    const Nbr n = make_nbr(g, id, p);
    const bool frozen = pcc && at_y0(g, n);
    for (int d = 0; d < 3; d++) {
      if (d != DIR_Y && frozen)
        put(links, d, p, id, q_one<double>());
      else
        put(links, d, p, id, random_link(&st));
    }
  }
  R.store(id, &st);
}

// ------------------------------------------------------- re-projection --
// normalize (lattice_setup.h:202-207): every link divided by its norm.
__global__ void __launch_bounds__(kBlock) normalize64(Links64 L, int vh) {
  const int id = blockIdx.x * kBlock + threadIdx.x;
  if (id >= vh) return;
  for (int p = 0; p < 2; p++)
    for (int d = 0; d < 3; d++) L.st(d, p, id, q_normalize(L.ld_own(d, p, id)));
}
__global__ void __launch_bounds__(kBlock) normalize32(Links32 L, int vh) {
  const int id = blockIdx.x * kBlock + threadIdx.x;
  if (id >= vh) return;
  for (int p = 0; p < 2; p++)
    for (int d = 0; d < 3; d++) L.st(d, p, id, renorm_fast(L.ld_own(d, p, id)));
}

// ----------------------------------------------------- layout changes ---
// reference AoS: phi[(p*Vh + id)*12 + d*4 + c]
__global__ void __launch_bounds__(kBlock) aos_to_soa64(const double* __restrict__ aos, Links64 L, int vh) {
  const int id = blockIdx.x * kBlock + threadIdx.x;
  if (id >= vh) return;
  for (int p = 0; p < 2; p++) {
    const double* s = aos + ((size_t)p * vh + id) * 12;
    for (int d = 0; d < 3; d++)
      L.st(d, p, id, Quat<double>{s[d * 4 + 0], s[d * 4 + 1], s[d * 4 + 2], s[d * 4 + 3]});
  }
}
__global__ void __launch_bounds__(kBlock) soa_to_aos64(Links64 L, double* __restrict__ aos, int vh) {
  const int id = blockIdx.x * kBlock + threadIdx.x;
  if (id >= vh) return;
  for (int p = 0; p < 2; p++) {
    double* s = aos + ((size_t)p * vh + id) * 12;
    for (int d = 0; d < 3; d++) {
      Quat<double> u = L.ld_own(d, p, id);
      s[d * 4 + 0] = u.w;
      s[d * 4 + 1] = u.x;
      s[d * 4 + 2] = u.y;
      s[d * 4 + 3] = u.z;
    }
  }
}
__global__ void __launch_bounds__(kBlock) aos_to_soa32(const double* __restrict__ aos, Links32 L, int vh) {
  const int id = blockIdx.x * kBlock + threadIdx.x;
  if (id >= vh) return;
  for (int p = 0; p < 2; p++) {
    const double* s = aos + ((size_t)p * vh + id) * 12;
    for (int d = 0; d < 3; d++)
      L.st(d, p, id, Quat<float>{(float)s[d * 4 + 0], (float)s[d * 4 + 1], (float)s[d * 4 + 2],
                                 (float)s[d * 4 + 3]});
  }
}
__global__ void __launch_bounds__(kBlock) soa_to_aos32(Links32 L, double* __restrict__ aos, int vh) {
  const int id = blockIdx.x * kBlock + threadIdx.x;
  if (id >= vh) return;
  for (int p = 0; p < 2; p++) {
    double* s = aos + ((size_t)p * vh + id) * 12;
    for (int d = 0; d < 3; d++) {
      Quat<float> u = L.ld_own(d, p, id);
      s[d * 4 + 0] = u.w;
      s[d * 4 + 1] = u.x;
      s[d * 4 + 2] = u.y;
      s[d * 4 + 3] = u.z;
    }
  }
}

// en_av<PMC> (observables.h:99-141): energy = mean of -(1 - P_xt), plaquette
// = mean of (P_yx + P_yt + P_xt)/3; with PMC the y plaquettes at y = Ly-1 count
// as 1.  out[0] = energy, out[1] = plaquette.
template <class L, int PMC>
__global__ void __launch_bounds__(kBlock) measure(L links, Geo g, double2* partials,
                                                  unsigned int* counter, double* out) {
  double e = 0, pl = 0;
  measure_sites<L, PMC != 0>(links, g, blockIdx.x, gridDim.x, e, pl);  // grid: measure_blocks(V/2)
  double se, sp;
  block_sum2(e, pl * (1.0 / 3.0), &se, &sp);
  if (threadIdx.x == 0) partials[blockIdx.x] = make_double2(se, sp);
  finish_sum2(partials, counter, 1.0 / (2.0 * (double)g.vh), out);
}

// Unitarity: out[0] = mean det, out[1] = number of links with |det-1| > tol
// or not finite (print_det, lattice_setup.h:176-183, plus a NaN/Inf check).
template <class L>
__global__ void __launch_bounds__(kBlock) unitarity(L links, int vh, double tol, double2* partials,
                                                    unsigned int* counter, double* out) {
  const int id = blockIdx.x * kBlock + threadIdx.x;
  double s = 0, bad = 0;
  if (id < vh) {
    for (int p = 0; p < 2; p++)
      for (int d = 0; d < 3; d++) {
        double det = q_det(ld64(links, d, p, id));
        s += det;
        if (!(fabs(det - 1.0) <= tol)) bad += 1;
      }
  }
  double ss, sb;
  block_sum2(s, bad, &ss, &sb);
  if (threadIdx.x == 0) partials[blockIdx.x] = make_double2(ss, sb);
  finish_sum2(partials, counter, 1.0, out);
}

// ----------------------------------------------------------- RNG tape ----
struct TapeRec {
  double ud;
  float uf, log_uf, cospi_2uf, sc_sin, sc_cos;
  unsigned int same_step;
};

__global__ void __launch_bounds__(kBlock) rng_tape(unsigned long long seed, long long first, int n_streams,
                                                   int n_draws, TapeRec* out) {
  const int i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n_streams) return;
  curandStateMRG32k3a_t st;
  curand_init(seed, (unsigned long long)(first + i), 0ull, &st);
  for (int k = 0; k < n_draws; k++) {
    curandStateMRG32k3a_t cp = st;
    float f = curand_uniform(&cp);
    double d = curand_uniform_double(&st);
    unsigned int same = 1;
    for (int j = 0; j < 3; j++) same &= (cp.s1[j] == st.s1[j]) & (cp.s2[j] == st.s2[j]);
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

}  // namespace qcd
