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

namespace qcd {

constexpr int kBlock = 256;

struct PhaseArgs {
  float beta;
  float eps;
  int upd;
  int* err;     // device error word
  int* accept;  // V ints, reference site order; only for Metropolis
  int renorm;   // FP32: re-project each updated link (in double) before it is stored
};

// ------------------------------------------------------- one link update --
// Update U_MU at site n of sublattice PAR: the body of the six launches of
// mc_up_per/pcc/pmc (mc_updates.h:129-465, mc_updates_pcc.h:4-214,
// mc_updates_pmc.h:4-247).  Shared by the per-phase kernels (CG = false) and
// the wavefront kernel (CG = true).
template <bool CG>
__device__ __forceinline__ void add_accept(int* p, int v) {
  if (CG)
    atomicAdd(p, v);  // at L2: the counter may sit in a stale L1 line
  else
    *p += v;
}

template <int MU, int PAR, int BC, int KIND, bool CG>
__device__ __forceinline__ void site64(const Links64T<CG>& L, const RngStoreT<CG>& R, const Geo& g,
                                       const PhaseArgs& a, const Nbr& n) {
  if (BC == BC_PCC && MU != DIR_Y && at_y0(g, n)) return;
  const int id = n.id;
  Quat<double> A = staple_sum<MU, BC, Links64T<CG>, double>(L, g, n, PAR);
  if (KIND == KIND_HB) {
    curandStateMRG32k3a_t st;
    R.load(id, &st);
    Quat<double> U = heatbath_ref(A, (double)a.beta, &st, a.err);
    L.st(MU, PAR, id, U);
    R.store(id, &st);
  } else if (KIND == KIND_METRO) {
    curandStateMRG32k3a_t st;
    R.load(id, &st);
    Quat<double> U = L.ld_own(MU, PAR, id);
    int acc = metropolis_ref(U, A, (double)a.beta, (double)a.eps, a.upd, &st);
    L.st(MU, PAR, id, U);
    R.store(id, &st);
    add_accept<CG>(a.accept + PAR * g.vh + id, acc);
  } else {
    Quat<double> U = L.ld_own(MU, PAR, id);
    L.st(MU, PAR, id, overrelax_ref(A, U));
  }
}

template <int MU, int PAR, int BC, int KIND, bool CG>
__device__ __forceinline__ void site32(const Links32T<CG>& L, const RngStoreT<CG>& R, const Geo& g,
                                       const PhaseArgs& a, const Nbr& n, int renorm) {
  if (BC == BC_PCC && MU != DIR_Y && at_y0(g, n)) return;
  const int id = n.id;
  Quat<float> A = staple_sum<MU, BC, Links32T<CG>, float>(L, g, n, PAR);
  Quat<float> U;
  if (KIND == KIND_HB) {
    curandStateMRG32k3a_t st;
    R.load(id, &st);
    U = heatbath_fast(A, a.beta, &st, a.err);
    R.store(id, &st);
  } else if (KIND == KIND_METRO) {
    curandStateMRG32k3a_t st;
    R.load(id, &st);
    U = L.ld_own(MU, PAR, id);
    int acc = metropolis_fast(U, A, a.beta, a.eps, a.upd, &st);
    R.store(id, &st);
    add_accept<CG>(a.accept + PAR * g.vh + id, acc);
  } else {
    U = overrelax_fast(A, L.ld_own(MU, PAR, id));
  }
  L.st(MU, PAR, id, renorm ? renorm_fast(U) : U);
}

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
// curand_init(seed, id, 0) per half-lattice site (lattice_setup.h:15-21).
__global__ void __launch_bounds__(kBlock) rng_setup(RngStore R, unsigned long long seed, int vh) {
  const int id = blockIdx.x * kBlock + threadIdx.x;
  if (id >= vh) return;
  curandStateMRG32k3a_t st;
  curand_init(seed, (unsigned long long)id, 0ull, &st);
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

// ---------------------------------------------------------- reductions --
// Deterministic FP64 sums: each CTA writes its partial (fixed tree order),
// the last CTA to finish adds the partials in index order and resets the
// arrival counter.  No floating-point atomics, so the result does not depend
// on CTA scheduling (the reference's en_av uses atomicAdd, observables.h:137-140).
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Sums two values over the CTA into out2 (valid in thread 0).
__device__ __forceinline__ void block_sum2(double v0, double v1, double* out0, double* out1) {
  __shared__ double sh[2][kBlock / 32];
  v0 = warp_sum(v0);
  v1 = warp_sum(v1);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sh[0][w] = v0;
    sh[1][w] = v1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int i = 0; i < kBlock / 32; i++) {
      a += sh[0][i];
      b += sh[1][i];
    }
    *out0 = a;
    *out1 = b;
  }
}

// After thread 0 of every CTA stored its partial pair: the last CTA adds all
// partials in order, scales them and writes out[0..1].
__device__ __forceinline__ void finish_sum2(double2* partials, unsigned int* counter, double scale,
                                            double* out) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned int prev = atomicAdd(counter, 1u);
    last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  // fixed-order sum over partials: per-thread strided chunks, then the CTA tree
  double a = 0, b = 0;
  for (unsigned int i = threadIdx.x; i < gridDim.x; i += kBlock) {
    double2 v = __ldcg(partials + i);  // L2: written by other CTAs
    a += v.x;
    b += v.y;
  }
  __syncthreads();
  double sa, sb;
  block_sum2(a, b, &sa, &sb);
  if (threadIdx.x == 0) {
    out[0] = sa * scale;
    out[1] = sb * scale;
    *counter = 0u;
  }
}

// 1 - 1/2 Re tr of the plaquettes at one site, in the reference's product
// order (plaquette_yx/yt/xt, observables.h:1-21):
//   P_yx = U_y(x) U_x(x+y) U_y(x+x)^+ U_x(x)^+  and alike.
template <class L>
__device__ __forceinline__ Quat<double> ld64(const L& links, int d, int p, int id);
template <>
__device__ __forceinline__ Quat<double> ld64<Links64>(const Links64& links, int d, int p, int id) {
  return links.ld(d, p, id);
}
template <>
__device__ __forceinline__ Quat<double> ld64<Links32>(const Links32& links, int d, int p, int id) {
  Quat<float> u = links.ld(d, p, id);
  return Quat<double>{u.w, u.x, u.y, u.z};
}

template <class L>
__device__ __forceinline__ double plaq(const L& links, int mu, int nu, int p, int id, int omu,
                                       int onu) {
  // U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
  Quat<double> A = q_mul(ld64(links, mu, p, id), ld64(links, nu, p ^ 1, id + omu));
  Quat<double> B = q_mul_bd(A, ld64(links, mu, p ^ 1, id + onu));
  A = q_mul_bd(B, ld64(links, nu, p, id));
  return 1 - A.w;
}

// en_av<PMC> (observables.h:99-141): energy = mean of -(1 - P_xt), plaquette
// = mean of (P_yx + P_yt + P_xt)/3; with PMC the y plaquettes at y = Ly-1 count
// as 1.  out[0] = energy, out[1] = plaquette.
template <class L, int PMC>
__global__ void __launch_bounds__(kBlock) measure(L links, Geo g, double2* partials,
                                                  unsigned int* counter, double* out) {
  const int id = blockIdx.x * kBlock + threadIdx.x;
  double e = 0, pl = 0;
  if (id < g.vh) {
    for (int p = 0; p < 2; p++) {
      const Nbr n = make_nbr(g, id, p);
      double a = plaq(links, DIR_Y, DIR_X, p, id, n.yp, n.xp);
      double b = plaq(links, DIR_Y, DIR_T, p, id, n.yp, n.tp);
      double c = plaq(links, DIR_X, DIR_T, p, id, n.xp, n.tp);
      if (PMC && at_ytop(g, n)) {
        a = 0;
        b = 0;
      }
      e += -c;
      pl += (3 - a - b - c) / 3;
    }
  }
  double se, sp;
  block_sum2(e, pl, &se, &sp);
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
