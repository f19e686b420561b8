// Device building blocks shared by the single-lattice kernels (kernels.cuh)
// and the batched-replica kernels (batch.cu): the per-link update of one
// checkerboard phase and the deterministic FP64 block reductions.  Templates
// and inline functions only, so several translation units can include it.
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
  // FP32 draws (counter-based): the key, the device word holding the number
  // of drawing phases run before this launch (advanced on the device, so a
  // captured graph draws fresh numbers on every replay), this phase's offset
  // from it, and the offset added to the site index (a replica's stream
  // offset in a batch)
  unsigned long long seed;
  const unsigned long long* phase_ptr;
  unsigned int phase_off;
  unsigned int site_off;
  PhiloxKeys keys;  // round keys of `seed` (philox_keys), set by whoever fills the arguments
};

// The drawing-phase counter of the FP32 draws lives on the device and is
// advanced by this one-thread launch after every heat-bath or Metropolis pass
// (inside a captured graph too).  Internal linkage: each translation unit
// that includes this header has its own copy.
static __global__ void advance_counter(unsigned long long* c, unsigned long long n) { *c += n; }

// the drawing-phase number of this launch
__device__ __forceinline__ unsigned long long draw_phase(const PhaseArgs& a) {
  return __ldg(a.phase_ptr) + a.phase_off;
}

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

// FP32: the same updates with FP32 links and FP64 fix-ups; the heat-bath and
// Metropolis draw from the counter-based Philox stream of (site, phase), so
// no generator state is read or written.
// The new value of FP32 link U_MU at a site of sublattice PAR whose global
// sublattice index is gid (the Philox site counter and the accept slot);
// `links` and `n` address the staple links (global memory here, a
// shared-memory tile in the fused-pair kernel).  Metropolis accept counts are
// added only when count_accept is set.
template <int MU, int PAR, int BC, int KIND, class L>
__device__ __forceinline__ Quat<float> link_update32(const L& links, const Geo& g, const PhaseArgs& a, const Nbr& n,
                                                     int gid, int renorm, bool count_accept) {
  Quat<float> A = staple_sum<MU, BC, L, float>(links, g, n, PAR);
  Quat<float> U;
  if (KIND == KIND_HB) {
    PhiloxStream st(a.keys, a.site_off + (unsigned int)gid, draw_phase(a));
    U = heatbath_fast(A, a.beta, st, a.err);
  } else if (KIND == KIND_METRO) {
    PhiloxStream st(a.keys, a.site_off + (unsigned int)gid, draw_phase(a));
    U = links.ld_own(MU, PAR, n.id);
    int acc = metropolis_fast(U, A, a.beta, a.eps, a.upd, st);
    if (count_accept) atomicAdd(a.accept + PAR * g.vh + gid, acc);
  } else {
    U = overrelax_fast(A, links.ld_own(MU, PAR, n.id));
  }
  return renorm ? renorm_fast(U) : U;
}

template <int MU, int PAR, int BC, int KIND, bool CG>
__device__ __forceinline__ void site32(const Links32T<CG>& L, const RngStoreT<CG>& R, const Geo& g,
                                       const PhaseArgs& a, const Nbr& n, int renorm) {
  if (BC == BC_PCC && MU != DIR_Y && at_y0(g, n)) return;
  const int id = n.id;
  Quat<float> A = staple_sum<MU, BC, Links32T<CG>, float>(L, g, n, PAR);
  Quat<float> U;
  if (KIND == KIND_HB) {
    PhiloxStream st(a.keys, a.site_off + (unsigned int)id, draw_phase(a));
    U = heatbath_fast(A, a.beta, st, a.err);
  } else if (KIND == KIND_METRO) {
    PhiloxStream st(a.keys, a.site_off + (unsigned int)id, draw_phase(a));
    U = L.ld_own(MU, PAR, id);
    int acc = metropolis_fast(U, A, a.beta, a.eps, a.upd, st);
    add_accept<CG>(a.accept + PAR * g.vh + id, acc);
  } else {
    U = overrelax_fast(A, L.ld_own(MU, PAR, id));
  }
  L.st(MU, PAR, id, renorm ? renorm_fast(U) : U);
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
  const unsigned int ctas = gridDim.x;
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned int prev = atomicAdd(counter, 1u);
    last = (prev == ctas - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  // fixed-order sum over partials: per-thread strided chunks, then the CTA tree
  double a = 0, b = 0;
  for (unsigned int i = threadIdx.x; i < ctas; i += kBlock) {
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

// FP32 links: the three products in FP32 (the link's own precision), the
// result handed to the FP64 sums
__device__ __forceinline__ double plaq(const Links32& links, int mu, int nu, int p, int id, int omu, int onu) {
  Quat<float> A = q_mul(links.ld(mu, p, id), links.ld(nu, p ^ 1, id + omu));
  Quat<float> B = q_mul_bd(A, links.ld(mu, p ^ 1, id + onu));
  A = q_mul_bd(B, links.ld(nu, p, id));
  return 1.0 - (double)A.w;
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

// CTAs of a measurement: one per 1024 half-lattice sites (each thread then
// sums at least four sites of each parity, which amortises the CTA's
// reduction) up to a fixed cap, the threads striding over the sites, so a
// large lattice makes a few thousand partial sums (added by the last CTA).
// The count depends on the lattice only, so the summation order is the same
// on every device and for a lattice measured alone or in a batch.
constexpr long long kMeasureMaxBlocks = 4096;
constexpr long long kMeasureSitesPerBlock = 4 * kBlock;
__host__ __device__ __forceinline__ unsigned int measure_blocks(long long vh) {
  const long long nb = (vh + kMeasureSitesPerBlock - 1) / kMeasureSitesPerBlock;
  return (unsigned int)(nb < kMeasureMaxBlocks ? nb : kMeasureMaxBlocks);
}

// Energy and plaquette sums of the items k = c*256 + tid, + nb*256, ... of
// CTA c of nb, item k < V being the site of sublattice p = k / (V/2) with
// sublattice index k - p V/2: -(1 - P_xt) and 3 - the sum of the three 1 - P.
// One site of one parity per item keeps few links live per thread.  A
// multiply-high finds the site's t-slice; the neighbours come from the slice
// position (multiply-high).
template <class L, bool PMC>
__device__ __forceinline__ void measure_sites(const L& links, const Geo& g, int c, int nb, double& e, double& pl) {
  const unsigned int items = 2u * (unsigned int)g.vh;
  for (unsigned int k = (unsigned int)c * kBlock + threadIdx.x; k < items; k += (unsigned int)nb * kBlock) {
    const int p = k >= (unsigned int)g.vh;
    const int id = (int)k - p * g.vh;
    const int t = div_by((unsigned int)id, g.slice_m);
    const int s = id - t * g.slice;
    const Nbr n = make_nbr_slice(g, s, t, p);
    double a = plaq(links, DIR_Y, DIR_X, p, id, n.yp, n.xp);
    double b = plaq(links, DIR_Y, DIR_T, p, id, n.yp, n.tp);
    double cc = plaq(links, DIR_X, DIR_T, p, id, n.xp, n.tp);
    if (PMC && at_ytop(g, n)) {
      a = 0;
      b = 0;
    }
    e += -cc;
    pl += 3 - a - b - cc;  // the 1/3 of the plaquette average is applied once per thread
  }
}

}  // namespace qcd
