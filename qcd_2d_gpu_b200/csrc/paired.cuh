// FP32 link store in site pairs, and the kernels that use it.
//
// For a lattice with Lt divisible by 4 the FP32 links are stored in pairs:
// sublattice site id (t < Lt/2, lane 0) and site id + V/4 (t + Lt/2, lane 1)
// of the same plane share one 32-B record
//     (w0, w1, x0, x1) (y0, y1, z0, z1)
// (measured faster than a lo and a hi half-plane per class), so one thread updates both sites with packed two-lane FP32 arithmetic
// (fma.rn.f32x2 through __ffma2_rn): a quaternion product is 8 packed
// multiply-adds for two sites instead of 16 per site, and the neighbour
// offsets are worked out once for the pair.  Lt/2 is even, so both sites of
// a pair have the same q = ((t + x) mod 2) xor parity and therefore the same
// neighbour offsets inside the half lattice of "rows" r = t mod Lt/2; the
// only difference is at the row seam: going +t from row Lt/2 - 1 (or -t from
// row 0) lands on row 0 (Lt/2 - 1) with the two lanes exchanged, so the
// loaded pair is swapped there.  The seam is a whole row, so the swap is
// uniform over a CTA (a CTA works on one row).
//
// The per-link arithmetic is the FP32 path's (updates.cuh): staples in FP32,
// the heat-bath with its FP64 accept test and the Metropolis exact decision
// per lane, over-relaxation by the reflection identity, re-projection in
// double.  A site draws from the counter-based stream of its own sublattice
// index, so it draws exactly the numbers it draws in the unpaired store.
#pragma once
#include "sites.cuh"

namespace qcd {

// ------------------------------------------------------ two-lane floats --
struct Q2 {
  float2 w, x, y, z;
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 swap2(float2 a) { return make_float2(a.y, a.x); }
__device__ __forceinline__ Q2 swap_lanes(const Q2& q) { return Q2{swap2(q.w), swap2(q.x), swap2(q.y), swap2(q.z)}; }
__device__ __forceinline__ Quat<float> lane0(const Q2& q) { return Quat<float>{q.w.x, q.x.x, q.y.x, q.z.x}; }
__device__ __forceinline__ Quat<float> lane1(const Q2& q) { return Quat<float>{q.w.y, q.x.y, q.y.y, q.z.y}; }
__device__ __forceinline__ Q2 join(const Quat<float>& a, const Quat<float>& b) {
  return Q2{f2(a.w, b.w), f2(a.x, b.x), f2(a.y, b.y), f2(a.z, b.z)};
}

// The quaternion products of su2.cuh on both lanes.  Each subtracted term is
// written as a multiply-add with a negated copy of one factor's component,
// formed once per product, so every packed instruction is a plain
// multiply-add.
// a b^+
__device__ __forceinline__ Q2 p2_mul_bd(const Q2& a, const Q2& b) {
  const float2 nx = neg2(b.x), ny = neg2(b.y), nz = neg2(b.z);
  Q2 c;
  c.w = fma2(a.z, b.z, fma2(a.y, b.y, fma2(a.x, b.x, mul2(a.w, b.w))));
  c.x = fma2(a.z, b.y, fma2(a.y, nz, fma2(a.w, nx, mul2(a.x, b.w))));
  c.y = fma2(a.x, b.z, fma2(a.w, ny, fma2(a.z, nx, mul2(a.y, b.w))));
  c.z = fma2(a.x, ny, fma2(a.w, nz, fma2(a.y, b.x, mul2(a.z, b.w))));
  return c;
}
// A + a b^+
__device__ __forceinline__ Q2 p2_acc_mul_bd(const Q2& A, const Q2& a, const Q2& b) {
  const float2 nx = neg2(b.x), ny = neg2(b.y), nz = neg2(b.z);
  Q2 c;
  c.w = fma2(a.z, b.z, fma2(a.y, b.y, fma2(a.x, b.x, fma2(a.w, b.w, A.w))));
  c.x = fma2(a.z, b.y, fma2(a.y, nz, fma2(a.w, nx, fma2(a.x, b.w, A.x))));
  c.y = fma2(a.x, b.z, fma2(a.w, ny, fma2(a.z, nx, fma2(a.y, b.w, A.y))));
  c.z = fma2(a.x, ny, fma2(a.w, nz, fma2(a.y, b.x, fma2(a.z, b.w, A.z))));
  return c;
}
// a b
__device__ __forceinline__ Q2 p2_mul(const Q2& a, const Q2& b) {
  const float2 nx = neg2(b.x), ny = neg2(b.y), nz = neg2(b.z);
  Q2 c;
  c.w = fma2(a.z, nz, fma2(a.y, ny, fma2(a.x, nx, mul2(a.w, b.w))));
  c.x = fma2(a.z, ny, fma2(a.y, b.z, fma2(a.w, b.x, mul2(a.x, b.w))));
  c.y = fma2(a.x, nz, fma2(a.w, b.y, fma2(a.z, b.x, mul2(a.y, b.w))));
  c.z = fma2(a.x, b.y, fma2(a.w, b.z, fma2(a.y, nx, mul2(a.z, b.w))));
  return c;
}
// A + P^+ c
__device__ __forceinline__ Q2 p2_acc_mul_ad(const Q2& A, const Q2& P, const Q2& c) {
  const float2 nw = neg2(c.w), nx = neg2(c.x), ny = neg2(c.y), nz = neg2(c.z);
  Q2 r;
  r.w = fma2(P.z, c.z, fma2(P.y, c.y, fma2(P.x, c.x, fma2(P.w, c.w, A.w))));
  r.x = fma2(P.z, c.y, fma2(P.y, nz, fma2(P.w, c.x, fma2(P.x, nw, A.x))));
  r.y = fma2(P.x, c.z, fma2(P.w, c.y, fma2(P.z, nx, fma2(P.y, nw, A.y))));
  r.z = fma2(P.x, ny, fma2(P.w, c.z, fma2(P.y, c.x, fma2(P.z, nw, A.z))));
  return r;
}
// Re of a b^+ (the w component alone): 1/2 Re tr(a b^+)
__device__ __forceinline__ float2 p2_retr_bd(const Q2& a, const Q2& b) {
  return fma2(a.z, b.z, fma2(a.y, b.y, fma2(a.x, b.x, mul2(a.w, b.w))));
}

// ------------------------------------------------------------- the store --
// One pair record in one 32-B access (sm_100 global loads and stores of
// eight 32-bit words; the record is 32-B aligned): half the load
// instructions and L1 wavefronts of two float4 accesses.
__device__ __forceinline__ Q2 ld_pair_nc(const float4* p) {
  float a0, a1, a2, a3, b0, b1, b2, b3;
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(a0), "=f"(a1), "=f"(a2), "=f"(a3), "=f"(b0), "=f"(b1), "=f"(b2), "=f"(b3)
      : "l"(p));
  return Q2{f2(a0, a1), f2(a2, a3), f2(b0, b1), f2(b2, b3)};
}
__device__ __forceinline__ Q2 ld_pair(const float4* p) {
  float a0, a1, a2, a3, b0, b1, b2, b3;
  asm volatile("ld.global.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=f"(a0), "=f"(a1), "=f"(a2), "=f"(a3), "=f"(b0), "=f"(b1), "=f"(b2), "=f"(b3)
               : "l"(p)
               : "memory");
  return Q2{f2(a0, a1), f2(a2, a3), f2(b0, b1), f2(b2, b3)};
}
__device__ __forceinline__ void st_pair(float4* p, const Q2& u) {
  asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(u.w.x), "f"(u.w.y), "f"(u.x.x),
               "f"(u.x.y), "f"(u.y.x), "f"(u.y.y), "f"(u.z.x), "f"(u.z.y)
               : "memory");
}

struct Pair32 {
  float4* q;  // 6 planes (plane_of(dir, parity)) of vhp pairs, each pair two float4
  int vhp;    // V/4: pairs per plane
  // first float4 of pair j (the second follows it)
  __device__ __forceinline__ float4* at(int dir, int par, int j) const {
    return q + ((size_t)plane_of(dir, par) * vhp + j) * 2;
  }
  // a neighbour pair (not written by the launch that reads it)
  __device__ __forceinline__ Q2 ld(int dir, int par, int j) const { return ld_pair_nc(at(dir, par, j)); }
  // the pair a thread rewrites
  __device__ __forceinline__ Q2 ld_own(int dir, int par, int j) const { return ld_pair(at(dir, par, j)); }
  __device__ __forceinline__ void st(int dir, int par, int j, const Q2& u) const { st_pair(at(dir, par, j), u); }
  // one site, by its sublattice index (the one-off kernels: starts, layout changes)
  __device__ __forceinline__ Quat<float> ld_site(int dir, int par, int id) const {
    const int lane = id >= vhp, j = id - lane * vhp;
    const float* lo = reinterpret_cast<const float*>(at(dir, par, j));
    const float* hi = reinterpret_cast<const float*>(at(dir, par, j) + 1);
    return Quat<float>{lo[lane], lo[2 + lane], hi[lane], hi[2 + lane]};
  }
  __device__ __forceinline__ void st_site(int dir, int par, int id, const Quat<float>& u) const {
    const int lane = id >= vhp, j = id - lane * vhp;
    float* lo = reinterpret_cast<float*>(at(dir, par, j));
    float* hi = reinterpret_cast<float*>(at(dir, par, j) + 1);
    lo[lane] = u.w;
    lo[2 + lane] = u.x;
    hi[lane] = u.y;
    hi[2 + lane] = u.z;
  }
};

// starts (init_cold / init_hot of kernels.cuh) write one site at a time
__device__ __forceinline__ void put(const Pair32& L, int d, int p, int id, const Quat<double>& u) {
  L.st_site(d, p, id, Quat<float>{(float)u.w, (float)u.x, (float)u.y, (float)u.z});
}

// ------------------------------------------------------------- staples --
// The staple sum of both lanes of pair n (n from the half geometry gh, whose
// t-slices are the rows); sp: this row is the last (+t crosses the seam), sm:
// this row is the first (-t crosses the seam).  Same staples, order and PMC
// masks as add_staples (updates.cuh); the backward product a^+ b^+ is formed
// as (b a)^+.
// PS: the store accessor (Pair32, or a variant with other load paths)
template <int MU, int NU, int BC, class PS>
__device__ __forceinline__ void add_staples2(const PS& P, const Geo& gh, const Nbr& n, int par, bool sp, bool sm,
                                             Q2& A) {
  const int o = par ^ 1;
  const bool drop_fwd = BC == BC_PMC && NU == DIR_Y && at_ytop(gh, n);
  const bool drop_bwd = BC == BC_PMC && NU == DIR_Y && at_y0(gh, n);
  if (!drop_fwd) {
    Q2 a = P.ld(NU, o, n.id + off_plus(n, MU));
    if (MU == DIR_T && sp) a = swap_lanes(a);
    Q2 b = P.ld(MU, o, n.id + off_plus(n, NU));
    if (NU == DIR_T && sp) b = swap_lanes(b);
    const Q2 c = P.ld(NU, par, n.id);
    A = p2_acc_mul_bd(A, p2_mul_bd(a, b), c);
  }
  if (!drop_bwd) {
    const int m = n.id + off_minus(n, NU);
    const bool sw = NU == DIR_T && sm;  // the backward sites lie across the -t seam
    Q2 a = P.ld(NU, par, m + off_plus(n, MU));
    if ((MU == DIR_T && sp) || sw) a = swap_lanes(a);
    Q2 b = P.ld(MU, o, m);
    Q2 c = P.ld(NU, o, m);
    if (sw) {
      b = swap_lanes(b);
      c = swap_lanes(c);
    }
    A = p2_acc_mul_ad(A, p2_mul(b, a), c);
  }
}

template <int MU, int BC, class PS>
__device__ __forceinline__ Q2 staple_sum2(const PS& P, const Geo& gh, const Nbr& n, int par, bool sp, bool sm) {
  Q2 A{f2(0.f, 0.f), f2(0.f, 0.f), f2(0.f, 0.f), f2(0.f, 0.f)};
  add_staples2<MU, Planes<MU>::NU1, BC>(P, gh, n, par, sp, sm, A);
  add_staples2<MU, Planes<MU>::NU2, BC>(P, gh, n, par, sp, sm, A);
  return A;
}

// U' = 2 (<A, Ubar> / |A|^2) Abar - U on both lanes (overrelax_fast)
__device__ __forceinline__ Q2 overrelax2(const Q2& A, const Q2& U) {
  const float2 rt = fma2(A.z, neg2(U.z), fma2(A.y, neg2(U.y), fma2(A.x, neg2(U.x), mul2(A.w, U.w))));
  const float2 dt = fma2(A.z, A.z, fma2(A.y, A.y, fma2(A.x, A.x, mul2(A.w, A.w))));
  const float2 c = f2(__fdividef(2.f * rt.x, dt.x), __fdividef(2.f * rt.y, dt.y));
  const float2 nc = neg2(c);
  return Q2{fma2(c, A.w, neg2(U.w)), fma2(nc, A.x, neg2(U.x)), fma2(nc, A.y, neg2(U.y)), fma2(nc, A.z, neg2(U.z))};
}

// ------------------------------------------------------------ one phase --
// The new links of both lanes of pair n (sublattice PAR); gid0 is lane 0's
// sublattice index (lane 1's is gid0 + V/4), used for the counter-based
// draws and the Metropolis accept counters.
template <int MU, int PAR, int BC, int KIND, class PS>
__device__ __forceinline__ Q2 pair_update(const PS& P, const Geo& gh, const PhaseArgs& a, const Nbr& n, bool sp,
                                          bool sm, int renorm) {
  const Q2 A = staple_sum2<MU, BC>(P, gh, n, PAR, sp, sm);
  const unsigned int gid0 = (unsigned int)n.id, gid1 = gid0 + (unsigned int)P.vhp;
  Q2 U;
  if (KIND == KIND_HB) {
    PhiloxStream s0(a.keys, a.site_off + gid0, draw_phase(a));
    PhiloxStream s1(a.keys, a.site_off + gid1, draw_phase(a));
    const Quat<float> u0 = heatbath_fast(lane0(A), a.beta, s0, a.err);
    const Quat<float> u1 = heatbath_fast(lane1(A), a.beta, s1, a.err);
    U = join(u0, u1);
  } else if (KIND == KIND_METRO) {
    const Q2 U0 = P.ld_own(MU, PAR, n.id);
    Quat<float> u0 = lane0(U0), u1 = lane1(U0);
    PhiloxStream s0(a.keys, a.site_off + gid0, draw_phase(a));
    PhiloxStream s1(a.keys, a.site_off + gid1, draw_phase(a));
    const int acc0 = metropolis_fast(u0, lane0(A), a.beta, a.eps, a.upd, s0);
    const int acc1 = metropolis_fast(u1, lane1(A), a.beta, a.eps, a.upd, s1);
    int* acc = a.accept + PAR * 2 * P.vhp;
    acc[gid0] += acc0;
    acc[gid1] += acc1;
    U = join(u0, u1);
  } else {
    U = overrelax2(A, P.ld_own(MU, PAR, n.id));
  }
  if (renorm) U = join(renorm_fast(lane0(U)), renorm_fast(lane1(U)));
  return U;
}

// Launch grid (ceil(slice / kBlock), Lt/2): blockIdx.y is the row.  The
// heat-bath and over-relaxation phases run spill-free at four CTAs per SM (64
// registers), measured 3-5% faster than five with small spills; Metropolis
// keeps five.
template <int MU, int PAR, int BC, int KIND>
__global__ void __launch_bounds__(kBlock, KIND == KIND_METRO ? 5 : 4) phase32p(Pair32 P, Geo gh, PhaseArgs a) {
  const int s = blockIdx.x * kBlock + threadIdx.x;
  if (s >= gh.slice) return;
  const int r = blockIdx.y;
  const Nbr n = make_nbr_slice(gh, s, r, PAR);
  if (BC == BC_PCC && MU != DIR_Y && at_y0(gh, n)) return;
  P.st(MU, PAR, n.id, pair_update<MU, PAR, BC, KIND>(P, gh, a, n, r == gh.lt - 1, r == 0, a.renorm));
}

// ------------------------------------------------------- measurement ----
// 1/2 Re tr U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+ on both lanes
// (plaquette_yx/yt/xt, observables.h:1-21), products in FP32; the caller
// forms 1 - P in double, as the unpaired measurement does
__device__ __forceinline__ float2 plaq2(const Pair32& P, int mu, int nu, int p, int id, int omu, int onu, bool swmu,
                                        bool swnu) {
  Q2 b = P.ld(nu, p ^ 1, id + omu);
  if (swmu) b = swap_lanes(b);
  Q2 c = P.ld(mu, p ^ 1, id + onu);
  if (swnu) c = swap_lanes(c);
  const Q2 A = p2_mul(P.ld(mu, p, id), b);
  const Q2 B = p2_mul_bd(A, c);
  return p2_retr_bd(B, P.ld(nu, p, id));
}

// Items k = c*256 + tid, + nb*256, ... below 2 V/4: pair k - p V/4 of
// sublattice p = k / (V/4), both lanes; deterministic per-CTA partials as
// in measure (kernels.cuh).
template <bool PMC>
__device__ __forceinline__ void measure_pairs(const Pair32& P, const Geo& gh, int c, int nb, double& e, double& pl) {
  const unsigned int items = 2u * (unsigned int)gh.vh;
  for (unsigned int k = (unsigned int)c * kBlock + threadIdx.x; k < items; k += (unsigned int)nb * kBlock) {
    const int p = k >= (unsigned int)gh.vh;
    const int id = (int)k - p * gh.vh;
    const int r = div_by((unsigned int)id, gh.slice_m);
    const int s = id - r * gh.slice;
    const Nbr n = make_nbr_slice(gh, s, r, p);
    const bool sp = r == gh.lt - 1;
    const float2 a = plaq2(P, DIR_Y, DIR_X, p, id, n.yp, n.xp, false, false);
    const float2 b = plaq2(P, DIR_Y, DIR_T, p, id, n.yp, n.tp, false, sp);
    const float2 cc = plaq2(P, DIR_X, DIR_T, p, id, n.xp, n.tp, false, sp);
    double ay = (1.0 - (double)a.x) + (1.0 - (double)a.y), by = (1.0 - (double)b.x) + (1.0 - (double)b.y);
    const double cs = (1.0 - (double)cc.x) + (1.0 - (double)cc.y);
    if (PMC && at_ytop(gh, n)) {
      ay = 0;
      by = 0;
    }
    e += -cs;
    pl += 6 - ay - by - cs;
  }
}

template <int PMC>
__global__ void __launch_bounds__(kBlock) measure_p(Pair32 P, Geo gh, double2* partials, unsigned int* counter,
                                                    double* out) {
  double e = 0, pl = 0;
  measure_pairs<PMC != 0>(P, gh, blockIdx.x, gridDim.x, e, pl);  // grid: measure_blocks(V/2)
  double se, sp;
  block_sum2(e, pl * (1.0 / 3.0), &se, &sp);
  if (threadIdx.x == 0) partials[blockIdx.x] = make_double2(se, sp);
  finish_sum2(partials, counter, 1.0 / (4.0 * (double)gh.vh), out);
}

// ------------------------------------------------ whole-store kernels ----
// (internal linkage: each translation unit that includes this header and
// launches them has its own copy)
// thread per pair: re-projection of both lanes of all six planes (normalize)
static __global__ void __launch_bounds__(kBlock) normalize32p(Pair32 P) {
  const int j = blockIdx.x * kBlock + threadIdx.x;
  if (j >= P.vhp) return;
  for (int p = 0; p < 2; p++)
    for (int d = 0; d < 3; d++) {
      const Q2 u = P.ld_own(d, p, j);
      P.st(d, p, j, join(renorm_fast(lane0(u)), renorm_fast(lane1(u))));
    }
}

// unitarity (kernels.cuh): thread per pair
static __global__ void __launch_bounds__(kBlock) unitarity_p(Pair32 P, double tol, double2* partials, unsigned int* counter,
                                                      double* out) {
  const int j = blockIdx.x * kBlock + threadIdx.x;
  double s = 0, bad = 0;
  if (j < P.vhp) {
    for (int p = 0; p < 2; p++)
      for (int d = 0; d < 3; d++) {
        const Q2 u = P.ld_own(d, p, j);
        for (int l = 0; l < 2; l++) {
          const Quat<float> v = l ? lane1(u) : lane0(u);
          const double det = q_det(Quat<double>{v.w, v.x, v.y, v.z});
          s += det;
          if (!(fabs(det - 1.0) <= tol)) bad += 1;
        }
      }
  }
  double ss, sb;
  block_sum2(s, bad, &ss, &sb);
  if (threadIdx.x == 0) partials[blockIdx.x] = make_double2(ss, sb);
  finish_sum2(partials, counter, 1.0, out);
}

// reference AoS (phi[(p*Vh + id)*12 + d*4 + c]) <-> paired store, thread per site
static __global__ void __launch_bounds__(kBlock) aos_to_pair32(const double* __restrict__ aos, Pair32 P, int vh) {
  const int id = blockIdx.x * kBlock + threadIdx.x;
  if (id >= vh) return;
  for (int p = 0; p < 2; p++) {
    const double* s = aos + ((size_t)p * vh + id) * 12;
    for (int d = 0; d < 3; d++)
      P.st_site(d, p, id,
                Quat<float>{(float)s[d * 4 + 0], (float)s[d * 4 + 1], (float)s[d * 4 + 2], (float)s[d * 4 + 3]});
  }
}
static __global__ void __launch_bounds__(kBlock) pair32_to_aos(Pair32 P, double* __restrict__ aos, int vh) {
  const int id = blockIdx.x * kBlock + threadIdx.x;
  if (id >= vh) return;
  for (int p = 0; p < 2; p++) {
    double* s = aos + ((size_t)p * vh + id) * 12;
    for (int d = 0; d < 3; d++) {
      const Quat<float> u = P.ld_site(d, p, id);
      s[d * 4 + 0] = u.w;
      s[d * 4 + 1] = u.x;
      s[d * 4 + 2] = u.y;
      s[d * 4 + 3] = u.z;
    }
  }
}

// one float4 plane store (Links32) <-> paired store, thread per pair
static __global__ void __launch_bounds__(kBlock) plain_to_pair32(const float4* __restrict__ src, Pair32 P) {
  const int j = blockIdx.x * kBlock + threadIdx.x;
  if (j >= P.vhp) return;
  for (int k = 0; k < 6; k++) {
    const float4 a = src[(size_t)k * 2 * P.vhp + j], b = src[(size_t)k * 2 * P.vhp + j + P.vhp];
    float4* d = P.q + ((size_t)k * P.vhp + j) * 2;
    d[0] = make_float4(a.x, b.x, a.y, b.y);
    d[1] = make_float4(a.z, b.z, a.w, b.w);
  }
}
static __global__ void __launch_bounds__(kBlock) pair32_to_plain(Pair32 P, float4* __restrict__ dst) {
  const int j = blockIdx.x * kBlock + threadIdx.x;
  if (j >= P.vhp) return;
  for (int k = 0; k < 6; k++) {
    const float4* s = P.q + ((size_t)k * P.vhp + j) * 2;
    const float4 u = s[0], v = s[1];
    dst[(size_t)k * 2 * P.vhp + j] = make_float4(u.x, u.z, v.x, v.z);
    dst[(size_t)k * 2 * P.vhp + j + P.vhp] = make_float4(u.y, u.w, v.y, v.w);
  }
}

}  // namespace qcd
