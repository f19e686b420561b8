// Checkerboard geometry and the SoA link store in HBM.
//
// Sites are split by parity p = (t + x + y) mod 2 into two sublattices of
// Vh = V/2 sites.  A sublattice index is id = y' + Lyh*(x + Lx*t) with
// Lyh = Ly/2 (the reference's half-lattice index, mc_updates.h:130-134);
// the physical y of the site is 2y' + q with q = ((t + x) mod 2) xor p.
// Stream id of the random-number generator is this id for both parities
// (lattice_setup.h:15-21; even and odd kernels share state + id).
//
// Link store: one plane per (direction mu, parity p), plane index mu*2 + p,
// mu = 0 (y), 1 (x), 2 (t); inside a plane the links are contiguous in id.
//   FP64: two double2 planes (w, x) and (y, z) -> every warp load is 512 B
//         contiguous (coalesced), no partial sectors.
//   FP32: one float4 plane -> one 16-B load per link.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "su2.cuh"

namespace qcd {

enum { DIR_Y = 0, DIR_X = 1, DIR_T = 2 };
enum { BC_PER = 0, BC_PCC = 1, BC_PMC = 2 };

struct Geo {
  int lt, lx, ly;  // physical extents (all even)
  int lyh;         // Ly / 2
  int slice;       // Lyh * Lx : sublattice sites per t-slice
  int vh;          // Lyh * Lx * Lt
  // s / lyh for 0 <= s < slice as (s * lyh_magic) >> 32, lyh_magic = ceil(2^32 / lyh):
  // exact when lyh^2 * lx < 2^32 (fastdiv = 1), otherwise a hardware division is used
  unsigned long long lyh_magic;
  int fastdiv;
  // n / slice for any 32-bit n as the high word of n * slice_m (0: slice = 1)
  unsigned long long slice_m;
};

// m = ceil(2^64 / d) for 2 <= d < 2^32 (0 for d = 1): floor(n * m / 2^64) =
// floor(n / d) for every n < 2^32, because m * d - 2^64 < d
__host__ __forceinline__ unsigned long long div_magic(unsigned long long d) { return ~0ull / d + 1; }
__device__ __forceinline__ int div_by(unsigned int n, unsigned long long m) {
  return m ? (int)__umul64hi((unsigned long long)n, m) : (int)n;
}

__host__ __forceinline__ Geo make_geo(int lt, int lx, int ly) {
  Geo g;
  g.lt = lt;
  g.lx = lx;
  g.ly = ly;
  g.lyh = ly / 2;
  g.slice = g.lyh * lx;
  g.vh = g.slice * lt;
  g.lyh_magic = ((1ull << 32) + (unsigned long long)g.lyh - 1) / (unsigned long long)g.lyh;
  g.fastdiv = (unsigned long long)g.lyh * (unsigned long long)g.lyh * (unsigned long long)lx < (1ull << 32);
  g.slice_m = div_magic((unsigned long long)g.slice);
  return g;
}

// Decoded sublattice site plus the offsets (in sublattice index units) of its
// six neighbours, which all lie on the other sublattice.  Offsets add: the
// site x + mu - nu is id + off_plus(mu) + off_minus(nu) on the same
// sublattice, because moving in x or t does not change q and moving in y does
// not change x or t.
struct Nbr {
  int id, yq, x, t, q;
  int yp, ym, xp, xm, tp, tm;
};

__device__ __forceinline__ void finish_nbr(const Geo& g, int parity, Nbr& n);

// From the sublattice index (two divisions).
__device__ __forceinline__ Nbr make_nbr(const Geo& g, int id, int parity) {
  Nbr n;
  n.id = id;
  n.yq = id % g.lyh;
  int r = id / g.lyh;
  n.x = r % g.lx;
  n.t = r / g.lx;
  finish_nbr(g, parity, n);
  return n;
}

// From the position s inside t-slice t (launch grid (slice, Lt)): one
// multiply-high instead of two divisions.
__device__ __forceinline__ Nbr make_nbr_slice(const Geo& g, int s, int t, int parity) {
  Nbr n;
  n.t = t;
  n.x = g.fastdiv ? (int)(((unsigned long long)(unsigned)s * g.lyh_magic) >> 32) : s / g.lyh;
  n.yq = s - n.x * g.lyh;
  n.id = s + t * g.slice;
  finish_nbr(g, parity, n);
  return n;
}

// From the sublattice index: the t-slice by a multiply-high, the rest as in
// make_nbr_slice; the same offsets as make_nbr.
__device__ __forceinline__ Nbr make_nbr_fast(const Geo& g, int id, int parity) {
  const int t = div_by((unsigned int)id, g.slice_m);
  return make_nbr_slice(g, id - t * g.slice, t, parity);
}

__device__ __forceinline__ void finish_nbr(const Geo& g, int parity, Nbr& n) {
  n.q = ((n.t + n.x) & 1) ^ parity;
  // +y: a site with odd physical y moves to the next y' (wrapping), an even
  // one stays at the same y' (mc_updates.h:139-141, 195-197)
  n.yp = n.q ? (n.yq == g.lyh - 1 ? -(g.lyh - 1) : 1) : 0;
  // -y: the mirror image (mc_updates.h:252-254, 309-311)
  n.ym = n.q ? 0 : (n.yq == 0 ? g.lyh - 1 : -1);
  n.xp = n.x == g.lx - 1 ? -(g.lx - 1) * g.lyh : g.lyh;
  n.xm = n.x == 0 ? (g.lx - 1) * g.lyh : -g.lyh;
  n.tp = n.t == g.lt - 1 ? -(g.lt - 1) * g.slice : g.slice;
  n.tm = n.t == 0 ? (g.lt - 1) * g.slice : -g.slice;
}

__device__ __forceinline__ int off_plus(const Nbr& n, int dir) {
  return dir == DIR_Y ? n.yp : dir == DIR_X ? n.xp : n.tp;
}
__device__ __forceinline__ int off_minus(const Nbr& n, int dir) {
  return dir == DIR_Y ? n.ym : dir == DIR_X ? n.xm : n.tm;
}

// physical y of the site is 0 / Ly-1
__device__ __forceinline__ bool at_y0(const Geo& g, const Nbr& n) { return n.yq == 0 && n.q == 0; }
__device__ __forceinline__ bool at_ytop(const Geo& g, const Nbr& n) {
  return n.yq == g.lyh - 1 && n.q == 1;
}

__host__ __device__ __forceinline__ size_t plane_of(int dir, int parity) { return (size_t)(dir * 2 + parity); }

// Load/store policy: CG = false uses the read-only path (__ldg) for neighbour
// links, which is safe inside one phase launch because no link a phase reads
// is written in that launch.  CG = true (the wavefront kernel) reads and
// writes at L2 (.cg): there, other CTAs of the same launch rewrite links, and
// a line left in this SM's L1 by an earlier task could be stale.
template <class T, bool CG>
__device__ __forceinline__ T ld_nb(const T* p) {
  if (CG) return __ldcg(p);
  return __ldg(p);
}
template <class T, bool CG>
__device__ __forceinline__ T ld_rw(const T* p) {
  if (CG) return __ldcg(p);
  return *p;
}
template <class T, bool CG>
__device__ __forceinline__ void st_rw(T* p, const T& v) {
  if (CG)
    __stcg(p, v);
  else
    *p = v;
}

// ---------------------------------------------------------------- FP64 ----
template <bool CG>
struct Links64T {
  double2* lo;  // (w, x)
  double2* hi;  // (y, z)
  int vh;
  __device__ __forceinline__ Quat<double> ld(int dir, int parity, int id) const {
    size_t i = plane_of(dir, parity) * vh + id;
    double2 a = ld_nb<double2, CG>(lo + i), b = ld_nb<double2, CG>(hi + i);
    return Quat<double>{a.x, a.y, b.x, b.y};
  }
  // the link this thread rewrites
  __device__ __forceinline__ Quat<double> ld_own(int dir, int parity, int id) const {
    size_t i = plane_of(dir, parity) * vh + id;
    double2 a = ld_rw<double2, CG>(lo + i), b = ld_rw<double2, CG>(hi + i);
    return Quat<double>{a.x, a.y, b.x, b.y};
  }
  __device__ __forceinline__ void st(int dir, int parity, int id, const Quat<double>& u) const {
    size_t i = plane_of(dir, parity) * vh + id;
    st_rw<double2, CG>(lo + i, make_double2(u.w, u.x));
    st_rw<double2, CG>(hi + i, make_double2(u.y, u.z));
  }
};
typedef Links64T<false> Links64;

// ---------------------------------------------------------------- FP32 ----
template <bool CG>
struct Links32T {
  float4* q;
  int vh;
  __device__ __forceinline__ Quat<float> ld(int dir, int parity, int id) const {
    float4 a = ld_nb<float4, CG>(q + plane_of(dir, parity) * vh + id);
    return Quat<float>{a.x, a.y, a.z, a.w};
  }
  __device__ __forceinline__ Quat<float> ld_own(int dir, int parity, int id) const {
    float4 a = ld_rw<float4, CG>(q + plane_of(dir, parity) * vh + id);
    return Quat<float>{a.x, a.y, a.z, a.w};
  }
  __device__ __forceinline__ void st(int dir, int parity, int id, const Quat<float>& u) const {
    st_rw<float4, CG>(q + plane_of(dir, parity) * vh + id, make_float4(u.w, u.x, u.y, u.z));
  }
};
typedef Links32T<false> Links32;

}  // namespace qcd
