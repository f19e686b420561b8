// Fused even/odd pairs of the FP32 sweep, streamed through shared memory by
// bulk asynchronous copies (the TMA engine), for B200 (sm_100a).
//
// The six phases of a pass come in pairs (MU, even), (MU, odd).  Within a
// pair, U_MU couples only to sites displaced perpendicular to MU, so a pair
// can be run as a stream: one CTA owns a tile of rows x y' and walks along a
// streamed direction S (t for MU = y, x; x for MU = t).  At step j it updates
// the even U_MU of slice e and the odd U_MU of slice e - 2; the odd update
// needs the new even links of slices e-3 .. e-1, all made at earlier steps, so
// the two halves of a step are independent and one block barrier per step
// suffices.  The third direction R (y for MU = x, t; x for MU = y) has no
// streaming order: the even links of a one-site ring around the tile are
// recomputed by each CTA that needs them (their inputs are old links, so the
// recomputation is exact).
//
// Data flow per CTA (one per SM; 227 KB of shared memory):
//   * seven planes of NS x NR x W float4: the six link classes (direction,
//     parity) of NS consecutive slices of the tile and its halo, each slice of
//     a class one tensor copy (cp.async.bulk.tensor, a 5-D box of the link
//     store) from HBM/L2, and the new even U_MU of the same slices; boxes that
//     cross the lattice edge read zeros there and the CTA patches those cells
//     with their periodic images;
//   * NS mbarriers, one per slice slot; a slot is refilled with the slice NS
//     ahead once the block barrier shows nobody reads it, so every load is
//     issued two steps before it is needed;
//   * results go straight from registers to the other copy of the link store:
//     the pair reads the current store and writes U_MU into the second one,
//     so a CTA recomputing a ring never sees a neighbour's new links.
//
// Every link update is the one of the per-phase kernels (link_update32, same
// draws: the Philox counter is the site's global sublattice index and the
// phase number), the staples now gathered from shared memory.
//
// Tensor copies: the innermost coordinate is the quaternion component, always
// 0, so every box starts on a 16-byte boundary; the store comes from
// cudaMalloc and each slot is padded to 128 bytes.  No copy uses cluster
// multicast.
#pragma once
#include <cuda.h>
#include <stdint.h>
#include "sites.cuh"

namespace qcd {

constexpr int kPairNS = 7;      // slice slots
constexpr int kPairNR = 17;     // staged rows
constexpr int kPairW = 17;      // staged y' window
constexpr int kPairPlanes = 7;  // six link classes + the new even links of MU
// float4 per slot of a plane: the NR x W box of one slice, padded to 128 bytes
// (the alignment of a tensor copy's shared-memory destination)
constexpr int kPairSlotStride = (kPairNR * kPairW + 7) / 8 * 8;
constexpr int kPairPlane = kPairNS * kPairSlotStride;  // float4 per plane
constexpr size_t kPairSmemBytes = (size_t)kPairPlanes * kPairPlane * sizeof(float4) + kPairNS * sizeof(uint64_t);
constexpr unsigned int kPairFillBytes = 6u * kPairNR * kPairW * sizeof(float4);  // one slice of six classes
// within the 227 KB a block may opt in to, with room for the static variables
static_assert(kPairSmemBytes + 256 <= 232448, "pair kernel shared memory");
constexpr unsigned long long kPairWaitNs = 200000000ull;  // bound of one wait: 0.2 s, far above any real load

// Frame of the pair kernel for direction MU.
//   S      streamed direction
//   ROW    direction of the staged rows (the other one of x, t)
//   TR     tile rows;  ROW0: staged row of the first tile row
//   TY     tile y' per row;  W0: window column of the first tile y'
//   YRING  the ring is in y (MU = x, t) or in the rows (MU = y)
//   NT     threads: one per site update of a step
template <int MU>
struct PairCfg;
template <>
struct PairCfg<DIR_X> {
  static constexpr int S = DIR_T, ROW = DIR_X, TR = 16, ROW0 = 0, TY = 15, W0 = 1, NT = 512;
  static constexpr bool YRING = true;
};
template <>
struct PairCfg<DIR_T> {
  static constexpr int S = DIR_X, ROW = DIR_T, TR = 16, ROW0 = 0, TY = 15, W0 = 1, NT = 512;
  static constexpr bool YRING = true;
};
template <>
struct PairCfg<DIR_Y> {
  static constexpr int S = DIR_T, ROW = DIR_X, TR = 13, ROW0 = 2, TY = 16, W0 = 0, NT = 448;
  static constexpr bool YRING = false;
};
// even items (tile + ring) and odd items (tile) of a full tile fit one per thread
static_assert(16 * 16 + 16 * 15 <= 512, "x/t pair items");
static_assert(15 * 16 + 13 * 16 <= 448, "y pair items");
// staged rows and window cover the stencil: +1 row (MU = x, t) or ring +-1 and
// stencil +-1 rows (MU = y); ring +-1 and stencil +-1 in y' (MU = x, t) or +y (MU = y)
static_assert(16 + 1 <= kPairNR && 13 + 4 <= kPairNR, "rows");
static_assert(15 + 2 <= kPairW && 16 + 1 <= kPairW, "window");

struct PairPlanes {
  const float4* src[6];  // the current link classes, plane d*2 + p
  float4* dst_e;         // U_MU(even) of the other store
  float4* dst_o;         // U_MU(odd) of the other store
  int alt_mask;          // bit p: class p is read from the second store (tensor map tm_alt)
};

struct PairGrid {
  int n_row_tiles;  // tiles along ROW
  int seg;          // streamed slices per CTA
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ int pmod(int a, int n) {
  a %= n;
  return a < 0 ? a + n : a;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned int bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_test(uint32_t addr, unsigned int parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(addr), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait for the completion of the phase with the given parity: false
// after kPairWaitNs of wall time, or as soon as any CTA has flagged a timeout
// in the device error word (so one stuck load ends the whole launch quickly).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned int parity, const int* err) {
  const uint32_t addr = smem_u32(bar);
  unsigned long long t0 = 0;
  for (unsigned int i = 0;; i++) {
    if (mbar_test(addr, parity)) return true;
    if ((i & 63) == 63) {
      if (*(const volatile int*)err & DEVERR_TIMEOUT) return false;
      const unsigned long long t = global_ns();
      if (t0 == 0)
        t0 = t;
      else if (t - t0 > kPairWaitNs)
        return false;
    }
  }
}
// Bounded wait for this CTA's own copies before it exits after a timeout.
__device__ __forceinline__ void mbar_drain(uint64_t* bar, unsigned int parity) {
  const uint32_t addr = smem_u32(bar);
  const unsigned long long t0 = global_ns();
  while (!mbar_test(addr, parity) && global_ns() - t0 < kPairWaitNs) {
  }
}
// One box of a 5-D tensor map (component, y', x, t, class) into shared memory,
// completing on bar.  Coordinates outside the tensor read as zero.
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c1, int c2, int c3, int c4,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
      : "memory");
}

// The links of a step as the staple gather sees them: plane d*2 + p of the
// staged slices; in the odd half, U_MU(even) comes from the new-link plane.
template <int MU, bool ODD>
struct PairSmem {
  const float4* base;
  __device__ __forceinline__ Quat<float> ld(int dir, int par, int idx) const {
    const int plane = (ODD && dir == MU && par == 0) ? 6 : dir * 2 + par;
    const float4 v = base[plane * kPairPlane + idx];
    return Quat<float>{v.x, v.y, v.z, v.w};
  }
  __device__ __forceinline__ Quat<float> ld_own(int dir, int par, int idx) const { return ld(dir, par, idx); }
};

// Fill slot `slot` with unwrapped slice sx of the tile's rows and window: one
// tensor copy per link class (the box NR rows x W y' of one slice), issued by
// one thread.  Rows and y' are given unwrapped: where the box crosses the
// lattice edge it reads zeros, and the CTA patches those cells (pair_patch).
template <int MU>
__device__ __forceinline__ void pair_fill(float4* sm, uint64_t* bar, int slot, int sx, const PairPlanes& P,
                                          const CUtensorMap* tm_cur, const CUtensorMap* tm_alt, const Geo& g,
                                          int R0, int Y0h) {
  typedef PairCfg<MU> C;
  const int ls = C::S == DIR_T ? g.lt : g.lx;
  const int s = pmod(sx, ls);
  const int row0 = R0 - C::ROW0, y0 = Y0h - C::W0;
  const int cx = C::S == DIR_T ? row0 : s, ct = C::S == DIR_T ? s : row0;
  // the generic-proxy reads of this slot (before the block barrier) come
  // before the asynchronous writes that refill it
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mbar_expect_tx(bar, kPairFillBytes);
#pragma unroll
  for (int p = 0; p < 6; p++)
    tma_load_5d(sm + p * kPairPlane + slot * kPairSlotStride, (P.alt_mask >> p) & 1 ? tm_alt : tm_cur, y0, cx, ct,
                p, bar);
}

// The cells of a staged slice that lie beyond the lattice edge in the rows or
// in y' (the box read zeros there), with their periodic images: up to four
// per thread, fixed for the CTA except for the slice.
struct PairPatch {
  const float4* src[4];  // link of the image in its class, slice term excluded
  int soff[4];           // shared-memory index without the slot term
  int valid;             // bit m: cell m is an edge cell
};

// Cell m of this thread is k = tid + m * NT of the 6 x NR x W cells of a slice
// (every cell has a thread: 6 * 17 * 17 <= 4 * 448).
template <int MU>
__device__ __forceinline__ PairPatch pair_patch_cells(const PairPlanes& P, const Geo& g, int R0, int Y0h, int tid) {
  typedef PairCfg<MU> C;
  static_assert(6 * kPairNR * kPairW <= 4 * C::NT, "patch cells per thread");
  const int lrow = C::ROW == DIR_T ? g.lt : g.lx;
  PairPatch pp;
  pp.valid = 0;
#pragma unroll
  for (int m = 0; m < 4; m++) {
    pp.src[m] = P.src[0];
    pp.soff[m] = 0;
    const int k = tid + m * C::NT;
    if (k >= 6 * kPairNR * kPairW) continue;
    const int p = k / (kPairNR * kPairW), rem = k - p * (kPairNR * kPairW);
    const int r = rem / kPairW, w = rem - r * kPairW;
    const int gr_u = R0 - C::ROW0 + r, y_u = Y0h - C::W0 + w;
    if (gr_u >= 0 && gr_u < lrow && y_u >= 0 && y_u < g.lyh) continue;
    const int gr = pmod(gr_u, lrow), yq = pmod(y_u, g.lyh);
    // the row coordinate is x (slice = t) or t (slice = x)
    const size_t off = C::S == DIR_T ? (size_t)yq + (size_t)g.lyh * gr : (size_t)yq + (size_t)g.lyh * g.lx * gr;
    const float4* base = P.src[0];
    switch (p) {
      case 1: base = P.src[1]; break;
      case 2: base = P.src[2]; break;
      case 3: base = P.src[3]; break;
      case 4: base = P.src[4]; break;
      case 5: base = P.src[5]; break;
      default: break;
    }
    pp.src[m] = base + off;
    pp.soff[m] = p * kPairPlane + r * kPairW + w;
    pp.valid |= 1 << m;
  }
  return pp;
}

// Overwrite the thread's edge cells of slot `slot` (unwrapped slice sx) with
// their periodic images, after the slot's tensor copies completed.
template <int MU>
__device__ __forceinline__ void pair_patch(float4* sm, const PairPatch& pp, int slot, int sx, const Geo& g) {
  typedef PairCfg<MU> C;
  const int ls = C::S == DIR_T ? g.lt : g.lx;
  const size_t sterm = C::S == DIR_T ? (size_t)pmod(sx, ls) * g.lyh * g.lx : (size_t)pmod(sx, ls) * g.lyh;
#pragma unroll
  for (int m = 0; m < 4; m++)
    if ((pp.valid >> m) & 1) sm[pp.soff[m] + slot * kPairSlotStride] = __ldcg(pp.src[m] + sterm);
}

// One fused pair (MU, even) + (MU, odd) over one segment of the streamed
// direction for one tile.  Grid: (row tiles x y tiles, segments).
template <int MU, int BC, int KIND>
__global__ void __launch_bounds__(PairCfg<MU>::NT, 1)
    pair32(const __grid_constant__ CUtensorMap tm_cur, const __grid_constant__ CUtensorMap tm_alt, PairPlanes P,
           Geo g, PhaseArgs a, PairGrid pg) {
  typedef PairCfg<MU> C;
  extern __shared__ __align__(128) float4 sm[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kPairPlanes * kPairPlane);
  __shared__ int abort_flag;

  const int ls = C::S == DIR_T ? g.lt : g.lx, lrow = C::ROW == DIR_T ? g.lt : g.lx;
  const int rt = blockIdx.x % pg.n_row_tiles, yt = blockIdx.x / pg.n_row_tiles;
  const int R0 = rt * C::TR, Y0h = yt * C::TY;
  const int nr = min(C::TR, lrow - R0), ny = min(C::TY, g.lyh - Y0h);
  const int s0 = blockIdx.y * pg.seg, s1 = min(s0 + pg.seg, ls);
  const int first = s0 - 2, last = s1 + 1;  // unwrapped slices staged
  const int tid = threadIdx.x;

  if (tid == 0) {
    abort_flag = 0;
    for (int i = 0; i < kPairNS; i++) mbar_init(&bars[i], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0)
    for (int x = first; x <= last && x < first + kPairNS; x++)
      pair_fill<MU>(sm, &bars[x - first], x - first, x, P, &tm_cur, &tm_alt, g, R0, Y0h);
  // a tile whose staged rows or y' window cross the lattice edge patches the
  // cells its boxes read as zeros
  const bool edge = R0 - C::ROW0 < 0 || R0 - C::ROW0 + kPairNR > lrow || Y0h - C::W0 < 0 ||
                    Y0h - C::W0 + kPairW > g.lyh;
  PairPatch pp;
  pp.valid = 0;
  if (edge) pp = pair_patch_cells<MU>(P, g, R0, Y0h, tid);

  // this thread's item: an even site (tile + ring) or an odd site (tile)
  const int ne_row = C::YRING ? ny + 1 : ny;                  // even items per row
  const int ne_rows = C::YRING ? nr : nr + 2;                 // even rows
  const int n_even = ne_row * ne_rows, n_odd = ny * nr;
  const bool is_even = tid < n_even, is_odd = !is_even && tid < n_even + n_odd;
  int r = 0, i = 0;
  if (is_even) {
    r = tid / ne_row;
    i = tid - r * ne_row;
    r += C::YRING ? C::ROW0 : C::ROW0 - 1;
  } else if (is_odd) {
    const int u = tid - n_even;
    r = u / ny;
    i = u - r * ny;
    r += C::ROW0;
  }
  const int grow = pmod(R0 - C::ROW0 + r, lrow);  // global row coordinate
  const bool tile_row = r >= C::ROW0 && r < C::ROW0 + nr;
  int issued = min(last, first + kPairNS - 1);  // last slice whose fill was issued

  // Per-thread state along the stream, advanced by one slice per step: the
  // unwrapped slice of this thread's update, its slot, its global slice, the
  // parity q of its physical y (which flips from slice to slice) and the
  // global index term of the slice.  The window column, y' and tile test take
  // one of two values, for q = 0 and q = 1.
  const int par = is_even ? 0 : 1;
  int sx = is_even ? s0 - 1 : s0 - 3;
  int slot = pmod(sx - first, kPairNS);
  int gs = pmod(sx, ls);
  int q = ((sx + grow) & 1) ^ par;
  const int s_stride = C::S == DIR_T ? g.lyh * g.lx : g.lyh;
  int s_term = gs * s_stride;
  const int row_term = C::S == DIR_T ? g.lyh * grow : g.lyh * g.lx * grow;
  // window column: even items of a y-ring row start one column early when
  // their physical y is odd
  const int w_0 = C::YRING ? C::W0 + i : i;
  const int w_1 = C::YRING ? (is_even ? C::W0 - 1 + i : C::W0 + i) : i;
  const int yq_0 = pmod(Y0h - C::W0 + w_0, g.lyh), yq_1 = pmod(Y0h - C::W0 + w_1, g.lyh);
  const bool in_tile_0 = C::YRING ? (w_0 >= C::W0 && w_0 < C::W0 + ny) : tile_row;
  const bool in_tile_1 = C::YRING ? (w_1 >= C::W0 && w_1 < C::W0 + ny) : tile_row;
  const int row_off = r * kPairW;
  PhaseArgs ap = a;
  ap.phase_off = a.phase_off + (unsigned int)par;

  const int J = s1 - s0 + 3;
  for (int j = 0; j < J; j++) {
    const int e = s0 - 1 + j;
    // wait for the slices first read at this step
    bool ok = true;
    if (j == 0) {
      for (int x = first; x <= e && ok; x++) ok = mbar_wait(&bars[(x - first) % kPairNS], ((x - first) / kPairNS) & 1, a.err);
    }
    if (ok && e + 1 <= last) ok = mbar_wait(&bars[(e + 1 - first) % kPairNS], ((e + 1 - first) / kPairNS) & 1, a.err);
    if (!ok) {
      atomicOr(a.err, DEVERR_TIMEOUT);
      abort_flag = 1;
    }
    if (edge) {
      if (ok) {
        if (j == 0)
          for (int x = first; x <= e; x++) pair_patch<MU>(sm, pp, (x - first) % kPairNS, x, g);
        if (e + 1 <= last) pair_patch<MU>(sm, pp, (e + 1 - first) % kPairNS, e + 1, g);
      }
      __syncthreads();
    }
    const bool active = is_even ? (sx <= s1) : (is_odd && sx >= s0);
    if (ok && active) {
      const int w = q ? w_1 : w_0, yq = q ? yq_1 : yq_0;
      const int gid = yq + row_term + s_term;
      Nbr n;
      n.id = slot * kPairSlotStride + row_off + w;
      n.yq = yq;
      n.q = q;
      n.x = 0;
      n.t = 0;
      n.yp = q ? 1 : 0;
      n.ym = q ? 0 : -1;
      const int sp = slot == kPairNS - 1 ? -(kPairNS - 1) * kPairSlotStride : kPairSlotStride;
      const int sm_ = slot == 0 ? (kPairNS - 1) * kPairSlotStride : -kPairSlotStride;
      if (C::ROW == DIR_X) {
        n.xp = kPairW;
        n.xm = -kPairW;
        n.tp = sp;
        n.tm = sm_;
      } else {
        n.tp = kPairW;
        n.tm = -kPairW;
        n.xp = sp;
        n.xm = sm_;
      }
      const bool in_tile = q ? in_tile_1 : in_tile_0;
      const bool in_seg = sx >= s0 && sx < s1;
      Quat<float> U;
      if (is_even) {
        const PairSmem<MU, false> L{sm};
        if (BC == BC_PCC && MU != DIR_Y && at_y0(g, n))
          U = L.ld_own(MU, 0, n.id);  // frozen: the old link carries over
        else
          U = link_update32<MU, 0, BC, KIND>(L, g, ap, n, gid, a.renorm, in_tile && in_seg);
        sm[6 * kPairPlane + n.id] = make_float4(U.w, U.x, U.y, U.z);
        if (in_tile && in_seg) P.dst_e[gid] = make_float4(U.w, U.x, U.y, U.z);
      } else {
        const PairSmem<MU, true> L{sm};
        if (BC == BC_PCC && MU != DIR_Y && at_y0(g, n))
          U = L.ld_own(MU, 1, n.id);
        else
          U = link_update32<MU, 1, BC, KIND>(L, g, ap, n, gid, a.renorm, true);
        P.dst_o[gid] = make_float4(U.w, U.x, U.y, U.z);
      }
    }
    // the next slice
    sx++;
    q ^= 1;
    if (++slot == kPairNS) slot = 0;
    if (++gs == ls) {
      gs = 0;
      s_term = 0;
    } else {
      s_term += s_stride;
    }
    __syncthreads();
    if (abort_flag) break;
    // the slot of slice e - 3 is free: refill it with slice e - 3 + NS
    const int fx = e - 3 + kPairNS;
    if (e - 3 >= first && fx <= last) {
      if (tid == 0)
        pair_fill<MU>(sm, &bars[(fx - first) % kPairNS], (fx - first) % kPairNS, fx, P, &tm_cur, &tm_alt, g, R0, Y0h);
      issued = fx;
    }
  }
  if (abort_flag && tid == 0) {
    // leave no copy in flight into this CTA's shared memory: wait (bounded)
    // for the latest fill of every slot
    for (int x = max(first, issued - kPairNS + 1); x <= issued; x++)
      mbar_drain(&bars[(x - first) % kPairNS], ((x - first) / kPairNS) & 1);
  }
}

}  // namespace qcd
