// Random numbers.  The FP64 sweep and every hot start draw from per-site
// MRG32k3a streams, stored compactly; the FP32 sweep draws from the
// counter-based Philox4x32-10 below and stores nothing.
//
// The reference keeps one curandStateMRG32k3a_t (48 B, AoS) per half-lattice
// site and seeds stream id with curand_init(seed, id, 0) (lattice_setup.h:15-21,
// kernel.cu:77-79).  Uniform draws only read and write the six 32-bit words of
// the two component generators, so the store here keeps just those, as six
// u32 planes of Vh words (24 B per stream, coalesced), and rebuilds the cuRAND
// state in registers around each update.  The draws themselves are cuRAND's
// own curand_uniform / curand_uniform_double, so the sequence per stream is
// the reference's by construction.
#pragma once
#include <curand_kernel.h>
#include <stdint.h>

namespace qcd {

template <bool CG>
struct RngStoreT {
  uint32_t* w;  // w[j * vh + id], j = 0..2 -> s1[j], j = 3..5 -> s2[j-3]
  int vh;

  __device__ __forceinline__ uint32_t get(int j, int id) const {
    const uint32_t* p = w + (size_t)j * vh + id;
    return CG ? __ldcg(p) : *p;
  }
  __device__ __forceinline__ void put(int j, int id, uint32_t v) const {
    uint32_t* p = w + (size_t)j * vh + id;
    if (CG)
      __stcg(p, v);
    else
      *p = v;
  }
  __device__ __forceinline__ void load(int id, curandStateMRG32k3a_t* s) const {
    s->s1[0] = get(0, id);
    s->s1[1] = get(1, id);
    s->s1[2] = get(2, id);
    s->s2[0] = get(3, id);
    s->s2[1] = get(4, id);
    s->s2[2] = get(5, id);
    s->boxmuller_flag = 0;
    s->boxmuller_flag_double = 0;
    s->boxmuller_extra = 0.f;
    s->boxmuller_extra_double = 0.0;
  }
  __device__ __forceinline__ void store(int id, const curandStateMRG32k3a_t* s) const {
    put(0, id, s->s1[0]);
    put(1, id, s->s1[1]);
    put(2, id, s->s1[2]);
    put(3, id, s->s2[0]);
    put(4, id, s->s2[1]);
    put(5, id, s->s2[2]);
  }
};
typedef RngStoreT<false> RngStore;

// ------------------------------------------------- seeding many streams ----
// curand_init(seed, id, 0) places stream id 2^76 steps after stream id - 1
// (it truncates the subsequence to 51 bits to stay inside one 2^127-step
// sequence: L'Ecuyer's substreams).  Its skip-ahead costs about a millisecond
// per call for the ids of a large lattice, so the streams are seeded here
// from curand_init(seed, 0, 0) alone: stream id is J^id applied to it, with J
// = A^(2^76) and A the transition matrix of each MRG32k3a component
// (L'Ecuyer, "Good parameters and implementations for combined multiple
// recursive random number generators", Operations Research 47(1), 1999:
// x_n = 1403580 x_{n-2} - 810728 x_{n-3} mod m1,
// y_n = 527612 y_{n-1} - 1370589 y_{n-3} mod m2, state (s[0], s[1], s[2]) =
// oldest to newest).  id is taken in base-256 digits, J^id = prod_k
// (J^(256^k))^(d_k), from tables of J^(j 256^k), j < 256, k < 5 (ids below
// 2^40) built on the host by repeated squaring.  Thread 0 of a CTA jumps to the
// CTA's first stream, every thread on by its index.  The states equal
// curand_init's word for word (the FP64 path's bit-for-bit tests against the
// reference depend on it).
constexpr uint64_t kMrgM1 = 4294967087ull, kMrgM2 = 4294944443ull;
constexpr int kMrgSubseqLog2 = 76;  // steps between consecutive subsequences: 2^76
constexpr int kMrgDigits = 5;       // base-256 digits of a stream number: ids < 2^40
constexpr int kMrgJumps = 256;
constexpr int kMrgJumpWords = kMrgDigits * kMrgJumps * 18;  // [digit][j]: component 1 then 2, 3x3 row-major
constexpr long long kMrgMaxStreams = 1ll << 40;

inline void mrg_jump_table(uint32_t* out) {
  typedef unsigned __int128 u128;
  struct M3 {
    uint64_t a[9];
  };
  auto mul = [](const M3& x, const M3& y, uint64_t m) {
    M3 r;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        u128 s = 0;
        for (int k = 0; k < 3; k++) s += (u128)x.a[3 * i + k] * y.a[3 * k + j];
        r.a[3 * i + j] = (uint64_t)(s % m);
      }
    return r;
  };
  M3 a1 = {{0, 1, 0, 0, 0, 1, kMrgM1 - 810728, 1403580, 0}};
  M3 a2 = {{0, 1, 0, 0, 0, 1, kMrgM2 - 1370589, 0, 527612}};
  for (int i = 0; i < kMrgSubseqLog2; i++) {  // J = A^(2^76)
    a1 = mul(a1, a1, kMrgM1);
    a2 = mul(a2, a2, kMrgM2);
  }
  for (int d = 0; d < kMrgDigits; d++) {  // a = J^(256^d)
    M3 p1 = {{1, 0, 0, 0, 1, 0, 0, 0, 1}}, p2 = p1;
    for (int j = 0; j < kMrgJumps; j++) {
      uint32_t* o = out + ((size_t)d * kMrgJumps + j) * 18;
      for (int k = 0; k < 9; k++) {
        o[k] = (uint32_t)p1.a[k];
        o[9 + k] = (uint32_t)p2.a[k];
      }
      p1 = mul(p1, a1, kMrgM1);
      p2 = mul(p2, a2, kMrgM2);
    }
    a1 = p1;  // J^(256^(d+1))
    a2 = p2;
  }
}

// The table on the host, built once per process.
inline const uint32_t* mrg_jump_host() {
  struct T {
    uint32_t w[kMrgJumpWords];
    T() { mrg_jump_table(w); }
  };
  static const T t;
  return t.w;
}

// s <- M s mod m for one component (M: 9 words, row-major)
__device__ __forceinline__ void mrg_mat_vec(const uint32_t* __restrict__ M, unsigned int s[3], uint64_t m) {
  uint64_t r[3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    uint64_t acc = 0;
#pragma unroll
    for (int k = 0; k < 3; k++) acc += ((uint64_t)__ldg(M + 3 * i + k) * s[k]) % m;  // terms < m < 2^32
    r[i] = acc % m;
  }
  s[0] = (unsigned int)r[0];
  s[1] = (unsigned int)r[1];
  s[2] = (unsigned int)r[2];
}

// s (s1 then s2) <- J^id s for 0 <= id < 2^40, from digit `first_digit` on
__device__ __forceinline__ void mrg_jump(unsigned int s[6], const uint32_t* table, unsigned long long id,
                                        int first_digit = 0) {
  id >>= 8 * first_digit;
  for (int d = first_digit; d < kMrgDigits && id; d++, id >>= 8) {
    const int j = (int)(id & 255u);
    if (!j) continue;
    const uint32_t* M = table + ((size_t)d * kMrgJumps + j) * 18;
    mrg_mat_vec(M, s, kMrgM1);
    mrg_mat_vec(M + 9, s + 3, kMrgM2);
  }
}

// The CTA's thread 0 puts the state of stream `first` (curand_init(seed,
// first, 0)) in base[6]; the CTA then reads it with mrg_jump_from.
__device__ __forceinline__ void mrg_cta_base(unsigned int base[6], const uint32_t* table, unsigned long long seed,
                                             unsigned long long first) {
  curandStateMRG32k3a_t s0;
  curand_init(seed, 0ull, 0ull, &s0);
  unsigned int s[6] = {s0.s1[0], s0.s1[1], s0.s1[2], s0.s2[0], s0.s2[1], s0.s2[2]};
  mrg_jump(s, table, first);
  for (int i = 0; i < 6; i++) base[i] = s[i];
}

// The state of stream (the CTA's first stream) + j, 0 <= j < 256.
__device__ __forceinline__ void mrg_jump_from(const unsigned int base[6], const uint32_t* table, int j,
                                              curandStateMRG32k3a_t* st) {
  unsigned int s[6] = {base[0], base[1], base[2], base[3], base[4], base[5]};
  if (j) {
    const uint32_t* M = table + (size_t)j * 18;
    mrg_mat_vec(M, s, kMrgM1);
    mrg_mat_vec(M + 9, s + 3, kMrgM2);
  }
  for (int i = 0; i < 3; i++) {
    st->s1[i] = s[i];
    st->s2[i] = s[3 + i];
  }
  st->boxmuller_flag = 0;
  st->boxmuller_flag_double = 0;
  st->boxmuller_extra = 0.f;
  st->boxmuller_extra_double = 0.0;
}

// ------------------------------------------------ counter-based stream ----
// Philox4x32-10 (J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11): a 4 x 32-bit counter
// and a 2 x 32-bit key go through ten rounds of two 32 x 32 -> 64-bit
// multiplies with the round keys bumped by the Weyl increments between
// rounds.  It keeps no state in memory: the FP32 sweep draws from the counter
// (site, block, phase counter) under the key (seed), which removes the 2 x 24 B
// of generator-state traffic per site and phase that a stored generator costs.
struct Philox4x32 {
  static constexpr uint32_t kM0 = 0xD2511F53u, kM1 = 0xCD9E8D57u;  // round multipliers
  static constexpr uint32_t kW0 = 0x9E3779B9u, kW1 = 0xBB67AE85u;  // key increments
  __host__ __device__ __forceinline__ static void block(const uint32_t ctr[4], const uint32_t key[2],
                                                        uint32_t out[4]) {
    uint32_t x0 = ctr[0], x1 = ctr[1], x2 = ctr[2], x3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
#pragma unroll
    for (int r = 0; r < 10; r++) {
      if (r) {
        k0 += kW0;
        k1 += kW1;
      }
      const uint64_t p0 = (uint64_t)kM0 * x0, p1 = (uint64_t)kM1 * x2;
      const uint32_t y0 = (uint32_t)(p1 >> 32) ^ x1 ^ k0;
      const uint32_t y2 = (uint32_t)(p0 >> 32) ^ x3 ^ k1;
      x1 = (uint32_t)p1;
      x3 = (uint32_t)p0;
      x0 = y0;
      x2 = y2;
    }
    out[0] = x0;
    out[1] = x1;
    out[2] = x2;
    out[3] = x3;
  }
};

// The ten round keys of a Philox4x32-10 key (the key bumped by the Weyl
// increments before each round after the first): they depend on the seed
// only, so a kernel receives them precomputed (in its parameters, read as
// constant operands) instead of adding them again in every block.
struct PhiloxKeys {
  uint32_t k[20];  // round r: k[2r], k[2r + 1]
};
__host__ __device__ __forceinline__ PhiloxKeys philox_keys(unsigned long long seed) {
  PhiloxKeys s;
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  for (int r = 0; r < 10; r++) {
    s.k[2 * r] = k0;
    s.k[2 * r + 1] = k1;
    k0 += Philox4x32::kW0;
    k1 += Philox4x32::kW1;
  }
  return s;
}
// The same block as Philox4x32::block, with the round keys given.
__host__ __device__ __forceinline__ void philox_block_rk(const uint32_t ctr[4], const PhiloxKeys& ks,
                                                         uint32_t out[4]) {
  uint32_t x0 = ctr[0], x1 = ctr[1], x2 = ctr[2], x3 = ctr[3];
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint64_t p0 = (uint64_t)Philox4x32::kM0 * x0, p1 = (uint64_t)Philox4x32::kM1 * x2;
    const uint32_t y0 = (uint32_t)(p1 >> 32) ^ x1 ^ ks.k[2 * r];
    const uint32_t y2 = (uint32_t)(p0 >> 32) ^ x3 ^ ks.k[2 * r + 1];
    x1 = (uint32_t)p1;
    x3 = (uint32_t)p0;
    x0 = y0;
    x2 = y2;
  }
  out[0] = x0;
  out[1] = x1;
  out[2] = x2;
  out[3] = x3;
}

// The draws of one link update: counter (site, block, phase lo, phase hi),
// block = 0, 1, ... as the update consumes 32-bit words in order.  `phase`
// numbers the drawing phases of the lattice (6 per heat-bath or Metropolis
// pass), so no two updates share a counter.
struct PhiloxStream {
  const PhiloxKeys& ks;  // round keys of the key (the seed)
  uint32_t ctr[4];
  uint32_t b0, b1, b2, b3;
  int left;
  __device__ __forceinline__ PhiloxStream(const PhiloxKeys& keys, uint32_t site, unsigned long long phase)
      : ks(keys) {
    ctr[0] = site;
    ctr[1] = 0;
    ctr[2] = (uint32_t)phase;
    ctr[3] = (uint32_t)(phase >> 32);
    left = 0;
  }
  __device__ __forceinline__ uint32_t next() {
    if (left == 0) {
      uint32_t o[4];
      philox_block_rk(ctr, ks, o);
      ctr[1]++;
      b0 = o[0];
      b1 = o[1];
      b2 = o[2];
      b3 = o[3];
      left = 4;
    }
    const uint32_t v = b0;  // rotate through registers (no indexed local array)
    b0 = b1;
    b1 = b2;
    b2 = b3;
    left--;
    return v;
  }
  // The next whole block of four words (for a consumer whose draws come in
  // fours; a stream is read either this way or word by word, not both).
  __device__ __forceinline__ void block(uint32_t o[4]) {
    philox_block_rk(ctr, ks, o);
    ctr[1]++;
  }
  // (k + 1) / 2^24 for the top 24 bits k of a word: exact floats in (0, 1]
  __device__ __forceinline__ static float u24(uint32_t w) { return (float)((w >> 8) + 1u) * 5.9604644775390625e-8f; }
  __device__ __forceinline__ float uniform() { return u24(next()); }
  // (k + 1) / 2^53 from 53 bits of two words: exact doubles in (0, 1]
  __device__ __forceinline__ double uniform_double() {
    const uint64_t hi = next(), lo = next();
    return (double)(((hi << 21) | (lo >> 11)) + 1ull) * 1.1102230246251565e-16;
  }
};

}  // namespace qcd
