// Per-site MRG32k3a streams, stored compactly.
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

}  // namespace qcd
