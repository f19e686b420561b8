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

struct RngStore {
  uint32_t* w;  // w[j * vh + id], j = 0..2 -> s1[j], j = 3..5 -> s2[j-3]
  int vh;

  __device__ __forceinline__ void load(int id, curandStateMRG32k3a_t* s) const {
    s->s1[0] = w[0 * (size_t)vh + id];
    s->s1[1] = w[1 * (size_t)vh + id];
    s->s1[2] = w[2 * (size_t)vh + id];
    s->s2[0] = w[3 * (size_t)vh + id];
    s->s2[1] = w[4 * (size_t)vh + id];
    s->s2[2] = w[5 * (size_t)vh + id];
    s->boxmuller_flag = 0;
    s->boxmuller_flag_double = 0;
    s->boxmuller_extra = 0.f;
    s->boxmuller_extra_double = 0.0;
  }
  __device__ __forceinline__ void store(int id, const curandStateMRG32k3a_t* s) const {
    w[0 * (size_t)vh + id] = s->s1[0];
    w[1 * (size_t)vh + id] = s->s1[1];
    w[2 * (size_t)vh + id] = s->s1[2];
    w[3 * (size_t)vh + id] = s->s2[0];
    w[4 * (size_t)vh + id] = s->s2[1];
    w[5 * (size_t)vh + id] = s->s2[2];
  }
};

}  // namespace qcd
