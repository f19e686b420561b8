// Host entry of the fused-pair schedule of the FP32 sweep (pairs.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include "lattice.cuh"

namespace qcd {

struct PhaseArgs;

// Tensor maps of one FP32 link store (5-D: component, y', x, t, class) with
// the boxes the pair kernels copy: NR rows of x (pairs y, x) or of t (pair t)
// by W y', one slice.
struct PairMaps {
  CUtensorMap rows_x, rows_t;
};

// Encode the maps of `store` (six classes of vh float4).
cudaError_t pair_encode_maps(const float4* store, const Geo& g, PairMaps* out);

// Streamed slices per CTA for a pair whose streamed direction has `ls`
// slices and whose perpendicular plane has `tiles` tiles: enough segments to
// give every SM several CTAs, at least 16 slices each (fewer only when the
// lattice is shorter).
int pair_segment(int ls, int tiles, int sms);

// One pass of the FP32 sweep as three fused pairs (y, x, t) with update
// `kind`: reads the link store `cur` (six planes of vh float4), writes every
// new link into `alt` (maps_cur / maps_alt: their tensor maps); `seg` streamed slices per CTA (0: pair_segment).  The
// caller swaps the two stores afterwards.  Returns the first launch error.
cudaError_t pair_pass32(const float4* cur, float4* alt, const PairMaps& maps_cur, const PairMaps& maps_alt, const Geo& g,
                        int bc, int kind, const PhaseArgs& a, int seg, int sms, cudaStream_t stream);

}  // namespace qcd
