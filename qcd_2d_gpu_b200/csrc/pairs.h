// Host entry of the fused-pair schedule of the FP32 sweep (pairs.cu).
#pragma once
#include <cuda_runtime.h>
#include "lattice.cuh"

namespace qcd {

struct PhaseArgs;

// Streamed slices per CTA for a pair whose streamed direction has `ls`
// slices and whose perpendicular plane has `tiles` tiles: enough segments to
// give every SM several CTAs, at least 16 slices each (fewer only when the
// lattice is shorter).
int pair_segment(int ls, int tiles, int sms);

// One pass of the FP32 sweep as three fused pairs (y, x, t) with update
// `kind`: reads the link store `cur` (six planes of vh float4), writes every
// new link into `alt`; `seg` streamed slices per CTA (0: pair_segment).  The
// caller swaps the two stores afterwards.  Returns the first launch error.
cudaError_t pair_pass32(const float4* cur, float4* alt, const Geo& g, int bc, int kind, const PhaseArgs& a, int seg,
                        int sms, cudaStream_t stream);

}  // namespace qcd
