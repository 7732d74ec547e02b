// Auto-tuner of ALGO_INTERP_LORENZO (reference api/impl/FalconsAlgoInterp.hpp:273-544).
#pragma once
#include "../../include/falcons_b200.h"
#include "context.cuh"

namespace fb2 {

// Resolves the interpolation settings for ALGO_INTERP_LORENZO on the device-resident field d_x
// and sets c.cmprAlgo = ALGO_INTERP.  Sampled blocks are cut and trial-compressed with the
// tuning sweeps on the device; candidates are ranked by the zstd size of their codes and
// unpredictable values, exactly as the reference ranks them.  max_abs is the field's largest
// |value| (InterpParams::max_abs).
template <class T>
void tune_interp(Context &ctx, falcons_config &c, const T *d_x, cudaStream_t st, double max_abs);

}  // namespace fb2
