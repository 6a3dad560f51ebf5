// Flat FP32 split-precision kernels for 3-D grids (internal to the library).
#pragma once

#include "s32_tiled.h"

namespace miso_b200 {

// One RK stage, one thread per cell; `prev` is the previous stage state.
void launch_s32_rk_flat(const CFSet &prev, const RkArgs &a, int stage, int grid, cudaStream_t st);
// One artificial-viscosity sweep (dir 0, 1, 2); the z sweep (dir 2) writes
// per-block CFL minima to a.partial[0..grid) when a.partial is set.
void launch_s32_av_flat(const AvArgs &a, int dir, int grid, cudaStream_t st);

}  // namespace miso_b200
