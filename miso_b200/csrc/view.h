// Views: the tiled 3-D FP32-split step of one grid over field arrays that
// another owner holds (internal to the library).  The batched solver runs
// each of its 3-D instances through a view, so that they take the same
// pipelined kernels -- TMA plane tiles, line sweeps -- as a single grid,
// each on its own stream (concurrent branches of the step's graph).
#pragma once

#include <cuda_runtime.h>

#include "../../include/miso_b200.h"
#include "common.cuh"

namespace miso_b200 {

// hi / lo: the two state sets, stg: the two stage sets, each set 9 arrays
// at one pitch of `pitch_bytes`; cc the characteristic speed; sc the
// instance's step scalars (its dt and error bits).  Returns ERR_STATE when
// the grid cannot take the tiled path.
int b200_view_create(const miso_b200_grid_desc &gd, const miso_b200_params &pp,
                     cudaStream_t stream, float *const hi[2][NF], float *const lo[2][NF],
                     float *const stg[2][NF], float *cc, size_t pitch_bytes, StepScalars *sc,
                     miso_b200_handle **out);
// One step (CFL, then the update) with the state in set `cur` (cur < 0: the
// set the view's last step, fill or upload left it in); returns the set that
// holds the new state.  A view keeps its own set: with the fused y and z
// pass a step swaps the sets twice, while the batch's other instances swap
// once per sweep.
int b200_view_step(miso_b200_handle *h, int cur, int *cur_out);
// The set that holds the view's current state, and its reset (after a
// graph capture, which records steps without leaving their effect).
int b200_view_cur(const miso_b200_handle *h);
void b200_view_set_cur(miso_b200_handle *h, int cur);
// The state in set `cur` was replaced: fill its ghosts, forget the CFL minima.
int b200_view_fill(miso_b200_handle *h, int cur);
// Bring the lo ghost images up to date (before a download).
int b200_view_fresh_lo(miso_b200_handle *h, int cur);
long long b200_view_launches(const miso_b200_handle *h);

}  // namespace miso_b200
