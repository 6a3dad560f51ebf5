// Tiled FP32 split-precision kernels for 3-D grids (internal to the library).
#pragma once

#include "common.cuh"

namespace miso_b200 {

// The 9 field arrays of one state set.
using FSet = FieldPtrs<float>;
using CFSet = FieldPtrs<const float>;

// Arguments of one Runge-Kutta stage launch.
struct RkArgs {
  Geom g;
  CFSet u0;     // U^n (hi words), read at the cell itself
  FSet hi, lo;  // stage 3: state updated in place
  FSet out;     // stages 0-2: stage state written here
  float *cc;    // stage 3: characteristic speed of the new state
  const StepScalars *sc;
  unsigned int *err;
  float gm, gm1, cs_fac, vv_fac, ca_fac;
  int L;  // planes per work item along i
  int i0, i1;  // the planes [i0, i1) this launch finishes (a shard's interior / boundary part)
  int tiles_j, tiles_k, items;
  Source src;           // built-in source term (kind 0: none)
  const float *src_ro;  // density of the stage's argument state (the source's ro)
  long long wait_limit;  // bound (cycles) of the waits for each plane's copy
  // > 0 (pipelined stage only, a test of the timeout path): before its first
  // plane every thread waits, with this bound, on a barrier phase that
  // nothing completes, so the wait runs out and the timeout path is taken
  long long stall_limit;
};

// Arguments of one artificial-viscosity sweep launch.
struct AvArgs {
  Geom g;
  CFSet hi, lo;
  FSet hi2, lo2;
  const float *cc;
  const StepScalars *sc;
  unsigned int *err;
  float *partial;  // z sweep: per-block CFL minima of the new state (nullable)
  float ep, fh, gm, gm1, cfl_dx;
  int L;  // cells per work item along the sweep axis (x, y sweeps)
  int r0, r1;  // x / y sweeps: the cells [r0, r1) of the sweep axis this launch finishes
  // x sweep with the last RK update deferred into it: hi / lo hold U^n, and
  // the speed of U^{n+1} = (hi, lo) - dt_4 D goes to cc_out
  float *cc_out;
  float cs_fac, vv_fac, ca_fac;
  long long wait_limit;  // bound (cycles) of the consumer waits for each plane's copy
  // z sweep (nullable): per-block FP64 sums of the new state's ro, mx, my,
  // mz, et and ph^2 (6 per block), the monitors folded into the last sweep
  double *mon;
};

// Arrays whose interior shell gets its ghost images (s32_shell.cu); f[n] is
// the field index that selects the mirror sign (NF: never negated).
struct ShellArgs {
  float *p[2 * NF + 1];
  int f[2 * NF + 1];
  unsigned m[2 * NF + 1];  // per array: images to write, bit (m-1) for image mask m
                           // (1 = i, 2 = j, 4 = k, sums = edges and corners)
  int n;
  int slab;  // >= 0: every mask lies on the faces of this axis (enumerate its slabs only)
};
// image masks: the faces of one axis set (no edges or corners), or everything
constexpr unsigned SHELL_FACES_I = 1u << 0, SHELL_FACES_J = 1u << 1, SHELL_FACES_K = 1u << 3;
constexpr unsigned SHELL_FACES = SHELL_FACES_I | SHELL_FACES_J | SHELL_FACES_K;
constexpr unsigned SHELL_ALL = 0x7fu;
void launch_s32_shell(const Geom &g, const ShellArgs &a, int grid, cudaStream_t st);
long long s32_shell_cells(const Geom &g);  // interior cells within the margin of a face
long long s32_shell_count(const Geom &g, int slab);  // cells a shell launch visits

bool s32_tiled_supported(const Geom &g);
// 4-D tensor maps (k, j, i, field) over 9 arrays at `pitch_bytes`:
//   kind 0: RK plane tile (k 36, j 12, i 1, 9 fields)
//   kind 1: AV line (k 132, j 1, i 1, 9 fields)
int s32_make_tmap(const Geom &g, const float *field0, size_t pitch_bytes, int kind, void *tm_out);
//   kind 2: the z line sweep's wrap copies (k 8, j 1, i 1, 9 fields)
// 3-D tensor map of one array for the AV line (k kbox, j 1, i 1)
int s32_make_tmap_cc(const Geom &g, const float *cc, void *tm_out, int kbox = 132);
int s32_configure();
void s32_rk_items(const Geom &g, int L, int &tiles_j, int &tiles_k, int &items);
// work items of an RK stage launch over the planes [i0, i1)
int s32_rk_items_range(const Geom &g, int L, int i0, int i1);
void launch_s32_rk_tiled(const void *tm, const RkArgs &a, int stage, int grid, cudaStream_t st);
// Pipelined RK stage (s32_rk.cu): same tensor map and work items as the
// tiled kernel, one barrier per plane, packed FP32x2 differences.
int s32_rk_pipe_configure();
void launch_s32_rk_pipe(const void *tm, const RkArgs &a, int stage, int grid, cudaStream_t st);

// tm3: the characteristic speed (3-D map), or with `defer` (x sweep only)
// the deferred last RK stage's right-hand side D (4-D map, kind 1)
void launch_s32_av_line(const void *tm_hi, const void *tm_lo, const void *tm3, const AvArgs &a,
                        int dir, bool defer, int grid, cudaStream_t st);
void launch_s32_av_z(const AvArgs &a, int grid, cudaStream_t st);
// work items of the x (dir 0) / y (dir 1) line sweep over the cells [r0, r1)
// of its axis: k blocks x lines x chunks of L
int s32_av_line_items(const Geom &g, int dir, int L, int r0, int r1);

// z sweep as a streaming line (TMA rows of 132 k cells, wrap copies of 8 for
// periodic k faces); writes a.partial[blockIdx.x]
int s32_zline_per_sm();  // resident z line CTAs per SM (after s32_configure)
void launch_s32_av_zline(const void *tm_hi, const void *tm_lo, const void *tm_cc,
                         const void *tm_wh, const void *tm_wc, const AvArgs &a, int grid,
                         cudaStream_t st);
// y and z sweeps in one pass (y sweep variant 3): the z line sweep's rows
// and wrap copies (of hi, lo and the speed) with the y sweep run down each
// column; writes a.partial[blockIdx.x] and, with a.mon, the monitor sums
int s32_yz_per_sm();  // resident fused-sweep CTAs per SM (after s32_configure)
void launch_s32_av_yz(const void *tm_hi, const void *tm_lo, const void *tm_cc, const void *tm_wh,
                      const void *tm_wl, const void *tm_wc, const AvArgs &a, int grid,
                      cudaStream_t st);
// x / y sweep, one warp per 32-cell line segment marching along the sweep
// axis (s32_av.cu): no shared memory, no CTA barrier; interior-only writes
void launch_s32_av_march(const AvArgs &a, int dir, int grid, cudaStream_t st);

}  // namespace miso_b200
