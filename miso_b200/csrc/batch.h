// Batched advance of many independent grids (internal to the library).
//
// All instances of a batch live in the same field arrays, one after the
// other; a table gives each instance its geometry, parameters and the
// element offset of its cell 0.  The interior cells of every instance are
// cut into tiles of BATCH_TILE consecutive cells; every pass of the step is
// ONE launch of a persistent grid that walks the tile list, so instances of
// any size share the GPU evenly.  Each instance keeps its own time step:
// the CFL pass reduces per tile and folds the tile minima per instance
// (segmented minimum).
#pragma once

#include "common.cuh"

namespace miso_b200 {

constexpr int BATCH_TILE = 256;  // cells per tile = threads per CTA

struct BatchInst {
  Geom g;
  long long base;  // element offset of this instance's cell 0 in every array
  long long nint;  // interior cells
  double gm, cfl_number, ep, fh, cs_fac, ca_fac, vv_fac;
  double min_dxyz, cfl_dx;
  // block-tile axes of the FP32 kernels: R = the last non-degenerate axis
  // (unit stride), C = the one before it, P = the first of three (-1: none)
  int ax_r, ax_c, ax_p;
  // 1: a 3-D FP32-split instance stepped through a view (view.h) on the
  // pipelined kernels; the batch-wide kernels and lists leave it out
  int view;
};

struct BatchTile {
  int inst;   // instance index
  int start;  // first interior linear index of the tile
};

// Block tile of the FP32 kernels: BATCH_TC x BATCH_TR interior cells in the
// (C, R) axes at one P coordinate (1 x BATCH_TILE for 1-D instances).
constexpr int BATCH_TC = 8, BATCH_TR = 32;
struct BlockTile {
  int inst, p, c0, r0;
};

// Geometry of one block tile, precomputed on the host so every thread of a
// CTA can pick it up with one parallel copy.
struct TileGeo {
  int idx;               // instance
  int tc, tr;            // tile extent (BATCH_TC x BATCH_TR, or 1 x BATCH_TILE)
  int nc, nr;            // cells of the tile inside the interior
  int hc;                // halo width along C (0 when the instance has no C axis)
  long long cell0;       // element index (instance-relative) of the tile's first cell
  long long sP, sC, sR;  // strides of the P, C, R axes (0 when absent)
  int oC, oR;            // total coordinate of the tile origin along C, R
  int tC, tR;            // total extent along C, R
  int x[3];              // interior coordinates of the tile origin per array axis
  int pad;
};
TileGeo make_tile_geo(const BatchInst &in, int idx, const BlockTile &bt);

// Row segment of a 1-D or 2-D instance for the warp kernels (batch32_rows.cu):
// rows [c0, c1) along C (0, 1 for 1-D) and cells from r0 along R.
struct RowItem {
  int inst, c0, c1, r0;
};
constexpr int ROW_OUT = 28;    // cells a warp finishes along R (shuffle stencils)
constexpr int ROW_CHUNK = 32;  // rows a warp marches along C

struct BatchArgs {
  const BatchInst *insts;
  const BatchTile *tiles;
  int ntiles;
  const TileGeo *btiles;  // FP32 block tiles
  int nbtiles;
  int count;
  StepScalars *sc;       // per instance
  unsigned int *dtmin;   // per instance: float bits of the running CFL minimum
  unsigned int *err;     // error bits (shared)
};

// FP64 (primitive state, bit-faithful per cell to the single-grid kernels)
void b64_cfl(const BatchArgs &a, const FieldPtrs<const double> &q, int grid, cudaStream_t st);
void b_finalize(const BatchArgs &a, cudaStream_t st);
void b64_rhs(const BatchArgs &a, const FieldPtrs<const double> &o,
             const FieldPtrs<const double> &ar, const FieldPtrs<double> &r, int stage, int grid,
             cudaStream_t st);
void b64_cc(const BatchArgs &a, const FieldPtrs<const double> &q, double *cc, int grid,
            cudaStream_t st);
void b64_av(const BatchArgs &a, const FieldPtrs<const double> &q, const FieldPtrs<double> &r,
            const double *cc, int dir, int grid, cudaStream_t st);
void b64_fill(const BatchArgs &a, const FieldPtrs<double> &q, int grid, cudaStream_t st);
// the sweep along the own axes of the 1-D / 2-D instances (b64_av leaves
// them out): R by warp shuffles over `rows`, C by a march over `rows_c`
void b64_av_rows(const BatchArgs &a, const RowItem *rows, int nrows, const RowItem *rows_c,
                 int nrows_c, const FieldPtrs<const double> &q, const FieldPtrs<double> &r,
                 const double *cc, int dir, int grid, cudaStream_t st);

// FP32 split (conserved hi/lo state)
void b32_cfl(const BatchArgs &a, const FieldPtrs<const float> &hi, int grid, cudaStream_t st);
void b32_rk(const BatchArgs &a, const FieldPtrs<const float> &prev,
            const FieldPtrs<const float> &u0, const FieldPtrs<float> &hi,
            const FieldPtrs<float> &lo, const FieldPtrs<float> &out, float *cc, int stage,
            int grid, cudaStream_t st);
// fuse_cfl: also fold the next step's CFL candidate of the new state into
// the per-instance minima (the last sweep of a step)
void b32_av(const BatchArgs &a, const FieldPtrs<const float> &hi, const FieldPtrs<const float> &lo,
            const FieldPtrs<float> &hi2, const FieldPtrs<float> &lo2, const float *cc, int dir,
            int fuse_cfl, int grid, cudaStream_t st);
void b32_fill(const BatchArgs &a, const FieldPtrs<float> &q, int nfields, int grid,
              cudaStream_t st);
// ghost images of the listed near-boundary cells (instance, x0, x1, x2)
void b32_shell_fill(const BatchArgs &a, const int4 *cells, int n, const FieldPtrs<float> &q,
                    int nfields, int ftag, cudaStream_t st);
// warp-per-row kernels for 1-D / 2-D instances
// `combo` (b32_row_combo) selects the axis pair of every item in `items`
int b32_row_combo(int ax_r, int ax_c);
constexpr int ROW_COMBOS = 6;
// defer (stage 3): write the stage's right-hand side D to `out` and leave
// the update to the step's first sweep
void b32_rk_rows(const BatchArgs &a, const RowItem *items, int n, int combo,
                 const FieldPtrs<const float> &prev, const FieldPtrs<const float> &u0,
                 const FieldPtrs<float> &hi, const FieldPtrs<float> &lo,
                 const FieldPtrs<float> &out, float *cc, int stage, int defer, int grid,
                 cudaStream_t st);
// d4.f[0] != nullptr: the first sweep of a step whose last update was
// deferred -- every cell read is U^{n+1} = (hi, lo) - dt_4 D, and the sweep
// writes the speed of U^{n+1} to cc_out for the later sweeps
void b32_av_rows_r(const BatchArgs &a, const RowItem *items, int n,
                   const FieldPtrs<const float> &hi, const FieldPtrs<const float> &lo,
                   const FieldPtrs<float> &hi2, const FieldPtrs<float> &lo2, const float *cc,
                   int dir, int fuse_cfl, const FieldPtrs<const float> &d4, float *cc_out,
                   int grid, cudaStream_t st);
void b32_av_rows_c(const BatchArgs &a, const RowItem *items, int n,
                   const FieldPtrs<const float> &hi, const FieldPtrs<const float> &lo,
                   const FieldPtrs<float> &hi2, const FieldPtrs<float> &lo2, const float *cc,
                   int dir, int fuse_cfl, const FieldPtrs<const float> &d4, float *cc_out,
                   int grid, cudaStream_t st);
// resident CTAs of the block-tile kernels on `sms` SMs (their persistent grid)
int b32_block_grid(int sms);

}  // namespace miso_b200
