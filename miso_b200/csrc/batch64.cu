// Batched FP64 kernels: one persistent launch per pass over the tile list of
// all instances.  Compiled with --fmad=false; each cell goes through the
// same per-cell functions as the single-grid FP64 kernels (fp64_device.cuh),
// so every instance evolves bit for bit as it would alone.  Results are
// written with their ghost images (images.cuh).
#include "batch.h"
#include "fp64_device.cuh"
#include "images.cuh"

namespace miso_b200 {
namespace b64 {

// A tile's instance record, read by every thread of the CTA from the same
// addresses (one L1 broadcast): no shared copy and no barrier per tile.
__device__ __forceinline__ const BatchInst &tile_of(const BatchArgs &a, int t, int &idx,
                                                    int &start) {
  const BatchTile bt = a.tiles[t];
  idx = bt.inst;
  start = bt.start;
  return a.insts[bt.inst];
}

// interior coordinates and local cell index of linear interior index lin
// (32-bit: an instance holds fewer than 2^31 interior cells, as its tiles'
// int start indices do)
__device__ __forceinline__ long long decode(const Geom &g, int lin, int &x0, int &x1, int &x2) {
  x2 = lin % g.n[2];
  const int r = lin / g.n[2];
  x1 = r % g.n[1];
  x0 = r / g.n[1];
  return (long long)(x0 + g.m[0]) * g.st[0] + (long long)(x1 + g.m[1]) * g.st[1] + x2 + g.m[2];
}

template <typename P>
__device__ __forceinline__ P shift(const P &p, long long base) {
  P r;
#pragma unroll
  for (int f = 0; f < NF; ++f) r.f[f] = p.f[f] + base;
  return r;
}

__global__ void __launch_bounds__(BATCH_TILE)
cfl_kernel(BatchArgs a, FieldPtrs<const double> q) {
  __shared__ float red[BATCH_TILE / 32];
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    int idx, start;
    const BatchInst &in = tile_of(a, t, idx, start);
    const int lin = start + threadIdx.x;
    float best = 1.e10f;
    if (lin < in.nint) {
      int x0, x1, x2;
      const long long c = decode(in.g, lin, x0, x1, x2);
      bool bad;
      best = fminf(best, fp64::cfl_cell(shift(q, in.base), c, in.gm, in.cfl_dx, bad));
      if (bad) atomicOr(a.err, ERRBIT_NONFINITE);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
      float b = red[0];
      for (int w = 1; w < BATCH_TILE / 32; ++w) b = fminf(b, red[w]);
      // non-negative floats order as their bit patterns
      atomicMin(a.dtmin + idx, __float_as_uint(b));
    }
    __syncthreads();
  }
}

// Per instance: time step from the folded minimum and the step scalars
// (divb_parameters_set, mhd_integrator_host.hpp:337-341; stage factors,
// 258-277); the running minimum is reset for the next CFL pass.
__global__ void finalize_kernel(BatchArgs a) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < a.count; n += gridDim.x * blockDim.x) {
    const BatchInst &in = a.insts[n];
    if (in.view) continue;  // its view keeps its own step scalars
    const double dt = (double)__uint_as_float(a.dtmin[n]);
    StepScalars &sc = a.sc[n];
    sc.dt = dt;
    sc.dts[0] = dt / 4.0;
    sc.dts[1] = dt / 3.0;
    sc.dts[2] = dt / 2.0;
    sc.dts[3] = dt;
    const double ch = 0.8 * in.cfl_number * in.min_dxyz / dt;
    sc.ch2 = ch * ch;
    sc.tau = 2.0 * dt;
    for (int s = 0; s < 4; ++s) sc.ph_decay[s] = exp(-sc.dts[s] / sc.tau);
    a.dtmin[n] = __float_as_uint(1.e10f);
  }
}

// The right-hand side and viscosity kernels run 128-thread CTAs, each thread
// on two cells of a 256-cell tile: at their ~170 registers three CTAs (12
// warps) fit an SM, as for the single grid's per-cell kernels, where one
// 256-thread CTA (8 warps) did.
constexpr int HALF = BATCH_TILE / 2;

__global__ void __launch_bounds__(HALF, 3)
rhs_kernel(BatchArgs a, FieldPtrs<const double> o, FieldPtrs<const double> ar,
           FieldPtrs<double> r, int stage) {
  for (int t2 = blockIdx.x; t2 < 2 * a.ntiles; t2 += gridDim.x) {
    const int t = t2 >> 1;
    int idx, start;
    const BatchInst &in = tile_of(a, t, idx, start);
    const int lin = start + (t2 & 1) * HALF + threadIdx.x;
    if (lin < in.nint) {
      const Geom &g = in.g;
      int x0, x1, x2;
      const long long c = decode(g, lin, x0, x1, x2);
      const StepScalars &sc = a.sc[idx];
      double out[NF];
      fp64::rhs_cell(g, shift(o, in.base), shift(ar, in.base), c, sc.dts[stage], sc.ch2,
                     sc.ph_decay[stage], in.gm, out);
      const bool nb = near_boundary(g, x0, x1, x2);
      Img im;
      if (nb) make_img(g, x0, x1, x2, im);
#pragma unroll
      for (int f = 0; f < NF; ++f) store_cell(r.f[f] + in.base, c, nb, im, f, out[f]);
    }
  }
}

__global__ void __launch_bounds__(BATCH_TILE)
cc_kernel(BatchArgs a, FieldPtrs<const double> q, double *cc) {
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    int idx, start;
    const BatchInst &in = tile_of(a, t, idx, start);
    const int lin = start + threadIdx.x;
    if (lin < in.nint) {
      const Geom &g = in.g;
      int x0, x1, x2;
      const long long c = decode(g, lin, x0, x1, x2);
      const double v = fp64::cc_cell(shift(q, in.base), c, in.gm, in.cs_fac, in.vv_fac, in.ca_fac);
      const bool nb = near_boundary(g, x0, x1, x2);
      Img im;
      if (nb) make_img(g, x0, x1, x2, im);
      store_cell(cc + in.base, c, nb, im, NF, v);
    }
  }
}

__global__ void __launch_bounds__(HALF, 3)
av_kernel(BatchArgs a, FieldPtrs<const double> q, FieldPtrs<double> r, const double *cc,
          int dir) {
  for (int t2 = blockIdx.x; t2 < 2 * a.ntiles; t2 += gridDim.x) {
    const int t = t2 >> 1;
    int idx, start;
    const BatchInst &in = tile_of(a, t, idx, start);
    const int lin = start + (t2 & 1) * HALF + threadIdx.x;
    if (lin < in.nint) {
      const Geom &g = in.g;
      int x0, x1, x2;
      const long long c = decode(g, lin, x0, x1, x2);
      double out[NF];
      fp64::av_cell(g, shift(q, in.base), cc + in.base, c, dir, a.sc[idx].dt, in.ep, in.fh,
                    out);
      const bool nb = near_boundary(g, x0, x1, x2);
      Img im;
      if (nb) make_img(g, x0, x1, x2, im);
#pragma unroll
      for (int f = 0; f < NF; ++f) store_cell(r.f[f] + in.base, c, nb, im, f, out[f]);
    }
  }
}

// Write the ghost images of every interior value (after an upload).
__global__ void __launch_bounds__(BATCH_TILE)
fill_kernel(BatchArgs a, FieldPtrs<double> q) {
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    int idx, start;
    const BatchInst &in = tile_of(a, t, idx, start);
    const int lin = start + threadIdx.x;
    if (lin < in.nint) {
      const Geom &g = in.g;
      int x0, x1, x2;
      const long long c = decode(g, lin, x0, x1, x2);
      if (near_boundary(g, x0, x1, x2)) {
        Img im;
        make_img(g, x0, x1, x2, im);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          double *p = q.f[f] + in.base;
          store_img(p, c, im, f, p[c]);
        }
      }
    }
  }
}

}  // namespace b64

void b64_cfl(const BatchArgs &a, const FieldPtrs<const double> &q, int grid, cudaStream_t st) {
  b64::cfl_kernel<<<grid, BATCH_TILE, 0, st>>>(a, q);
}
void b_finalize(const BatchArgs &a, cudaStream_t st) {
  b64::finalize_kernel<<<(a.count + 255) / 256, 256, 0, st>>>(a);
}
void b64_rhs(const BatchArgs &a, const FieldPtrs<const double> &o,
             const FieldPtrs<const double> &ar, const FieldPtrs<double> &r, int stage, int grid,
             cudaStream_t st) {
  b64::rhs_kernel<<<2 * grid, b64::HALF, 0, st>>>(a, o, ar, r, stage);
}
void b64_cc(const BatchArgs &a, const FieldPtrs<const double> &q, double *cc, int grid,
            cudaStream_t st) {
  b64::cc_kernel<<<grid, BATCH_TILE, 0, st>>>(a, q, cc);
}
void b64_av(const BatchArgs &a, const FieldPtrs<const double> &q, const FieldPtrs<double> &r,
            const double *cc, int dir, int grid, cudaStream_t st) {
  b64::av_kernel<<<2 * grid, b64::HALF, 0, st>>>(a, q, r, cc, dir);
}
void b64_fill(const BatchArgs &a, const FieldPtrs<double> &q, int grid, cudaStream_t st) {
  b64::fill_kernel<<<grid, BATCH_TILE, 0, st>>>(a, q);
}

}  // namespace miso_b200
