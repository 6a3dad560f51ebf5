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

// The viscosity update of cell c from its limited quantities w (as
// av_load_w forms them) and the flux difference dF: av_cell's expressions in
// its operand order, so every kernel that reaches them gives its bits.
__device__ __forceinline__ void av_finish(const FieldPtrs<const double> &q, long long c,
                                          const double w[NF], const double dF[NF], double dsi,
                                          double dt, double out[NF]) {
  const double ro_c = w[0];
  const double ro = ro_c - dF[0] * dsi * dt;
  double v[3], b[3];
#pragma unroll
  for (int e = 0; e < 3; ++e) v[e] = (w[1 + e] - dF[1 + e] * dsi * dt) / ro;
#pragma unroll
  for (int e = 0; e < 3; ++e) b[e] = w[4 + e] - dF[4 + e] * dsi * dt;
  const double ph = w[7] - dF[7] * dsi * dt;
  const double ei_c = __ldg(q.f[EI] + c);
  const double vx_c = __ldg(q.f[VX] + c), vy_c = __ldg(q.f[VY] + c), vz_c = __ldg(q.f[VZ] + c);
  const double Et = ro_c * ei_c + 0.5 * ro_c * (vx_c * vx_c + vy_c * vy_c + vz_c * vz_c) +
                    PII8 * (w[4] * w[4] + w[5] * w[5] + w[6] * w[6]);
  const double ei = (Et - dF[8] * dsi * dt - 0.5 * ro * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) -
                     PII8 * (b[0] * b[0] + b[1] * b[1] + b[2] * b[2])) / ro;
  out[RO] = ro;
  out[VX] = v[0];
  out[VY] = v[1];
  out[VZ] = v[2];
  out[BX] = b[0];
  out[BY] = b[1];
  out[BZ] = b[2];
  out[EI] = ei;
  out[PH] = ph;
}

// Viscosity sweep `dir` on the tile list: a 3-D instance per cell (av_cell);
// an instance degenerate along dir in closed form -- its five stencil points
// are the cell itself, so the two face fluxes come from identical arguments
// and their difference is +0 (finite state), and av_cell reduces to the
// conversion to conserved quantities and back (the reference's round-off
// step) -- and the own axes of a 1-D / 2-D instance are left to the row
// kernels below.
__global__ void __launch_bounds__(HALF, 3)
av_kernel(BatchArgs a, FieldPtrs<const double> q, FieldPtrs<double> r, const double *cc,
          int dir) {
  for (int t2 = blockIdx.x; t2 < 2 * a.ntiles; t2 += gridDim.x) {
    const int t = t2 >> 1;
    int idx, start;
    const BatchInst &in = tile_of(a, t, idx, start);
    const bool degen = !in.g.s[dir];
    if (!degen && in.ax_p < 0) continue;  // a 1-D / 2-D instance's own axis: rows
    const int lin = start + (t2 & 1) * HALF + threadIdx.x;
    if (lin < in.nint) {
      const Geom &g = in.g;
      int x0, x1, x2;
      const long long c = decode(g, lin, x0, x1, x2);
      double out[NF];
      if (degen) {
        double w[NF], ccv;
        const FieldPtrs<const double> qs = shift(q, in.base);
        fp64::av_load_w(qs, cc + in.base, c, w, ccv);
        const double dF[NF] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        av_finish(qs, c, w, dF, g.dsi[dir], a.sc[idx].dt, out);
      } else {
        fp64::av_cell(g, shift(q, in.base), cc + in.base, c, dir, a.sc[idx].dt, in.ep, in.fh,
                      out);
      }
      const bool nb = near_boundary(g, x0, x1, x2);
      Img im;
      if (nb) make_img(g, x0, x1, x2, im);
#pragma unroll
      for (int f = 0; f < NF; ++f) store_cell(r.f[f] + in.base, c, nb, im, f, out[f]);
    }
  }
}

// Cell of a 1-D / 2-D instance at R coordinate r (ghosts included) and C
// coordinate c; the other axes are degenerate.
__device__ __forceinline__ long long row_cell(const BatchInst &in, int r, int c, int &x0, int &x1,
                                              int &x2) {
  int x[3] = {0, 0, 0};
  x[in.ax_r] = r;
  if (in.ax_c >= 0) x[in.ax_c] = c;
  x0 = x[0];
  x1 = x[1];
  x2 = x[2];
  const Geom &g = in.g;
  return (long long)(x0 + g.m[0]) * g.st[0] + (long long)(x1 + g.m[1]) * g.st[1] + x2 + g.m[2];
}

// Sweep along R, the unit-stride axis of a 1-D / 2-D instance: a warp loads
// 32 consecutive cells of a row (ghost cells at the ends, whose images the
// previous pass wrote) and updates the inner 28; each lane forms the slope
// and the upper face flux of its own cell once and takes its neighbours' by
// warp shuffles -- the per-cell sweep's dqq_eval and flux_core arguments, so
// every output is av_cell's bit for bit.  Row items: C rows [c0, c1) from
// R cell r0.
__global__ void __launch_bounds__(128)
av_rows_r_kernel(BatchArgs a, const RowItem *__restrict__ items, int n,
                 FieldPtrs<const double> q, FieldPtrs<double> r, const double *cc, int dir) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int wi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; wi < n; wi += nw) {
    const RowItem it = items[wi];
    const BatchInst &in = a.insts[it.inst];
    if (in.ax_r != dir) continue;
    const Geom &g = in.g;
    const FieldPtrs<const double> qs = shift(q, in.base);
    const double *ccs = cc + in.base;
    const double dt = a.sc[it.inst].dt, dsi = g.dsi[dir], ep = in.ep, fh = in.fh;
    const int nr = g.n[dir];
    const int rr = it.r0 + lane - 2;  // -2 .. nr+1 read
    const int rc = min(rr, nr + 1);
    for (int c = it.c0; c < it.c1; ++c) {
      int x0, x1, x2;
      const long long cell = row_cell(in, rc, c, x0, x1, x2);
      double w[NF], ccv;
      fp64::av_load_w(qs, ccs, cell, w, ccv);
      const double cc_up = __shfl_down_sync(0xffffffffu, ccv, 1);
      double dF[NF];
#pragma unroll
      for (int m = 0; m < NF; ++m) {
        const double wm = __shfl_up_sync(0xffffffffu, w[m], 1);
        const double wp = __shfl_down_sync(0xffffffffu, w[m], 1);
        const double dq = fp64::dqq_eval(wm, w[m], wp, ep);
        const double dq_up = __shfl_down_sync(0xffffffffu, dq, 1);
        const double Fup = fp64::flux_core(w[m], wp, dq, dq_up, 0.5 * (ccv + cc_up), fh);
        const double Fdw = __shfl_up_sync(0xffffffffu, Fup, 1);
        dF[m] = Fup - Fdw;
      }
      if (lane >= 2 && lane < 30 && rr < nr) {
        double out[NF];
        av_finish(qs, cell, w, dF, dsi, dt, out);
        const bool nb = near_boundary(g, x0, x1, x2);
        Img im;
        if (nb) make_img(g, x0, x1, x2, im);
#pragma unroll
        for (int f = 0; f < NF; ++f) store_cell(r.f[f] + in.base, cell, nb, im, f, out[f]);
      }
    }
  }
}

// Sweep along C, the other axis of a 2-D instance: a warp on 32 consecutive
// R cells marches along C over the rows [c0, c1) (two ghost rows at each
// end read as they lie), carrying the slopes and the lower face flux from
// cell to cell, so each is formed once -- av_cell's arguments again.
__global__ void __launch_bounds__(128)
av_rows_c_kernel(BatchArgs a, const RowItem *__restrict__ items, int n,
                 FieldPtrs<const double> q, FieldPtrs<double> r, const double *cc, int dir) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int wi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; wi < n; wi += nw) {
    const RowItem it = items[wi];
    const BatchInst &in = a.insts[it.inst];
    if (in.ax_c != dir) continue;
    const Geom &g = in.g;
    const FieldPtrs<const double> qs = shift(q, in.base);
    const double *ccs = cc + in.base;
    const double dt = a.sc[it.inst].dt, dsi = g.dsi[dir], ep = in.ep, fh = in.fh;
    const int nr = g.n[in.ax_r];
    const int rl = it.r0 + lane;
    const bool active = rl < nr;
    const int rcl = min(rl, nr - 1);  // idle lanes shadow the last cell; their values go unused
    const long long sC = g.st[dir];
    int x0, x1, x2;
    const long long base = row_cell(in, rcl, 0, x0, x1, x2);  // cell at C = 0
    double w0[NF], w1[NF], dq0[NF], F0[NF], cc0, cc1;
    {
      double wa[NF], wb[NF], cca, ccb;
      fp64::av_load_w(qs, ccs, base + (long long)(it.c0 - 2) * sC, wa, cca);
      fp64::av_load_w(qs, ccs, base + (long long)(it.c0 - 1) * sC, wb, ccb);
      fp64::av_load_w(qs, ccs, base + (long long)it.c0 * sC, w0, cc0);
      fp64::av_load_w(qs, ccs, base + (long long)(it.c0 + 1) * sC, w1, cc1);
#pragma unroll
      for (int m = 0; m < NF; ++m) {
        const double dqm = fp64::dqq_eval(wa[m], wb[m], w0[m], ep);
        dq0[m] = fp64::dqq_eval(wb[m], w0[m], w1[m], ep);
        F0[m] = fp64::flux_core(wb[m], w0[m], dqm, dq0[m], 0.5 * (ccb + cc0), fh);
      }
    }
    for (int c = it.c0; c < it.c1; ++c) {
      const long long cell = base + (long long)c * sC;
      double wp[NF], ccp;
      fp64::av_load_w(qs, ccs, cell + 2 * sC, wp, ccp);
      double dF[NF];
#pragma unroll
      for (int m = 0; m < NF; ++m) {
        const double dq1 = fp64::dqq_eval(w0[m], w1[m], wp[m], ep);
        const double F1 = fp64::flux_core(w0[m], w1[m], dq0[m], dq1, 0.5 * (cc0 + cc1), fh);
        dF[m] = F1 - F0[m];
        F0[m] = F1;
        dq0[m] = dq1;
      }
      if (active) {
        double out[NF];
        av_finish(qs, cell, w0, dF, dsi, dt, out);
        int y[3] = {x0, x1, x2};
        y[dir] = c;
        const bool nb = near_boundary(g, y[0], y[1], y[2]);
        Img im;
        if (nb) make_img(g, y[0], y[1], y[2], im);
#pragma unroll
        for (int f = 0; f < NF; ++f) store_cell(r.f[f] + in.base, cell, nb, im, f, out[f]);
      }
#pragma unroll
      for (int m = 0; m < NF; ++m) {
        w0[m] = w1[m];
        w1[m] = wp[m];
      }
      cc0 = cc1;
      cc1 = ccp;
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
void b64_av_rows(const BatchArgs &a, const RowItem *rows, int nrows, const RowItem *rows_c,
                 int nrows_c, const FieldPtrs<const double> &q, const FieldPtrs<double> &r,
                 const double *cc, int dir, int grid, cudaStream_t st) {
  if (nrows > 0) b64::av_rows_r_kernel<<<grid, 128, 0, st>>>(a, rows, nrows, q, r, cc, dir);
  if (nrows_c > 0) b64::av_rows_c_kernel<<<grid, 128, 0, st>>>(a, rows_c, nrows_c, q, r, cc, dir);
}
void b64_fill(const BatchArgs &a, const FieldPtrs<double> &q, int grid, cudaStream_t st) {
  b64::fill_kernel<<<grid, BATCH_TILE, 0, st>>>(a, q);
}

}  // namespace miso_b200
