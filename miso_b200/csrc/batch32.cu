// Batched FP32 split-precision kernels: one persistent launch per pass over
// the tile list of all instances (1-D, 2-D or 3-D, any mix).  Per cell the
// arithmetic is the flux form used by the single-grid split kernels
// (s32_common.cuh): the 4th-order difference of each axis pairs its points
// symmetrically, the state is updated with two-sums, results are written
// with their ghost images.
#include "batch.h"
#include "s32_common.cuh"

namespace miso_b200 {
namespace b32 {

using namespace s32t;

struct TileState {
  BatchInst inst;
  int idx;
  int start;
};

__device__ __forceinline__ void load_tile(const BatchArgs &a, int t, TileState &ts) {
  if (threadIdx.x == 0) {
    const BatchTile bt = a.tiles[t];
    ts.idx = bt.inst;
    ts.start = bt.start;
    ts.inst = a.insts[bt.inst];
  }
  __syncthreads();
}

__device__ __forceinline__ long long decode(const Geom &g, long long lin, int &x0, int &x1,
                                            int &x2) {
  x2 = (int)(lin % g.n[2]);
  const long long r = lin / g.n[2];
  x1 = (int)(r % g.n[1]);
  x0 = (int)(r / g.n[1]);
  return (long long)(x0 + g.m[0]) * g.st[0] + (long long)(x1 + g.m[1]) * g.st[1] + x2 + g.m[2];
}

__device__ __forceinline__ void load_u(const FieldPtrs<const float> &s, long long base,
                                       long long c, float u[NF]) {
#pragma unroll
  for (int f = 0; f < NF; ++f) u[f] = __ldg(s.f[f] + base + c);
}

template <int D>
__device__ __forceinline__ void flux_at(const FieldPtrs<const float> &s, long long base,
                                        long long c, float gm1, float ch2, float F[NF]) {
  float u[NF];
  load_u(s, base, c, u);
  PrimF p;
  prim(u, gm1, p);
  flux_dir<D>(u, p, ch2, F);
}

template <int D>
__device__ __forceinline__ void diff_dir(const FieldPtrs<const float> &s, long long base,
                                         long long c, long long S, float w, float gm1, float ch2,
                                         float acc[NF]) {
  float A[NF], Fa[NF], Fb[NF];
  flux_at<D>(s, base, c - 2 * S, gm1, ch2, Fa);
  flux_at<D>(s, base, c + 2 * S, gm1, ch2, Fb);
#pragma unroll
  for (int f = 0; f < NF; ++f) A[f] = Fa[f] - Fb[f];
  flux_at<D>(s, base, c + S, gm1, ch2, Fa);
  flux_at<D>(s, base, c - S, gm1, ch2, Fb);
#pragma unroll
  for (int f = 0; f < NF; ++f) acc[f] += w * (A[f] + 8.0f * (Fa[f] - Fb[f]));
}

__global__ void __launch_bounds__(BATCH_TILE)
cfl_kernel(BatchArgs a, FieldPtrs<const float> hi) {
  __shared__ TileState ts;
  __shared__ float red[BATCH_TILE / 32];
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    load_tile(a, t, ts);
    const BatchInst &in = ts.inst;
    const long long lin = ts.start + threadIdx.x;
    float best = 1.e10f;
    if (lin < in.nint) {
      int x0, x1, x2;
      const long long c = decode(in.g, lin, x0, x1, x2);
      float u[NF];
      load_u(hi, in.base, c, u);
      float cs, vv, ca, ein;
      speeds(u, (float)in.gm, (float)(in.gm - 1.0), cs, vv, ca, ein);
      const float tv = cs + vv + ca;
      best = fminf(best, (float)in.cfl_dx / tv);
      if (!(u[RO] > 0.0f) || !(ein >= 0.0f) || !isfinite(tv)) atomicOr(a.err, ERRBIT_NONFINITE);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
      float b = red[0];
      for (int w = 1; w < BATCH_TILE / 32; ++w) b = fminf(b, red[w]);
      atomicMin(a.dtmin + ts.idx, __float_as_uint(b));
    }
    __syncthreads();
  }
}

// Runge-Kutta stage `stage` for every instance (see rk_flat_kernel).
__global__ void __launch_bounds__(BATCH_TILE)
rk_kernel(BatchArgs a, FieldPtrs<const float> prev, FieldPtrs<const float> u0,
          FieldPtrs<float> hi, FieldPtrs<float> lo, FieldPtrs<float> out, float *cc, int stage) {
  __shared__ TileState ts;
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    load_tile(a, t, ts);
    const BatchInst &in = ts.inst;
    const long long lin = ts.start + threadIdx.x;
    if (lin < in.nint) {
      const Geom &g = in.g;
      int x0, x1, x2;
      const long long c = decode(g, lin, x0, x1, x2);
      const StepScalars &sc = a.sc[ts.idx];
      const float ch2 = (float)sc.ch2, dt = (float)sc.dts[stage];
      const float decay = (float)sc.ph_decay[stage];
      const float gm1 = (float)(in.gm - 1.0);
      float D[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) D[f] = 0.0f;
      if (g.s[0]) diff_dir<0>(prev, in.base, c, g.st[0], (float)(g.dsi[0] * INV12), gm1, ch2, D);
      if (g.s[1]) diff_dir<1>(prev, in.base, c, g.st[1], (float)(g.dsi[1] * INV12), gm1, ch2, D);
      if (g.s[2]) diff_dir<2>(prev, in.base, c, 1, (float)(g.dsi[2] * INV12), gm1, ch2, D);
      const bool nb = near_boundary(g, x0, x1, x2);
      Img im;
      if (nb) make_img(g, x0, x1, x2, im);
      if (stage < 3) {
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          float v = __ldg(u0.f[f] + in.base + c) - dt * D[f];
          if (f == PH) v *= decay;
          store_cell(out.f[f] + in.base, c, nb, im, f, v);
        }
      } else {
        float sv[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          float *hp = hi.f[f] + in.base;
          float *lp = lo.f[f] + in.base;
          const float h = hp[c], l = lp[c];
          float e;
          if (f == PH) {
            float tt;
            two_sum(h, l - dt * D[f], sv[f], tt);
            const float pr = sv[f] * decay;
            const float pe = fmaf(sv[f], decay, -pr);
            two_sum(pr, pe + tt * decay, sv[f], e);
          } else {
            two_sum(h, l - dt * D[f], sv[f], e);
          }
          store_cell(hp, c, nb, im, f, sv[f]);
          store_cell(lp, c, nb, im, f, e);
        }
        float cs, vv, ca, ein;
        speeds(sv, (float)in.gm, gm1, cs, vv, ca, ein);
        store_cell(cc + in.base, c, nb, im, NF,
                   cs * (float)in.cs_fac + vv * (float)in.vv_fac + ca * (float)in.ca_fac);
      }
    }
    __syncthreads();
  }
}

// One viscosity sweep along `dir` for every instance.  An instance for which
// `dir` is degenerate gets an exact copy (every difference is zero).
__global__ void __launch_bounds__(BATCH_TILE)
av_kernel(BatchArgs a, FieldPtrs<const float> hi, FieldPtrs<const float> lo,
          FieldPtrs<float> hi2, FieldPtrs<float> lo2, const float *cc, int dir) {
  __shared__ TileState ts;
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    load_tile(a, t, ts);
    const BatchInst &in = ts.inst;
    const long long lin = ts.start + threadIdx.x;
    if (lin < in.nint) {
      const Geom &g = in.g;
      int x0, x1, x2;
      const long long c = decode(g, lin, x0, x1, x2);
      const long long S = g.st[dir] * g.s[dir];
      const float fac = (float)(g.dsi[dir] * a.sc[ts.idx].dt);
      const float ep = (float)in.ep, fh = (float)in.fh;
      float w[5][NW], hic[NF];
#pragma unroll
      for (int p = 0; p < 5; ++p) {
        float u[NF];
        load_u(hi, in.base, c + (p - 2) * S, u);
        limited_vars(u, w[p]);
        if (p == 2) {
#pragma unroll
          for (int f = 0; f < NF; ++f) hic[f] = u[f];
        }
      }
      const float ccl = __ldg(cc + in.base + c - S), ccc = __ldg(cc + in.base + c);
      const float ccr = __ldg(cc + in.base + c + S);
      const float cdw = 0.5f * (ccl + ccc), cup = 0.5f * (ccc + ccr);
      const bool nb = near_boundary(g, x0, x1, x2);
      Img im;
      if (nb) make_img(g, x0, x1, x2, im);
#pragma unroll
      for (int n = 0; n < NW; ++n) {
        const float d0 = dqq_eval(w[0][n], w[1][n], w[2][n], ep);
        const float d1 = dqq_eval(w[1][n], w[2][n], w[3][n], ep);
        const float d2 = dqq_eval(w[2][n], w[3][n], w[4][n], ep);
        const float fdw = flux_core(w[1][n], w[2][n], d0, d1, cdw, fh);
        const float fup = flux_core(w[2][n], w[3][n], d1, d2, cup, fh);
        const int f = field_of(n);
        float s, e;
        two_sum(hic[f], __ldg(lo.f[f] + in.base + c) - (fup - fdw) * fac, s, e);
        store_cell(hi2.f[f] + in.base, c, nb, im, f, s);
        store_cell(lo2.f[f] + in.base, c, nb, im, f, e);
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(BATCH_TILE)
fill_kernel(BatchArgs a, FieldPtrs<float> q, int nfields) {
  __shared__ TileState ts;
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    load_tile(a, t, ts);
    const BatchInst &in = ts.inst;
    const long long lin = ts.start + threadIdx.x;
    if (lin < in.nint) {
      const Geom &g = in.g;
      int x0, x1, x2;
      const long long c = decode(g, lin, x0, x1, x2);
      if (near_boundary(g, x0, x1, x2)) {
        Img im;
        make_img(g, x0, x1, x2, im);
        for (int f = 0; f < nfields; ++f) {
          float *p = q.f[f] + in.base;
          store_img(p, c, im, f, p[c]);
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace b32

void b32_cfl(const BatchArgs &a, const FieldPtrs<const float> &hi, int grid, cudaStream_t st) {
  b32::cfl_kernel<<<grid, BATCH_TILE, 0, st>>>(a, hi);
}
void b32_rk(const BatchArgs &a, const FieldPtrs<const float> &prev,
            const FieldPtrs<const float> &u0, const FieldPtrs<float> &hi,
            const FieldPtrs<float> &lo, const FieldPtrs<float> &out, float *cc, int stage,
            int grid, cudaStream_t st) {
  b32::rk_kernel<<<grid, BATCH_TILE, 0, st>>>(a, prev, u0, hi, lo, out, cc, stage);
}
void b32_av(const BatchArgs &a, const FieldPtrs<const float> &hi, const FieldPtrs<const float> &lo,
            const FieldPtrs<float> &hi2, const FieldPtrs<float> &lo2, const float *cc, int dir,
            int grid, cudaStream_t st) {
  b32::av_kernel<<<grid, BATCH_TILE, 0, st>>>(a, hi, lo, hi2, lo2, cc, dir);
}
void b32_fill(const BatchArgs &a, const FieldPtrs<float> &q, int nfields, int grid,
              cudaStream_t st) {
  b32::fill_kernel<<<grid, BATCH_TILE, 0, st>>>(a, q, nfields);
}

}  // namespace miso_b200
