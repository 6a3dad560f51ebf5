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

// ---------------------------------------------------------------------------
// Block-tile kernels.  A tile is BATCH_TC x BATCH_TR interior cells in the
// instance's (C, R) axes at one P coordinate, or 1 x BATCH_TILE cells of a
// 1-D instance.  The tile's input state with a 2-cell halo along R and C is
// staged in shared memory once; flux vectors (RK) and limited variables
// (viscosity) along R and C are formed once per point there, so each cell
// reads its neighbours from shared memory.  The P axis of 3-D instances
// keeps per-cell neighbour evaluation from global memory.  These kernels
// write interior cells only; shell_fill_kernel then writes the ghost images
// of the near-boundary cells.
// ---------------------------------------------------------------------------
constexpr int TC = BATCH_TC, TR = BATCH_TR;
constexpr int U_PTS = (TC + 4) * (TR + 4) > BATCH_TILE + 4 ? (TC + 4) * (TR + 4) : BATCH_TILE + 4;
constexpr int FR_PTS = TC * (TR + 4) > BATCH_TILE + 4 ? TC * (TR + 4) : BATCH_TILE + 4;
constexpr int FC_PTS = (TC + 4) * TR;
constexpr int W_PTS = (TC + 4) * TR > U_PTS ? (TC + 4) * TR : U_PTS;

struct BlockGeo : TileGeo {
  BatchInst in;
};

// The tile's geometry and its instance's record, copied into shared memory
// by the CTA's threads in parallel (one word each).
__device__ __forceinline__ void load_block(const BatchArgs &a, int t, BlockGeo &bg) {
  constexpr int NT = (int)(sizeof(TileGeo) / 4), NI = (int)(sizeof(BatchInst) / 4);
  const int inst = __ldg(&a.btiles[t].idx);
  const int *st = reinterpret_cast<const int *>(a.btiles + t);
  const int *si = reinterpret_cast<const int *>(a.insts + inst);
  int *dt = reinterpret_cast<int *>(static_cast<TileGeo *>(&bg));
  int *di = reinterpret_cast<int *>(&bg.in);
  for (int w = threadIdx.x; w < NT + NI; w += blockDim.x) {
    if (w < NT)
      dt[w] = __ldg(st + w);
    else
      di[w - NT] = __ldg(si + w - NT);
  }
  __syncthreads();
}

// element index of tile point (c, r) in halo coordinates (c in [0, tc+2hc),
// r in [0, tr+4)), clamped into the instance's array
__device__ __forceinline__ long long block_point(const BlockGeo &bg, int c, int r) {
  const int ct = min(max(bg.oC + c - bg.hc, 0), bg.tC - 1);
  const int rt = min(max(bg.oR + r - 2, 0), bg.tR - 1);
  return bg.cell0 + (long long)(ct - bg.oC) * bg.sC + (long long)(rt - bg.oR) * bg.sR;
}

template <int D>
__device__ __forceinline__ void flux_pt(const float (&U)[NF][U_PTS], int m, float gm1, float ch2,
                                        float F[NF]) {
  float u[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) u[f] = U[f][m];
  PrimF p;
  prim(u, gm1, p);
  flux_dir<D>(u, p, ch2, F);
}

__device__ __forceinline__ void flux_pt_axis(const float (&U)[NF][U_PTS], int m, int axis,
                                             float gm1, float ch2, float F[NF]) {
  if (axis == 0)
    flux_pt<0>(U, m, gm1, ch2, F);
  else if (axis == 1)
    flux_pt<1>(U, m, gm1, ch2, F);
  else
    flux_pt<2>(U, m, gm1, ch2, F);
}

// 4th-order difference along the P axis (axis 0 of a 3-D instance) from
// global memory, as the per-cell kernels form it
__device__ __forceinline__ void diff_p(const FieldPtrs<const float> &s, long long base,
                                       long long c, long long S, float w, float gm1, float ch2,
                                       float acc[NF]) {
  diff_dir<0>(s, base, c, S, w, gm1, ch2, acc);
}

// Runge-Kutta stage `stage` for every instance (flux form; see rk_flat_kernel).
// LAST: the fourth stage (updates hi / lo and writes the speed), an
// instantiation of its own so the first three carry no lo words.
template <bool LAST>
__global__ void __launch_bounds__(BATCH_TILE, 3)
rk_block_kernel(BatchArgs a, FieldPtrs<const float> prev, FieldPtrs<const float> u0,
                FieldPtrs<float> hi, FieldPtrs<float> lo, FieldPtrs<float> out, float *cc,
                int stage) {
  __shared__ BlockGeo bg;
  __shared__ float U[NF][U_PTS];
  __shared__ float FR[NF][FR_PTS];
  __shared__ float FC[NF][FC_PTS];
  const int tid = threadIdx.x;
  for (int t = blockIdx.x; t < a.nbtiles; t += gridDim.x) {
    load_block(a, t, bg);
    const BatchInst &in = bg.in;
    const Geom &g = in.g;
    const int R = in.ax_r, C = in.ax_c, P = in.ax_p;
    const StepScalars &sc = a.sc[bg.idx];
    const float ch2 = (float)sc.ch2, dt = (float)sc.dts[stage];
    const float decay = (float)sc.ph_decay[stage];
    const float gm1 = (float)(in.gm - 1.0);
    const int W = bg.tr + 4, H = bg.tc + 2 * bg.hc;
    const int tcl = tid / bg.tr, trl = tid % bg.tr;
    const bool mine = tcl < bg.nc && trl < bg.nr;
    const long long c = bg.cell0 + (long long)tcl * bg.sC + (long long)trl * bg.sR;
    // centre values of this thread's cell, loaded before the staging waits
    float A0[NF], A1[NF];
    if (mine) {
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        if (!LAST) {
          A0[f] = __ldg(u0.f[f] + in.base + c);
        } else {
          A0[f] = hi.f[f][in.base + c];
          A1[f] = lo.f[f][in.base + c];
        }
      }
    }
    // 1. stage input with halos
    for (int m = tid; m < H * W; m += BATCH_TILE) {
      const long long e = in.base + block_point(bg, m / W, m % W);
#pragma unroll
      for (int f = 0; f < NF; ++f) U[f][m] = __ldg(prev.f[f] + e);
    }
    __syncthreads();
    // 2. flux vectors along R (tile rows, R halo) and C (tile columns, C halo)
    for (int m = tid; m < bg.tc * W; m += BATCH_TILE) {
      float F[NF];
      flux_pt_axis(U, m + bg.hc * W, R, gm1, ch2, F);
#pragma unroll
      for (int f = 0; f < NF; ++f) FR[f][m] = F[f];
    }
    if (C >= 0) {
      for (int m = tid; m < H * bg.tr; m += BATCH_TILE) {
        const int c = m / bg.tr, r = m % bg.tr;
        float F[NF];
        flux_pt_axis(U, c * W + r + 2, C, gm1, ch2, F);
#pragma unroll
        for (int f = 0; f < NF; ++f) FC[f][m] = F[f];
      }
    }
    __syncthreads();
    // 3. the tile's cells
    if (mine) {
      const float wR = (float)(g.dsi[R] * INV12);
      float D[NF];
      {
        const int m = tcl * W + trl;
#pragma unroll
        for (int f = 0; f < NF; ++f)
          D[f] = wR * ((FR[f][m] - FR[f][m + 4]) + 8.0f * (FR[f][m + 3] - FR[f][m + 1]));
      }
      if (C >= 0) {
        const float wC = (float)(g.dsi[C] * INV12);
        const int m = tcl * bg.tr + trl, S = bg.tr;
#pragma unroll
        for (int f = 0; f < NF; ++f)
          D[f] += wC * ((FC[f][m] - FC[f][m + 4 * S]) + 8.0f * (FC[f][m + 3 * S] - FC[f][m + S]));
      }
      if (P >= 0) diff_p(prev, in.base, c, bg.sP, (float)(g.dsi[P] * INV12), gm1, ch2, D);
      // interior only: the edge-tile fill writes the ghost images
      if (!LAST) {
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          float v = A0[f] - dt * D[f];
          if (f == PH) v *= decay;
          out.f[f][in.base + c] = v;
        }
      } else {
        float sv[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          float *hp = hi.f[f] + in.base;
          float *lp = lo.f[f] + in.base;
          const float h = A0[f], l = A1[f];
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
          hp[c] = sv[f];
          lp[c] = e;
        }
        float cs, vv, ca, ein;
        speeds(sv, (float)in.gm, gm1, cs, vv, ca, ein);
        cc[in.base + c] = cs * (float)in.cs_fac + vv * (float)in.vv_fac + ca * (float)in.ca_fac;
      }
    }
    __syncthreads();
  }
}

// One viscosity sweep along `dir` for every instance.  Along R or C the
// limited variables of the tile (halo 2 along the sweep) and the
// characteristic speed (halo 1) are staged in shared memory; along P (3-D)
// the cell reads its neighbours from global memory; an instance for which
// `dir` is degenerate gets its state copied (every difference is zero).
__global__ void __launch_bounds__(BATCH_TILE, 3)
av_block_kernel(BatchArgs a, FieldPtrs<const float> hi, FieldPtrs<const float> lo,
                FieldPtrs<float> hi2, FieldPtrs<float> lo2, const float *cc, int dir,
                int fuse_cfl) {
  __shared__ BlockGeo bg;
  __shared__ float Wv[NW][W_PTS];
  __shared__ float CCs[W_PTS];
  __shared__ float red[BATCH_TILE / 32];
  const int tid = threadIdx.x;
  for (int t = blockIdx.x; t < a.nbtiles; t += gridDim.x) {
    load_block(a, t, bg);
    const BatchInst &in = bg.in;
    const Geom &g = in.g;
    const int R = in.ax_r, C = in.ax_c;
    const bool along_r = dir == R, along_c = dir == C && C >= 0;
    const bool staged = along_r || along_c;
    // staged region: rows x cols with a 2-cell halo along the sweep axis
    const int rows = along_c ? bg.tc + 4 : bg.tc;
    const int cols = along_r ? bg.tr + 4 : bg.tr;
    const int tcl = tid / bg.tr, trl = tid % bg.tr;
    const bool mine = tcl < bg.nc && trl < bg.nr;
    const long long c = bg.cell0 + (long long)tcl * bg.sC + (long long)trl * bg.sR;
    float best = 1.e10f;
    float H0[NW], L0[NW];  // centre hi / lo in limited-variable order
    if (mine) {
#pragma unroll
      for (int n = 0; n < NW; ++n) {
        H0[n] = __ldg(hi.f[field_of(n)] + in.base + c);
        L0[n] = __ldg(lo.f[field_of(n)] + in.base + c);
      }
    }
    if (staged) {
      for (int m = tid; m < rows * cols; m += BATCH_TILE) {
        const int c = m / cols, r = m % cols;
        // halo coordinates: C halo only when sweeping C, R halo only along R
        const long long e = in.base + block_point(bg, c + (along_c ? 0 : bg.hc), r + (along_r ? 0 : 2));
        float u[NF], w[NW];
#pragma unroll
        for (int f = 0; f < NF; ++f) u[f] = __ldg(hi.f[f] + e);
        limited_vars(u, w);
#pragma unroll
        for (int n = 0; n < NW; ++n) Wv[n][m] = w[n];
        CCs[m] = __ldg(cc + e);
      }
    }
    __syncthreads();
    if (mine) {
      const float fac = (float)(g.dsi[dir] * a.sc[bg.idx].dt);
      const float ep = (float)in.ep, fh = (float)in.fh;
      float dF[NW];
      if (staged) {
        // centre at (tcl + 2, trl) along C or (tcl, trl + 2) along R
        const int S = along_r ? 1 : cols;
        const int m0 = along_r ? tcl * cols + trl + 2 : (tcl + 2) * cols + trl;
        const float cdw = 0.5f * (CCs[m0 - S] + CCs[m0]);
        const float cup = 0.5f * (CCs[m0] + CCs[m0 + S]);
#pragma unroll
        for (int n = 0; n < NW; ++n) {
          const float w0 = Wv[n][m0 - 2 * S], w1 = Wv[n][m0 - S], w2 = Wv[n][m0];
          const float w3 = Wv[n][m0 + S], w4 = Wv[n][m0 + 2 * S];
          const float d0 = dqq_eval(w0, w1, w2, ep);
          const float d1 = dqq_eval(w1, w2, w3, ep);
          const float d2 = dqq_eval(w2, w3, w4, ep);
          dF[n] = flux_core(w2, w3, d1, d2, cup, fh) - flux_core(w1, w2, d0, d1, cdw, fh);
        }
      } else if (g.s[dir]) {
        const long long S = g.st[dir];
        float w[5][NW];
#pragma unroll
        for (int p = 0; p < 5; ++p) {
          float u[NF];
          load_u(hi, in.base, c + (p - 2) * S, u);
          limited_vars(u, w[p]);
        }
        const float ccl = __ldg(cc + in.base + c - S), ccc = __ldg(cc + in.base + c);
        const float ccr = __ldg(cc + in.base + c + S);
        const float cdw = 0.5f * (ccl + ccc), cup = 0.5f * (ccc + ccr);
#pragma unroll
        for (int n = 0; n < NW; ++n) {
          const float d0 = dqq_eval(w[0][n], w[1][n], w[2][n], ep);
          const float d1 = dqq_eval(w[1][n], w[2][n], w[3][n], ep);
          const float d2 = dqq_eval(w[2][n], w[3][n], w[4][n], ep);
          dF[n] = flux_core(w[2][n], w[3][n], d1, d2, cup, fh) -
                  flux_core(w[1][n], w[2][n], d0, d1, cdw, fh);
        }
      } else {
#pragma unroll
        for (int n = 0; n < NW; ++n) dF[n] = 0.0f;
      }
      float sv[NF];
#pragma unroll
      for (int n = 0; n < NW; ++n) {
        const int f = field_of(n);
        float e;
        two_sum(H0[n], L0[n] - dF[n] * fac, sv[f], e);
        hi2.f[f][in.base + c] = sv[f];  // interior only (edge-tile fill follows)
        lo2.f[f][in.base + c] = e;
      }
      if (fuse_cfl) {
        // CFL candidate of the new state for the next step (as cfl_kernel)
        float cs, vv, ca, ein;
        speeds(sv, (float)in.gm, (float)(in.gm - 1.0), cs, vv, ca, ein);
        const float tv = cs + vv + ca;
        best = fminf(best, (float)in.cfl_dx / tv);
        if (!(sv[RO] > 0.0f) || !(ein >= 0.0f) || !isfinite(tv)) atomicOr(a.err, ERRBIT_NONFINITE);
      }
    }
    if (fuse_cfl) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, o));
      if ((tid & 31) == 0) red[tid >> 5] = best;
    }
    __syncthreads();
    if (fuse_cfl && tid == 0) {
      float b = red[0];
      for (int w = 1; w < BATCH_TILE / 32; ++w) b = fminf(b, red[w]);
      // non-negative floats order as their bit patterns
      atomicMin(a.dtmin + bg.idx, __float_as_uint(b));
    }
  }
}

// Ghost images of the listed near-boundary interior cells (instance, x0,
// x1, x2) of every instance, one cell per thread, for `nfields` arrays;
// ftag >= 0 selects one mirror-sign field for all of them (NF: never
// negated).  The cell's values are loaded before any image is stored.
__global__ void __launch_bounds__(BATCH_TILE)
shell_fill_kernel(BatchArgs a, const int4 *cells, int n, FieldPtrs<float> q, int nfields,
                  int ftag) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int4 w = __ldg(cells + e);
    const BatchInst &in = a.insts[w.x];
    const Geom &g = in.g;
    const long long base = in.base;
    const int c = cell_of(g, w.y, w.z, w.w);
    float v[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f)
      if (f < nfields) v[f] = q.f[f][base + c];
    Img im;
    make_img(g, w.y, w.z, w.w, im);
#pragma unroll
    for (int f = 0; f < NF; ++f)
      if (f < nfields) store_img(q.f[f] + base, (long long)c, im, ftag >= 0 ? ftag : f, v[f]);
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

TileGeo make_tile_geo(const BatchInst &in, int idx, const BlockTile &bt) {
  const Geom &g = in.g;
  const int R = in.ax_r, C = in.ax_c, P = in.ax_p;
  TileGeo tg{};
  tg.idx = idx;
  tg.tc = C >= 0 ? BATCH_TC : 1;
  tg.tr = C >= 0 ? BATCH_TR : BATCH_TILE;
  tg.hc = C >= 0 ? 2 : 0;
  tg.nr = g.n[R] - bt.r0 < tg.tr ? g.n[R] - bt.r0 : tg.tr;
  tg.nc = C >= 0 ? (g.n[C] - bt.c0 < tg.tc ? g.n[C] - bt.c0 : tg.tc) : 1;
  tg.sR = g.st[R];
  tg.sC = C >= 0 ? g.st[C] : 0;
  tg.sP = P >= 0 ? g.st[P] : 0;
  tg.oR = bt.r0 + g.m[R];
  tg.oC = C >= 0 ? bt.c0 + g.m[C] : 0;
  tg.tR = g.t[R];
  tg.tC = C >= 0 ? g.t[C] : 1;
  tg.x[0] = tg.x[1] = tg.x[2] = 0;
  tg.x[R] = bt.r0;
  if (C >= 0) tg.x[C] = bt.c0;
  if (P >= 0) tg.x[P] = bt.p;
  tg.cell0 = (P >= 0 ? (long long)(bt.p + g.m[P]) * tg.sP : 0) + (long long)tg.oC * tg.sC +
             (long long)tg.oR * tg.sR;
  return tg;
}

void b32_cfl(const BatchArgs &a, const FieldPtrs<const float> &hi, int grid, cudaStream_t st) {
  b32::cfl_kernel<<<grid, BATCH_TILE, 0, st>>>(a, hi);
}
void b32_rk(const BatchArgs &a, const FieldPtrs<const float> &prev,
            const FieldPtrs<const float> &u0, const FieldPtrs<float> &hi,
            const FieldPtrs<float> &lo, const FieldPtrs<float> &out, float *cc, int stage,
            int grid, cudaStream_t st) {
  if (stage == 3)
    b32::rk_block_kernel<true><<<grid, BATCH_TILE, 0, st>>>(a, prev, u0, hi, lo, out, cc, stage);
  else
    b32::rk_block_kernel<false><<<grid, BATCH_TILE, 0, st>>>(a, prev, u0, hi, lo, out, cc, stage);
}
void b32_av(const BatchArgs &a, const FieldPtrs<const float> &hi, const FieldPtrs<const float> &lo,
            const FieldPtrs<float> &hi2, const FieldPtrs<float> &lo2, const float *cc, int dir,
            int fuse_cfl, int grid, cudaStream_t st) {
  b32::av_block_kernel<<<grid, BATCH_TILE, 0, st>>>(a, hi, lo, hi2, lo2, cc, dir, fuse_cfl);
}
void b32_shell_fill(const BatchArgs &a, const int4 *cells, int n, const FieldPtrs<float> &q,
                    int nfields, int ftag, cudaStream_t st) {
  if (n <= 0) return;
  int grid = (n + BATCH_TILE - 1) / BATCH_TILE;
  if (grid > 4096) grid = 4096;
  b32::shell_fill_kernel<<<grid, BATCH_TILE, 0, st>>>(a, cells, n, q, nfields, ftag);
}
int b32_block_grid(int sms) {
  int rk = 0, av = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rk, b32::rk_block_kernel<true>, BATCH_TILE,
                                                    0) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&av, b32::av_block_kernel, BATCH_TILE, 0) !=
          cudaSuccess)
    return 2 * sms;
  const int per = rk < av ? rk : av;
  return (per > 0 ? per : 1) * sms;
}
void b32_fill(const BatchArgs &a, const FieldPtrs<float> &q, int nfields, int grid,
              cudaStream_t st) {
  b32::fill_kernel<<<grid, BATCH_TILE, 0, st>>>(a, q, nfields);
}

}  // namespace miso_b200
