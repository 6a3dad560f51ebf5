// Flat FP32 split-precision kernels for 3-D grids: one thread per cell,
// 32 x 8 (k, j) thread tiles so that k and j neighbours are served from L1,
// no shared-memory staging and no barriers, a small register footprint for
// high occupancy.  Flux vectors of the stencil points are recomputed per
// cell; each 4th-order difference pairs the points symmetrically,
// (F[-2] - F[+2]) + 8 (F[+1] - F[-1]), so a locally constant flux cancels
// exactly.  Results are written with their ghost images, the last RK stage
// writes the characteristic speed, and the z sweep folds the next step's CFL
// candidate into per-block minima.
//
// Physics as in fp32s_kernels.cu (flux form of mhd_integrator_host.hpp:
// 57-247; limiter.hpp:11-37; mhd_artificial_viscosity_host.hpp:51-348).
#include "common.cuh"
#include "s32_common.cuh"
#include "s32_flat.h"

namespace miso_b200 {
namespace s32f {

using namespace s32t;

constexpr int BK = 32, BJ = 8;

// Work item: a 32 x 8 (k, j) column tile over a chunk of L planes along i.
// Items are chunk-major, and the grid is one resident wave, so the CTAs in
// flight cover one band of planes; a thread marches down its column and the
// planes it touched a step earlier are still in L1.
struct Item {
  int j, k, i0, i1;
};

__device__ __forceinline__ int item_count(const Geom &g, int L) {
  return ((g.n[2] + BK - 1) / BK) * ((g.n[1] + BJ - 1) / BJ) * ((g.n[0] + L - 1) / L);
}

__device__ __forceinline__ Item item_of(const Geom &g, int it, int L) {
  const int tk = (g.n[2] + BK - 1) / BK, tj = (g.n[1] + BJ - 1) / BJ;
  const int per = tk * tj;
  const int ch = it / per, rem = it % per;
  Item r;
  r.j = (rem / tk) * BJ + (int)threadIdx.y;
  r.k = (rem % tk) * BK + (int)threadIdx.x;
  r.i0 = ch * L;
  r.i1 = min(g.n[0], r.i0 + L);
  return r;
}

__device__ __forceinline__ void load_state(const CFSet &s, int c, float u[NF]) {
#pragma unroll
  for (int f = 0; f < NF; ++f) u[f] = __ldg(s.f[f] + c);
}

template <int D>
__device__ __forceinline__ void flux_at(const CFSet &s, int c, float gm1, float ch2, float F[NF]) {
  float u[NF];
  load_state(s, c, u);
  PrimF p;
  prim(u, gm1, p);
  flux_dir<D>(u, p, ch2, F);
}

template <int D>
__device__ __forceinline__ void diff_dir(const CFSet &s, int c, int S, float w, float gm1,
                                         float ch2, float acc[NF]) {
  float A[NF], Fa[NF], Fb[NF];
  flux_at<D>(s, c - 2 * S, gm1, ch2, Fa);
  flux_at<D>(s, c + 2 * S, gm1, ch2, Fb);
#pragma unroll
  for (int f = 0; f < NF; ++f) A[f] = Fa[f] - Fb[f];
  flux_at<D>(s, c + S, gm1, ch2, Fa);
  flux_at<D>(s, c - S, gm1, ch2, Fb);
#pragma unroll
  for (int f = 0; f < NF; ++f) acc[f] += w * (A[f] + 8.0f * (Fa[f] - Fb[f]));
}

template <int STAGE>
__global__ void __launch_bounds__(BK * BJ, 3)
rk_flat_kernel(const CFSet prev, const RkArgs a) {
  const Geom &g = a.g;
  const float ch2 = (float)a.sc->ch2;
  const float dt = (float)a.sc->dts[STAGE];
  const float decay = (float)a.sc->ph_decay[STAGE];
  const float wx = (float)(g.dsi[0] * INV12);
  const float wy = (float)(g.dsi[1] * INV12);
  const float wz = (float)(g.dsi[2] * INV12);
  const int Si = (int)g.st[0], Sj = (int)g.st[1];
  const int items = item_count(g, a.L);
  for (int it = blockIdx.x; it < items; it += gridDim.x) {
    const Item itm = item_of(g, it, a.L);
    if (itm.j >= g.n[1] || itm.k >= g.n[2]) continue;
    const bool nbjk = itm.j < g.m[1] || itm.j >= g.n[1] - g.m[1] || itm.k < g.m[2] ||
                      itm.k >= g.n[2] - g.m[2];
    int cell = cell_of(g, itm.i0, itm.j, itm.k);
    for (int i = itm.i0; i < itm.i1; ++i, cell += Si) {
    float D[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) D[f] = 0.0f;
    diff_dir<2>(prev, cell, 1, wz, a.gm1, ch2, D);
    diff_dir<1>(prev, cell, Sj, wy, a.gm1, ch2, D);
    diff_dir<0>(prev, cell, Si, wx, a.gm1, ch2, D);
    const bool nb = nbjk || i < g.m[0] || i >= g.n[0] - g.m[0];
    Img im;
    if (nb) make_img(g, i, itm.j, itm.k, im);
    if (STAGE < 3) {
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        float v = __ldg(a.u0.f[f] + cell) - dt * D[f];
        if (f == PH) v *= decay;
        store_cell(a.out.f[f], cell, nb, im, f, v);
      }
    } else {
      float sv[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        float *hp = a.hi.f[f];
        float *lp = a.lo.f[f];
        const float h = hp[cell], l = lp[cell];
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
        store_cell(hp, cell, nb, im, f, sv[f]);
        store_cell(lp, cell, nb, im, f, e);
      }
      float cs, vv, ca, ein;
      speeds(sv, a.gm, a.gm1, cs, vv, ca, ein);
      store_cell(a.cc, cell, nb, im, NF, cs * a.cs_fac + vv * a.vv_fac + ca * a.ca_fac);
    }
    }
  }
}

// One artificial-viscosity sweep along DIR for one cell per thread.
template <int DIR>
__global__ void __launch_bounds__(BK * BJ, 3)
av_flat_kernel(const AvArgs a) {
  const Geom &g = a.g;
  const int S = (int)g.st[DIR];
  const float fac = (float)(g.dsi[DIR] * a.sc->dt);
  const int Si = (int)g.st[0];
  const int items = item_count(g, a.L);
  float best = 1.e10f;
  bool bad = false;
  for (int it = blockIdx.x; it < items; it += gridDim.x) {
    const Item itm = item_of(g, it, a.L);
    if (itm.j >= g.n[1] || itm.k >= g.n[2]) continue;
    const bool nbjk = itm.j < g.m[1] || itm.j >= g.n[1] - g.m[1] || itm.k < g.m[2] ||
                      itm.k >= g.n[2] - g.m[2];
    int cell = cell_of(g, itm.i0, itm.j, itm.k);
    for (int i = itm.i0; i < itm.i1; ++i, cell += Si) {
    float w[5][NW];
    float hic[NF];
#pragma unroll
    for (int p = 0; p < 5; ++p) {
      float u[NF];
      load_state(a.hi, cell + (p - 2) * S, u);
      limited_vars(u, w[p]);
      if (p == 2) {
#pragma unroll
        for (int f = 0; f < NF; ++f) hic[f] = u[f];
      }
    }
    const float ccl = __ldg(a.cc + cell - S), ccc = __ldg(a.cc + cell), ccr = __ldg(a.cc + cell + S);
    const float cdw = 0.5f * (ccl + ccc), cup = 0.5f * (ccc + ccr);
    const bool nb = nbjk || i < g.m[0] || i >= g.n[0] - g.m[0];
    Img im;
    if (nb) make_img(g, i, itm.j, itm.k, im);
    float s[NF];
#pragma unroll
    for (int n = 0; n < NW; ++n) {
      const float d0 = dqq_eval(w[0][n], w[1][n], w[2][n], a.ep);
      const float d1 = dqq_eval(w[1][n], w[2][n], w[3][n], a.ep);
      const float d2 = dqq_eval(w[2][n], w[3][n], w[4][n], a.ep);
      const float fdw = flux_core(w[1][n], w[2][n], d0, d1, cdw, a.fh);
      const float fup = flux_core(w[2][n], w[3][n], d1, d2, cup, a.fh);
      const int f = field_of(n);
      float e;
      two_sum(hic[f], __ldg(a.lo.f[f] + cell) - (fup - fdw) * fac, s[f], e);
      store_cell(a.hi2.f[f], cell, nb, im, f, s[f]);
      store_cell(a.lo2.f[f], cell, nb, im, f, e);
    }
    if (DIR == 2 && a.partial) {
      float cs, vv, ca, ein;
      speeds(s, a.gm, a.gm1, cs, vv, ca, ein);
      const float tv = cs + vv + ca;
      best = fminf(best, a.cfl_dx / tv);
      bad |= !(s[RO] > 0.0f) || !(ein >= 0.0f) || !isfinite(tv);
    }
    }
  }
  if (DIR == 2 && a.partial) {
    const int lane = (threadIdx.y * BK + threadIdx.x) & 31;
    const int wid = (threadIdx.y * BK + threadIdx.x) >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, o));
    __shared__ float red[BK * BJ / 32];
    if (lane == 0) red[wid] = best;
    if (bad) atomicOr(a.err, ERRBIT_NONFINITE);
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
      float b = red[0];
      for (int w2 = 1; w2 < BK * BJ / 32; ++w2) b = fminf(b, red[w2]);
      a.partial[blockIdx.x] = b;
    }
  }
}

}  // namespace s32f

void launch_s32_rk_flat(const CFSet &prev, const RkArgs &a, int stage, int grid,
                        cudaStream_t st) {
  const dim3 blk(s32f::BK, s32f::BJ);
  switch (stage) {
    case 0: s32f::rk_flat_kernel<0><<<grid, blk, 0, st>>>(prev, a); break;
    case 1: s32f::rk_flat_kernel<1><<<grid, blk, 0, st>>>(prev, a); break;
    case 2: s32f::rk_flat_kernel<2><<<grid, blk, 0, st>>>(prev, a); break;
    default: s32f::rk_flat_kernel<3><<<grid, blk, 0, st>>>(prev, a); break;
  }
}

void launch_s32_av_flat(const AvArgs &a, int dir, int grid, cudaStream_t st) {
  const dim3 blk(s32f::BK, s32f::BJ);
  switch (dir) {
    case 0: s32f::av_flat_kernel<0><<<grid, blk, 0, st>>>(a); break;
    case 1: s32f::av_flat_kernel<1><<<grid, blk, 0, st>>>(a); break;
    default: s32f::av_flat_kernel<2><<<grid, blk, 0, st>>>(a); break;
  }
}

}  // namespace miso_b200
