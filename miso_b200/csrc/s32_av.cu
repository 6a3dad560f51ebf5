// FP32 split-precision viscosity sweep along x or y for 3-D grids: one
// warp per line segment, marching along the sweep axis, with no shared
// memory, no TMA and no CTA barrier.
//
// A warp owns 32 consecutive k cells of one line (fixed j for the x sweep,
// fixed i for the y sweep) and marches along the sweep axis over a chunk of
// planes.  Per plane each lane loads the conserved hi words and the
// characteristic speed of its cell (coalesced 128-byte rows), forms the
// limited variables, the slope of the previous cell and the limited face
// flux, and finishes the cell two planes back, whose hi and lo words it
// loaded at the start of the plane.  The slope and face flux of the
// previous plane are carried in registers.  No neighbour along k is needed,
// so every lane finishes a cell.  The interior is written; the ghost images
// come from the shell kernel.
//
// Physics: mhd_artificial_viscosity_host.hpp:70-348 with limiter.hpp:11-37,
// in the compensated split form (two-sum update of the hi/lo pair).
#include "common.cuh"
#include "s32_common.cuh"
#include "s32_tiled.h"

namespace miso_b200 {
namespace s32v {

using namespace s32t;

template <int DIR>
__global__ void __launch_bounds__(256, 2)
av_march_kernel(const AvArgs a) {
  const Geom &g = a.g;
  constexpr int OTH = DIR == 0 ? 1 : 0;
  const int lane = threadIdx.x & 31;
  const int kblocks = (g.n[2] + 31) / 32;
  const int nu = g.n[OTH];
  const int chunks = (g.n[DIR] + a.L - 1) / a.L;
  const int items = kblocks * nu * chunks;
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  const float fac = (float)(g.dsi[DIR] * a.sc->dt);
  const float ep = a.ep, fh = a.fh;
  const int S = (int)g.st[DIR];  // element stride along the sweep axis
  for (int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); w < items; w += nw) {
    // chunk-major order: warps in flight cover one band of planes
    const int kb = w % kblocks;
    const int r1 = w / kblocks;
    const int u = r1 % nu;
    const int t0 = (r1 / nu) * a.L;
    const int t1 = min(g.n[DIR], t0 + a.L);
    const int k = kb * 32 + lane;
    const bool active = k < g.n[2];
    const int kc = min(k, g.n[2] + 1);  // stay inside the array
    // cell of interior coordinate t along the sweep axis
    const int x0b = DIR == 0 ? 0 : u, x1b = DIR == 0 ? u : 0;
    const int cell0 = cell_of(g, x0b, x1b, kc);  // t = 0
    auto load_w = [&](int t, float wv[NW], float &ccv) {
      // a plane across a face: the interior plane it images, with the
      // mirror signs of that face
      int side;
      const int cell = cell0 + ghost_src(g, DIR, t, side) * S;
      float uu[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) uu[f] = __ldg(a.hi.f[f] + cell);
      if (side >= 0) {
        const unsigned neg = g.negmask[DIR][side];
#pragma unroll
        for (int f = 0; f < NF; ++f)
          if ((neg >> f) & 1u) uu[f] = -uu[f];
      }
      limited_vars(uu, wv);
      ccv = __ldg(a.cc + cell);
    };
    // prologue: planes t0-2 .. t0+1 give the slope at t0 and the face flux
    // between t0-1 and t0
    float w0[NW], w1[NW], dq0[NW], F0[NW];
    float cc0, cc1;
    {
      float wa[NW], wb[NW], cca, ccb;
      load_w(t0 - 2, wa, cca);
      load_w(t0 - 1, wb, ccb);
      load_w(t0, w0, cc0);
      load_w(t0 + 1, w1, cc1);
#pragma unroll
      for (int n = 0; n < NW; ++n) {
        const float dqm = dqq_eval(wa[n], wb[n], w0[n], ep);
        dq0[n] = dqq_eval(wb[n], w0[n], w1[n], ep);
        F0[n] = flux_core(wb[n], w0[n], dqm, dq0[n], 0.5f * (ccb + cc0), fh);
      }
    }
    for (int t = t0; t < t1; ++t) {
      // cell t: its hi / lo words, and plane t+2 for the slope at t+1
      const int cell = cell0 + t * S;
      float H[NF], Lo[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        H[f] = __ldg(a.hi.f[f] + cell);
        Lo[f] = __ldg(a.lo.f[f] + cell);
      }
      float wp[NW], ccp;
      load_w(t + 2, wp, ccp);
      float dF[NW];
#pragma unroll
      for (int n = 0; n < NW; ++n) {
        const float dq1 = dqq_eval(w0[n], w1[n], wp[n], ep);
        const float F1 = flux_core(w0[n], w1[n], dq0[n], dq1, 0.5f * (cc0 + cc1), fh);
        dF[n] = F1 - F0[n];
        F0[n] = F1;
        dq0[n] = dq1;
        w0[n] = w1[n];
        w1[n] = wp[n];
      }
      cc0 = cc1;
      cc1 = ccp;
      if (active) {
#pragma unroll
        for (int n = 0; n < NW; ++n) {
          const int f = field_of(n);
          float sv, e;
          two_sum(H[f], Lo[f] - dF[n] * fac, sv, e);
          a.hi2.f[f][cell] = sv;
          a.lo2.f[f][cell] = e;
        }
      }
    }
  }
}

}  // namespace s32v

void launch_s32_av_march(const AvArgs &a, int dir, int grid, cudaStream_t st) {
  if (dir == 0)
    s32v::av_march_kernel<0><<<grid, 256, 0, st>>>(a);
  else
    s32v::av_march_kernel<1><<<grid, 256, 0, st>>>(a);
}

}  // namespace miso_b200
