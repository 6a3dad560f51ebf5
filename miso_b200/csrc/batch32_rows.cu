// Batched FP32 split-precision kernels for 1-D and 2-D instances: one warp
// per row segment, no shared memory and no CTA barrier.
//
// R is the instance's unit-stride axis, C the other non-degenerate one (2-D).
// A warp owns 32 consecutive cells along R.  Neighbours along R come from
// warp shuffles; for the Runge-Kutta stage and the sweep along R the two
// lanes at each end only feed their neighbours, so a warp finishes 28 cells.
// Along C a warp marches over a chunk of rows: the Runge-Kutta stage keeps
// the C flux in a three-deep register ring (rotated by unrolling the row
// loop three times), the sweep along C carries the limited variables, slope
// and face flux of the previous rows.  Results are
// written to the interior; the ghost images come from shell_fill_kernel.
//
// Arithmetic as the single-grid split kernels (flux form of
// mhd_integrator_host.hpp:57-247; limiter.hpp:11-37;
// mhd_artificial_viscosity_host.hpp:70-348): the 4th-order difference of C
// is split into P = F(c-2) - 8 F(c-1) and N = F(c+2) - 8 F(c+1) and
// finished as (wC*P + D_R) - wC*N with separately rounded products, so a
// locally constant flux cancels exactly.
#include "batch.h"
#include "s32_common.cuh"

namespace miso_b200 {
namespace b32r {

using namespace s32t;

constexpr unsigned FULL = 0xffffffffu;

struct RowGeo {
  long long base;
  int sR, sC, mR, mC, nR, nC, tR, R, C;
  float wR, wC;
};

__device__ __forceinline__ RowGeo row_geo(const BatchInst &in) {
  const Geom &g = in.g;
  RowGeo q;
  q.base = in.base;
  q.R = in.ax_r;
  q.C = in.ax_c;
  q.sR = (int)g.st[q.R];
  q.mR = g.m[q.R];
  q.nR = g.n[q.R];
  q.tR = g.t[q.R];
  q.wR = (float)(g.dsi[q.R] * INV12);
  if (q.C >= 0) {
    q.sC = (int)g.st[q.C];
    q.mC = g.m[q.C];
    q.nC = g.n[q.C];
    q.wC = (float)(g.dsi[q.C] * INV12);
  } else {
    q.sC = q.mC = 0;
    q.nC = 1;
    q.wC = 0.f;
  }
  return q;
}

// element index (instance-relative) of interior row c, total R coordinate rt
__device__ __forceinline__ int row_cell(const RowGeo &q, int c, int rt) {
  return (c + q.mC) * q.sC + rt * q.sR;
}

template <int D>
__device__ __forceinline__ void flux_of(const float u[NF], float gm1, float ch2, float F[NF]) {
  PrimF p;
  prim(u, gm1, p);
  flux_dir<D>(u, p, ch2, F);
}

// 4th-order difference along R of a lane-distributed flux: (F[-2] - F[+2]) +
// 8 (F[+1] - F[-1])
__device__ __forceinline__ float dR(float F) {
  const float m2 = __shfl_up_sync(FULL, F, 2), m1 = __shfl_up_sync(FULL, F, 1);
  const float p1 = __shfl_down_sync(FULL, F, 1), p2 = __shfl_down_sync(FULL, F, 2);
  return fmaf(8.0f, p1 - m1, m2 - p2);
}

struct StageK {
  float dt, decay, ch2, gm, gm1, cs_fac, vv_fac, ca_fac;
};

// The last stage's update U^{n+1} = (h, l) - dt D of one cell as a
// compensated pair (sv, e), the GLM damping on ph, and the speed of the new
// state, with explicitly rounded operations: the fourth stage forms it, or
// -- with the update deferred -- the first sweep of the step, for every
// cell it reads, with the same bits.
__device__ __forceinline__ void last_update(float dt, float decay, const float h[NF],
                                            const float l[NF], const float D[NF], float sv[NF],
                                            float e[NF]) {
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    const float t = __fmaf_rn(-dt, D[f], l[f]);
    if (f == PH) {
      float tt;
      two_sum(h[f], t, sv[f], tt);
      const float pr = __fmul_rn(sv[f], decay);
      const float pe = __fmaf_rn(sv[f], decay, -pr);
      two_sum(pr, __fmaf_rn(tt, decay, pe), sv[f], e[f]);
    } else {
      two_sum(h[f], t, sv[f], e[f]);
    }
  }
}
__device__ __forceinline__ float last_speed(const float sv[NF], float gm, float gm1,
                                            float cs_fac, float vv_fac, float ca_fac) {
  float cs, vv, ca, ein;
  speeds(sv, gm, gm1, cs, vv, ca, ein);
  return __fmaf_rn(ca, ca_fac, __fmaf_rn(vv, vv_fac, __fmul_rn(cs, cs_fac)));
}

// write the finished cell `cell` of a stage (centre values A0 / A1; LAST: the
// fourth stage, which updates hi / lo and writes the speed -- or with DEFER
// writes its right-hand side D to `out` and leaves the update to the step's
// first sweep)
template <bool LAST, bool DEFER>
__device__ __forceinline__ void rk_finish(const StageK &k, long long base, int cell,
                                          const float D[NF], const float A0[NF],
                                          const float A1[NF], const FieldPtrs<float> &hi,
                                          const FieldPtrs<float> &lo, const FieldPtrs<float> &out,
                                          float *cc) {
  if (DEFER) {
#pragma unroll
    for (int f = 0; f < NF; ++f) out.f[f][base + cell] = D[f];
  } else if (!LAST) {
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      float v = A0[f] - k.dt * D[f];
      if (f == PH) v *= k.decay;
      out.f[f][base + cell] = v;
    }
  } else {
    float sv[NF], e[NF];
    last_update(k.dt, k.decay, A0, A1, D, sv, e);
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      hi.f[f][base + cell] = sv[f];
      lo.f[f][base + cell] = e[f];
    }
    cc[base + cell] = last_speed(sv, k.gm, k.gm1, k.cs_fac, k.vv_fac, k.ca_fac);
  }
}

template <bool LAST>
__device__ __forceinline__ void load_centre(long long base, int cell,
                                            const FieldPtrs<const float> &u0,
                                            const FieldPtrs<float> &hi, const FieldPtrs<float> &lo,
                                            float A0[NF], float A1[NF]) {
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    if (!LAST) {
      A0[f] = __ldg(u0.f[f] + base + cell);
    } else {
      A0[f] = hi.f[f][base + cell];
      A1[f] = lo.f[f][base + cell];
    }
  }
}

// One row q of a 2-D march: F(q) -> Fn, F(q-1) in F1, F(q-2) in F2;
// R(q) -> Rn, R(q-2) in R2 (see the file comment for P, N and R).
template <int AR, int AC, bool LAST, bool DEFER>
__device__ __forceinline__ void rk_row(const StageK &k, const RowGeo &q,
                                       const RowItem &it, int qrow, int rt, bool lane_out,
                                       const FieldPtrs<const float> &prev,
                                       const FieldPtrs<const float> &u0,
                                       const FieldPtrs<float> &hi, const FieldPtrs<float> &lo,
                                       const FieldPtrs<float> &out, float *cc, float Fn[NF],
                                       const float F1[NF], const float F2[NF], float Rn[NF],
                                       const float R2[NF]) {
  const int c = qrow - 2;
  const bool fin = lane_out && c >= it.c0 && c < it.c1;
  const int ccell = row_cell(q, c, rt);
  float u[NF];
  const int cell = row_cell(q, qrow, rt);
#pragma unroll
  for (int f = 0; f < NF; ++f) u[f] = __ldg(prev.f[f] + q.base + cell);
  PrimF pv;
  prim(u, k.gm1, pv);
  flux_dir<AC>(u, pv, k.ch2, Fn);
  const bool mid = qrow >= it.c0 && qrow < it.c1;
  float FR[NF];
  flux_dir<AR>(u, pv, k.ch2, FR);
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    const float d = dR(FR[f]);  // every lane takes part in the shuffles
    if (mid) {
      const float P = fmaf(-8.f, F1[f], F2[f]);
      Rn[f] = __fadd_rn(__fmul_rn(q.wC, P), q.wR * d);
    }
  }
  if (fin) {
    float A0[NF], A1[NF], D[NF];
    if (!DEFER) load_centre<LAST>(q.base, ccell, u0, hi, lo, A0, A1);
#pragma unroll
    for (int f = 0; f < NF; ++f)
      D[f] = __fsub_rn(R2[f], __fmul_rn(q.wC, fmaf(-8.f, F1[f], Fn[f])));
    rk_finish<LAST, DEFER>(k, q.base, ccell, D, A0, A1, hi, lo, out, cc);
  }
}

// One item of the Runge-Kutta stage: axes AR (unit stride) and AC (-1: 1-D)
template <int AR, int AC, bool LAST, bool DEFER>
__device__ __forceinline__ void rk_item(const RowItem &it, const RowGeo &q, const StageK &k,
                                        const FieldPtrs<const float> &prev,
                                        const FieldPtrs<const float> &u0,
                                        const FieldPtrs<float> &hi, const FieldPtrs<float> &lo,
                                        const FieldPtrs<float> &out, float *cc) {
  const int lane = threadIdx.x & 31;
  const int r = it.r0 - 2 + lane;  // interior coordinate along R
  const int rt = min(max(r + q.mR, 0), q.tR - 1);
  const bool lane_out = lane >= 2 && lane < 30 && r < q.nR;
  if (AC < 0) {
    // 1-D: one row
    const int cell = rt * q.sR;
    float A0[NF], A1[NF];
    if (lane_out && !DEFER) load_centre<LAST>(q.base, cell, u0, hi, lo, A0, A1);
    float u[NF], F[NF], D[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) u[f] = __ldg(prev.f[f] + q.base + cell);
    flux_of<AR < 0 ? 0 : AR>(u, k.gm1, k.ch2, F);
#pragma unroll
    for (int f = 0; f < NF; ++f) D[f] = q.wR * dR(F[f]);
    if (lane_out) rk_finish<LAST, DEFER>(k, q.base, cell, D, A0, A1, hi, lo, out, cc);
    return;
  }
  constexpr int CC = AC < 0 ? 0 : AC;
  float FA[NF], FB[NF], FC[NF], RA[NF], RB[NF], RC[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) FA[f] = FB[f] = FC[f] = RA[f] = RB[f] = RC[f] = 0.f;
  const int qe = it.c1 + 1;
  for (int qr = it.c0 - 2; qr <= qe; qr += 3) {
    rk_row<AR, CC, LAST, DEFER>(k, q, it, qr, rt, lane_out, prev, u0, hi, lo, out, cc, FA, FC,
                                FB, RA, RB);
    if (qr + 1 > qe) break;
    rk_row<AR, CC, LAST, DEFER>(k, q, it, qr + 1, rt, lane_out, prev, u0, hi, lo, out, cc, FB,
                                FA, FC, RB, RC);
    if (qr + 2 > qe) break;
    rk_row<AR, CC, LAST, DEFER>(k, q, it, qr + 2, rt, lane_out, prev, u0, hi, lo, out, cc, FC,
                                FB, FA, RC, RA);
  }
}

// Runge-Kutta stage over the items of one axis pair (AR unit-stride axis,
// AC the other one, -1 for 1-D instances)
template <int AR, int AC, bool LAST, bool DEFER>
__global__ void __launch_bounds__(256, 2)
rk_rows_kernel(BatchArgs a, const RowItem *items, int nitems, FieldPtrs<const float> prev,
               FieldPtrs<const float> u0, FieldPtrs<float> hi, FieldPtrs<float> lo,
               FieldPtrs<float> out, float *cc, int stage) {
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  for (int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); w < nitems; w += nw) {
    const RowItem it = items[w];
    const BatchInst &in = a.insts[it.inst];
    const RowGeo q = row_geo(in);
    const StepScalars &sc = a.sc[it.inst];
    StageK k;
    k.dt = (float)sc.dts[stage];
    k.decay = (float)sc.ph_decay[stage];
    k.ch2 = (float)sc.ch2;
    k.gm = (float)in.gm;
    k.gm1 = (float)(in.gm - 1.0);
    k.cs_fac = (float)in.cs_fac;
    k.vv_fac = (float)in.vv_fac;
    k.ca_fac = (float)in.ca_fac;
    rk_item<AR, AC, LAST, DEFER>(it, q, k, prev, u0, hi, lo, out, cc);
  }
}

// CFL candidate of a new state (mhd_integrator_host.hpp:303-334), folded
// into the warp's running minimum
__device__ __forceinline__ void cfl_fold(const float s[NF], const BatchInst &in, float &best,
                                         bool &bad) {
  float cs, vv, ca, ein;
  speeds(s, (float)in.gm, (float)(in.gm - 1.0), cs, vv, ca, ein);
  const float tv = cs + vv + ca;
  best = fminf(best, (float)in.cfl_dx / tv);
  bad |= !(s[RO] > 0.0f) || !(ein >= 0.0f) || !isfinite(tv);
}

__device__ __forceinline__ void cfl_commit(const BatchArgs &a, int inst, float best, bool bad) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_xor_sync(FULL, best, o));
  if (__any_sync(FULL, bad) && (threadIdx.x & 31) == 0) atomicOr(a.err, ERRBIT_NONFINITE);
  if ((threadIdx.x & 31) == 0) atomicMin(a.dtmin + inst, __float_as_uint(best));
}

// The first sweep of a step whose last Runge-Kutta update was deferred: the
// stage's right-hand side D and the speed array the sweep writes for the
// later sweeps (d4.f[0] == nullptr: no deferred update).
struct Defer {
  FieldPtrs<const float> d4;
  float *cc_out;
};

// The words of one cell as the sweep reads them: hi / lo of the state, or
// with a deferred update U^{n+1} formed from them and D, with its speed.
__device__ __forceinline__ void sweep_cell(const BatchArgs &a, const BatchInst &in, int inst,
                                           long long at, const FieldPtrs<const float> &hi,
                                           const FieldPtrs<const float> &lo, const Defer &df,
                                           const float *cc, float u[NF], float l[NF],
                                           float &ccv) {
  if (df.d4.f[0]) {
    float h[NF], lw[NF], d[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      h[f] = __ldg(hi.f[f] + at);
      lw[f] = __ldg(lo.f[f] + at);
      d[f] = __ldg(df.d4.f[f] + at);
    }
    const StepScalars &sc = a.sc[inst];
    last_update((float)sc.dts[3], (float)sc.ph_decay[3], h, lw, d, u, l);
    ccv = last_speed(u, (float)in.gm, (float)(in.gm - 1.0), (float)in.cs_fac, (float)in.vv_fac,
                     (float)in.ca_fac);
  } else {
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      u[f] = __ldg(hi.f[f] + at);
      l[f] = __ldg(lo.f[f] + at);
    }
    ccv = cc ? __ldg(cc + at) : 0.f;
  }
}

// Viscosity sweep along R (shuffles), or -- for an instance whose axis
// `dir` is degenerate -- the state copied through unchanged.
__global__ void __launch_bounds__(256)
av_rows_r_kernel(BatchArgs a, const RowItem *items, int nitems, FieldPtrs<const float> hi,
                 FieldPtrs<const float> lo, FieldPtrs<float> hi2, FieldPtrs<float> lo2,
                 const float *cc, int dir, int fuse_cfl, Defer df) {
  const int lane = threadIdx.x & 31;
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  for (int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); w < nitems; w += nw) {
    const RowItem it = items[w];
    const BatchInst &in = a.insts[it.inst];
    const RowGeo q = row_geo(in);
    if (dir == q.C) continue;       // the sweep along C has its own kernel
    const bool sweep = dir == q.R;  // otherwise: degenerate along dir
    const float fac = sweep ? (float)(in.g.dsi[dir] * a.sc[it.inst].dt) : 0.f;
    const float ep = (float)in.ep, fh = (float)in.fh;
    const int r = it.r0 - 2 + lane;
    const int rt = min(max(r + q.mR, 0), q.tR - 1);
    const bool lane_out = lane >= 2 && lane < 30 && r < q.nR;
    float best = 1.e10f;
    bool bad = false;
    for (int c = it.c0; c < it.c1; ++c) {
      const int cell = row_cell(q, c, rt);
      float u[NF], l[NF], w[NW], ccc;
      sweep_cell(a, in, it.inst, q.base + cell, hi, lo, df, sweep ? cc : nullptr, u, l, ccc);
      if (df.d4.f[0] && lane_out) df.cc_out[q.base + cell] = ccc;  // read by the later sweeps
      float dF[NW];
      if (sweep) {
        limited_vars(u, w);
        const float cup = 0.5f * (ccc + __shfl_down_sync(FULL, ccc, 1));
#pragma unroll
        for (int n = 0; n < NW; ++n) {
          const float wm = __shfl_up_sync(FULL, w[n], 1);
          const float wp = __shfl_down_sync(FULL, w[n], 1);
          const float dq = dqq_eval(wm, w[n], wp, ep);
          const float dq_up = __shfl_down_sync(FULL, dq, 1);
          const float Fup = flux_core(w[n], wp, dq, dq_up, cup, fh);
          dF[n] = Fup - __shfl_up_sync(FULL, Fup, 1);
        }
      } else {
#pragma unroll
        for (int n = 0; n < NW; ++n) dF[n] = 0.f;
      }
      if (lane_out) {
        float s[NF];
#pragma unroll
        for (int n = 0; n < NW; ++n) {
          const int f = field_of(n);
          float e;
          two_sum(u[f], l[f] - dF[n] * fac, s[f], e);
          hi2.f[f][q.base + cell] = s[f];
          lo2.f[f][q.base + cell] = e;
        }
        if (fuse_cfl) cfl_fold(s, in, best, bad);
      }
    }
    if (fuse_cfl) cfl_commit(a, it.inst, best, bad);
  }
}

// Viscosity sweep along C: a warp marches over the rows of a chunk with all
// 32 lanes finishing cells (no halo along R is needed).
__global__ void __launch_bounds__(256, 2)
av_rows_c_kernel(BatchArgs a, const RowItem *items, int nitems, FieldPtrs<const float> hi,
                 FieldPtrs<const float> lo, FieldPtrs<float> hi2, FieldPtrs<float> lo2,
                 const float *cc, int dir, int fuse_cfl, Defer df) {
  const int lane = threadIdx.x & 31;
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  for (int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); w < nitems; w += nw) {
    const RowItem it = items[w];
    const BatchInst &in = a.insts[it.inst];
    const RowGeo q = row_geo(in);
    if (q.C != dir) continue;  // R and degenerate sweeps: av_rows_r_kernel
    const float fac = (float)(in.g.dsi[q.C] * a.sc[it.inst].dt);
    const float ep = (float)in.ep, fh = (float)in.fh;
    const int r = it.r0 + lane;
    const bool active = r < q.nR;
    const int rt = min(r + q.mR, q.tR - 1);
    auto load_w = [&](int row, float w[NW], float &ccv) {
      const int cell = row_cell(q, row, rt);
      float u[NF];
      if (df.d4.f[0]) {
        float l[NF];
        sweep_cell(a, in, it.inst, q.base + cell, hi, lo, df, cc, u, l, ccv);
      } else {
#pragma unroll
        for (int f = 0; f < NF; ++f) u[f] = __ldg(hi.f[f] + q.base + cell);
        ccv = __ldg(cc + q.base + cell);
      }
      limited_vars(u, w);
    };
    // prologue: rows c0-2 .. c0+1 give the slope at c0 and the face flux
    // between c0-1 and c0
    float w0[NW], w1[NW], dq0[NW], F0[NW];
    float cc0, cc1;
    {
      float wa[NW], wb[NW], cca, ccb;
      load_w(it.c0 - 2, wa, cca);
      load_w(it.c0 - 1, wb, ccb);
      load_w(it.c0, w0, cc0);
      load_w(it.c0 + 1, w1, cc1);
#pragma unroll
      for (int n = 0; n < NW; ++n) {
        const float dqm = dqq_eval(wa[n], wb[n], w0[n], ep);
        dq0[n] = dqq_eval(wb[n], w0[n], w1[n], ep);
        F0[n] = flux_core(wb[n], w0[n], dqm, dq0[n], 0.5f * (ccb + cc0), fh);
      }
    }
    float best = 1.e10f;
    bool bad = false;
    for (int c = it.c0; c < it.c1; ++c) {
      // cell c: its centre words, and row c+2 for the slope at c+1
      const int ccell = row_cell(q, c, rt);
      float H[NF], L[NF];
      if (active) {
        float ccv;
        sweep_cell(a, in, it.inst, q.base + ccell, hi, lo, df, nullptr, H, L, ccv);
        if (df.d4.f[0]) df.cc_out[q.base + ccell] = ccv;  // read by the later sweeps
      }
      float wp[NW], ccp;
      load_w(c + 2, wp, ccp);
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
        float s[NF];
#pragma unroll
        for (int n = 0; n < NW; ++n) {
          const int f = field_of(n);
          float e;
          two_sum(H[f], L[f] - dF[n] * fac, s[f], e);
          hi2.f[f][q.base + ccell] = s[f];
          lo2.f[f][q.base + ccell] = e;
        }
        if (fuse_cfl) cfl_fold(s, in, best, bad);
      }
    }
    if (fuse_cfl) cfl_commit(a, it.inst, best, bad);
  }
}

}  // namespace b32r

void b32_rk_rows(const BatchArgs &a, const RowItem *items, int n, int combo,
                 const FieldPtrs<const float> &prev, const FieldPtrs<const float> &u0,
                 const FieldPtrs<float> &hi, const FieldPtrs<float> &lo,
                 const FieldPtrs<float> &out, float *cc, int stage, int defer, int grid,
                 cudaStream_t st) {
  if (n <= 0) return;
#define MISO_RK_ROWS(R, C)                                                                    \
  if (stage == 3 && defer)                                                                  \
    b32r::rk_rows_kernel<R, C, true, true><<<grid, 256, 0, st>>>(a, items, n, prev, u0, hi,   \
                                                                 lo, out, cc, stage);         \
  else if (stage == 3)                                                                      \
    b32r::rk_rows_kernel<R, C, true, false><<<grid, 256, 0, st>>>(a, items, n, prev, u0, hi,  \
                                                                  lo, out, cc, stage);        \
  else                                                                                      \
    b32r::rk_rows_kernel<R, C, false, false><<<grid, 256, 0, st>>>(a, items, n, prev, u0, hi, \
                                                                   lo, out, cc, stage)
  switch (combo) {
    case 0: MISO_RK_ROWS(0, -1); break;
    case 1: MISO_RK_ROWS(1, -1); break;
    case 2: MISO_RK_ROWS(2, -1); break;
    case 3: MISO_RK_ROWS(1, 0); break;
    case 4: MISO_RK_ROWS(2, 0); break;
    default: MISO_RK_ROWS(2, 1); break;
  }
#undef MISO_RK_ROWS
}

int b32_row_combo(int ax_r, int ax_c) {
  if (ax_c < 0) return ax_r;                 // 1-D: 0, 1, 2
  return ax_r == 1 ? 3 : (ax_c == 0 ? 4 : 5);  // 2-D: (1,0), (2,0), (2,1)
}

void b32_av_rows_r(const BatchArgs &a, const RowItem *items, int n,
                   const FieldPtrs<const float> &hi, const FieldPtrs<const float> &lo,
                   const FieldPtrs<float> &hi2, const FieldPtrs<float> &lo2, const float *cc,
                   int dir, int fuse_cfl, const FieldPtrs<const float> &d4, float *cc_out,
                   int grid, cudaStream_t st) {
  if (n > 0)
    b32r::av_rows_r_kernel<<<grid, 256, 0, st>>>(a, items, n, hi, lo, hi2, lo2, cc, dir,
                                                 fuse_cfl, b32r::Defer{d4, cc_out});
}

void b32_av_rows_c(const BatchArgs &a, const RowItem *items, int n,
                   const FieldPtrs<const float> &hi, const FieldPtrs<const float> &lo,
                   const FieldPtrs<float> &hi2, const FieldPtrs<float> &lo2, const float *cc,
                   int dir, int fuse_cfl, const FieldPtrs<const float> &d4, float *cc_out,
                   int grid, cudaStream_t st) {
  if (n > 0)
    b32r::av_rows_c_kernel<<<grid, 256, 0, st>>>(a, items, n, hi, lo, hi2, lo2, cc, dir,
                                                 fuse_cfl, b32r::Defer{d4, cc_out});
}

}  // namespace miso_b200
