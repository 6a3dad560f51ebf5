// Device helpers shared by the FP32 split-precision kernels: ghost images,
// flux vectors, compensated sums and the limiter (internal to the library).
#pragma once

#include "common.cuh"
#include "images.cuh"

namespace miso_b200 {
namespace s32t {

using miso_b200::cell_of;
using miso_b200::Img;
using miso_b200::make_img;
using miso_b200::near_boundary;
using miso_b200::store_cell;
using miso_b200::store_img;

constexpr float FPII4 = (float)PII4;
constexpr float FPII8 = (float)PII8;

// ---------------------------------------------------------------------------
// Fluxes (flux form of mhd_integrator_host.hpp:106-244)
// ---------------------------------------------------------------------------
struct PrimF {
  float v[3], ptot, e_tot, vb;
};

__device__ __forceinline__ void prim(const float u[NF], float gm1, PrimF &p) {
  const float inv = 1.0f / u[RO];
  p.v[0] = u[MX] * inv;
  p.v[1] = u[MY] * inv;
  p.v[2] = u[MZ] * inv;
  const float bb = u[BX] * u[BX] + u[BY] * u[BY] + u[BZ] * u[BZ];
  const float pm = bb * FPII8;
  const float vm = p.v[0] * u[MX] + p.v[1] * u[MY] + p.v[2] * u[MZ];
  const float pr = gm1 * (u[ET] - 0.5f * vm - pm);
  p.ptot = pr + pm;
  p.e_tot = u[ET] + p.ptot;
  p.vb = p.v[0] * u[BX] + p.v[1] * u[BY] + p.v[2] * u[BZ];
}

template <int D>
__device__ __forceinline__ void flux_dir(const float u[NF], const PrimF &p, float ch2,
                                         float F[NF]) {
  const float vd = p.v[D], bd = u[BX + D];
  const float bd4 = bd * FPII4;
  F[RO] = u[MX + D];
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    float fm = u[MX + e] * vd - u[BX + e] * bd4;
    if (e == D) fm += p.ptot;
    F[MX + e] = fm;
    F[BX + e] = (e == D) ? u[PH] : (vd * u[BX + e] - p.v[e] * bd);
  }
  F[ET] = p.e_tot * vd - p.vb * bd4;
  F[PH] = ch2 * bd;
}

__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
  s = a + b;
  const float bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

// characteristic-speed pieces of a conserved state
__device__ __forceinline__ void speeds(const float s[NF], float gm, float gm1, float &cs,
                                       float &vv, float &ca, float &ein) {
  const float inv = 1.0f / s[RO];
  const float mm = s[MX] * s[MX] + s[MY] * s[MY] + s[MZ] * s[MZ];
  const float bb = s[BX] * s[BX] + s[BY] * s[BY] + s[BZ] * s[BZ];
  ein = (s[ET] - 0.5f * mm * inv - bb * FPII8) * inv;
  cs = sqrtf(fmaxf(gm * gm1 * ein, 0.0f));
  vv = sqrtf(mm) * inv;
  ca = sqrtf(bb * inv * FPII4);
}

// ---------------------------------------------------------------------------
// Artificial viscosity helpers (limiter.hpp:11-37)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float dqq_eval(float qq_dw, float qq_cn, float qq_up, float ep) {
  const float d_dw = qq_cn - qq_dw;
  const float d_up = qq_up - qq_cn;
  const float d_cn = (qq_up - qq_dw) * 0.5f;
  const float mx = fmaxf(fmaxf(ep * d_dw, ep * d_up), d_cn);
  const float mn = fminf(fminf(ep * d_dw, ep * d_up), d_cn);
  return fminf(0.0f, mx) + fmaxf(0.0f, mn);
}

__device__ __forceinline__ float flux_core(float qq_dw, float qq_up, float dqq_dw, float dqq_up,
                                           float cc, float fh) {
  const float qql = qq_dw + 0.5f * dqq_dw;
  const float qqr = qq_up - 0.5f * dqq_up;
  float dqq = qq_up - qq_dw;
  dqq = copysignf(fmaxf(fabsf(dqq), 1e-20f), dqq);
  const float ra = fminf(1.0f, __fdividef(qqr - qql, dqq));
  const float pp = (0.5f + copysignf(0.5f, ra)) * fmaxf(0.0f, 1.0f + fh * (ra - 1.0f));
  return -0.5f * cc * pp * (qqr - qql);
}

// limited quantities of a point: ro, mx, my, mz, bx, by, bz, ph, ro*e
constexpr int NW = 9;
__device__ __forceinline__ constexpr int field_of(int n) {
  return n == 7 ? PH : (n == 8 ? ET : n);
}
__device__ __forceinline__ void limited_vars(const float u[NF], float w[NW]) {
#pragma unroll
  for (int n = 0; n < 7; ++n) w[n] = u[n];
  w[7] = u[PH];
  const float inv = 1.0f / u[RO];
  w[8] = u[ET] - 0.5f * (u[MX] * u[MX] + u[MY] * u[MY] + u[MZ] * u[MZ]) * inv -
         (u[BX] * u[BX] + u[BY] * u[BY] + u[BZ] * u[BZ]) * FPII8;
}

}  // namespace s32t
}  // namespace miso_b200
