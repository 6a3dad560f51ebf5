// Device helpers shared by the FP32 split-precision kernels: ghost images,
// flux vectors, compensated sums and the limiter (internal to the library).
#pragma once

#include "common.cuh"

namespace miso_b200 {
namespace s32t {

constexpr float FPII4 = (float)PII4;
constexpr float FPII8 = (float)PII8;

// ---------------------------------------------------------------------------
// Ghost images of an interior cell (faces, edges, corners): at most one
// image coordinate per axis (axis sizes >= 2 * margin), so at most 7.
// ---------------------------------------------------------------------------
struct Img {
  int off[7];             // element offset of image (mask-1) from the cell
  unsigned short neg[7];  // fields whose image is negated
  unsigned valid;         // bit (mask-1): image exists
};

__device__ __forceinline__ bool near_boundary(const Geom &g, int x0, int x1, int x2) {
  return x0 < g.m[0] || x0 >= g.n[0] - g.m[0] || x1 < g.m[1] || x1 >= g.n[1] - g.m[1] ||
         x2 < g.m[2] || x2 >= g.n[2] - g.m[2];
}

__device__ __forceinline__ void make_img(const Geom &g, int x0, int x1, int x2, Img &im) {
  const int xs[3] = {x0, x1, x2};
  int d[3];
  unsigned short nm[3];
  bool h[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int m = g.m[a], n = g.n[a], X = xs[a] + m;
    h[a] = false;
    d[a] = 0;
    nm[a] = 0;
    if (xs[a] < m) {
      h[a] = true;
      d[a] = ((g.periodic[a] ? X + n : 2 * m - 1 - X) - X) * (int)g.st[a];
      nm[a] = g.negmask[a][0];
    } else if (xs[a] >= n - m) {
      h[a] = true;
      d[a] = ((g.periodic[a] ? X - n : 2 * (m + n) - 1 - X) - X) * (int)g.st[a];
      nm[a] = g.negmask[a][1];
    }
  }
  im.valid = 0;
#pragma unroll
  for (int mask = 1; mask < 8; ++mask) {
    const bool ok = (!(mask & 1) || h[0]) && (!(mask & 2) || h[1]) && (!(mask & 4) || h[2]);
    im.off[mask - 1] = ((mask & 1) ? d[0] : 0) + ((mask & 2) ? d[1] : 0) + ((mask & 4) ? d[2] : 0);
    im.neg[mask - 1] = (unsigned short)(((mask & 1) ? nm[0] : 0) ^ ((mask & 2) ? nm[1] : 0) ^
                                        ((mask & 4) ? nm[2] : 0));
    if (ok) im.valid |= 1u << (mask - 1);
  }
}

// p[cell] = v and every ghost image; field f picks the mirror sign.
__device__ __forceinline__ void store_img(float *p, int cell, const Img &im, int f, float v) {
  p[cell] = v;
#pragma unroll
  for (int m = 0; m < 7; ++m)
    if ((im.valid >> m) & 1u) p[cell + im.off[m]] = ((im.neg[m] >> f) & 1u) ? -v : v;
}

__device__ __forceinline__ void store_cell(float *p, int cell, bool nb, const Img &im, int f,
                                           float v) {
  if (nb)
    store_img(p, cell, im, f, v);
  else
    p[cell] = v;
}

__device__ __forceinline__ int cell_of(const Geom &g, int x0, int x1, int x2) {
  return (x0 + g.m[0]) * (int)g.st[0] + (x1 + g.m[1]) * (int)g.st[1] + (x2 + g.m[2]);
}

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
