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

// Every product and sum below is rounded as written (no contraction left to
// the compiler): a point's primitive variables and fluxes then get the same
// bits wherever a kernel forms them -- for a tile's own points and for its
// halo rows alike -- so that the step does not depend on where tiles, or the
// shards of a decomposed grid, begin.
__device__ __forceinline__ void prim(const float u[NF], float gm1, PrimF &p) {
  const float inv = 1.0f / u[RO];
  p.v[0] = __fmul_rn(u[MX], inv);
  p.v[1] = __fmul_rn(u[MY], inv);
  p.v[2] = __fmul_rn(u[MZ], inv);
  const float bb = __fmaf_rn(u[BZ], u[BZ], __fmaf_rn(u[BY], u[BY], __fmul_rn(u[BX], u[BX])));
  const float pm = __fmul_rn(bb, FPII8);
  const float vm =
      __fmaf_rn(p.v[2], u[MZ], __fmaf_rn(p.v[1], u[MY], __fmul_rn(p.v[0], u[MX])));
  // p_tot = (gm - 1) (et - vm / 2 - pm) + pm
  p.ptot = __fmaf_rn(gm1, __fsub_rn(__fmaf_rn(-0.5f, vm, u[ET]), pm), pm);
  p.e_tot = __fadd_rn(u[ET], p.ptot);
  p.vb = __fmaf_rn(p.v[2], u[BZ], __fmaf_rn(p.v[1], u[BY], __fmul_rn(p.v[0], u[BX])));
}

template <int D>
__device__ __forceinline__ void flux_dir(const float u[NF], const PrimF &p, float ch2,
                                         float F[NF]) {
  const float vd = p.v[D], bd = u[BX + D];
  const float bd4 = __fmul_rn(bd, FPII4);
  F[RO] = u[MX + D];
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    float fm = __fmaf_rn(u[MX + e], vd, -__fmul_rn(u[BX + e], bd4));
    if (e == D) fm = __fadd_rn(fm, p.ptot);
    F[MX + e] = fm;
    F[BX + e] = (e == D) ? u[PH] : __fmaf_rn(vd, u[BX + e], -__fmul_rn(p.v[e], bd));
  }
  F[ET] = __fmaf_rn(p.e_tot, vd, -__fmul_rn(p.vb, bd4));
  F[PH] = __fmul_rn(ch2, bd);
}

// ---------------------------------------------------------------------------
// One arithmetic for a single field (float) and for a pair of fields
// (float2, the packed FP32x2 add / mul / fma of sm_100: component-wise,
// round to nearest, so each component gets the bits the scalar operation
// gives).  Products are never contracted behind the caller's back: every
// fma is written out.
// ---------------------------------------------------------------------------
template <class V>
__device__ __forceinline__ V vs(float x);
template <>
__device__ __forceinline__ float vs<float>(float x) { return x; }
template <>
__device__ __forceinline__ float2 vs<float2>(float x) { return make_float2(x, x); }

__device__ __forceinline__ float vadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float2 vadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float vmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float2 vmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float vfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b, rounded once ((-1) * b is exact)
__device__ __forceinline__ float vsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float2 vsub(float2 a, float2 b) {
  return __ffma2_rn(make_float2(-1.f, -1.f), b, a);
}
__device__ __forceinline__ float vmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ float2 vmax(float2 a, float2 b) {
  return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y));
}
__device__ __forceinline__ float vmin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ float2 vmin(float2 a, float2 b) {
  return make_float2(fminf(a.x, b.x), fminf(a.y, b.y));
}
// approximate reciprocal (PTX rcp.approx.ftz.f32) of d held at |d| >= 1e-20
// with its sign: the divisor of the limiter ratio
__device__ __forceinline__ float guard_rcp(float d) {
  const float g = copysignf(fmaxf(fabsf(d), 1e-20f), d);
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(g));
  return r;
}
__device__ __forceinline__ float2 guard_rcp(float2 d) {
  return make_float2(guard_rcp(d.x), guard_rcp(d.y));
}
// H(ra) * max(0, t), H the step (0 where ra carries a sign bit, else 1)
__device__ __forceinline__ float hstep(float ra, float t) {
  return signbit(ra) ? 0.0f : fmaxf(0.0f, t);
}
__device__ __forceinline__ float2 hstep(float2 ra, float2 t) {
  return make_float2(hstep(ra.x, t.x), hstep(ra.y, t.y));
}

template <class V>
__device__ __forceinline__ void two_sum(V a, V b, V &s, V &e) {
  s = vadd(a, b);
  const V bb = vsub(s, a);
  e = vadd(vsub(a, vsub(s, bb)), vsub(b, bb));
}

// The last Runge-Kutta stage's closing pieces, written with explicitly
// rounded operations so that every kernel that forms them (the stage
// itself, or the x sweep it is deferred into) gets the same bits.
//   ph: (sv, t) = two_sum(hi, lo - dt D) is damped by `decay` into the pair
//   (sv, e) = two_sum(sv * decay, fma(sv, decay, -sv * decay) + t * decay)
__device__ __forceinline__ void ph_damp(float sv, float t, float decay, float &s, float &e) {
  const float pr = __fmul_rn(sv, decay);
  const float pe = __fmaf_rn(sv, decay, -pr);
  two_sum(pr, __fmaf_rn(t, decay, pe), s, e);
}
// characteristic speed cs_fac cs + vv_fac |v| + ca_fac ca of a state with
// density ro, |m|^2 = mm, |B|^2 = bb and total energy et
__device__ __forceinline__ float char_speed(float ro, float mm, float bb, float et, float gm,
                                            float gm1, float cs_fac, float vv_fac,
                                            float ca_fac) {
  const float inv = 1.0f / ro;
  const float kin = __fmul_rn(__fmul_rn(0.5f, mm), inv);
  const float mag = __fmul_rn(bb, FPII8);
  const float ein = __fmul_rn(__fsub_rn(__fsub_rn(et, kin), mag), inv);
  const float cs = sqrtf(fmaxf(__fmul_rn(__fmul_rn(gm, gm1), ein), 0.0f));
  const float vv = __fmul_rn(sqrtf(mm), inv);
  const float ca = sqrtf(__fmul_rn(__fmul_rn(bb, inv), FPII4));
  return __fmaf_rn(ca, ca_fac, __fmaf_rn(vv, vv_fac, __fmul_rn(cs, cs_fac)));
}

// |a|^2 of a 3-vector, rounded as written
__device__ __forceinline__ float norm2(float x, float y, float z) {
  return __fmaf_rn(z, z, __fmaf_rn(y, y, __fmul_rn(x, x)));
}

// characteristic-speed pieces of a conserved state (rounded as written, so
// that the CFL pass and a sweep that folds the CFL minima in agree)
__device__ __forceinline__ void speeds(const float s[NF], float gm, float gm1, float &cs,
                                       float &vv, float &ca, float &ein) {
  const float inv = 1.0f / s[RO];
  const float mm = norm2(s[MX], s[MY], s[MZ]);
  const float bb = norm2(s[BX], s[BY], s[BZ]);
  // (et - |m|^2 / (2 ro) - |B|^2 / (8 pi)) / ro
  ein = __fmul_rn(__fmaf_rn(-bb, FPII8, __fmaf_rn(__fmul_rn(-0.5f, mm), inv, s[ET])), inv);
  cs = sqrtf(fmaxf(__fmul_rn(__fmul_rn(gm, gm1), ein), 0.0f));
  vv = __fmul_rn(sqrtf(mm), inv);
  ca = sqrtf(__fmul_rn(__fmul_rn(bb, inv), FPII4));
}

// ---------------------------------------------------------------------------
// Artificial viscosity helpers (limiter.hpp:11-37)
// ---------------------------------------------------------------------------
// The point-gravity force per volume -ro g x / |x|^3 in FP32 at array
// indices (i, j, k) (Source, common.cuh; demo/mhd3d_magnetosphere/src/
// src.hpp:17-44).
__device__ __forceinline__ void gravity_force(const Source &s, float ro, int i, int j, int k,
                                              float &fx, float &fy, float &fz) {
  const float X = (float)s.x[i], Y = (float)s.y[j], Z = (float)s.z[k];
  const float rr = sqrtf(norm2(X, Y, Z));
  const float a = __fmul_rn(-ro, (float)s.g) / __fmul_rn(__fmul_rn(rr, rr), rr);
  fx = __fmul_rn(a, X);
  fy = __fmul_rn(a, Y);
  fz = __fmul_rn(a, Z);
}

// generalized minmod slope of the centre point (limiter.hpp:11-20)
template <class V>
__device__ __forceinline__ V dqq_t(V qq_dw, V qq_cn, V qq_up, V ep) {
  const V d_dw = vsub(qq_cn, qq_dw);
  const V d_up = vsub(qq_up, qq_cn);
  const V d_cn = vmul(vsub(qq_up, qq_dw), vs<V>(0.5f));
  const V a = vmul(ep, d_dw), b = vmul(ep, d_up);
  const V mx = vmax(vmax(a, b), d_cn);
  const V mn = vmin(vmin(a, b), d_cn);
  return vadd(vmin(vs<V>(0.0f), mx), vmax(vs<V>(0.0f), mn));
}

// limited face flux (limiter.hpp:22-37); hcc = -1/2 of the face speed
template <class V>
__device__ __forceinline__ V flux_t(V qq_dw, V qq_up, V dqq_dw, V dqq_up, V hcc, V fh) {
  const V qql = vfma(vs<V>(0.5f), dqq_dw, qq_dw);
  const V qqr = vfma(vs<V>(-0.5f), dqq_up, qq_up);
  const V diff = vsub(qqr, qql);
  const V ra = vmin(vs<V>(1.0f), vmul(diff, guard_rcp(vsub(qq_up, qq_dw))));
  const V pp = hstep(ra, vfma(fh, vadd(ra, vs<V>(-1.0f)), vs<V>(1.0f)));
  return vmul(vmul(hcc, pp), diff);
}

__device__ __forceinline__ float dqq_eval(float qq_dw, float qq_cn, float qq_up, float ep) {
  return dqq_t<float>(qq_dw, qq_cn, qq_up, ep);
}

// cc: the face speed
__device__ __forceinline__ float flux_core(float qq_dw, float qq_up, float dqq_dw, float dqq_up,
                                           float cc, float fh) {
  return flux_t<float>(qq_dw, qq_up, dqq_dw, dqq_up, -0.5f * cc, fh);
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
  // ro e = et - |m|^2 / (2 ro) - |B|^2 / (8 pi), rounded as written
  const float et_k = __fmaf_rn(__fmul_rn(-0.5f, norm2(u[MX], u[MY], u[MZ])), inv, u[ET]);
  w[8] = __fmaf_rn(-norm2(u[BX], u[BY], u[BZ]), FPII8, et_k);
}

// the limited quantities as pairs (ro, mx) (my, mz) (bx, by) (bz, ph) and
// ro*e alone; pair i component c is limited quantity 2i + c
struct W9 {
  float2 p[4];
  float s;
};
__device__ __forceinline__ void limited_w9(const float u[NF], W9 &w) {
  float t[NW];
  limited_vars(u, t);
#pragma unroll
  for (int i = 0; i < 4; ++i) w.p[i] = make_float2(t[2 * i], t[2 * i + 1]);
  w.s = t[8];
}

// Flux difference F(k+1/2) - F(k-1/2) of the z sweep for the cells of a
// warp that holds 32 consecutive cells of a row, one per lane (hi words u
// and characteristic speed cc of the lane's cell); neighbours come from
// warp shuffles, so lanes 2..29 get a complete difference.
__device__ __forceinline__ void z_flux_diff(const float u[NF], float cc, float ep, float fh,
                                            W9 &dF) {
  W9 w;
  limited_w9(u, w);
  const float cc_up = __shfl_down_sync(0xffffffffu, cc, 1);
  const float hcc = -0.25f * (cc + cc_up);  // -1/2 of the face speed
  const float2 hcc2 = vs<float2>(hcc), ep2 = vs<float2>(ep), fh2 = vs<float2>(fh);
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    const float2 wm = make_float2(__shfl_up_sync(0xffffffffu, w.p[n].x, 1),
                                  __shfl_up_sync(0xffffffffu, w.p[n].y, 1));
    const float2 wp = make_float2(__shfl_down_sync(0xffffffffu, w.p[n].x, 1),
                                  __shfl_down_sync(0xffffffffu, w.p[n].y, 1));
    const float2 dq = dqq_t(wm, w.p[n], wp, ep2);
    const float2 dq_up = make_float2(__shfl_down_sync(0xffffffffu, dq.x, 1),
                                     __shfl_down_sync(0xffffffffu, dq.y, 1));
    const float2 Fup = flux_t(w.p[n], wp, dq, dq_up, hcc2, fh2);
    const float2 Fdw = make_float2(__shfl_up_sync(0xffffffffu, Fup.x, 1),
                                   __shfl_up_sync(0xffffffffu, Fup.y, 1));
    dF.p[n] = vsub(Fup, Fdw);
  }
  const float wm = __shfl_up_sync(0xffffffffu, w.s, 1);
  const float wp = __shfl_down_sync(0xffffffffu, w.s, 1);
  const float dq = dqq_t(wm, w.s, wp, ep);
  const float dq_up = __shfl_down_sync(0xffffffffu, dq, 1);
  const float Fup = flux_t(w.s, wp, dq, dq_up, hcc, fh);
  const float Fdw = __shfl_up_sync(0xffffffffu, Fup, 1);
  dF.s = vsub(Fup, Fdw);
}

// (hi, lo) - fac * dF as compensated pairs into s (hi words) and e (lo words)
__device__ __forceinline__ void av_update(const float u[NF], const float l[NF], const W9 &dF,
                                          float fac, float s[NF], float e[NF]) {
  const float2 mfac2 = vs<float2>(-fac);
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    const int f0 = field_of(2 * n), f1 = field_of(2 * n + 1);
    float2 sv, ev;
    two_sum(make_float2(u[f0], u[f1]), vfma(dF.p[n], mfac2, make_float2(l[f0], l[f1])), sv, ev);
    s[f0] = sv.x;
    s[f1] = sv.y;
    e[f0] = ev.x;
    e[f1] = ev.y;
  }
  two_sum(u[ET], vfma(dF.s, -fac, l[ET]), s[ET], e[ET]);
}

}  // namespace s32t
}  // namespace miso_b200
