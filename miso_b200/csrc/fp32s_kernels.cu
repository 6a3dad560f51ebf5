// FP32 split-precision form of the MHD step.
//
// State: the conserved set (ro, mx, my, mz, bx, by, bz, et, ph) as FP32
// hi/lo pairs (value = hi + lo).  The right-hand side and the artificial
// viscosity are computed in FP32 from the hi words; every update of the
// state is accumulated with a two-sum so the rounding of each update is
// carried in lo instead of being lost.  Intermediate Runge-Kutta stage
// states are plain FP32.
//
// The physics is the reference's (mhd_integrator_host.hpp:57-247 and
// mhd_artificial_viscosity_host.hpp:51-348) written in flux form: the sum
// of the reference's product derivatives along an axis equals the 4th-order
// difference of the ideal-MHD flux vector along that axis
//   F(ro) = m_d
//   F(m_e) = m_e v_d - b_e b_d / 4pi + delta_ed (p + |B|^2 / 8pi)
//   F(b_e) = v_d b_e - v_e b_d  (e != d),   F(b_d) = ph
//   F(ph)  = ch^2 b_d
//   F(et)  = (et + p + |B|^2 / 8pi) v_d - (v.B) b_d / 4pi
// with Gaussian units (constants.hpp:8-16), p = (gamma-1) rho e.
// The GLM damping keeps the reference's form ph = (ph0 + dt R) exp(-dt/tau).
#include "common.cuh"
#include "kernels_s32.h"
#include "s32_common.cuh"

namespace miso_b200 {
namespace s32 {

constexpr float FPII4 = (float)PII4;
constexpr float FPII8 = (float)PII8;
constexpr float FINV12 = (float)INV12;

struct Cons {
  float ro, m[3], b[3], et, ph;
};

__device__ __forceinline__ Cons load_cons(const FieldPtrs<const float> &u, long long c) {
  Cons q;
  q.ro = __ldg(u.f[RO] + c);
  q.m[0] = __ldg(u.f[MX] + c);
  q.m[1] = __ldg(u.f[MY] + c);
  q.m[2] = __ldg(u.f[MZ] + c);
  q.b[0] = __ldg(u.f[BX] + c);
  q.b[1] = __ldg(u.f[BY] + c);
  q.b[2] = __ldg(u.f[BZ] + c);
  q.et = __ldg(u.f[ET] + c);
  q.ph = __ldg(u.f[PH] + c);
  return q;
}

// Flux vector along axis d at one point.
__device__ __forceinline__ void flux(const Cons &q, int d, float gm1, float ch2, float F[NF]) {
  const float inv = 1.0f / q.ro;
  const float v0 = q.m[0] * inv, v1 = q.m[1] * inv, v2 = q.m[2] * inv;
  const float v[3] = {v0, v1, v2};
  const float bb = q.b[0] * q.b[0] + q.b[1] * q.b[1] + q.b[2] * q.b[2];
  const float pm = bb * FPII8;
  const float vm = v0 * q.m[0] + v1 * q.m[1] + v2 * q.m[2];
  const float roe = q.et - 0.5f * vm - pm;
  const float p = gm1 * roe;
  const float ptot = p + pm;
  const float vd = v[d], bd = q.b[d];
  const float vbd = (v0 * q.b[0] + v1 * q.b[1] + v2 * q.b[2]);
  F[RO] = q.m[d];
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    float fm = q.m[e] * vd - q.b[e] * bd * FPII4;
    if (e == d) fm += ptot;
    F[MX + e] = fm;
    F[BX + e] = (e == d) ? q.ph : (vd * q.b[e] - v[e] * bd);
  }
  F[ET] = (q.et + ptot) * vd - vbd * bd * FPII4;
  F[PH] = ch2 * bd;
}

__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
  s = a + b;
  const float bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

__device__ __forceinline__ void decode_index(const Geom &g, long long lin, int &i, int &j,
                                             int &k) {
  k = (int)(lin % g.n[2]) + g.m[2];
  const long long r1 = lin / g.n[2];
  j = (int)(r1 % g.n[1]) + g.m[1];
  i = (int)(r1 / g.n[1]) + g.m[0];
}

// Runge-Kutta stage `stage` (0..3): U_s = U_n + dts[stage] * R(U_{s-1}).
// Stages 0-2 write the FP32 stage buffer `out`; stage 3 accumulates into the
// hi/lo state in place (each cell reads only its own hi/lo).
__global__ void __launch_bounds__(128)
rk_stage_kernel(Geom g, FieldPtrs<const float> prev, FieldPtrs<float> hi, FieldPtrs<float> lo,
                FieldPtrs<float> out, const StepScalars *__restrict__ sc, int stage, float gm1,
                Source src) {
  const long long nint = (long long)g.n[0] * g.n[1] * g.n[2];
  const float dt = (float)sc->dts[stage];
  const float ch2 = (float)sc->ch2;
  const float decay = (float)sc->ph_decay[stage];
  for (long long lin = blockIdx.x * (long long)blockDim.x + threadIdx.x; lin < nint;
       lin += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode_index(g, lin, i, j, k);
    const long long c = i * g.st[0] + j * g.st[1] + k;
    float R[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) R[f] = 0.0f;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (!g.s[d]) continue;
      const long long s = g.st[d];
      const float w = (float)g.dsi[d] * FINV12;
      float P2[NF], P1[NF], M1[NF], M2[NF];
      flux(load_cons(prev, c + 2 * s), d, gm1, ch2, P2);
      flux(load_cons(prev, c + s), d, gm1, ch2, P1);
      flux(load_cons(prev, c - s), d, gm1, ch2, M1);
      flux(load_cons(prev, c - 2 * s), d, gm1, ch2, M2);
#pragma unroll
      for (int f = 0; f < NF; ++f) R[f] -= ((M2[f] - P2[f]) + 8.0f * (P1[f] - M1[f])) * w;
    }
    // a caller's source functor: its heating enters the new total energy
    // outside the dt factor (mhd_integrator_host.hpp:241)
    float heat = 0.0f;
    if (src.kind == 1) {  // point gravity on the argument state's density
      const float X = (float)src.x[i], Y = (float)src.y[j], Z = (float)src.z[k];
      const float rr = sqrtf(X * X + Y * Y + Z * Z);
      const float a = -prev.f[RO][c] * (float)src.g / (rr * rr * rr);
      R[MX] += a * X;
      R[MY] += a * Y;
      R[MZ] += a * Z;
    } else if (src.kind == 2) {  // the functor's terms, filled before the stage
      R[MX] += (float)src.arr[0][c];
      R[MY] += (float)src.arr[1][c];
      R[MZ] += (float)src.arr[2][c];
      heat = (float)src.arr[3][c];
    }
    if (stage < 3) {
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const float u0 = hi.f[f][c];
        float v = u0 + dt * R[f];
        if (f == PH) v = (u0 + dt * R[f]) * decay;
        if (f == ET && src.kind == 2) v += heat;
        out.f[f][c] = v;
      }
    } else {
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const float h = hi.f[f][c], l = lo.f[f][c];
        float s, e;
        if (f == PH) {
          // (h + l + dt R) * decay, with the product's rounding kept in lo
          float t;
          two_sum(h, l + dt * R[f], s, t);
          const float p = s * decay;
          const float pe = fmaf(s, decay, -p);
          two_sum(p, pe + t * decay, s, e);
        } else if (f == ET && src.kind == 2) {
          two_sum(h, (l + dt * R[f]) + heat, s, e);
        } else {
          two_sum(h, l + dt * R[f], s, e);
        }
        hi.f[f][c] = s;
        lo.f[f][c] = e;
      }
    }
  }
}

// Characteristic speed cs_fac*cs + vv_fac*|v| + ca_fac*ca on every cell
// (mhd_artificial_viscosity_host.hpp:51-68), from the hi words.
__global__ void __launch_bounds__(256)
char_velocity_kernel(Geom g, FieldPtrs<const float> u, float *__restrict__ cc, float gm,
                     float cs_fac, float vv_fac, float ca_fac) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < g.cells;
       n += (long long)gridDim.x * blockDim.x) {
    const Cons q = load_cons(u, n);
    const float inv = 1.0f / q.ro;
    const float mm = q.m[0] * q.m[0] + q.m[1] * q.m[1] + q.m[2] * q.m[2];
    const float bb = q.b[0] * q.b[0] + q.b[1] * q.b[1] + q.b[2] * q.b[2];
    const float e = (q.et - 0.5f * mm * inv - bb * FPII8) * inv;
    const float cs = sqrtf(fmaxf(gm * (gm - 1.0f) * e, 0.0f));
    const float vv = sqrtf(mm) * inv;
    const float ca = sqrtf(bb * inv * FPII4);
    cc[n] = cs * cs_fac + vv * vv_fac + ca * ca_fac;
  }
}

// limiter.hpp:11-21 in FP32
__device__ __forceinline__ float dqq_eval(float qq_dw, float qq_cn, float qq_up, float ep) {
  const float d_dw = qq_cn - qq_dw;
  const float d_up = qq_up - qq_cn;
  const float d_cn = (qq_up - qq_dw) * 0.5f;
  const float mx = fmaxf(fmaxf(ep * d_dw, ep * d_up), d_cn);
  const float mn = fminf(fminf(ep * d_dw, ep * d_up), d_cn);
  return fminf(0.0f, mx) + fmaxf(0.0f, mn);
}

// limiter.hpp:25-37 in FP32
__device__ __forceinline__ float flux_core(float qq_dw, float qq_up, float dqq_dw, float dqq_up,
                                           float cc, float fh) {
  const float qql = qq_dw + 0.5f * dqq_dw;
  const float qqr = qq_up - 0.5f * dqq_up;
  float dqq = qq_up - qq_dw;
  dqq = copysignf(fmaxf(fabsf(dqq), 1e-20f), dqq);
  const float ra = fminf(1.0f, (qqr - qql) / dqq);
  const float pp = (0.5f + copysignf(0.5f, ra)) * fmaxf(0.0f, 1.0f + fh * (ra - 1.0f));
  return -0.5f * cc * pp * (qqr - qql);
}

__device__ __forceinline__ float av_dflux(const float w[5], float ccl, float ccc, float ccr,
                                          float ep, float fh) {
  const float a = dqq_eval(w[0], w[1], w[2], ep);
  const float b = dqq_eval(w[1], w[2], w[3], ep);
  const float c = dqq_eval(w[2], w[3], w[4], ep);
  const float f_dw = flux_core(w[1], w[2], a, b, 0.5f * (ccl + ccc), fh);
  const float f_up = flux_core(w[2], w[3], b, c, 0.5f * (ccc + ccr), fh);
  return f_up - f_dw;
}

// One artificial-viscosity sweep along `dir`: (hi, lo) -> (hi2, lo2).
__global__ void __launch_bounds__(128)
av_sweep_kernel(Geom g, FieldPtrs<const float> hi, FieldPtrs<const float> lo,
                FieldPtrs<float> hi2, FieldPtrs<float> lo2, const float *__restrict__ cc,
                const StepScalars *__restrict__ sc, int dir, float ep, float fh) {
  const long long nint = (long long)g.n[0] * g.n[1] * g.n[2];
  const long long s = g.st[dir] * g.s[dir];
  const float fac = (float)(g.dsi[dir] * sc->dt);
  for (long long lin = blockIdx.x * (long long)blockDim.x + threadIdx.x; lin < nint;
       lin += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode_index(g, lin, i, j, k);
    const long long c = i * g.st[0] + j * g.st[1] + k;
    const float ccl = __ldg(cc + c - s), ccc = __ldg(cc + c), ccr = __ldg(cc + c + s);
    Cons q[5];
#pragma unroll
    for (int t = 0; t < 5; ++t) q[t] = load_cons(hi, c + (t - 2) * s);
    float w[5];
    float dF[NF];
#define MISO_AV(F_, expr)                 \
  _Pragma("unroll") for (int t = 0; t < 5; ++t) w[t] = (expr); \
  dF[F_] = av_dflux(w, ccl, ccc, ccr, ep, fh);
    MISO_AV(RO, q[t].ro)
    MISO_AV(MX, q[t].m[0])
    MISO_AV(MY, q[t].m[1])
    MISO_AV(MZ, q[t].m[2])
    MISO_AV(BX, q[t].b[0])
    MISO_AV(BY, q[t].b[1])
    MISO_AV(BZ, q[t].b[2])
    MISO_AV(PH, q[t].ph)
    // internal energy density ro*e = et - |m|^2/(2 ro) - |B|^2/(8 pi)
    MISO_AV(ET, q[t].et -
                    0.5f * (q[t].m[0] * q[t].m[0] + q[t].m[1] * q[t].m[1] + q[t].m[2] * q[t].m[2]) /
                        q[t].ro -
                    (q[t].b[0] * q[t].b[0] + q[t].b[1] * q[t].b[1] + q[t].b[2] * q[t].b[2]) * FPII8)
#undef MISO_AV
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      float sh, se;
      two_sum(hi.f[f][c], lo.f[f][c] - dF[f] * fac, sh, se);
      hi2.f[f][c] = sh;
      lo2.f[f][c] = se;
    }
  }
}

// With the magnetosphere boundary the state is read in FP64 from hi + lo:
// its strong dipole field makes the magnetic energy dwarf the thermal one
// near the body, and the internal energy formed from the FP32 hi words
// alone can cancel below zero where hi + lo holds a positive one.
__device__ __forceinline__ float cfl_cell64(const FieldPtrs<const float> &u,
                                            const FieldPtrs<const float> &lo, long long c,
                                            double gm, bool &bad) {
  double q[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) q[f] = (double)__ldg(u.f[f] + c) + (double)__ldg(lo.f[f] + c);
  const double inv = 1.0 / q[RO];
  const double mm = q[MX] * q[MX] + q[MY] * q[MY] + q[MZ] * q[MZ];
  const double bb = q[BX] * q[BX] + q[BY] * q[BY] + q[BZ] * q[BZ];
  const double e = (q[ET] - 0.5 * mm * inv - bb * PII8) * inv;
  const double tv = sqrt(gm * (gm - 1.0) * e) + sqrt(mm) * inv + sqrt(bb * inv * PII4);
  bad |= !(q[RO] > 0.0) || !(e >= 0.0) || !isfinite(tv);
  return (float)tv;
}

__global__ void __launch_bounds__(256)
cfl_partial_kernel(Geom g, FieldPtrs<const float> u, float *__restrict__ partial,
                   unsigned int *__restrict__ err, float gm, float gm1, float cfl_dx,
                   Magneto mg, FieldPtrs<const float> lo) {
  const long long nint = (long long)g.n[0] * g.n[1] * g.n[2];
  float best = 1.e10f;
  bool bad = false;
  for (long long lin = blockIdx.x * (long long)blockDim.x + threadIdx.x; lin < nint;
       lin += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode_index(g, lin, i, j, k);
    const long long c = i * g.st[0] + j * g.st[1] + k;
    float tv;
    if (mg.on) {
      tv = cfl_cell64(u, lo, c, (double)gm, bad);
    } else {
      // the speed as the sweeps that fold the CFL minima in form it
      float q[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) q[f] = u.f[f][c];
      float cs, vv, ca, e;
      s32t::speeds(q, gm, gm1, cs, vv, ca, e);
      tv = cs + vv + ca;
      bad |= !(q[RO] > 0.0f) || !(e >= 0.0f) || !isfinite(tv);
    }
    if (mg.mask_cfl) {
      // the magnetosphere demo's CFL (timestep.hpp:15-49): the sphere
      // r <= r_inner moves at 1e-10
      const double x = mg.x[i], y = mg.y[j], z = mg.z[k];
      if (sqrt(x * x + y * y + z * z) <= mg.r_inner) tv = 1.e-10f;
    }
    best = fminf(best, cfl_dx / tv);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, o));
  __shared__ float red[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = best;
  if (bad) atomicOr(err, ERRBIT_NONFINITE);
  __syncthreads();
  if (wid == 0) {
    best = lane < (int)(blockDim.x >> 5) ? red[lane] : 1.e10f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (lane == 0) partial[blockIdx.x] = best;
  }
}

// The magnetosphere demo's boundary (demo/mhd3d_magnetosphere/src/bc.hpp:
// 39-158) on the split state, every cell, ghosts included, after the
// mirror fill: the FP64 form's steps (magneto_bc_kernel) on the cell's
// primitive variables formed in FP64 from the conserved state -- hi + lo
// (PAIR) or a stage buffer's single words -- written back in the same form.
template <bool PAIR>
__global__ void __launch_bounds__(256)
magneto_split_kernel(Geom g, FieldPtrs<float> hi, FieldPtrs<float> lo, Magneto mg, double gm) {
  const bool inflow = g.s[0] && !g.periodic[0] && !g.ext[0][0];
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.cells;
       c += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(c % g.t[2]);
    const long long r1 = c / g.t[2];
    const int j = (int)(r1 % g.t[1]);
    const int i = (int)(r1 / g.t[1]);
    double u[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f)
      u[f] = PAIR ? (double)hi.f[f][c] + (double)lo.f[f][c] : (double)hi.f[f][c];
    // conserved -> primitive
    double p[NF];
    p[RO] = u[RO];
    p[VX] = u[MX] / u[RO];
    p[VY] = u[MY] / u[RO];
    p[VZ] = u[MZ] / u[RO];
    p[BX] = u[BX];
    p[BY] = u[BY];
    p[BZ] = u[BZ];
    p[EI] = (u[ET] - 0.5 * u[RO] * (p[VX] * p[VX] + p[VY] * p[VY] + p[VZ] * p[VZ]) -
             PII8 * (u[BX] * u[BX] + u[BY] * u[BY] + u[BZ] * u[BZ])) /
            u[RO];
    p[PH] = u[PH];
    if (inflow && i < g.m[0]) {
      p[RO] = mg.ro_sw;
      p[VX] = mg.vx_sw;
      p[EI] = mg.pr_sw / (gm - 1.0) / p[RO];
      p[BZ] = mg.bz_sw;
    }
    const double x = mg.x[i], y = mg.y[j], z = mg.z[k];
    const double rr = sqrt(x * x + y * y + z * z);
    const double r1n = rr / mg.r_inner;
    const double hh = fmax2f(0.0, r1n * r1n - 1.0);
    const double w = mg.a0 * hh / (mg.a0 * hh + 1.0);
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      const double b = mg.blend[f] ? mg.blend[f][c] : 0.0;
      p[f] = p[f] * w + b * (1.0 - w);
    }
    p[RO] = fmax2f(p[RO], mg.ro_floor);
    p[EI] = fmax2f(p[EI], mg.pr_floor / (gm - 1.0) / p[RO]);
    // primitive -> conserved
    u[RO] = p[RO];
    u[MX] = p[RO] * p[VX];
    u[MY] = p[RO] * p[VY];
    u[MZ] = p[RO] * p[VZ];
    u[BX] = p[BX];
    u[BY] = p[BY];
    u[BZ] = p[BZ];
    u[ET] = p[RO] * p[EI] + 0.5 * p[RO] * (p[VX] * p[VX] + p[VY] * p[VY] + p[VZ] * p[VZ]) +
            PII8 * (p[BX] * p[BX] + p[BY] * p[BY] + p[BZ] * p[BZ]);
    u[PH] = p[PH];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      const float h = __double2float_rn(u[f]);
      hi.f[f][c] = h;
      if (PAIR) lo.f[f][c] = __double2float_rn(u[f] - (double)h);
    }
  }
}

// FP64 primitives -> conserved hi/lo (every cell).
__global__ void __launch_bounds__(256)
to_split_kernel(long long cells, FieldPtrs<const double> q, FieldPtrs<float> hi,
                FieldPtrs<float> lo) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < cells;
       n += (long long)gridDim.x * blockDim.x) {
    const double ro = q.f[RO][n], vx = q.f[VX][n], vy = q.f[VY][n], vz = q.f[VZ][n];
    const double bx = q.f[BX][n], by = q.f[BY][n], bz = q.f[BZ][n];
    const double ei = q.f[EI][n], ph = q.f[PH][n];
    double u[NF];
    u[RO] = ro;
    u[MX] = ro * vx;
    u[MY] = ro * vy;
    u[MZ] = ro * vz;
    u[BX] = bx;
    u[BY] = by;
    u[BZ] = bz;
    u[ET] = ro * ei + 0.5 * ro * (vx * vx + vy * vy + vz * vz) + PII8 * (bx * bx + by * by + bz * bz);
    u[PH] = ph;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      const float h = __double2float_rn(u[f]);
      hi.f[f][n] = h;
      lo.f[f][n] = __double2float_rn(u[f] - (double)h);
    }
  }
}

// conserved hi/lo -> FP64 primitives (every cell).
__global__ void __launch_bounds__(256)
from_split_kernel(long long cells, FieldPtrs<const float> hi, FieldPtrs<const float> lo,
                  FieldPtrs<double> q) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < cells;
       n += (long long)gridDim.x * blockDim.x) {
    double u[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) u[f] = (double)hi.f[f][n] + (lo.f[f] ? (double)lo.f[f][n] : 0.0);
    const double ro = u[RO];
    const double vx = u[MX] / ro, vy = u[MY] / ro, vz = u[MZ] / ro;
    const double bb = u[BX] * u[BX] + u[BY] * u[BY] + u[BZ] * u[BZ];
    q.f[RO][n] = ro;
    q.f[VX][n] = vx;
    q.f[VY][n] = vy;
    q.f[VZ][n] = vz;
    q.f[BX][n] = u[BX];
    q.f[BY][n] = u[BY];
    q.f[BZ][n] = u[BZ];
    q.f[EI][n] = (u[ET] - 0.5 * ro * (vx * vx + vy * vy + vz * vz) - PII8 * bb) / ro;
    q.f[PH][n] = u[PH];
  }
}

}  // namespace s32

static int blocks_for(long long work, int threads, int sms, int per_sm) {
  long long b = (work + threads - 1) / threads;
  long long cap = (long long)sms * per_sm;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

void launch_s32_rk_stage(const Geom &g, const FieldPtrs<const float> &prev,
                         const FieldPtrs<float> &hi, const FieldPtrs<float> &lo,
                         const FieldPtrs<float> &out, const StepScalars *sc, int stage, double gm,
                         const Source &src, int sms, cudaStream_t st) {
  const long long nint = (long long)g.n[0] * g.n[1] * g.n[2];
  s32::rk_stage_kernel<<<blocks_for(nint, 128, sms, 16), 128, 0, st>>>(
      g, prev, hi, lo, out, sc, stage, (float)(gm - 1.0), src);
}

void launch_s32_char_velocity(const Geom &g, const FieldPtrs<const float> &u, float *cc,
                              double gm, double cs_fac, double vv_fac, double ca_fac, int sms,
                              cudaStream_t st) {
  s32::char_velocity_kernel<<<blocks_for(g.cells, 256, sms, 8), 256, 0, st>>>(
      g, u, cc, (float)gm, (float)cs_fac, (float)vv_fac, (float)ca_fac);
}

void launch_s32_av_sweep(const Geom &g, const FieldPtrs<const float> &hi,
                         const FieldPtrs<const float> &lo, const FieldPtrs<float> &hi2,
                         const FieldPtrs<float> &lo2, const float *cc, const StepScalars *sc,
                         int dir, double ep, double fh, int sms, cudaStream_t st) {
  const long long nint = (long long)g.n[0] * g.n[1] * g.n[2];
  s32::av_sweep_kernel<<<blocks_for(nint, 128, sms, 16), 128, 0, st>>>(
      g, hi, lo, hi2, lo2, cc, sc, dir, (float)ep, (float)fh);
}

void launch_s32_cfl_partial(const Geom &g, const FieldPtrs<const float> &u, float *partial,
                            int nparts, StepScalars *sc, double gm, double cfl_dx,
                            cudaStream_t st, const Magneto &mg,
                            const FieldPtrs<const float> &lo) {
  s32::cfl_partial_kernel<<<nparts, 256, 0, st>>>(g, u, partial, &sc->err, (float)gm,
                                                  (float)(gm - 1.0), (float)cfl_dx, mg, lo);
}

void launch_s32_magneto(const Geom &g, const FieldPtrs<float> &hi, const FieldPtrs<float> &lo,
                        bool pair, const Magneto &mg, double gm, int sms, cudaStream_t st) {
  const int grid = blocks_for(g.cells, 256, sms, 8);
  if (pair)
    s32::magneto_split_kernel<true><<<grid, 256, 0, st>>>(g, hi, lo, mg, gm);
  else
    s32::magneto_split_kernel<false><<<grid, 256, 0, st>>>(g, hi, lo, mg, gm);
}

void launch_s32_to_split(long long cells, const FieldPtrs<const double> &q,
                         const FieldPtrs<float> &hi, const FieldPtrs<float> &lo, int sms,
                         cudaStream_t st) {
  s32::to_split_kernel<<<blocks_for(cells, 256, sms, 8), 256, 0, st>>>(cells, q, hi, lo);
}

void launch_s32_from_split(long long cells, const FieldPtrs<const float> &hi,
                           const FieldPtrs<const float> &lo, const FieldPtrs<double> &q, int sms,
                           cudaStream_t st) {
  s32::from_split_kernel<<<blocks_for(cells, 256, sms, 8), 256, 0, st>>>(cells, hi, lo, q);
}

}  // namespace miso_b200
