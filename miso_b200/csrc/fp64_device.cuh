// FP64 per-cell arithmetic of the MHD step, shared by the single-grid and
// the batched kernels (internal to the library).  Every translation unit
// that includes it is compiled with --fmad=false, so each multiply and add
// rounds separately in the reference's operand order, as the x86-64 host
// build of the reference does.
//
//   RHS + stage update   miso/include/miso/mhd_integrator_host.hpp:57-247
//   central difference   miso/include/miso/mhd_integrator.hpp:14-58
//   EOS                  miso/include/miso/eos.hpp:25-42
//   AV                   miso/include/miso/mhd_artificial_viscosity_host.hpp:51-348
//   limiter              miso/include/miso/limiter.hpp:11-37
//   CFL                  miso/include/miso/mhd_integrator_host.hpp:303-334
#pragma once

#include "common.cuh"

namespace miso_b200 {
namespace fp64 {

struct Prim {
  double ro, vx, vy, vz, bx, by, bz, ei, ph;
};

__device__ __forceinline__ Prim load_prim(const FieldPtrs<const double> &a, long long c) {
  Prim p;
  p.ro = __ldg(a.f[RO] + c);
  p.vx = __ldg(a.f[VX] + c);
  p.vy = __ldg(a.f[VY] + c);
  p.vz = __ldg(a.f[VZ] + c);
  p.bx = __ldg(a.f[BX] + c);
  p.by = __ldg(a.f[BY] + c);
  p.bz = __ldg(a.f[BZ] + c);
  p.ei = __ldg(a.f[EI] + c);
  p.ph = __ldg(a.f[PH] + c);
  return p;
}

// Point values whose 4th-order differences enter the RHS along one
// direction d (velocity component vd, field component bd).  Products keep
// the reference's factor order ((q1*q2)*q3); a*b == b*a exactly.
struct PointTerms {
  double ro_v;          // ro*vd
  double mx_v, my_v, mz_v;  // (ro*vx)*vd, (ro*vy)*vd, (ro*vz)*vd
  double pr, bb;        // gas pressure, |B|^2
  double bx_b, by_b, bz_b;  // bx*bd, by*bd, bz*bd
  double ph, b;         // ph, bd
  double ht_v, vb_b;    // ht*vd, vb*bd
  double vd_be[3];      // vd*be (e != d)
  double ve_bd[3];      // ve*bd (e != d)
};

__device__ __forceinline__ void point_terms(const Prim &p, int d, double gm, PointTerms &t) {
  const double v[3] = {p.vx, p.vy, p.vz};
  const double b[3] = {p.bx, p.by, p.bz};
  // eos.hpp:25-31
  const double pr = (gm - 1.0) * p.ro * p.ei;
  // mhd_integrator_host.hpp:64-89
  const double bb = p.bx * p.bx + p.by * p.by + p.bz * p.bz;
  const double ht = +p.ro * p.ei + pr + bb * PII4 +
                    0.5 * p.ro * (+p.vx * p.vx + p.vy * p.vy + p.vz * p.vz);
  const double vb = +p.vx * p.bx + p.vy * p.by + p.vz * p.bz;
  const double vd = v[d], bd = b[d];
  t.ro_v = p.ro * vd;
  t.mx_v = p.ro * p.vx * vd;
  t.my_v = p.ro * p.vy * vd;
  t.mz_v = p.ro * p.vz * vd;
  t.pr = pr;
  t.bb = bb;
  t.bx_b = p.bx * bd;
  t.by_b = p.by * bd;
  t.bz_b = p.bz * bd;
  t.ph = p.ph;
  t.b = bd;
  t.ht_v = ht * vd;
  t.vb_b = vb * bd;
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    t.vd_be[e] = vd * b[e];
    t.ve_bd[e] = v[e] * bd;
  }
}

// mhd_integrator.hpp:14-58: (-q[+2] + 8 q[+1] - 8 q[-1] + q[-2]) * inv12 * dsi
__device__ __forceinline__ double d4(double p2, double p1, double m1, double m2, double dsi) {
  return (-p2 + 8.0 * p1 - 8.0 * m1 + m2) * INV12 * dsi;
}

struct DirTerms {
  double ro_v, mx_v, my_v, mz_v, pr, bb, bx_b, by_b, bz_b, ph, b, ht_v, vb_b;
  double vd_be[3], ve_bd[3];
};

__device__ __forceinline__ void dir_terms(const FieldPtrs<const double> &a, long long c,
                                          long long s, int d, double dsi, double gm,
                                          DirTerms &D) {
  PointTerms P2, P1, M1, M2;
  point_terms(load_prim(a, c + 2 * s), d, gm, P2);
  point_terms(load_prim(a, c + s), d, gm, P1);
  point_terms(load_prim(a, c - s), d, gm, M1);
  point_terms(load_prim(a, c - 2 * s), d, gm, M2);
#define MISO_D4(m) D.m = d4(P2.m, P1.m, M1.m, M2.m, dsi)
  MISO_D4(ro_v);
  MISO_D4(mx_v);
  MISO_D4(my_v);
  MISO_D4(mz_v);
  MISO_D4(pr);
  MISO_D4(bb);
  MISO_D4(bx_b);
  MISO_D4(by_b);
  MISO_D4(bz_b);
  MISO_D4(ph);
  MISO_D4(b);
  MISO_D4(ht_v);
  MISO_D4(vb_b);
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    MISO_D4(vd_be[e]);
    MISO_D4(ve_bd[e]);
  }
#undef MISO_D4
}

// limiter.hpp:11-21
__device__ __forceinline__ double dqq_eval(double qq_dw, double qq_cn, double qq_up, double ep) {
  const double dqq_dw = qq_cn - qq_dw;
  const double dqq_up = qq_up - qq_cn;
  const double dqq_cn = (qq_up - qq_dw) * 0.5;
  const double dqq_max = fmax3f(ep * dqq_dw, ep * dqq_up, dqq_cn);
  const double dqq_min = fmin3f(ep * dqq_dw, ep * dqq_up, dqq_cn);
  return fmin2f(0.0, dqq_max) + fmax2f(0.0, dqq_min);
}

// limiter.hpp:25-37
__device__ __forceinline__ double flux_core(double qq_dw, double qq_up, double dqq_dw,
                                            double dqq_up, double cc, double fh) {
  const double qql = qq_dw + 0.5 * dqq_dw;
  const double qqr = qq_up - 0.5 * dqq_up;
  double dqq = qq_up - qq_dw;
  dqq = copysign(fmax2f(fabs(dqq), 1e-20), dqq);
  const double ra = fmin2f(1.0, (qqr - qql) / dqq);
  const double pp = (0.5 + copysign(0.5, ra)) * fmax2f(0.0, 1.0 + fh * (ra - 1.0));
  return -0.5 * cc * pp * (qqr - qql);
}

__device__ __forceinline__ double av_dflux(const double w[5], double ccl, double ccc, double ccr,
                                           double ep, double fh) {
  const double dqq_dw = dqq_eval(w[0], w[1], w[2], ep);
  const double dqq_cn = dqq_eval(w[1], w[2], w[3], ep);
  const double dqq_up = dqq_eval(w[2], w[3], w[4], ep);
  const double f_dw = flux_core(w[1], w[2], dqq_dw, dqq_cn, 0.5 * (ccl + ccc), fh);
  const double f_up = flux_core(w[2], w[3], dqq_cn, dqq_up, 0.5 * (ccc + ccr), fh);
  return f_up - f_dw;
}

// The limited quantities of cell c as av_cell forms them -- ro, the
// momenta ro v, B, ph and ro ei -- and its characteristic speed.
__device__ __forceinline__ void av_load_w(const FieldPtrs<const double> &q, const double *cc,
                                          long long c, double w[NF], double &ccv) {
  const double ro = __ldg(q.f[RO] + c);
  w[0] = ro;
  w[1] = ro * __ldg(q.f[VX] + c);
  w[2] = ro * __ldg(q.f[VY] + c);
  w[3] = ro * __ldg(q.f[VZ] + c);
  w[4] = __ldg(q.f[BX] + c);
  w[5] = __ldg(q.f[BY] + c);
  w[6] = __ldg(q.f[BZ] + c);
  w[7] = __ldg(q.f[PH] + c);
  w[8] = ro * __ldg(q.f[EI] + c);
  ccv = __ldg(cc + c);
}

// One Runge-Kutta stage for interior cell c: out = orgn + dt * R(argm)
// (mhd_integrator_host.hpp:106-244, expression by expression).
// The source's force per volume at cell (i, j, k) (array indices) from the
// stage's argument state (src.vx/vy/vz of the reference, evaluated on c_qq).
__device__ __forceinline__ void source_force(const Source &s, const FieldPtrs<const double> &a,
                                             long long c, int i, int j, int k, double &sx,
                                             double &sy, double &sz) {
  sx = sy = sz = 0.0;
  if (s.kind == 2) {
    sx = s.arr[0][c];
    sy = s.arr[1][c];
    sz = s.arr[2][c];
  } else if (s.kind == 1) {
    const double X = s.x[i], Y = s.y[j], Z = s.z[k];
    const double rr = sqrt(X * X + Y * Y + Z * Z);
    const double r3 = rr * rr * rr;  // util::pow3
    const double ro = a.f[RO][c];
    sx = -ro * s.g * X / r3;
    sy = -ro * s.g * Y / r3;
    sz = -ro * s.g * Z / r3;
  }
}

// The source's energy term src.ei (mhd_integrator_host.hpp:241, added to the
// new total energy outside the dt factor): 0 for every built-in source.
__device__ __forceinline__ double source_heat(const Source &s, long long c) {
  return s.kind == 2 ? s.arr[3][c] : 0.0;
}

__device__ __forceinline__ void rhs_cell(const Geom &g, const FieldPtrs<const double> &o,
                                         const FieldPtrs<const double> &a, long long c,
                                         double dt, double ch2, double decay, double gm,
                                         double out[NF], double sx = 0.0, double sy = 0.0,
                                         double sz = 0.0, double se = 0.0) {
  // sx, sy, sz: the source's force per volume, se its energy term (0 for
  // EmptySourceTerm, mhd_model_base.hpp:131-155)
  const double src = se;
    DirTerms X, Y, Z;
    dir_terms(a, c, g.st[0] * g.s[0], 0, g.dsi[0], gm, X);
    dir_terms(a, c, g.st[1] * g.s[1], 1, g.dsi[1], gm, Y);
    dir_terms(a, c, g.st[2] * g.s[2], 2, g.dsi[2], gm, Z);

    const double oro = o.f[RO][c], ovx = o.f[VX][c], ovy = o.f[VY][c], ovz = o.f[VZ][c];
    const double obx = o.f[BX][c], oby = o.f[BY][c], obz = o.f[BZ][c];
    const double oei = o.f[EI][c], oph = o.f[PH][c];

    const double ro = oro + dt * (-X.ro_v - Y.ro_v - Z.ro_v);

    const double vx = (oro * ovx + dt * (-X.mx_v - Y.mx_v - Z.mx_v - X.pr - X.bb * PII8 +
                                        PII4 * (+X.bx_b + Y.bx_b + Z.bx_b) + sx)) / ro;
    const double vy = (oro * ovy + dt * (-X.my_v - Y.my_v - Z.my_v - Y.pr - Y.bb * PII8 +
                                        PII4 * (+X.by_b + Y.by_b + Z.by_b) + sy)) / ro;
    const double vz = (oro * ovz + dt * (-X.mz_v - Y.mz_v - Z.mz_v - Z.pr - Z.bb * PII8 +
                                        PII4 * (+X.bz_b + Y.bz_b + Z.bz_b) + sz)) / ro;

    const double bx = obx + dt * (-Y.vd_be[0] - Z.vd_be[0] + Y.ve_bd[0] + Z.ve_bd[0] - X.ph);
    const double by = oby + dt * (-X.vd_be[1] - Z.vd_be[1] + X.ve_bd[1] + Z.ve_bd[1] - Y.ph);
    const double bz = obz + dt * (-X.vd_be[2] - Y.vd_be[2] + X.ve_bd[2] + Y.ve_bd[2] - Z.ph);

    const double ph = (oph + dt * ch2 * (-X.b - Y.b - Z.b)) * decay;

    const double Et = +oro * oei + 0.5 * oro * (+ovx * ovx + ovy * ovy + ovz * ovz) +
                      PII8 * (+obx * obx + oby * oby + obz * obz);
    const double ei = (Et + dt * (-X.ht_v - Y.ht_v - Z.ht_v + PII4 * (+X.vb_b + Y.vb_b + Z.vb_b)) -
                       0.5 * ro * (+vx * vx + vy * vy + vz * vz) -
                       PII8 * (+bx * bx + by * by + bz * bz) + src) / ro;

  out[RO] = ro;
  out[VX] = vx;
  out[VY] = vy;
  out[VZ] = vz;
  out[BX] = bx;
  out[BY] = by;
  out[BZ] = bz;
  out[EI] = ei;
  out[PH] = ph;
}

// One directional viscosity sweep for cell c
// (mhd_artificial_viscosity_host.hpp:70-348).
__device__ __forceinline__ void av_cell(const Geom &g, const FieldPtrs<const double> &q,
                                        const double *__restrict__ cc, long long c, int dir,
                                        double dt, double ep, double fh, double out[NF]) {
  const long long s = g.st[dir] * g.s[dir];
  const double dsi = g.dsi[dir];
    const double ccl = __ldg(cc + c - s), ccc = __ldg(cc + c), ccr = __ldg(cc + c + s);
    long long p[5];
#pragma unroll
    for (int t = 0; t < 5; ++t) p[t] = c + (t - 2) * s;
    double ro5[5], w[5];
#pragma unroll
    for (int t = 0; t < 5; ++t) ro5[t] = __ldg(q.f[RO] + p[t]);

    const double dro = av_dflux(ro5, ccl, ccc, ccr, ep, fh);
    const double ro_c = ro5[2];
    const double ro = ro_c - dro * dsi * dt;

    double v[3], m_old[3];
#pragma unroll
    for (int e = 0; e < 3; ++e) {
#pragma unroll
      for (int t = 0; t < 5; ++t) w[t] = ro5[t] * __ldg(q.f[VX + e] + p[t]);
      m_old[e] = w[2];
      const double dm = av_dflux(w, ccl, ccc, ccr, ep, fh);
      v[e] = (m_old[e] - dm * dsi * dt) / ro;
    }
    double b_old[3], b[3];
#pragma unroll
    for (int e = 0; e < 3; ++e) {
#pragma unroll
      for (int t = 0; t < 5; ++t) w[t] = __ldg(q.f[BX + e] + p[t]);
      b_old[e] = w[2];
      const double db = av_dflux(w, ccl, ccc, ccr, ep, fh);
      b[e] = b_old[e] - db * dsi * dt;
    }
#pragma unroll
    for (int t = 0; t < 5; ++t) w[t] = __ldg(q.f[PH] + p[t]);
    const double dph = av_dflux(w, ccl, ccc, ccr, ep, fh);
    const double ph = w[2] - dph * dsi * dt;

#pragma unroll
    for (int t = 0; t < 5; ++t) w[t] = ro5[t] * __ldg(q.f[EI] + p[t]);
    const double dei = av_dflux(w, ccl, ccc, ccr, ep, fh);
    const double ei_c = __ldg(q.f[EI] + c);
    const double vx_c = __ldg(q.f[VX] + c), vy_c = __ldg(q.f[VY] + c), vz_c = __ldg(q.f[VZ] + c);
    const double Et = ro_c * ei_c + 0.5 * ro_c * (vx_c * vx_c + vy_c * vy_c + vz_c * vz_c) +
                      PII8 * (b_old[0] * b_old[0] + b_old[1] * b_old[1] + b_old[2] * b_old[2]);
    const double ei = (Et - dei * dsi * dt - 0.5 * ro * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) -
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

// Characteristic speed cs_fac*cs + vv_fac*|v| + ca_fac*ca of cell n
// (mhd_artificial_viscosity_host.hpp:51-68 with eos.hpp:36-42).
__device__ __forceinline__ double cc_cell(const FieldPtrs<const double> &q, long long n,
                                          double gm, double cs_fac, double vv_fac,
                                          double ca_fac) {
  const double ro = q.f[RO][n], vx = q.f[VX][n], vy = q.f[VY][n], vz = q.f[VZ][n];
  const double bx = q.f[BX][n], by = q.f[BY][n], bz = q.f[BZ][n], ei = q.f[EI][n];
  const double cs = sqrt(gm * (gm - 1.0) * ei);
  const double vv = sqrt(vx * vx + vy * vy + vz * vz);
  const double ca = sqrt((bx * bx + by * by + bz * bz) / ro * PII4);
  return cs * cs_fac + vv * vv_fac + ca * ca_fac;
}

// CFL candidate of cell c, rounded to float as util::min2 does
// (mhd_integrator_host.hpp:303-334); `bad` flags a non-physical cell.
__device__ __forceinline__ float cfl_cell(const FieldPtrs<const double> &q, long long c,
                                          double gm, double cfl_dx, bool &bad) {
  const double ro = q.f[RO][c], vx = q.f[VX][c], vy = q.f[VY][c], vz = q.f[VZ][c];
  const double bx = q.f[BX][c], by = q.f[BY][c], bz = q.f[BZ][c], ei = q.f[EI][c];
  const double cs = sqrt(gm * (gm - 1.0) * ei);
  const double vv = sqrt(+vx * vx + vy * vy + vz * vz);
  const double ca = sqrt((+bx * bx + by * by + bz * bz) / ro * PII4);
  const double total_vel = cs + vv + ca;
  bad = !(ro > 0.0) || !(ei >= 0.0) || !isfinite(total_vel);
  return __double2float_rn(cfl_dx / total_vel);
}

}  // namespace fp64
}  // namespace miso_b200
