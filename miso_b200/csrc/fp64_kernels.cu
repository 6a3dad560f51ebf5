// FP64 kernels of the MHD step, written to reproduce the reference's
// double-precision host arithmetic bit for bit.
//
// This translation unit is compiled with --fmad=false: every multiply and add
// below rounds separately, in the reference's operand order, as the x86-64
// host build of the reference does (no FMA).  Division and square root are
// IEEE round-to-nearest (nvcc defaults), as on the host.
//
// Reference expressions followed (paths inside the MISO project):
//   RHS + stage update   miso/include/miso/mhd_integrator_host.hpp:57-247
//   central difference   miso/include/miso/mhd_integrator.hpp:14-58
//   EOS                  miso/include/miso/eos.hpp:25-42
//   AV                   miso/include/miso/mhd_artificial_viscosity_host.hpp:51-348
//   limiter              miso/include/miso/limiter.hpp:11-37
//   CFL                  miso/include/miso/mhd_integrator_host.hpp:303-334
//   ghost fill           boundary_condition.hpp:77-136, mhd_halo_exchange.hpp:51-265
#include "common.cuh"
#include "kernels.h"

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

// One Runge-Kutta stage: rslt = orgn + dt * R(argm) on interior cells,
// mhd_integrator_host.hpp:106-244 expression by expression.
__global__ void __launch_bounds__(128)
rhs_stage_kernel(Geom g, FieldPtrs<const double> o, FieldPtrs<const double> a,
                 FieldPtrs<double> r, const StepScalars *__restrict__ sc, int stage, double gm) {
  const long long nint = (long long)g.n[0] * g.n[1] * g.n[2];
  const double dt = sc->dts[stage];
  const double ch2 = sc->ch2;
  const double decay = sc->ph_decay[stage];
  const double src = 0.0;  // EmptySourceTerm (mhd_model_base.hpp:131-155)
  for (long long lin = blockIdx.x * (long long)blockDim.x + threadIdx.x; lin < nint;
       lin += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(lin % g.n[2]) + g.m[2];
    const long long r1 = lin / g.n[2];
    const int j = (int)(r1 % g.n[1]) + g.m[1];
    const int i = (int)(r1 / g.n[1]) + g.m[0];
    const long long c = i * g.st[0] + j * g.st[1] + k;

    DirTerms X, Y, Z;
    dir_terms(a, c, g.st[0] * g.s[0], 0, g.dsi[0], gm, X);
    dir_terms(a, c, g.st[1] * g.s[1], 1, g.dsi[1], gm, Y);
    dir_terms(a, c, g.st[2] * g.s[2], 2, g.dsi[2], gm, Z);

    const double oro = o.f[RO][c], ovx = o.f[VX][c], ovy = o.f[VY][c], ovz = o.f[VZ][c];
    const double obx = o.f[BX][c], oby = o.f[BY][c], obz = o.f[BZ][c];
    const double oei = o.f[EI][c], oph = o.f[PH][c];

    const double ro = oro + dt * (-X.ro_v - Y.ro_v - Z.ro_v);

    const double vx = (oro * ovx + dt * (-X.mx_v - Y.mx_v - Z.mx_v - X.pr - X.bb * PII8 +
                                        PII4 * (+X.bx_b + Y.bx_b + Z.bx_b) + src)) / ro;
    const double vy = (oro * ovy + dt * (-X.my_v - Y.my_v - Z.my_v - Y.pr - Y.bb * PII8 +
                                        PII4 * (+X.by_b + Y.by_b + Z.by_b) + src)) / ro;
    const double vz = (oro * ovz + dt * (-X.mz_v - Y.mz_v - Z.mz_v - Z.pr - Z.bb * PII8 +
                                        PII4 * (+X.bz_b + Y.bz_b + Z.bz_b) + src)) / ro;

    const double bx = obx + dt * (-Y.vd_be[0] - Z.vd_be[0] + Y.ve_bd[0] + Z.ve_bd[0] - X.ph);
    const double by = oby + dt * (-X.vd_be[1] - Z.vd_be[1] + X.ve_bd[1] + Z.ve_bd[1] - Y.ph);
    const double bz = obz + dt * (-X.vd_be[2] - Y.vd_be[2] + X.ve_bd[2] + Y.ve_bd[2] - Z.ph);

    const double ph = (oph + dt * ch2 * (-X.b - Y.b - Z.b)) * decay;

    const double Et = +oro * oei + 0.5 * oro * (+ovx * ovx + ovy * ovy + ovz * ovz) +
                      PII8 * (+obx * obx + oby * oby + obz * obz);
    const double ei = (Et + dt * (-X.ht_v - Y.ht_v - Z.ht_v + PII4 * (+X.vb_b + Y.vb_b + Z.vb_b)) -
                       0.5 * ro * (+vx * vx + vy * vy + vz * vz) -
                       PII8 * (+bx * bx + by * by + bz * bz) + src) / ro;

    r.f[RO][c] = ro;
    r.f[VX][c] = vx;
    r.f[VY][c] = vy;
    r.f[VZ][c] = vz;
    r.f[BX][c] = bx;
    r.f[BY][c] = by;
    r.f[BZ][c] = bz;
    r.f[EI][c] = ei;
    r.f[PH][c] = ph;
  }
}

// ----------------------------------------------------------------------
// Artificial viscosity
// ----------------------------------------------------------------------

// mhd_artificial_viscosity_host.hpp:51-68 with eos.hpp:36-42, on every cell.
__global__ void __launch_bounds__(256)
char_velocity_kernel(Geom g, FieldPtrs<const double> q, double *__restrict__ cc, double gm,
                     double cs_fac, double vv_fac, double ca_fac) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < g.cells;
       n += (long long)gridDim.x * blockDim.x) {
    const double ro = q.f[RO][n], vx = q.f[VX][n], vy = q.f[VY][n], vz = q.f[VZ][n];
    const double bx = q.f[BX][n], by = q.f[BY][n], bz = q.f[BZ][n], ei = q.f[EI][n];
    const double cs = sqrt(gm * (gm - 1.0) * ei);
    const double vv = sqrt(vx * vx + vy * vy + vz * vz);
    const double ca = sqrt((bx * bx + by * by + bz * bz) / ro * PII4);
    cc[n] = cs * cs_fac + vv * vv_fac + ca * ca_fac;
  }
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

// One directional sweep (mhd_artificial_viscosity_host.hpp:70-348) on the
// interior cells; ghost cells are refilled from their images afterwards.
__global__ void __launch_bounds__(128)
av_sweep_kernel(Geom g, FieldPtrs<const double> q, FieldPtrs<double> r,
                const double *__restrict__ cc, const StepScalars *__restrict__ sc, int dir,
                double ep, double fh) {
  const long long nint = (long long)g.n[0] * g.n[1] * g.n[2];
  const long long s = g.st[dir] * g.s[dir];
  const double dsi = g.dsi[dir];
  const double dt = sc->dt;
  for (long long lin = blockIdx.x * (long long)blockDim.x + threadIdx.x; lin < nint;
       lin += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(lin % g.n[2]) + g.m[2];
    const long long r1 = lin / g.n[2];
    const int j = (int)(r1 % g.n[1]) + g.m[1];
    const int i = (int)(r1 / g.n[1]) + g.m[0];
    const long long c = i * g.st[0] + j * g.st[1] + k;
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

    r.f[RO][c] = ro;
    r.f[VX][c] = v[0];
    r.f[VY][c] = v[1];
    r.f[VZ][c] = v[2];
    r.f[BX][c] = b[0];
    r.f[BY][c] = b[1];
    r.f[BZ][c] = b[2];
    r.f[EI][c] = ei;
    r.f[PH][c] = ph;
  }
}

// ----------------------------------------------------------------------
// CFL (mhd_integrator_host.hpp:303-334): per-block float-rounded minimum of
// cfl * min3(dx,dy,dz) / (cs + |v| + ca) over the interior, then one block
// folds the partials and derives the step scalars on the device.
// ----------------------------------------------------------------------
__global__ void __launch_bounds__(256)
cfl_partial_kernel(Geom g, FieldPtrs<const double> q, float *__restrict__ partial,
                   unsigned int *__restrict__ err, double gm, double cfl_dx) {
  const long long nint = (long long)g.n[0] * g.n[1] * g.n[2];
  float best = 1.e10f;
  bool bad = false;
  for (long long lin = blockIdx.x * (long long)blockDim.x + threadIdx.x; lin < nint;
       lin += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(lin % g.n[2]) + g.m[2];
    const long long r1 = lin / g.n[2];
    const int j = (int)(r1 % g.n[1]) + g.m[1];
    const int i = (int)(r1 / g.n[1]) + g.m[0];
    const long long c = i * g.st[0] + j * g.st[1] + k;
    const double ro = q.f[RO][c], vx = q.f[VX][c], vy = q.f[VY][c], vz = q.f[VZ][c];
    const double bx = q.f[BX][c], by = q.f[BY][c], bz = q.f[BZ][c], ei = q.f[EI][c];
    const double cs = sqrt(gm * (gm - 1.0) * ei);
    const double vv = sqrt(+vx * vx + vy * vy + vz * vz);
    const double ca = sqrt((+bx * bx + by * by + bz * bz) / ro * PII4);
    const double total_vel = cs + vv + ca;
    // util::min2(dt, x): both sides through float; fminf ignores a NaN side.
    best = fminf(best, __double2float_rn(cfl_dx / total_vel));
    bad |= !(ro > 0.0) || !(ei >= 0.0) || !isfinite(total_vel);
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

}  // namespace fp64

// Fold the per-block minima and derive every scalar of the step on the
// device (divb_parameters_set, mhd_integrator_host.hpp:337-341; stage
// factors, 258-277).  Shared by both precisions.
__global__ void __launch_bounds__(1024)
cfl_finalize_kernel(const float *__restrict__ partial, int nparts, StepScalars *sc,
                    double cfl_number, double min_dxyz) {
  float best = 1.e10f;
  for (int n = threadIdx.x; n < nparts; n += blockDim.x) best = fminf(best, partial[n]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, o));
  __shared__ float red[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = best;
  __syncthreads();
  if (wid == 0) {
    best = lane < (int)(blockDim.x >> 5) ? red[lane] : 1.e10f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (lane == 0) {
      const double dt = (double)best;
      sc->dt = dt;
      sc->dts[0] = dt / 4.0;
      sc->dts[1] = dt / 3.0;
      sc->dts[2] = dt / 2.0;
      sc->dts[3] = dt;
      const double ch = 0.8 * cfl_number * min_dxyz / dt;
      sc->ch2 = ch * ch;
      sc->tau = 2.0 * dt;
      for (int s = 0; s < 4; ++s) sc->ph_decay[s] = exp(-sc->dts[s] / sc->tau);
    }
  }
}

// ----------------------------------------------------------------------
// Ghost fill along one axis over the full extent of the other two axes
// (so edges and corners hold composed images).  Periodic faces wrap
// (mhd_halo_exchange.hpp:51-265 with the rank as its own neighbour);
// other faces mirror with a per-field sign (boundary_condition.hpp:77-136).
// ----------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256)
fill_axis_kernel(Geom g, FieldPtrs<T> q, int a, int nfields) {
  const int m = g.m[a], t = g.t[a];
  const int b = (a + 1) % 3, c = (a + 2) % 3;
  const long long plane = (long long)g.t[b] * g.t[c];
  const long long total = 2LL * m * plane;
  for (long long lin = blockIdx.x * (long long)blockDim.x + threadIdx.x; lin < total;
       lin += (long long)gridDim.x * blockDim.x) {
    const long long uv = lin % plane;
    const int layer = (int)(lin / plane);  // 0..2m-1
    const int side = layer / m, gi = layer % m;
    const int u = (int)(uv / g.t[c]), v = (int)(uv % g.t[c]);
    int dst, src;
    const bool per = g.periodic[a] != 0;
    if (per) {
      dst = side == 0 ? gi : t - m + gi;
      src = side == 0 ? t - 2 * m + gi : m + gi;
    } else {
      dst = side == 0 ? gi : t - m + gi;
      src = side == 0 ? 2 * m - gi - 1 : t - m - gi - 1;
    }
    const long long base = u * g.st[b] + (long long)v * g.st[c];
    const long long ld = base + dst * g.st[a];
    const long long ls = base + src * g.st[a];
    for (int f = 0; f < nfields; ++f) {
      const T val = q.f[f][ls];
      q.f[f][ld] = per ? val : (T)(g.sign[a][side][f] * val);
    }
  }
}

template __global__ void fill_axis_kernel<double>(Geom, FieldPtrs<double>, int, int);
template __global__ void fill_axis_kernel<float>(Geom, FieldPtrs<float>, int, int);

}  // namespace miso_b200

// ---------------------------------------------------------------------------
// Host-side launchers
// ---------------------------------------------------------------------------
namespace miso_b200 {

static int grid_blocks(long long work, int threads, int sms, int per_sm) {
  long long b = (work + threads - 1) / threads;
  long long cap = (long long)sms * per_sm;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

void launch_fp64_rhs_stage(const Geom &g, const FieldPtrs<const double> &o,
                           const FieldPtrs<const double> &a, const FieldPtrs<double> &r,
                           const StepScalars *sc, int stage, double gm, int sms,
                           cudaStream_t st) {
  const long long nint = (long long)g.n[0] * g.n[1] * g.n[2];
  fp64::rhs_stage_kernel<<<grid_blocks(nint, 128, sms, 16), 128, 0, st>>>(g, o, a, r, sc, stage,
                                                                            gm);
}

void launch_fp64_char_velocity(const Geom &g, const FieldPtrs<const double> &q, double *cc,
                               double gm, double cs_fac, double vv_fac, double ca_fac, int sms,
                               cudaStream_t st) {
  fp64::char_velocity_kernel<<<grid_blocks(g.cells, 256, sms, 8), 256, 0, st>>>(
      g, q, cc, gm, cs_fac, vv_fac, ca_fac);
}

void launch_fp64_av_sweep(const Geom &g, const FieldPtrs<const double> &q,
                          const FieldPtrs<double> &r, const double *cc, const StepScalars *sc,
                          int dir, double ep, double fh, int sms, cudaStream_t st) {
  const long long nint = (long long)g.n[0] * g.n[1] * g.n[2];
  fp64::av_sweep_kernel<<<grid_blocks(nint, 128, sms, 16), 128, 0, st>>>(g, q, r, cc, sc, dir,
                                                                           ep, fh);
}

int cfl_partial_blocks(int sms) { return sms * 4; }

void launch_fp64_cfl(const Geom &g, const FieldPtrs<const double> &q, float *partial,
                     StepScalars *sc, double gm, double cfl_number, double cfl_dx,
                     double min_dxyz, int sms, cudaStream_t st) {
  const int nb = cfl_partial_blocks(sms);
  fp64::cfl_partial_kernel<<<nb, 256, 0, st>>>(g, q, partial, &sc->err, gm, cfl_dx);
  cfl_finalize_kernel<<<1, 1024, 0, st>>>(partial, nb, sc, cfl_number, min_dxyz);
}

void launch_cfl_finalize(const float *partial, int nparts, StepScalars *sc, double cfl_number,
                         double min_dxyz, cudaStream_t st) {
  cfl_finalize_kernel<<<1, 1024, 0, st>>>(partial, nparts, sc, cfl_number, min_dxyz);
}

template <typename T>
void launch_fill_ghosts(const Geom &g, const FieldPtrs<T> &q, int nfields, int sms,
                        cudaStream_t st) {
  for (int a = 0; a < 3; ++a) {
    if (!g.s[a]) continue;
    const int b = (a + 1) % 3, c = (a + 2) % 3;
    const long long work = 2LL * g.m[a] * g.t[b] * g.t[c];
    fill_axis_kernel<T><<<grid_blocks(work, 256, sms, 8), 256, 0, st>>>(g, q, a, nfields);
  }
}

template void launch_fill_ghosts<double>(const Geom &, const FieldPtrs<double> &, int, int,
                                         cudaStream_t);
template void launch_fill_ghosts<float>(const Geom &, const FieldPtrs<float> &, int, int,
                                        cudaStream_t);

}  // namespace miso_b200
