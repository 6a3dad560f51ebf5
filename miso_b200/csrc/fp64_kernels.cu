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
#include "fp64_device.cuh"
#include "kernels.h"

namespace miso_b200 {
namespace fp64 {

// One Runge-Kutta stage: rslt = orgn + dt * R(argm) on interior cells,
// mhd_integrator_host.hpp:106-244 expression by expression.
__global__ void __launch_bounds__(128)
rhs_stage_kernel(Geom g, FieldPtrs<const double> o, FieldPtrs<const double> a,
                 FieldPtrs<double> r, const StepScalars *__restrict__ sc, int stage, double gm,
                 Source src) {
  const long long nint = (long long)g.n[0] * g.n[1] * g.n[2];
  const double dt = sc->dts[stage];
  const double ch2 = sc->ch2;
  const double decay = sc->ph_decay[stage];
  for (long long lin = blockIdx.x * (long long)blockDim.x + threadIdx.x; lin < nint;
       lin += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(lin % g.n[2]) + g.m[2];
    const long long r1 = lin / g.n[2];
    const int j = (int)(r1 % g.n[1]) + g.m[1];
    const int i = (int)(r1 / g.n[1]) + g.m[0];
    const long long c = i * g.st[0] + j * g.st[1] + k;

    double out[NF], sx, sy, sz;
    source_force(src, a, c, i, j, k, sx, sy, sz);
    rhs_cell(g, o, a, c, dt, ch2, decay, gm, out, sx, sy, sz, source_heat(src, c));
#pragma unroll
    for (int f = 0; f < NF; ++f) r.f[f][c] = out[f];
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

// One directional sweep (mhd_artificial_viscosity_host.hpp:70-348) on the
// interior cells; ghost cells are refilled from their images afterwards.
__global__ void __launch_bounds__(128)
av_sweep_kernel(Geom g, FieldPtrs<const double> q, FieldPtrs<double> r,
                const double *__restrict__ cc, const StepScalars *__restrict__ sc, int dir,
                double ep, double fh) {
  const long long nint = (long long)g.n[0] * g.n[1] * g.n[2];
  const double dt = sc->dt;
  for (long long lin = blockIdx.x * (long long)blockDim.x + threadIdx.x; lin < nint;
       lin += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(lin % g.n[2]) + g.m[2];
    const long long r1 = lin / g.n[2];
    const int j = (int)(r1 % g.n[1]) + g.m[1];
    const int i = (int)(r1 / g.n[1]) + g.m[0];
    const long long c = i * g.st[0] + j * g.st[1] + k;
    double out[NF];
    av_cell(g, q, cc, c, dir, dt, ep, fh, out);
#pragma unroll
    for (int f = 0; f < NF; ++f) r.f[f][c] = out[f];
  }
}


// A viscosity sweep marching along the sweep axis: a warp owns 32
// neighbouring lines (along `lane_ax`) and walks a chunk of L cells of them
// along `dir`, carrying the limited variables, their slopes and the face
// fluxes of the previous cells in registers, so each slope and each face
// flux is formed once instead of three and two times.  The arguments of
// every dqq_eval and flux_core call are the per-cell sweep's (av_cell), so
// every output is bit for bit the same.  Interior cells only; ghost cells
// along `dir` are read as neighbours.
__global__ void __launch_bounds__(128)
av_march_kernel(Geom g, FieldPtrs<const double> q, FieldPtrs<double> r,
                const double *__restrict__ cc, const StepScalars *__restrict__ sc, int dir,
                int lane_ax, int line_ax, double ep, double fh, int L) {
  const long long sD = g.st[dir], sL = g.st[lane_ax], sU = g.st[line_ax];
  const int nD = g.n[dir], nL = g.n[lane_ax], nU = g.n[line_ax];
  const int lane = threadIdx.x & 31;
  const int lblocks = (nL + 31) / 32;
  const int chunks = (nD + L - 1) / L;
  const long long items = (long long)lblocks * nU * chunks;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  const double dt = sc->dt, dsi = g.dsi[dir];
  for (long long wi = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; wi < items;
       wi += nw) {
    const int lb = (int)(wi % lblocks);
    const long long r1 = wi / lblocks;
    const int u = (int)(r1 % nU);
    const int t0 = (int)(r1 / nU) * L;
    const int t1 = min(nD, t0 + L);
    const int l = lb * 32 + lane;
    const bool active = l < nL;
    const int lc = min(l, nL - 1);  // idle lanes shadow the last line; their values go unused
    const long long base = (long long)(lc + g.m[lane_ax]) * sL +
                           (long long)(u + g.m[line_ax]) * sU + (long long)g.m[dir] * sD;
    // prologue: cells t0-2 .. t0+1 give the slopes at t0-1, t0 and the flux
    // through the face between t0-1 and t0
    double w0[NF], w1[NF], dq0[NF], F0[NF], cc0, cc1;
    {
      double wa[NF], wb[NF], cca, ccb;
      av_load_w(q, cc, base + (long long)(t0 - 2) * sD, wa, cca);
      av_load_w(q, cc, base + (long long)(t0 - 1) * sD, wb, ccb);
      av_load_w(q, cc, base + (long long)t0 * sD, w0, cc0);
      av_load_w(q, cc, base + (long long)(t0 + 1) * sD, w1, cc1);
#pragma unroll
      for (int n = 0; n < NF; ++n) {
        const double dqm = dqq_eval(wa[n], wb[n], w0[n], ep);
        dq0[n] = dqq_eval(wb[n], w0[n], w1[n], ep);
        F0[n] = flux_core(wb[n], w0[n], dqm, dq0[n], 0.5 * (ccb + cc0), fh);
      }
    }
    for (int t = t0; t < t1; ++t) {
      const long long c = base + (long long)t * sD;
      double wp[NF], ccp;
      av_load_w(q, cc, c + 2 * sD, wp, ccp);
      double dF[NF];
#pragma unroll
      for (int n = 0; n < NF; ++n) {
        const double dq1 = dqq_eval(w0[n], w1[n], wp[n], ep);
        const double F1 = flux_core(w0[n], w1[n], dq0[n], dq1, 0.5 * (cc0 + cc1), fh);
        dF[n] = F1 - F0[n];
        F0[n] = F1;
        dq0[n] = dq1;
      }
      if (active) {
        // the per-cell sweep's update (av_cell), cell t holding w0
        const double ro_c = w0[0];
        const double ro = ro_c - dF[0] * dsi * dt;
        double v[3], b[3];
#pragma unroll
        for (int e = 0; e < 3; ++e) v[e] = (w0[1 + e] - dF[1 + e] * dsi * dt) / ro;
#pragma unroll
        for (int e = 0; e < 3; ++e) b[e] = w0[4 + e] - dF[4 + e] * dsi * dt;
        const double ph = w0[7] - dF[7] * dsi * dt;
        const double ei_c = __ldg(q.f[EI] + c);
        const double vx_c = __ldg(q.f[VX] + c), vy_c = __ldg(q.f[VY] + c),
                     vz_c = __ldg(q.f[VZ] + c);
        const double Et = ro_c * ei_c + 0.5 * ro_c * (vx_c * vx_c + vy_c * vy_c + vz_c * vz_c) +
                          PII8 * (w0[4] * w0[4] + w0[5] * w0[5] + w0[6] * w0[6]);
        const double ei = (Et - dF[8] * dsi * dt -
                           0.5 * ro * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) -
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
#pragma unroll
      for (int n = 0; n < NF; ++n) {
        w0[n] = w1[n];
        w1[n] = wp[n];
      }
      cc0 = cc1;
      cc1 = ccp;
    }
  }
}

// The z sweep (the contiguous axis): a warp loads 32 consecutive cells of a
// row and updates the inner 28; each lane forms the slope and the upper
// face flux of its own cell once and takes its neighbours' by warp
// shuffles -- the same dqq_eval and flux_core arguments as the per-cell
// sweep, so every output is bit for bit the same.
__global__ void __launch_bounds__(128)
av_z_shfl_kernel(Geom g, FieldPtrs<const double> q, FieldPtrs<double> r,
                 const double *__restrict__ cc, const StepScalars *__restrict__ sc, double ep,
                 double fh) {
  const int lane = threadIdx.x & 31;
  const int nk = g.n[2];
  const int segs = (nk + 27) / 28;
  const long long work = (long long)g.n[0] * g.n[1] * segs;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  const double dt = sc->dt, dsi = g.dsi[2];
  for (long long wi = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; wi < work;
       wi += nw) {
    const int sg = (int)(wi % segs);
    const long long row = wi / segs;
    const int j = (int)(row % g.n[1]) + g.m[1];
    const int i = (int)(row / g.n[1]) + g.m[0];
    const int k = sg * 28 + lane - 2;  // interior k of this lane (-2 .. nk+1 read)
    const int kc = min(k, nk + 1);
    const long long c = i * g.st[0] + j * g.st[1] + kc + g.m[2];
    double w[NF], ccv;
    av_load_w(q, cc, c, w, ccv);
    const double cc_up = __shfl_down_sync(0xffffffffu, ccv, 1);
    double dF[NF];
#pragma unroll
    for (int n = 0; n < NF; ++n) {
      const double wm = __shfl_up_sync(0xffffffffu, w[n], 1);
      const double wp = __shfl_down_sync(0xffffffffu, w[n], 1);
      const double dq = dqq_eval(wm, w[n], wp, ep);
      const double dq_up = __shfl_down_sync(0xffffffffu, dq, 1);
      const double Fup = flux_core(w[n], wp, dq, dq_up, 0.5 * (ccv + cc_up), fh);
      const double Fdw = __shfl_up_sync(0xffffffffu, Fup, 1);
      dF[n] = Fup - Fdw;
    }
    if (lane >= 2 && lane < 30 && k < nk) {
      const double ro_c = w[0];
      const double ro = ro_c - dF[0] * dsi * dt;
      double v[3], b[3];
#pragma unroll
      for (int e = 0; e < 3; ++e) v[e] = (w[1 + e] - dF[1 + e] * dsi * dt) / ro;
#pragma unroll
      for (int e = 0; e < 3; ++e) b[e] = w[4 + e] - dF[4 + e] * dsi * dt;
      const double ph = w[7] - dF[7] * dsi * dt;
      const double ei_c = __ldg(q.f[EI] + c);
      const double vx_c = __ldg(q.f[VX] + c), vy_c = __ldg(q.f[VY] + c),
                   vz_c = __ldg(q.f[VZ] + c);
      const double Et = ro_c * ei_c + 0.5 * ro_c * (vx_c * vx_c + vy_c * vy_c + vz_c * vz_c) +
                        PII8 * (w[4] * w[4] + w[5] * w[5] + w[6] * w[6]);
      const double ei = (Et - dF[8] * dsi * dt -
                         0.5 * ro * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) -
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
}

// ----------------------------------------------------------------------
// CFL (mhd_integrator_host.hpp:303-334): per-block float-rounded minimum of
// cfl * min3(dx,dy,dz) / (cs + |v| + ca) over the interior, then one block
// folds the partials and derives the step scalars on the device.
// ----------------------------------------------------------------------
__global__ void __launch_bounds__(256)
cfl_partial_kernel(Geom g, FieldPtrs<const double> q, float *__restrict__ partial,
                   unsigned int *__restrict__ err, double gm, double cfl_dx, Magneto mg) {
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
    double total_vel = cs + vv + ca;
    bad |= !isfinite(total_vel);
    if (mg.mask_cfl) {
      // the magnetosphere demo's CFL (timestep.hpp:15-49): the sphere
      // r <= r_inner moves at slow_speed 1e-10
      const double x = mg.x[i], y = mg.y[j], z = mg.z[k];
      const double rr = sqrt(x * x + y * y + z * z);
      const double mask = rr > mg.r_inner ? 1.0 : 0.0;
      total_vel = total_vel * mask + 1.e-10 * (1.0 - mask);
    }
    // util::min2(dt, x): both sides through float; fminf ignores a NaN side.
    best = fminf(best, __double2float_rn(cfl_dx / total_vel));
    bad |= !(ro > 0.0) || !(ei >= 0.0);
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
    if (g.ext[a][side]) continue;  // a face shared with a neighbouring shard
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

// The magnetosphere demo's boundary after the mirror fill (bc.hpp:39-158):
// the x-inner ghosts of ro, vx, ei, bz take the solar wind (a physical face
// only), then every cell, ghosts included, is blended toward the reference
// state with weight f = a0 h / (a0 h + 1), h = max2(0, (r / r_inner)^2 - 1),
// and floored: ro = max2(ro, ro_floor), ei = max2(ei, pr_floor / (gm - 1) /
// ro).  max2 is the float-rounded util::max2 (utility.hpp:91-124).  The
// mirror faces come first in a different face order than the demo's; that
// changes edge and corner ghosts only, which no stencil reads.
__global__ void __launch_bounds__(256)
magneto_bc_kernel(Geom g, FieldPtrs<double> q, Magneto mg, double gm) {
  const long long cells = g.cells;
  const bool inflow = g.s[0] && !g.periodic[0] && !g.ext[0][0];
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < cells;
       c += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(c % g.t[2]);
    const long long r1 = c / g.t[2];
    const int j = (int)(r1 % g.t[1]);
    const int i = (int)(r1 / g.t[1]);
    double u[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) u[f] = q.f[f][c];
    if (inflow && i < g.m[0]) {
      u[RO] = mg.ro_sw;
      u[VX] = mg.vx_sw;
      u[EI] = mg.pr_sw / (gm - 1.0) / u[RO];
      u[BZ] = mg.bz_sw;
    }
    const double x = mg.x[i], y = mg.y[j], z = mg.z[k];
    const double rr = sqrt(x * x + y * y + z * z);
    const double r1n = rr / mg.r_inner;
    const double hh = fmax2f(0.0, r1n * r1n - 1.0);
    const double w = mg.a0 * hh / (mg.a0 * hh + 1.0);
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      const double b = mg.blend[f] ? mg.blend[f][c] : 0.0;
      u[f] = u[f] * w + b * (1.0 - w);
    }
    u[RO] = fmax2f(u[RO], mg.ro_floor);
    u[EI] = fmax2f(u[EI], mg.pr_floor / (gm - 1.0) / u[RO]);
#pragma unroll
    for (int f = 0; f < NF; ++f) q.f[f][c] = u[f];
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
                           const StepScalars *sc, int stage, double gm, const Source &src,
                           int sms, cudaStream_t st) {
  const long long nint = (long long)g.n[0] * g.n[1] * g.n[2];
  fp64::rhs_stage_kernel<<<grid_blocks(nint, 128, sms, 16), 128, 0, st>>>(g, o, a, r, sc, stage,
                                                                            gm, src);
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
  // the marching sweep wherever the sweep axis and a lane axis are real;
  // the per-cell sweep elsewhere (a degenerate sweep still rounds: v =
  // (ro v) / ro)
  const int lane_ax = dir == 2 ? -1 : (g.s[2] ? 2 : (dir == 0 ? 1 : 0));
  if (dir == 2 && g.s[2] && g.n[2] >= 4) {
    fp64::av_z_shfl_kernel<<<sms * 8, 128, 0, st>>>(g, q, r, cc, sc, ep, fh);
    return;
  }
  if (dir < 2 && g.s[dir] && lane_ax >= 0 && g.s[lane_ax] && g.n[dir] >= 4) {
    const int line_ax = 3 - dir - lane_ax;
    const int L = 64;
    fp64::av_march_kernel<<<sms * 8, 128, 0, st>>>(g, q, r, cc, sc, dir, lane_ax, line_ax, ep,
                                                   fh, L);
    return;
  }
  fp64::av_sweep_kernel<<<grid_blocks(nint, 128, sms, 16), 128, 0, st>>>(g, q, r, cc, sc, dir,
                                                                           ep, fh);
}

int cfl_partial_blocks(int sms) { return sms * 4; }

void launch_fp64_cfl(const Geom &g, const FieldPtrs<const double> &q, float *partial,
                     StepScalars *sc, double gm, double cfl_number, double cfl_dx,
                     double min_dxyz, const Magneto &mg, int sms, cudaStream_t st) {
  const int nb = cfl_partial_blocks(sms);
  fp64::cfl_partial_kernel<<<nb, 256, 0, st>>>(g, q, partial, &sc->err, gm, cfl_dx, mg);
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

void launch_magneto_bc(const Geom &g, const FieldPtrs<double> &q, const Magneto &mg, double gm,
                       int sms, cudaStream_t st) {
  magneto_bc_kernel<<<grid_blocks(g.cells, 256, sms, 8), 256, 0, st>>>(g, q, mg, gm);
}

template void launch_fill_ghosts<double>(const Geom &, const FieldPtrs<double> &, int, int,
                                         cudaStream_t);
template void launch_fill_ghosts<float>(const Geom &, const FieldPtrs<float> &, int, int,
                                        cudaStream_t);

}  // namespace miso_b200
