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
    rhs_cell(g, o, a, c, dt, ch2, decay, gm, out, sx, sy, sz);
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
