// Shared device-side definitions for the MISO B200 MHD step.
//
// Layout contract (miso/include/miso/array3d.hpp:54-60): every field is a
// separate (i_total, j_total, k_total) array with k fastest; axes of size 1
// are degenerate (margin 0, stride flag 0, inverse spacing 0;
// grid.hpp:67-90).  Field order: ro, vx, vy, vz, bx, by, bz, ei, ph
// (mhd_fields.hpp:17-18) for the primitive FP64 state; the FP32-split state
// holds the conserved set ro, mx, my, mz, bx, by, bz, et, ph.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace miso_b200 {

constexpr int NF = 9;
enum { RO = 0, VX, VY, VZ, BX, BY, BZ, EI, PH };
// conserved aliases used by the FP32-split form
enum { MX = 1, MY = 2, MZ = 3, ET = 7 };

// constants.hpp:8-16 (double values, the same literals the reference folds)
constexpr double INV12 = 1.0 / 12.0;
constexpr double PII4 = 1.0 / (4.0 * 3.14159265358979323846);
constexpr double PII8 = 1.0 / (8.0 * 3.14159265358979323846);

// Geometry of one grid, passed by value to every kernel.
struct Geom {
  int n[3];      // interior cells per axis
  int m[3];      // ghost width per axis (0 on a degenerate axis)
  int t[3];      // total cells per axis (n + 2m)
  int s[3];      // 1 if the axis is non-degenerate
  long long st[3];  // element strides of i, j, k
  long long cells;  // t0 * t1 * t2
  double dsi[3];    // inverse spacing per axis (0 on a degenerate axis)
  int periodic[3];
  float sign[3][2][NF];  // mirror sign on non-periodic faces
  unsigned short negmask[3][2];  // bit f set where sign[a][side][f] < 0 (0 on periodic axes)
  // 1 where the face is shared with a neighbouring shard of a decomposed
  // grid: its ghost layer is filled by the halo exchange, never by an image
  unsigned char ext[3][2];
};

// Built-in source term of the momentum and energy equations (the Source
// concept of mhd_model_base.hpp:131-155): none (EmptySourceTerm), or the
// point gravity at the coordinate origin of the magnetosphere demo
// (demo/mhd3d_magnetosphere/src/src.hpp:17-44).  x / y / z are the cell
// centres per axis (total cells, ghosts included), as grid.hpp:22-31 places
// them.
// The magnetosphere demo's boundary (demo/mhd3d_magnetosphere/src/bc.hpp:
// 39-158) and its masked CFL (timestep.hpp:15-49), for the FP64 form.
struct Magneto {
  int on;        // the boundary runs after every ghost fill
  int mask_cfl;  // the CFL gives the sphere r <= r_inner the speed 1e-10
  double ro_sw, pr_sw, vx_sw, bz_sw;  // solar wind held in the x-inner ghosts
  double r_inner, a0;                 // blend toward `blend` near the sphere
  double ro_floor, pr_floor;
  const double *blend[9];  // primitive state with ghosts (null: zeros)
  const double *x, *y, *z; // cell centres per axis, ghosts included
};

struct Source {
  int kind;  // 0 none, 1 point gravity, 2 a caller's functor (arrays filled per stage)
  double g;  // gravitational constant: force per volume -ro g x / |x|^3
  const double *x, *y, *z;
  // kind 2: src.vx, src.vy, src.vz and src.ei of every cell for the stage
  // at hand (arrays of the field layout), filled by the caller's functor
  const double *arr[4];
};

// Per-step scalars, resident in device memory so a whole step can run
// without a host round trip.  Written by the CFL finalisation kernel (device
// dt) or uploaded by the host (host dt, as Integrator::update(dt) receives
// it).  Mirrors Integrator::divb_parameters_set
// (mhd_integrator_host.hpp:337-341) and runge_kutta_4step's stage factors
// dt/4, dt/3, dt/2, dt (mhd_integrator_host.hpp:258-277).
struct StepScalars {
  double dt;
  double dts[4];
  double ch2;
  double tau;
  double ph_decay[4];  // exp(-dts[s] / tau)
  unsigned int err;    // error bits (MISO_B200_ERR_NONFINITE ...)
  unsigned int pad;
};

constexpr unsigned int ERRBIT_NONFINITE = 1u;
constexpr unsigned int ERRBIT_TIMEOUT = 2u;  // a bounded device-side wait ran out

// utility.hpp:91-124: util::min2/max2/min3/max3 only have float overloads,
// so double operands are rounded to float and the float result widened
// back.  These helpers keep that rounding in device code.
__device__ __forceinline__ double fmin2f(double a, double b) {
  return (double)fminf(__double2float_rn(a), __double2float_rn(b));
}
__device__ __forceinline__ double fmax2f(double a, double b) {
  return (double)fmaxf(__double2float_rn(a), __double2float_rn(b));
}
__device__ __forceinline__ double fmin3f(double a, double b, double c) {
  return (double)fminf(fminf(__double2float_rn(a), __double2float_rn(b)), __double2float_rn(c));
}
__device__ __forceinline__ double fmax3f(double a, double b, double c) {
  return (double)fmaxf(fmaxf(__double2float_rn(a), __double2float_rn(b)), __double2float_rn(c));
}

template <typename T>
struct FieldPtrs {
  T *f[NF];
};

}  // namespace miso_b200
