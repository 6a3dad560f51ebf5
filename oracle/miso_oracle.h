/*
 * miso_oracle.h -- CPU restatement of MISO's explicit ideal-MHD step.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is the checker for the CUDA path in
 * miso_b200/; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  Nothing in the product links or calls it.
 *
 * Parity is pinned: tests/test_oracle_vs_reference.py checks this
 * restatement bit-for-bit against the reference's own host integrator
 * (mhd::Integrator<double, backend::Host>) compiled from its headers into
 * oracle/_ref/, and tests/test_oracle_golden.py checks it against committed
 * fixtures generated from that build plus the reference's own test
 * statements (Sod shock tube accuracy, symmetric boundary index KATs).
 *
 * Layout contract (miso/include/miso/array3d.hpp:54-60): each of the 9
 * fields is a separate (i_total, j_total, k_total) array, k fastest, with
 * `margin` ghost cells on every axis whose size is > 1 (grid.hpp:67-75).
 * Field order: ro, vx, vy, vz, bx, by, bz, ei, ph (mhd_fields.hpp:17-18).
 */
#ifndef MISO_ORACLE_H
#define MISO_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct miso_oracle_desc {
  int i_size, j_size, k_size; /* interior cells per axis */
  int margin;                 /* ghost width on non-degenerate axes (2) */
  double x_min, x_max, y_min, y_max, z_min, z_max;
  int periodic[3];            /* 1 = periodic wrap, 0 = symmetric mirror */
  double sign[3][2][9];       /* mirror sign per axis, side (0 inner, 1 outer), field */
  double gm;                  /* ratio of specific heats */
  double cfl_number;
  double ep, fh;              /* limiter parameters (config_defaults.hpp:24-27) */
  double cs_fac, ca_fac, vv_fac;
  int source;                 /* 0 EmptySourceTerm, 1 point gravity at the origin, 2 a callback, 3 constants */
  double g_grav;              /* its gravitational constant (force -ro g x / |x|^3) */
  /* Boundary: 0 = the mirror / periodic faces above; 1 = the magnetosphere
   * demo's boundary (demo/mhd3d_magnetosphere/src/bc.hpp:39-158): mirror
   * faces, the solar-wind ro, vx, ei, bz fixed in the x-inner ghosts, then on
   * every cell a blend toward `blend` near the sphere r = r_inner and floors
   * on ro and ei.  Non-periodic axes only. */
  int boundary;
  double sw_ro, sw_pr, sw_vx, sw_bz; /* solar_wind: mass_density, gas_pressure, x_velocity_field, z_magnetic_field */
  double r_inner, a0;                /* magnetosphere: radius, a0 */
  double ro_floor, pr_floor;         /* floor: ro_floor, pr_floor */
  const double *blend[9];            /* primitive state with ghosts; NULL: zeros */
  int cfl_masked;                    /* 1: the demo's CFL with r <= r_inner masked (timestep.hpp:15-49) */
  /* source 2: a caller's source functor, evaluated before every stage on
   * its argument state (the 9 primitive arrays, ghosts included): it fills
   * src.vx, src.vy, src.vz and src.ei of every cell into s[0..3] (arrays of
   * the same layout) and returns 0.  source 3: the constants src_const
   * (vx, vy, vz, ei) in every cell. */
  int (*src_fn)(void *user, double *const q[9], double *const s[4]);
  void *src_user;
  double src_const[4];
} miso_oracle_desc;

/* Fill every ghost cell of q (9 arrays) from its periodic or mirror image. */
int miso_oracle_fill_ghosts(const miso_oracle_desc *d, double *const q[9]);

/* CFL time step with the reference's float-rounded minimum. */
double miso_oracle_cfl(const miso_oracle_desc *d, double *const q[9]);

/* One RHS stage: rslt = orgn + dt * R(argm) on interior cells. */
int miso_oracle_stage(const miso_oracle_desc *d, double *const orgn[9],
                      double *const argm[9], double *const rslt[9], double dt,
                      double ch_divb_square, double tau_divb);

/* Artificial viscosity (cc from q, sweeps x,y,z, ghost fill after each). */
int miso_oracle_av(const miso_oracle_desc *d, double *const q[9], double dt);

/* One full step with a given dt (RK4 + AV). */
int miso_oracle_update(const miso_oracle_desc *d, double *const q[9], double dt);

/* nsteps of (cfl, update); optionally fill ghosts first; dt_out[n] per step. */
int miso_oracle_run(const miso_oracle_desc *d, double *const q[9], int nsteps,
                    int fill_first, double *dt_out);

/* Grid axis (0=x,1=y,2=z): cell centres, spacings, inverse spacings. */
int miso_oracle_axis(const miso_oracle_desc *d, int axis, double *s,
                     double *ds, double *dsi);

/* Global minimum spacing as the reference forms it (float-rounded). */
double miso_oracle_min_dxyz(const miso_oracle_desc *d);

#ifdef __cplusplus
}
#endif
#endif
