/*
 * miso_oracle.c -- CPU restatement of MISO's explicit ideal-MHD step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): see
 * miso_oracle.h.  Every expression below keeps the reference's operand order
 * so that, compiled with -O2 -ffp-contract=off on x86-64 (no FMA), results
 * are bit-identical to the reference's own double-precision host path.
 *
 * Reference files (paths inside the MISO project):
 *   miso/include/miso/mhd_integrator.hpp:14-58            4th-order central difference
 *   miso/include/miso/mhd_integrator_host.hpp:57-247      update_sc4 (RHS + stage update)
 *   miso/include/miso/mhd_integrator_host.hpp:258-277     runge_kutta_4step
 *   miso/include/miso/mhd_integrator_host.hpp:280-300     apply_artificial_viscosity
 *   miso/include/miso/mhd_integrator_host.hpp:303-341     cfl, divb_parameters_set
 *   miso/include/miso/mhd_artificial_viscosity_host.hpp:51-348
 *   miso/include/miso/limiter.hpp:11-37                   dqq_eval, flux_core
 *   miso/include/miso/utility.hpp:91-124                  min/max through float
 *   miso/include/miso/eos.hpp:25-42                       gas_pressure, sound_speed
 *   miso/include/miso/boundary_condition.hpp:77-136       symmetric mirror
 *   miso/include/miso/mhd_halo_exchange.hpp:51-265        periodic wrap (1 rank)
 *   demo/mhd3d_magnetosphere/src/bc.hpp:39-158            magnetosphere boundary
 *   demo/mhd3d_magnetosphere/src/timestep.hpp:15-49       masked CFL
 *   miso/include/miso/grid.hpp:22-99,241                  axes, min_dxyz
 *   miso/include/miso/constants.hpp:8-16                  inv12, pii4, pii8
 */
#include "miso_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NF 9
enum { RO = 0, VX, VY, VZ, BX, BY, BZ, EI, PH };

static const double INV12 = 1.0 / 12.0;               /* constants.hpp:8-9 */
static const double PII4 = 1.0 / (4.0 * M_PI);        /* constants.hpp:13-14 */
static const double PII8 = 1.0 / (8.0 * M_PI);        /* constants.hpp:16-17 */

/* utility.hpp:91-124: util::min2/max2/min3/max3 resolve to the float-only
 * fmin_safe/fmax_safe, so double arguments are rounded to float first and
 * the float result is widened back. */
static inline double fmin2(double a, double b) { return (double)fminf((float)a, (float)b); }
static inline double fmax2(double a, double b) { return (double)fmaxf((float)a, (float)b); }
static inline double fmin3(double a, double b, double c) {
  return (double)fminf(fminf((float)a, (float)b), (float)c);
}
static inline double fmax3(double a, double b, double c) {
  return (double)fmaxf(fmaxf((float)a, (float)b), (float)c);
}

typedef struct {
  int n[3], m[3], t[3], s[3]; /* size, margin, total, stride flag per axis */
  long st[3];                 /* element strides i,j,k */
  long cells;
  double *ax[3], *dax[3], *daxi[3];
  double min_dxyz;
} geom;

/* grid.hpp:22-31 (UniformAxisProvider) and 53-99 (AxisGrid). */
static void axis_build(int size, int margin, double lo, double hi, double *s,
                       double *ds, double *dsi) {
  if (size == 1) {
    double sp = (hi - lo) / (double)size;
    s[0] = lo + ((double)0 + 0.5) * sp;
    ds[0] = 1.e30;
    dsi[0] = 0.0;
    return;
  }
  int total = size + 2 * margin;
  for (int i = 0; i < total; ++i) {
    int ig = i - margin;
    double sp = (hi - lo) / (double)size;
    s[i] = lo + ((double)ig + 0.5) * sp;
    ds[i] = sp;
    dsi[i] = 1.0 / ds[i];
  }
}

static int geom_init(geom *g, const miso_oracle_desc *d) {
  const int sz[3] = {d->i_size, d->j_size, d->k_size};
  const double lo[3] = {d->x_min, d->y_min, d->z_min};
  const double hi[3] = {d->x_max, d->y_max, d->z_max};
  if (d->margin < 1) return -1;
  for (int a = 0; a < 3; ++a) {
    if (sz[a] <= 0 || !(lo[a] < hi[a])) return -1;
    g->n[a] = sz[a];
    g->s[a] = sz[a] > 1 ? 1 : 0;
    g->m[a] = d->margin * g->s[a];
    g->t[a] = sz[a] + 2 * g->m[a];
    if (g->s[a] && sz[a] < g->m[a]) return -1;
  }
  g->st[2] = 1;
  g->st[1] = g->t[2];
  g->st[0] = (long)g->t[1] * g->t[2];
  g->cells = (long)g->t[0] * g->t[1] * g->t[2];
  for (int a = 0; a < 3; ++a) {
    g->ax[a] = (double *)malloc(sizeof(double) * g->t[a]);
    g->dax[a] = (double *)malloc(sizeof(double) * g->t[a]);
    g->daxi[a] = (double *)malloc(sizeof(double) * g->t[a]);
    axis_build(sz[a], d->margin, lo[a], hi[a], g->ax[a], g->dax[a], g->daxi[a]);
  }
  /* grid.hpp:241: min3 of the first spacing of each axis, through float. */
  g->min_dxyz = fmin3(g->dax[0][0], g->dax[1][0], g->dax[2][0]);
  return 0;
}

static void geom_free(geom *g) {
  for (int a = 0; a < 3; ++a) {
    free(g->ax[a]);
    free(g->dax[a]);
    free(g->daxi[a]);
  }
}

static inline long IDX(const geom *g, int i, int j, int k) {
  return ((long)i * g->t[1] + j) * g->t[2] + k;
}

/* ---------------------------------------------------------------------- */
/* Ghost fill.                                                              */
/* Symmetric faces (boundary_condition.hpp:77-136): ghost g on the inner    */
/* side takes sign * q[2m-g-1]; outer ghost total-m+g takes sign *          */
/* q[total-m-g-1].  Periodic faces (mhd_halo_exchange.hpp:51-265 with the   */
/* rank as its own neighbour): ghost g takes q[total-2m+g], outer ghost      */
/* total-m+g takes q[m+g].  Axes are filled x, then y, then z, each over    */
/* the full extent of the other axes, so edge and corner ghosts hold the    */
/* composed image.  The reference leaves those corners stale; no interior   */
/* update reads them (all stencils are axis-aligned), so interior results  */
/* are unaffected.                                                          */
/* ---------------------------------------------------------------------- */
/* One face (axis a, side 0 inner / 1 outer) for the fields in `mask`. */
static void fill_face(const geom *g, const miso_oracle_desc *d, double *const q[NF], int a,
                      int side, unsigned mask) {
  if (!g->s[a]) return;
  const int m = g->m[a], t = g->t[a];
  const int b = (a + 1) % 3, c = (a + 2) % 3;
  for (int gi = 0; gi < m; ++gi) {
    int dst, src;
    double sgn[NF];
    if (d->periodic[a]) {
      dst = side == 0 ? gi : t - m + gi;
      src = side == 0 ? t - 2 * m + gi : m + gi;
      for (int f = 0; f < NF; ++f) sgn[f] = 1.0;
    } else {
      dst = side == 0 ? gi : t - m + gi;
      src = side == 0 ? 2 * m - gi - 1 : t - m - gi - 1;
      for (int f = 0; f < NF; ++f) sgn[f] = d->sign[a][side][f];
    }
    for (int u = 0; u < g->t[b]; ++u) {
      for (int v = 0; v < g->t[c]; ++v) {
        int id[3], is_[3];
        id[a] = dst; id[b] = u; id[c] = v;
        is_[a] = src; is_[b] = u; is_[c] = v;
        long ld = IDX(g, id[0], id[1], id[2]);
        long ls = IDX(g, is_[0], is_[1], is_[2]);
        for (int f = 0; f < NF; ++f)
          if ((mask >> f) & 1u) q[f][ld] = sgn[f] * q[f][ls];
      }
    }
  }
}

static void fill_axis(const geom *g, const miso_oracle_desc *d, double *const q[NF], int a) {
  fill_face(g, d, q, a, 0, 0x1ffu);
  fill_face(g, d, q, a, 1, 0x1ffu);
}

/* ---------------------------------------------------------------------- */
/* The magnetosphere demo's boundary (demo/mhd3d_magnetosphere/src/bc.hpp: */
/* 39-158), in its order: mirror on x outer, y inner / outer, z inner /     */
/* outer (all fields), x inner (vy, vz, bx, by, ph); the x-inner ghosts of   */
/* ro, vx, ei, bz set to the solar wind; then on every cell, ghosts         */
/* included, ro..ph blended toward the `blend` state with weight f = a0 h / */
/* (a0 h + 1), h = max2(0, (r / r_inner)^2 - 1), and the floors             */
/* ro = max2(ro, ro_floor), ei = max2(ei, pr_floor / (gm - 1) / ro).  max2  */
/* is the reference's float-rounded util::max2.                             */
/* ---------------------------------------------------------------------- */
static void magnetosphere_bc(const geom *g, const miso_oracle_desc *d, double *const q[NF]) {
  fill_face(g, d, q, 0, 1, 0x1ffu);
  fill_face(g, d, q, 1, 0, 0x1ffu);
  fill_face(g, d, q, 1, 1, 0x1ffu);
  fill_face(g, d, q, 2, 0, 0x1ffu);
  fill_face(g, d, q, 2, 1, 0x1ffu);
  fill_face(g, d, q, 0, 0, (1u << VY) | (1u << VZ) | (1u << BX) | (1u << BY) | (1u << PH));
  if (g->s[0])
    for (int i = 0; i < g->m[0]; ++i)
      for (int j = 0; j < g->t[1]; ++j)
        for (int k = 0; k < g->t[2]; ++k) {
          const long c = IDX(g, i, j, k); /* the inner ghosts i < m (symmetric_index) */
          q[RO][c] = d->sw_ro;
          q[VX][c] = d->sw_vx;
          q[EI][c] = d->sw_pr / (d->gm - 1.0) / q[RO][c];
          q[BZ][c] = d->sw_bz;
        }
  for (int i = 0; i < g->t[0]; ++i)
    for (int j = 0; j < g->t[1]; ++j)
      for (int k = 0; k < g->t[2]; ++k) {
        const long c = IDX(g, i, j, k);
        const double x = g->ax[0][i], y = g->ax[1][j], z = g->ax[2][k];
        const double rr = sqrt(x * x + y * y + z * z);
        const double r1 = rr / d->r_inner;
        const double hh = fmax2(0.0, r1 * r1 - 1.0);
        const double f = d->a0 * hh / (d->a0 * hh + 1.0);
        for (int v = 0; v < NF; ++v) {
          const double b = d->blend[v] ? d->blend[v][c] : 0.0;
          q[v][c] = q[v][c] * f + b * (1.0 - f);
        }
        q[RO][c] = fmax2(q[RO][c], d->ro_floor);
        q[EI][c] = fmax2(q[EI][c], d->pr_floor / (d->gm - 1.0) / q[RO][c]);
      }
}

/* Integrator::apply_boundary_condition: the boundary functor, then the halo
 * exchange (periodic faces of one rank). */
static void fill_ghosts(const geom *g, const miso_oracle_desc *d, double *const q[NF]) {
  if (d->boundary == 1) {
    magnetosphere_bc(g, d, q);
    return;
  }
  for (int a = 0; a < 3; ++a) fill_axis(g, d, q, a);
}

/* ---------------------------------------------------------------------- */
/* 4th-order central difference (mhd_integrator.hpp:14-58).                 */
/* ---------------------------------------------------------------------- */
static inline double D1(const double *a, long c, long s, double dsi) {
  return (-a[c + 2 * s] + 8.0 * a[c + s] - 8.0 * a[c - s] + a[c - 2 * s]) * INV12 * dsi;
}
static inline double D2(const double *a, const double *b, long c, long s, double dsi) {
  return (-a[c + 2 * s] * b[c + 2 * s] + 8.0 * a[c + s] * b[c + s] -
          8.0 * a[c - s] * b[c - s] + a[c - 2 * s] * b[c - 2 * s]) * INV12 * dsi;
}
static inline double D3(const double *a, const double *b, const double *e, long c,
                        long s, double dsi) {
  return (-a[c + 2 * s] * b[c + 2 * s] * e[c + 2 * s] +
          8.0 * a[c + s] * b[c + s] * e[c + s] -
          8.0 * a[c - s] * b[c - s] * e[c - s] +
          a[c - 2 * s] * b[c - 2 * s] * e[c - 2 * s]) * INV12 * dsi;
}

/* mhd_integrator_host.hpp:57-247 with the derived arrays of eos.hpp:25-31
 * and lines 64-89.  The source term (src.vx/vy/vz inside dt * (...), src.ei
 * added to the new total energy, lines 134-168 and 241) is the empty one
 * (adds 0.0), the point gravity of the magnetosphere demo
 * (demo/mhd3d_magnetosphere/src/src.hpp:17-44): force per volume
 * -ro g x / |x|^3 on the stage's argument state, no heating -- or a
 * caller's functor (its four values per cell, from the argument state),
 * or four constants.  Returns the callback's nonzero status. */
static int stage(const geom *g, const miso_oracle_desc *d, double *const o[NF],
                 double *const a[NF], double *const r[NF], double dt, double ch2,
                 double tau, double *pr, double *bb, double *ht, double *vb) {
  const double gm = d->gm;
  double *s4[4] = {NULL, NULL, NULL, NULL};
  if (d->source == 2) {
    double *blk = (double *)malloc(sizeof(double) * 4 * (size_t)g->cells);
    if (!blk) return -1;
    for (int q = 0; q < 4; ++q) {
      s4[q] = blk + (size_t)q * g->cells;
      for (long n = 0; n < g->cells; ++n) s4[q][n] = 0.0;
    }
    const int rc = d->src_fn ? d->src_fn(d->src_user, a, s4) : -1;
    if (rc) {
      free(blk);
      return rc;
    }
  }
  for (long n = 0; n < g->cells; ++n) {
    pr[n] = (gm - 1.0) * a[RO][n] * a[EI][n];
    bb[n] = a[BX][n] * a[BX][n] + a[BY][n] * a[BY][n] + a[BZ][n] * a[BZ][n];
    ht[n] = +a[RO][n] * a[EI][n] + pr[n] + bb[n] * PII4 +
            0.5 * a[RO][n] * (+a[VX][n] * a[VX][n] + a[VY][n] * a[VY][n] + a[VZ][n] * a[VZ][n]);
    vb[n] = +a[VX][n] * a[BX][n] + a[VY][n] * a[BY][n] + a[VZ][n] * a[BZ][n];
  }
  const long si = g->st[0] * g->s[0], sj = g->st[1] * g->s[1], sk = g->st[2] * g->s[2];
  const double *ro = a[RO], *vx = a[VX], *vy = a[VY], *vz = a[VZ];
  const double *bx = a[BX], *by = a[BY], *bz = a[BZ], *ph = a[PH];
  const double src = 0.0; /* EmptySourceTerm (mhd_model_base.hpp:131-155), and src.ei */
  for (int i = g->m[0]; i < g->t[0] - g->m[0]; ++i) {
    const double dxi = g->daxi[0][i];
    for (int j = g->m[1]; j < g->t[1] - g->m[1]; ++j) {
      const double dyi = g->daxi[1][j];
      for (int k = g->m[2]; k < g->t[2] - g->m[2]; ++k) {
        const double dzi = g->daxi[2][k];
        const long c = IDX(g, i, j, k);
        double sx = src, sy = src, sz = src, se = src;
        if (d->source == 2) {
          sx = s4[0][c];
          sy = s4[1][c];
          sz = s4[2][c];
          se = s4[3][c];
        } else if (d->source == 3) {
          sx = d->src_const[0];
          sy = d->src_const[1];
          sz = d->src_const[2];
          se = d->src_const[3];
        } else if (d->source == 1) {
          const double X = g->ax[0][i], Y = g->ax[1][j], Z = g->ax[2][k];
          const double rr = sqrt(X * X + Y * Y + Z * Z);
          const double r3 = rr * rr * rr; /* util::pow3 */
          sx = -a[RO][c] * d->g_grav * X / r3;
          sy = -a[RO][c] * d->g_grav * Y / r3;
          sz = -a[RO][c] * d->g_grav * Z / r3;
        }

        r[RO][c] = o[RO][c] + dt * (-D2(ro, vx, c, si, dxi) - D2(ro, vy, c, sj, dyi) -
                                    D2(ro, vz, c, sk, dzi));

        r[VX][c] = (o[RO][c] * o[VX][c] +
                    dt * (-D3(ro, vx, vx, c, si, dxi) - D3(ro, vx, vy, c, sj, dyi) -
                          D3(ro, vx, vz, c, sk, dzi) - D1(pr, c, si, dxi) -
                          D1(bb, c, si, dxi) * PII8 +
                          PII4 * (+D2(bx, bx, c, si, dxi) + D2(bx, by, c, sj, dyi) +
                                  D2(bx, bz, c, sk, dzi)) +
                          sx)) / r[RO][c];

        r[VY][c] = (o[RO][c] * o[VY][c] +
                    dt * (-D3(ro, vy, vx, c, si, dxi) - D3(ro, vy, vy, c, sj, dyi) -
                          D3(ro, vy, vz, c, sk, dzi) - D1(pr, c, sj, dyi) -
                          D1(bb, c, sj, dyi) * PII8 +
                          PII4 * (+D2(by, bx, c, si, dxi) + D2(by, by, c, sj, dyi) +
                                  D2(by, bz, c, sk, dzi)) +
                          sy)) / r[RO][c];

        r[VZ][c] = (o[RO][c] * o[VZ][c] +
                    dt * (-D3(ro, vz, vx, c, si, dxi) - D3(ro, vz, vy, c, sj, dyi) -
                          D3(ro, vz, vz, c, sk, dzi) - D1(pr, c, sk, dzi) -
                          D1(bb, c, sk, dzi) * PII8 +
                          PII4 * (+D2(bz, bx, c, si, dxi) + D2(bz, by, c, sj, dyi) +
                                  D2(bz, bz, c, sk, dzi)) +
                          sz)) / r[RO][c];

        r[BX][c] = o[BX][c] + dt * (-D2(vy, bx, c, sj, dyi) - D2(vz, bx, c, sk, dzi) +
                                    D2(vx, by, c, sj, dyi) + D2(vx, bz, c, sk, dzi) -
                                    D1(ph, c, si, dxi));

        r[BY][c] = o[BY][c] + dt * (-D2(vx, by, c, si, dxi) - D2(vz, by, c, sk, dzi) +
                                    D2(vy, bx, c, si, dxi) + D2(vy, bz, c, sk, dzi) -
                                    D1(ph, c, sj, dyi));

        r[BZ][c] = o[BZ][c] + dt * (-D2(vx, bz, c, si, dxi) - D2(vy, bz, c, sj, dyi) +
                                    D2(vz, bx, c, si, dxi) + D2(vz, by, c, sj, dyi) -
                                    D1(ph, c, sk, dzi));

        r[PH][c] = (o[PH][c] + dt * ch2 * (-D1(bx, c, si, dxi) - D1(by, c, sj, dyi) -
                                           D1(bz, c, sk, dzi))) * exp(-dt / tau);

        const double Et = +o[RO][c] * o[EI][c] +
                          0.5 * o[RO][c] * (+o[VX][c] * o[VX][c] + o[VY][c] * o[VY][c] +
                                            o[VZ][c] * o[VZ][c]) +
                          PII8 * (+o[BX][c] * o[BX][c] + o[BY][c] * o[BY][c] +
                                  o[BZ][c] * o[BZ][c]);

        r[EI][c] = (Et +
                    dt * (-D2(ht, vx, c, si, dxi) - D2(ht, vy, c, sj, dyi) -
                          D2(ht, vz, c, sk, dzi) +
                          PII4 * (+D2(vb, bx, c, si, dxi) + D2(vb, by, c, sj, dyi) +
                                  D2(vb, bz, c, sk, dzi))) -
                    0.5 * r[RO][c] * (+r[VX][c] * r[VX][c] + r[VY][c] * r[VY][c] +
                                      r[VZ][c] * r[VZ][c]) -
                    PII8 * (+r[BX][c] * r[BX][c] + r[BY][c] * r[BY][c] +
                            r[BZ][c] * r[BZ][c]) +
                    se) / r[RO][c];
      }
    }
  }
  if (s4[0]) free(s4[0]);
  return 0;
}

/* ---------------------------------------------------------------------- */
/* Limiter (limiter.hpp:11-37).                                             */
/* ---------------------------------------------------------------------- */
static inline double dqq_eval(double qq_dw, double qq_cn, double qq_up, double ep) {
  double dqq_dw = qq_cn - qq_dw;
  double dqq_up = qq_up - qq_cn;
  double dqq_cn = (qq_up - qq_dw) * 0.5;
  double dqq_max = fmax3(ep * dqq_dw, ep * dqq_up, dqq_cn);
  double dqq_min = fmin3(ep * dqq_dw, ep * dqq_up, dqq_cn);
  return fmin2(0.0, dqq_max) + fmax2(0.0, dqq_min);
}

static inline double flux_core(double qq_dw, double qq_up, double dqq_dw,
                               double dqq_up, double cc, double fh) {
  double qql = qq_dw + 0.5 * dqq_dw;
  double qqr = qq_up - 0.5 * dqq_up;
  double dqq = qq_up - qq_dw;
  dqq = copysign(fmax2(fabs(dqq), 1e-20), dqq);
  double ra = fmin2(1.0, (qqr - qql) / dqq);
  double pp = (0.5 + copysign(0.5, ra)) * fmax2(0.0, 1.0 + fh * (ra - 1.0));
  return -0.5 * cc * pp * (qqr - qql);
}

/* mhd_artificial_viscosity_host.hpp:51-68 with eos.hpp:36-42. */
static void char_velocity(const geom *g, const miso_oracle_desc *d, double *const q[NF],
                          double *cc) {
  const double gm = d->gm;
  for (long n = 0; n < g->cells; ++n) {
    double cs = sqrt(gm * (gm - 1.0) * q[EI][n]);
    double vv = sqrt(q[VX][n] * q[VX][n] + q[VY][n] * q[VY][n] + q[VZ][n] * q[VZ][n]);
    double ca = sqrt((q[BX][n] * q[BX][n] + q[BY][n] * q[BY][n] + q[BZ][n] * q[BZ][n]) /
                     q[RO][n] * PII4);
    cc[n] = cs * d->cs_fac + vv * d->vv_fac + ca * d->ca_fac;
  }
}

/* Limited diffusive flux difference of the five values w[0..4] centred on
 * w[2] (mhd_artificial_viscosity_host.hpp:120-141 pattern, per field). */
static inline double av_dflux(const double w[5], double ccl, double ccc, double ccr,
                              double ep, double fh) {
  double dqq_dw = dqq_eval(w[0], w[1], w[2], ep);
  double dqq_cn = dqq_eval(w[1], w[2], w[3], ep);
  double dqq_up = dqq_eval(w[2], w[3], w[4], ep);
  double f_dw = flux_core(w[1], w[2], dqq_dw, dqq_cn, 0.5 * (ccl + ccc), fh);
  double f_up = flux_core(w[2], w[3], dqq_cn, dqq_up, 0.5 * (ccc + ccr), fh);
  return f_up - f_dw;
}

/* mhd_artificial_viscosity_host.hpp:70-348: one directional sweep. */
static void av_sweep(const geom *g, const miso_oracle_desc *d, double *const q[NF],
                     double *const r[NF], const double *cc, int dir, double dt) {
  int lo[3] = {0, 0, 0}, hi[3] = {g->t[0], g->t[1], g->t[2]};
  lo[dir] = 2 * g->s[dir];
  hi[dir] = g->t[dir] - 2 * g->s[dir];
  const long s = g->st[dir] * g->s[dir];
  const double *dsi_ax = g->daxi[dir];
  const double ep = d->ep, fh = d->fh;
  for (int i = lo[0]; i < hi[0]; ++i) {
    for (int j = lo[1]; j < hi[1]; ++j) {
      for (int k = lo[2]; k < hi[2]; ++k) {
        const long c = IDX(g, i, j, k);
        const int ia = dir == 0 ? i : (dir == 1 ? j : k);
        const double dsi = dsi_ax[ia * g->s[dir]];
        const double ccl = cc[c - s], ccc = cc[c], ccr = cc[c + s];
        double w[5];
        long p[5];
        for (int t = 0; t < 5; ++t) p[t] = c + (t - 2) * s;

        for (int t = 0; t < 5; ++t) w[t] = q[RO][p[t]];
        double dro = av_dflux(w, ccl, ccc, ccr, ep, fh);
        r[RO][c] = q[RO][c] - dro * dsi * dt;

        for (int t = 0; t < 5; ++t) w[t] = q[RO][p[t]] * q[VX][p[t]];
        double dmx = av_dflux(w, ccl, ccc, ccr, ep, fh);
        r[VX][c] = (q[RO][c] * q[VX][c] - dmx * dsi * dt) / r[RO][c];

        for (int t = 0; t < 5; ++t) w[t] = q[RO][p[t]] * q[VY][p[t]];
        double dmy = av_dflux(w, ccl, ccc, ccr, ep, fh);
        r[VY][c] = (q[RO][c] * q[VY][c] - dmy * dsi * dt) / r[RO][c];

        for (int t = 0; t < 5; ++t) w[t] = q[RO][p[t]] * q[VZ][p[t]];
        double dmz = av_dflux(w, ccl, ccc, ccr, ep, fh);
        r[VZ][c] = (q[RO][c] * q[VZ][c] - dmz * dsi * dt) / r[RO][c];

        for (int t = 0; t < 5; ++t) w[t] = q[BX][p[t]];
        double dbx = av_dflux(w, ccl, ccc, ccr, ep, fh);
        r[BX][c] = q[BX][c] - dbx * dsi * dt;

        for (int t = 0; t < 5; ++t) w[t] = q[BY][p[t]];
        double dby = av_dflux(w, ccl, ccc, ccr, ep, fh);
        r[BY][c] = q[BY][c] - dby * dsi * dt;

        for (int t = 0; t < 5; ++t) w[t] = q[BZ][p[t]];
        double dbz = av_dflux(w, ccl, ccc, ccr, ep, fh);
        r[BZ][c] = q[BZ][c] - dbz * dsi * dt;

        for (int t = 0; t < 5; ++t) w[t] = q[PH][p[t]];
        double dph = av_dflux(w, ccl, ccc, ccr, ep, fh);
        r[PH][c] = q[PH][c] - dph * dsi * dt;

        for (int t = 0; t < 5; ++t) w[t] = q[RO][p[t]] * q[EI][p[t]];
        double dei = av_dflux(w, ccl, ccc, ccr, ep, fh);
        double Et = q[RO][c] * q[EI][c] +
                    0.5 * q[RO][c] * (q[VX][c] * q[VX][c] + q[VY][c] * q[VY][c] +
                                      q[VZ][c] * q[VZ][c]) +
                    PII8 * (q[BX][c] * q[BX][c] + q[BY][c] * q[BY][c] + q[BZ][c] * q[BZ][c]);
        r[EI][c] = (Et - dei * dsi * dt -
                    0.5 * r[RO][c] * (r[VX][c] * r[VX][c] + r[VY][c] * r[VY][c] +
                                      r[VZ][c] * r[VZ][c]) -
                    PII8 * (r[BX][c] * r[BX][c] + r[BY][c] * r[BY][c] + r[BZ][c] * r[BZ][c])) /
                   r[RO][c];
      }
    }
  }
}

/* mhd_integrator_host.hpp:303-334 with eos.hpp:36-42. */
static double cfl(const geom *g, const miso_oracle_desc *d, double *const q[NF]) {
  double dt = 1.e10;
  const double gm = d->gm;
  for (int i = g->m[0]; i < g->t[0] - g->m[0]; ++i)
    for (int j = g->m[1]; j < g->t[1] - g->m[1]; ++j)
      for (int k = g->m[2]; k < g->t[2] - g->m[2]; ++k) {
        const long c = IDX(g, i, j, k);
        double cs = sqrt(gm * (gm - 1.0) * q[EI][c]);
        double vv = sqrt(+q[VX][c] * q[VX][c] + q[VY][c] * q[VY][c] + q[VZ][c] * q[VZ][c]);
        double ca = sqrt((+q[BX][c] * q[BX][c] + q[BY][c] * q[BY][c] + q[BZ][c] * q[BZ][c]) /
                         q[RO][c] * PII4);
        double total_vel = cs + vv + ca;
        if (d->cfl_masked) {
          /* demo/mhd3d_magnetosphere/src/timestep.hpp:15-49: the sphere
           * r <= r_inner moves at slow_speed 1e-10 */
          const double x = g->ax[0][i], y = g->ax[1][j], z = g->ax[2][k];
          const double rr = sqrt(x * x + y * y + z * z);
          const double mask = rr > d->r_inner ? 1.0 : 0.0;
          total_vel = total_vel * mask + 1.e-10 * (1.0 - mask);
        }
        dt = fmin2(dt, d->cfl_number * fmin3(g->dax[0][i], g->dax[1][j], g->dax[2][k]) /
                           total_vel);
      }
  return dt;
}

typedef struct {
  double *argm[NF], *rslt[NF];
  double *pr, *bb, *ht, *vb, *cc;
  double *block;
} work;

static int work_alloc(work *w, const geom *g) {
  const long n = g->cells;
  w->block = (double *)calloc((size_t)n * (2 * NF + 5), sizeof(double));
  if (!w->block) return -1;
  for (int f = 0; f < NF; ++f) {
    w->argm[f] = w->block + (long)f * n;
    w->rslt[f] = w->block + (long)(NF + f) * n;
  }
  w->pr = w->block + (long)(2 * NF) * n;
  w->bb = w->pr + n;
  w->ht = w->bb + n;
  w->vb = w->ht + n;
  w->cc = w->vb + n;
  return 0;
}

static void copy_fields(const geom *g, double *const dst[NF], double *const src[NF]) {
  for (int f = 0; f < NF; ++f) memcpy(dst[f], src[f], sizeof(double) * g->cells);
}

/* mhd_integrator_host.hpp:280-300. */
static void apply_av(const geom *g, const miso_oracle_desc *d, double *const q[NF],
                     work *w, double dt) {
  char_velocity(g, d, q, w->cc);
  for (int dir = 0; dir < 3; ++dir) {
    av_sweep(g, d, q, w->rslt, w->cc, dir, dt);
    copy_fields(g, q, w->rslt);
    fill_ghosts(g, d, q);
  }
}

/* mhd_integrator_host.hpp:258-277 and 337-350. */
static int update(const geom *g, const miso_oracle_desc *d, double *const q[NF], work *w,
                  double dt) {
  const double ch = 0.8 * d->cfl_number * g->min_dxyz / dt;
  const double ch2 = ch * ch;
  const double tau = 2.0 * dt;
  int rc;
  if ((rc = stage(g, d, q, q, w->rslt, dt / 4.0, ch2, tau, w->pr, w->bb, w->ht, w->vb))) return rc;
  copy_fields(g, w->argm, w->rslt);
  fill_ghosts(g, d, w->argm);
  if ((rc = stage(g, d, q, w->argm, w->rslt, dt / 3.0, ch2, tau, w->pr, w->bb, w->ht, w->vb)))
    return rc;
  copy_fields(g, w->argm, w->rslt);
  fill_ghosts(g, d, w->argm);
  if ((rc = stage(g, d, q, w->argm, w->rslt, dt / 2.0, ch2, tau, w->pr, w->bb, w->ht, w->vb)))
    return rc;
  copy_fields(g, w->argm, w->rslt);
  fill_ghosts(g, d, w->argm);
  if ((rc = stage(g, d, q, w->argm, w->rslt, dt, ch2, tau, w->pr, w->bb, w->ht, w->vb)))
    return rc;
  copy_fields(g, q, w->rslt);
  fill_ghosts(g, d, q);
  apply_av(g, d, q, w, dt);
  return 0;
}

/* ---------------------------------------------------------------------- */
/* Exported entry points.                                                   */
/* ---------------------------------------------------------------------- */
int miso_oracle_fill_ghosts(const miso_oracle_desc *d, double *const q[9]) {
  geom g;
  if (geom_init(&g, d)) return -1;
  fill_ghosts(&g, d, q);
  geom_free(&g);
  return 0;
}

double miso_oracle_cfl(const miso_oracle_desc *d, double *const q[9]) {
  geom g;
  if (geom_init(&g, d)) return -1.0;
  double dt = cfl(&g, d, q);
  geom_free(&g);
  return dt;
}

int miso_oracle_stage(const miso_oracle_desc *d, double *const orgn[9],
                      double *const argm[9], double *const rslt[9], double dt,
                      double ch_divb_square, double tau_divb) {
  geom g;
  if (geom_init(&g, d)) return -1;
  work w;
  if (work_alloc(&w, &g)) { geom_free(&g); return -2; }
  const int rc = stage(&g, d, orgn, argm, rslt, dt, ch_divb_square, tau_divb, w.pr, w.bb, w.ht,
                       w.vb);
  free(w.block);
  geom_free(&g);
  return rc;
}

int miso_oracle_av(const miso_oracle_desc *d, double *const q[9], double dt) {
  geom g;
  if (geom_init(&g, d)) return -1;
  work w;
  if (work_alloc(&w, &g)) { geom_free(&g); return -2; }
  copy_fields(&g, w.rslt, q);
  apply_av(&g, d, q, &w, dt);
  free(w.block);
  geom_free(&g);
  return 0;
}

int miso_oracle_update(const miso_oracle_desc *d, double *const q[9], double dt) {
  geom g;
  if (geom_init(&g, d)) return -1;
  work w;
  if (work_alloc(&w, &g)) { geom_free(&g); return -2; }
  copy_fields(&g, w.rslt, q);
  copy_fields(&g, w.argm, q);
  const int rc = update(&g, d, q, &w, dt);
  free(w.block);
  geom_free(&g);
  return rc;
}

int miso_oracle_run(const miso_oracle_desc *d, double *const q[9], int nsteps,
                    int fill_first, double *dt_out) {
  geom g;
  if (geom_init(&g, d)) return -1;
  work w;
  if (work_alloc(&w, &g)) { geom_free(&g); return -2; }
  if (fill_first) fill_ghosts(&g, d, q);
  copy_fields(&g, w.rslt, q);
  copy_fields(&g, w.argm, q);
  int rc = 0;
  for (int n = 0; n < nsteps && !rc; ++n) {
    double dt = cfl(&g, d, q);
    if (dt_out) dt_out[n] = dt;
    rc = update(&g, d, q, &w, dt);
  }
  free(w.block);
  geom_free(&g);
  return rc;
}

int miso_oracle_axis(const miso_oracle_desc *d, int axis, double *s, double *ds,
                     double *dsi) {
  geom g;
  if (axis < 0 || axis > 2) return -1;
  if (geom_init(&g, d)) return -1;
  for (int n = 0; n < g.t[axis]; ++n) {
    s[n] = g.ax[axis][n];
    ds[n] = g.dax[axis][n];
    dsi[n] = g.daxi[axis][n];
  }
  geom_free(&g);
  return 0;
}

double miso_oracle_min_dxyz(const miso_oracle_desc *d) {
  geom g;
  if (geom_init(&g, d)) return -1.0;
  double v = g.min_dxyz;
  geom_free(&g);
  return v;
}
