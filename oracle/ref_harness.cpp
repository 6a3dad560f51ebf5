/*
 * ref_harness.cpp -- drives the reference's OWN host integrator
 * (miso::mhd::Integrator<double, backend::Host>, compiled from the MISO
 * headers where they lie) behind the same C entry points as the oracle
 * restatement, so tests can check the restatement against the reference
 * bit for bit.  Built by oracle/Makefile into oracle/_ref/libmiso_ref.so.
 * TEST INFRASTRUCTURE ONLY: nothing in the product loads it.
 *
 * The boundary functor mirrors the demos' "outflow" condition
 * (demo/mhd1d_shock_tube/src/main.cpp:85-162): on every physical (non
 * periodic) face, boundary_condition::symmetric is applied to all 9 fields
 * with the per-field sign given in the descriptor.  Periodic faces are
 * handled by the reference's HaloExchanger through single-rank MPI.
 */
#include <miso/boundary_condition.hpp>
#include <miso/eos.hpp>
#include <miso/mhd_integrator.hpp>
#include <miso/mhd_model_base.hpp>

#include <cstdio>
#include <filesystem>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <unistd.h>

#include "miso_oracle.h"

using namespace miso;
// The reference is templated on Real: double by default, float for the
// build that mirrors its demos (compiled with -DMISO_REF_FLOAT).  The C
// entry points always exchange double arrays; a float build converts on the
// way in and out (float -> double -> float is exact).
#ifdef MISO_REF_FLOAT
using Real = float;
#else
using Real = double;
#endif
using B = backend::Host;

namespace {

struct DescBC {
  mpi::Shape &shape;
  double sign[3][2][9];

  DescBC(mpi::Shape &s, const miso_oracle_desc &d) : shape(s) {
    std::memcpy(sign, d.sign, sizeof(sign));
  }

  void apply(mhd::FieldsView<Real> qq, GridView<const Real> grid) const {
    namespace bc = miso::boundary_condition;
    Array3DView<Real> *f[9] = {&qq.ro, &qq.vx, &qq.vy, &qq.vz, &qq.bx,
                               &qq.by, &qq.bz, &qq.ei, &qq.ph};
    const Direction dirs[3] = {Direction::X, Direction::Y, Direction::Z};
    const Side sides[2] = {Side::INNER, Side::OUTER};
    for (int a = 0; a < 3; ++a)
      for (int s = 0; s < 2; ++s)
        if (bc::is_physical_boundary(dirs[a], sides[s], shape))
          for (int v = 0; v < 9; ++v)
            bc::symmetric(B{}, *f[v], grid, sign[a][s][v] < 0 ? Sign::Neg : Sign::Pos,
                          dirs[a], sides[s]);
  }
};

// The magnetosphere demo's boundary (demo/mhd3d_magnetosphere/src/bc.hpp:
// 39-158), restated as a boundary functor of the reference's concept on the
// reference's own boundary_condition helpers and util::max2: mirror faces
// (x outer, y inner / outer, z inner / outer for all fields; x inner for vy,
// vz, bx, by, ph), the solar wind fixed in the x-inner ghosts of ro, vx, ei,
// bz, then on every cell a blend toward the state qq_init and floors on ro
// and ei.  The demo allocates qq_init and never writes it; here it holds the
// descriptor's blend state (zeros where none is given).
struct MagnetoBC {
  mpi::Shape &shape;
  double sign[3][2][9];
  Real gm, ro_sw, pr_sw, vx_sw, bz_imf, rra, a0, ro_floor, pr_floor;
  mhd::Fields<Real, B> qq_init;

  MagnetoBC(mpi::Shape &s, const miso_oracle_desc &d, Grid<Real, B> &g)
      : shape(s), gm(d.gm), ro_sw(d.sw_ro), pr_sw(d.sw_pr), vx_sw(d.sw_vx), bz_imf(d.sw_bz),
        rra(d.r_inner), a0(d.a0), ro_floor(d.ro_floor), pr_floor(d.pr_floor),
        qq_init(g.i_total, g.j_total, g.k_total) {
    std::memcpy(sign, d.sign, sizeof(sign));
    Array3D<Real, B> *f[9] = {&qq_init.ro, &qq_init.vx, &qq_init.vy, &qq_init.vz, &qq_init.bx,
                              &qq_init.by, &qq_init.bz, &qq_init.ei, &qq_init.ph};
    for (int v = 0; v < 9; ++v)
      for (size_t n = 0; n < f[v]->size(); ++n)
        f[v]->data()[n] = d.blend[v] ? (Real)d.blend[v][n] : Real(0);
  }

  void mirror(mhd::FieldsView<Real> &qq, GridView<const Real> grid, int a, int s,
              unsigned mask) const {
    namespace bc = miso::boundary_condition;
    Array3DView<Real> *f[9] = {&qq.ro, &qq.vx, &qq.vy, &qq.vz, &qq.bx,
                               &qq.by, &qq.bz, &qq.ei, &qq.ph};
    const Direction dirs[3] = {Direction::X, Direction::Y, Direction::Z};
    const Side sides[2] = {Side::INNER, Side::OUTER};
    if (!bc::is_physical_boundary(dirs[a], sides[s], shape)) return;
    for (int v = 0; v < 9; ++v)
      if ((mask >> v) & 1u)
        bc::symmetric(B{}, *f[v], grid, sign[a][s][v] < 0 ? Sign::Neg : Sign::Pos, dirs[a],
                      sides[s]);
  }

  void apply(mhd::FieldsView<Real> qq, GridView<const Real> grid) const {
    namespace bc = miso::boundary_condition;
    mirror(qq, grid, 0, 1, 0x1ffu);
    mirror(qq, grid, 1, 0, 0x1ffu);
    mirror(qq, grid, 1, 1, 0x1ffu);
    mirror(qq, grid, 2, 0, 0x1ffu);
    mirror(qq, grid, 2, 1, 0x1ffu);
    if (bc::is_physical_boundary(Direction::X, Side::INNER, shape)) {
      mirror(qq, grid, 0, 0, (1u << 2) | (1u << 3) | (1u << 4) | (1u << 5) | (1u << 8));
      int i0, i1, j0, j1, k0, k1;
      bc::range_set(i0, i1, j0, j1, k0, k1, Direction::X, grid);
      for (int i = i0; i < i1; ++i)
        for (int j = j0; j < j1; ++j)
          for (int k = k0; k < k1; ++k) {
            int ig, it;
            bc::symmetric_index(i, grid.i_total, grid.i_margin, ig, it, Side::INNER);
            qq.ro(ig, j, k) = ro_sw;
            qq.vx(ig, j, k) = vx_sw;
            qq.ei(ig, j, k) = pr_sw / (gm - 1.0) / qq.ro(ig, j, k);
            qq.bz(ig, j, k) = bz_imf;
          }
    }
    auto qi = qq_init.const_view();
    for (int i = 0; i < grid.i_total; ++i)
      for (int j = 0; j < grid.j_total; ++j)
        for (int k = 0; k < grid.k_total; ++k) {
          const Real rr = util::sqrt(grid.x[i] * grid.x[i] + grid.y[j] * grid.y[j] +
                                     grid.z[k] * grid.z[k]);
          const Real hh = util::max2<Real>(0.0, util::pow2(rr / rra) - 1.0);
          const Real f = a0 * hh / (a0 * hh + 1.0);
          auto lerp = [f](Real a, Real b) { return a * f + b * (1.0 - f); };
          qq.ro(i, j, k) = lerp(qq.ro(i, j, k), qi.ro(i, j, k));
          qq.vx(i, j, k) = lerp(qq.vx(i, j, k), qi.vx(i, j, k));
          qq.vy(i, j, k) = lerp(qq.vy(i, j, k), qi.vy(i, j, k));
          qq.vz(i, j, k) = lerp(qq.vz(i, j, k), qi.vz(i, j, k));
          qq.bx(i, j, k) = lerp(qq.bx(i, j, k), qi.bx(i, j, k));
          qq.by(i, j, k) = lerp(qq.by(i, j, k), qi.by(i, j, k));
          qq.bz(i, j, k) = lerp(qq.bz(i, j, k), qi.bz(i, j, k));
          qq.ei(i, j, k) = lerp(qq.ei(i, j, k), qi.ei(i, j, k));
          qq.ph(i, j, k) = lerp(qq.ph(i, j, k), qi.ph(i, j, k));
          qq.ro(i, j, k) = util::max2<Real>(qq.ro(i, j, k), ro_floor);
          qq.ei(i, j, k) = util::max2<Real>(qq.ei(i, j, k), pr_floor / (gm - 1.0) / qq.ro(i, j, k));
        }
  }
};

// The demo's CFL with the sphere r <= radius masked
// (demo/mhd3d_magnetosphere/src/timestep.hpp:15-49), on the reference's own
// reduce and util::min2 / min3.
Real masked_cfl(const mhd::Fields<Real, B> &qq, const Grid<Real, B> &grid, Real gm,
                Real cfl_number, Real rra) {
  const Real slow_speed = 1.e-10;
  const Real dt_max = 1.e10;
  auto qq_v = qq.const_view();
  auto grid_v = grid.const_view();
  Range3D range{{grid.i_margin, grid.i_total - grid.i_margin},
                {grid.j_margin, grid.j_total - grid.j_margin},
                {grid.k_margin, grid.k_total - grid.k_margin}};
  const auto f = [=](int i, int j, int k) {
    Real cs = util::sqrt(gm * (gm - 1.0) * qq_v.ei(i, j, k));
    Real vv = util::sqrt(qq_v.vx(i, j, k) * qq_v.vx(i, j, k) + qq_v.vy(i, j, k) * qq_v.vy(i, j, k) +
                         qq_v.vz(i, j, k) * qq_v.vz(i, j, k));
    Real ca = util::sqrt((qq_v.bx(i, j, k) * qq_v.bx(i, j, k) + qq_v.by(i, j, k) * qq_v.by(i, j, k) +
                          qq_v.bz(i, j, k) * qq_v.bz(i, j, k)) /
                         qq_v.ro(i, j, k) * pii4<Real>);
    Real total_vel = (cs + vv + ca);
    Real rr = util::sqrt(util::pow2(grid_v.x[i]) + util::pow2(grid_v.y[j]) + util::pow2(grid_v.z[k]));
    Real mask = rr > rra ? 1.0 : 0.0;
    Real masked_vel = total_vel * mask + slow_speed * (1.0 - mask);
    Real dxyz = util::min3(grid_v.dx[i], grid_v.dy[j], grid_v.dz[k]);
    return cfl_number * dxyz / masked_vel;
  };
  const auto op = [](Real a, Real b) { return util::min2(a, b); };
  return reduce(B{}, range, dt_max, f, op);
}

// The point gravity of the magnetosphere demo
// (demo/mhd3d_magnetosphere/src/src.hpp:17-44), restated as a source
// functor of the reference's Source concept (mhd_model_base.hpp:131-155):
// force per volume -ro g x / |x|^3 from the stage's argument state, no
// heating.
struct PointGravity {
  GridView<const Real> grid;
  Real g_grav;
  PointGravity(Grid<Real, B> &g, Real gg) : grid(g.const_view()), g_grav(gg) {}
  Real r3(int i, int j, int k) const {
    return util::pow3(util::sqrt(grid.x[i] * grid.x[i] + grid.y[j] * grid.y[j] +
                                 grid.z[k] * grid.z[k]));
  }
  Real vx(mhd::FieldsView<const Real> qq, int i, int j, int k) const {
    return -qq.ro(i, j, k) * g_grav * grid.x[i] / r3(i, j, k);
  }
  Real vy(mhd::FieldsView<const Real> qq, int i, int j, int k) const {
    return -qq.ro(i, j, k) * g_grav * grid.y[j] / r3(i, j, k);
  }
  Real vz(mhd::FieldsView<const Real> qq, int i, int j, int k) const {
    return -qq.ro(i, j, k) * g_grav * grid.z[k] / r3(i, j, k);
  }
  Real ei(mhd::FieldsView<const Real>, int, int, int) const { return 0.0; }
};

// Four constants as a functor of the reference's Source concept
// (mhd_model_base.hpp:131-155): src.vx, src.vy, src.vz and src.ei of every
// cell, whatever the state -- the descriptor's source 3, which pins where
// update_sc4 adds each term (mhd_integrator_host.hpp:134, 151, 168, 241).
struct ConstSource {
  Real c[4];
  explicit ConstSource(const double *v) {
    for (int q = 0; q < 4; ++q) c[q] = (Real)v[q];
  }
  Real vx(mhd::FieldsView<const Real>, int, int, int) const { return c[0]; }
  Real vy(mhd::FieldsView<const Real>, int, int, int) const { return c[1]; }
  Real vz(mhd::FieldsView<const Real>, int, int, int) const { return c[2]; }
  Real ei(mhd::FieldsView<const Real>, int, int, int) const { return c[3]; }
};

struct Session {
  std::unique_ptr<Env> env;
  std::string path;
  std::unique_ptr<Config> config;
  std::unique_ptr<mpi::Shape> shape;
  std::unique_ptr<Grid<Real, B>> grid;
  std::unique_ptr<mhd::ExecContext<Real, B>> ctx;
  std::unique_ptr<mhd::Integrator<Real, B>> integ;
  std::unique_ptr<eos::IdealEOS<Real>> eos;
  std::unique_ptr<DescBC> bc;
  std::unique_ptr<MagnetoBC> mbc;
  mhd::EmptySourceTerm<Real> src;
  const miso_oracle_desc &desc;

  // f(boundary functor) with the descriptor's boundary
  template <class F> void with_bc(F &&f) {
    if (desc.boundary == 1)
      f(*mbc);
    else
      f(*bc);
  }
  // Integrator::update with the descriptor's boundary and source
  void update(Real dt, mhd::Fields<Real, B> &qq) {
    with_bc([&](auto &b) {
      if (desc.source == 1)
        integ->update(dt, *eos, b, PointGravity(*grid, (Real)desc.g_grav), qq);
      else if (desc.source == 3)
        integ->update(dt, *eos, b, ConstSource(desc.src_const), qq);
      else
        integ->update(dt, *eos, b, src, qq);
    });
  }
  Real cfl(const mhd::Fields<Real, B> &qq) {
    if (desc.cfl_masked)
      return masked_cfl(qq, *grid, eos->gm, (Real)desc.cfl_number, (Real)desc.r_inner);
    return integ->cfl(qq, *eos);
  }

  explicit Session(const miso_oracle_desc &d) : desc(d) {
    static Env *global_env = new Env();
    (void)global_env;
    char tmpl[] = "/tmp/miso_ref_cfgXXXXXX";
    int fd = mkstemp(tmpl);
    if (fd < 0) throw std::runtime_error("mkstemp failed");
    close(fd);
    path = tmpl;
    std::ostringstream y;
    y.precision(17);
    y << "io:\n  enabled: false\n  continue: false\n  save_dir: ./\n";
    y << "grid:\n  i_size: " << d.i_size << "\n  j_size: " << d.j_size
      << "\n  k_size: " << d.k_size << "\n  margin: " << d.margin << "\n  x_min: " << d.x_min
      << "\n  x_max: " << d.x_max << "\n  y_min: " << d.y_min << "\n  y_max: " << d.y_max
      << "\n  z_min: " << d.z_min << "\n  z_max: " << d.z_max << "\n";
    y << "mpi:\n  x_procs: 1\n  y_procs: 1\n  z_procs: 1\n";
    y << "domain:\n  periodic:\n    x: " << (d.periodic[0] ? "true" : "false")
      << "\n    y: " << (d.periodic[1] ? "true" : "false")
      << "\n    z: " << (d.periodic[2] ? "true" : "false") << "\n";
    y << "mhd:\n  cfl_number: " << d.cfl_number << "\n  artificial_viscosity:\n    ep: " << d.ep
      << "\n    fh: " << d.fh << "\n    cs_fac: " << d.cs_fac << "\n    ca_fac: " << d.ca_fac
      << "\n    vv_fac: " << d.vv_fac << "\n";
    y << "eos:\n  gm: " << d.gm << "\n";
    {
      std::ofstream f(path);
      f << y.str();
    }
    config.reset(new Config(path));
    shape.reset(new mpi::Shape(*config));
    grid.reset(new Grid<Real, B>(d.i_size, d.j_size, d.k_size, d.margin, d.x_min, d.x_max,
                                 d.y_min, d.y_max, d.z_min, d.z_max));
    ctx.reset(new mhd::ExecContext<Real, B>(*shape, *grid));
    integ.reset(new mhd::Integrator<Real, B>(*config, *grid, *ctx));
    eos.reset(new eos::IdealEOS<Real>(d.gm));
    bc.reset(new DescBC(*shape, d));
    if (d.boundary == 1) mbc.reset(new MagnetoBC(*shape, d, *grid));
  }
  ~Session() { std::remove(path.c_str()); }
};

void to_fields(mhd::Fields<Real, B> &qq, double *const q[9]) {
  Array3D<Real, B> *f[9] = {&qq.ro, &qq.vx, &qq.vy, &qq.vz, &qq.bx,
                            &qq.by, &qq.bz, &qq.ei, &qq.ph};
  for (int v = 0; v < 9; ++v)
    for (size_t n = 0; n < f[v]->size(); ++n) f[v]->data()[n] = (Real)q[v][n];
}

void from_fields(const mhd::Fields<Real, B> &qq, double *const q[9]) {
  const Array3D<Real, B> *f[9] = {&qq.ro, &qq.vx, &qq.vy, &qq.vz, &qq.bx,
                                  &qq.by, &qq.bz, &qq.ei, &qq.ph};
  for (int v = 0; v < 9; ++v)
    for (size_t n = 0; n < f[v]->size(); ++n) q[v][n] = (double)f[v]->data()[n];
}

} // namespace

extern "C" {

int miso_ref_run(const miso_oracle_desc *d, double *const q[9], int nsteps, int fill_first,
                 double *dt_out) {
  try {
    Session s(*d);
    mhd::Fields<Real, B> qq(*s.grid);
    to_fields(qq, q);
    if (fill_first) s.with_bc([&](auto &b) { s.integ->apply_boundary_condition(b, qq); });
    for (int n = 0; n < nsteps; ++n) {
      const Real dt = s.cfl(qq);
      if (dt_out) dt_out[n] = dt;
      s.update(dt, qq);
    }
    from_fields(qq, q);
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "miso_ref_run: %s\n", e.what());
    return -1;
  }
}

/* One step (update) with a given dt, as ModelBase::update does after cfl. */
int miso_ref_update(const miso_oracle_desc *d, double *const q[9], double dt) {
  try {
    Session s(*d);
    mhd::Fields<Real, B> qq(*s.grid);
    to_fields(qq, q);
    s.update((Real)dt, qq);
    from_fields(qq, q);
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "miso_ref_update: %s\n", e.what());
    return -1;
  }
}

double miso_ref_cfl(const miso_oracle_desc *d, double *const q[9]) {
  try {
    Session s(*d);
    mhd::Fields<Real, B> qq(*s.grid);
    to_fields(qq, q);
    return s.cfl(qq);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "miso_ref_cfl: %s\n", e.what());
    return -1.0;
  }
}

int miso_ref_stage(const miso_oracle_desc *d, double *const orgn[9], double *const argm[9],
                   double *const rslt[9], double dt, double ch_divb_square,
                   double tau_divb) {
  try {
    Session s(*d);
    mhd::Fields<Real, B> o(*s.grid), a(*s.grid), r(*s.grid);
    to_fields(o, orgn);
    to_fields(a, argm);
    to_fields(r, rslt);
    s.integ->ch_divb_square = ch_divb_square;
    s.integ->tau_divb = tau_divb;
    if (d->source == 1)
      s.integ->update_sc4(dt, *s.eos, PointGravity(*s.grid, d->g_grav), o, a, r);
    else if (d->source == 3)
      s.integ->update_sc4(dt, *s.eos, ConstSource(d->src_const), o, a, r);
    else
      s.integ->update_sc4(dt, *s.eos, s.src, o, a, r);
    from_fields(r, rslt);
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "miso_ref_stage: %s\n", e.what());
    return -1;
  }
}

int miso_ref_av(const miso_oracle_desc *d, double *const q[9], double dt) {
  try {
    Session s(*d);
    mhd::Fields<Real, B> qq(*s.grid);
    to_fields(qq, q);
    s.with_bc([&](auto &b) { s.integ->apply_artificial_viscosity(dt, *s.eos, b, qq); });
    from_fields(qq, q);
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "miso_ref_av: %s\n", e.what());
    return -1;
  }
}

int miso_ref_fill_ghosts(const miso_oracle_desc *d, double *const q[9]) {
  try {
    Session s(*d);
    mhd::Fields<Real, B> qq(*s.grid);
    to_fields(qq, q);
    s.with_bc([&](auto &b) { s.integ->apply_boundary_condition(b, qq); });
    from_fields(qq, q);
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "miso_ref_fill_ghosts: %s\n", e.what());
    return -1;
  }
}

double miso_ref_min_dxyz(const miso_oracle_desc *d) {
  try {
    Session s(*d);
    return s.grid->min_dxyz;
  } catch (const std::exception &e) {
    return -1.0;
  }
}

/* Symmetric-boundary index helper of the reference (boundary_condition.hpp:77-90),
 * exposed for the index known-answer test. */
void miso_ref_symmetric_index(int i, int i_total, int i_margin, int outer, int *ghst,
                              int *trgt) {
  boundary_condition::symmetric_index(i, i_total, i_margin, *ghst, *trgt,
                                      outer ? Side::OUTER : Side::INNER);
}

} // extern "C"
