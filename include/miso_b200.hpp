// miso_b200.hpp -- header-only C++17 drop-in for MISO's mhd::Integrator over
// the C ABI of libmiso_b200.so (include/miso_b200.h).
//
// miso_b200::Integrator<Real> has the member functions through which
// mhd::MHD and mhd::ModelBase drive the reference's integrator
// (miso/include/miso/mhd.hpp:28-45 calling
// miso/include/miso/mhd_integrator_host.hpp:303-350 /
// miso/include/miso/mhd_integrator_cuda.cuh:450-487):
//
//     Real cfl(const Fields &qq, const EOS &eos);
//     void update(Real dt, const EOS &eos, const BC &bc, const Src &src, Fields &qq);
//     void apply_boundary_condition(const BC &bc, Fields &qq);
//
// `Fields` is any type with the reference's members ro, vx, vy, vz, bx, by,
// bz, ei, ph, each with data() (mhd::Fields<Real, backend::Host> or
// <Real, backend::CUDA>, miso/include/miso/mhd_fields.hpp:55-181): host or
// device pointers both work for Real = double; Real = float fields are
// converted through host staging (host fields only).  `Grid` is any type
// with the reference Grid's i_size .. k_size, i_margin .. k_margin and
// x_min .. z_max (miso/include/miso/grid.hpp:146-211).
//
// The EOS, BC and source arguments are checked, not ignored: the EOS must
// have the ideal gas's `gm` equal to Physics::gm (else Error); the boundary
// must be the Boundary descriptor (periodic, or mirror with a sign per field
// as boundary_condition::symmetric, boundary_condition.hpp:109-136) -- a
// descriptor with other mirror signs than the last one is applied, another
// periodicity is an Error; the source must be NoSource (EmptySourceTerm,
// mhd_model_base.hpp:139-155) or PointGravity<Real>.  Any other boundary or
// source type is a compile-time error: reference functors run through the
// backend of include/miso_b200_backend.hpp instead.
//
// Residency.  By default cfl() copies qq to the device, an update() that
// directly follows a cfl() on the same fields (ModelBase::update's
// sequence) reuses that copy, and update() copies the result back, so qq
// always holds the state exactly as with the reference.  set_resident(true)
// keeps the state on the device between calls (qq is then read only by
// push() and written only by pull()), which is how a time loop should drive
// it.  Real = float fields must be host arrays (they are widened through
// host staging); device float fields are refused with an Error.
//
// Errors from the library are thrown as miso_b200::Error (with the status
// code and the library's message).
#ifndef MISO_B200_HPP
#define MISO_B200_HPP

#include <cstddef>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "miso_b200.h"

namespace miso_b200 {

#ifndef MISO_B200_ERROR_DEFINED
#define MISO_B200_ERROR_DEFINED
class Error : public std::runtime_error {
 public:
  Error(int code, const std::string &msg) : std::runtime_error(msg), code_(code) {}
  int code() const noexcept { return code_; }

 private:
  int code_;
};
#endif

inline void check(int rc, miso_b200_handle *h, const char *what) {
  if (rc != MISO_B200_OK)
    throw Error(rc, std::string(what) + ": " + miso_b200_last_error(h));
}

// Physics and numerics parameters (the config keys the reference reads:
// eos.gm, mhd.cfl_number, mhd.artificial_viscosity.*; defaults as
// miso/include/miso/config_defaults.hpp).
struct Physics {
  double gm = 5.0 / 3.0;
  double cfl_number = 0.4;
  double ep = 1.0, fh = 1.0;
  double cs_fac = 1.0, ca_fac = 1.0, vv_fac = 1.0;
};

// Built-in boundaries: per axis periodic, or mirror with a sign per side
// and field (field order ro, vx, vy, vz, bx, by, bz, ei, ph).
struct Boundary {
  int periodic[3] = {1, 1, 1};
  double sign[3][2][9];
  Boundary() {
    for (auto &a : sign)
      for (auto &s : a)
        for (double &v : s) v = 1.0;
  }
  static Boundary all_periodic() { return Boundary(); }
  // the demos' "outflow": symmetric with Sign::Pos on all 9 fields
  static Boundary all_mirror() {
    Boundary b;
    b.periodic[0] = b.periodic[1] = b.periodic[2] = 0;
    return b;
  }
};

// No source term (the reference's mhd::EmptySourceTerm).
struct NoSource {};

#ifndef MISO_B200_POINT_GRAVITY_DEFINED
#define MISO_B200_POINT_GRAVITY_DEFINED
// The magnetosphere demo's point gravity (demo/mhd3d_magnetosphere/src/
// src.hpp:17-44): force per volume -ro g x / |x|^3 about the origin.
template <typename Real>
struct PointGravity {
  Real g;
};
#endif

template <class T>
struct is_boundary_descriptor : std::is_same<T, Boundary> {};

template <class Real>
class Integrator {
  static_assert(std::is_same<Real, double>::value || std::is_same<Real, float>::value,
                "Real must be float or double");

 public:
  template <class Grid>
  Integrator(const Grid &grid, const Physics &phys, const Boundary &bc,
             int precision = MISO_B200_FP64, void *stream = nullptr) {
    miso_b200_grid_desc gd{};
    gd.i_size = grid.i_size;
    gd.j_size = grid.j_size;
    gd.k_size = grid.k_size;
    // the reference forces margin 0 on size-1 axes; the largest margin is
    // the grid's margin
    gd.margin = grid.i_margin > grid.j_margin ? grid.i_margin : grid.j_margin;
    if (grid.k_margin > gd.margin) gd.margin = grid.k_margin;
    gd.x_min = grid.x_min;
    gd.x_max = grid.x_max;
    gd.y_min = grid.y_min;
    gd.y_max = grid.y_max;
    gd.z_min = grid.z_min;
    gd.z_max = grid.z_max;
    for (int a = 0; a < 3; ++a) {
      gd.periodic[a] = bc.periodic[a];
      for (int s = 0; s < 2; ++s)
        for (int f = 0; f < 9; ++f) gd.sign[a][s][f] = bc.sign[a][s][f];
    }
    miso_b200_params pp{};
    pp.gm = phys.gm;
    pp.cfl_number = phys.cfl_number;
    pp.ep = phys.ep;
    pp.fh = phys.fh;
    pp.cs_fac = phys.cs_fac;
    pp.ca_fac = phys.ca_fac;
    pp.vv_fac = phys.vv_fac;
    pp.precision = precision;
    check(miso_b200_create(&gd, &pp, stream, &h_), nullptr, "miso_b200_create");
    gm_ = phys.gm;
    bc_ = bc;
    cells_ = (size_t)(grid.i_size + 2 * grid.i_margin) * (grid.j_size + 2 * grid.j_margin) *
             (grid.k_size + 2 * grid.k_margin);
  }
  ~Integrator() {
    if (h_) miso_b200_destroy(h_);
  }
  Integrator(const Integrator &) = delete;
  Integrator &operator=(const Integrator &) = delete;

  // -- the reference's integrator interface ---------------------------------
  template <class Fields, class EOS>
  Real cfl(const Fields &qq, const EOS &eos) {
    check_eos(eos);
    if (!resident_) push(qq);
    double dt = 0.0;
    check(miso_b200_cfl(h_, &dt), h_, "miso_b200_cfl");
    // the state on the device is qq's: a following update() needs no copy
    pushed_ = qq.ro.data();
    return (Real)dt;
  }

  template <class EOS, class BC, class Src, class Fields>
  void update(Real dt, const EOS &eos, const BC &bc, const Src &src, Fields &qq) {
    check_eos(eos);
    set_boundary(bc);
    set_source(src);
    if (!resident_ && pushed_ != (const void *)qq.ro.data()) push(qq);
    pushed_ = nullptr;
    check(miso_b200_update(h_, (double)dt), h_, "miso_b200_update");
    if (!resident_) pull(qq);
  }

  template <class BC, class Fields>
  void apply_boundary_condition(const BC &bc, Fields &qq) {
    set_boundary(bc);
    pushed_ = nullptr;
    if (!resident_) push(qq);
    check(miso_b200_fill_ghosts(h_), h_, "miso_b200_fill_ghosts");
    if (!resident_) pull(qq);
  }

  // -- residency and transfers ----------------------------------------------
  void set_resident(bool on) { resident_ = on; }
  bool resident() const { return resident_; }

  template <class Fields>
  void push(const Fields &qq) {
    const Real *src[9] = {qq.ro.data(), qq.vx.data(), qq.vy.data(), qq.vz.data(), qq.bx.data(),
                          qq.by.data(), qq.bz.data(), qq.ei.data(), qq.ph.data()};
    const double *q[9];
    stage_in(src, q);
    check(miso_b200_upload(h_, q), h_, "miso_b200_upload");
  }

  template <class Fields>
  void pull(Fields &qq) {
    Real *dst[9] = {qq.ro.data(), qq.vx.data(), qq.vy.data(), qq.vz.data(), qq.bx.data(),
                    qq.by.data(), qq.bz.data(), qq.ei.data(), qq.ph.data()};
    double *q[9];
    stage_out_ptrs(dst, q);
    check(miso_b200_download(h_, q), h_, "miso_b200_download");
    stage_out(dst);
  }

  // -- source and boundary descriptors ---------------------------------------
  // the magnetosphere demo's point gravity (demo/mhd3d_magnetosphere/src/
  // src.hpp:17-44): force per volume -ro g x / |x|^3, both forms
  void set_point_gravity(double g) {
    check(miso_b200_set_source(h_, MISO_B200_SOURCE_POINT_GRAVITY, &g, 1), h_,
          "miso_b200_set_source");
  }
  // the magnetosphere demo's boundary and masked CFL (bc.hpp:39-158,
  // timestep.hpp:15-49), FP64 form: the config's solar_wind, magnetosphere
  // and floor entries
  struct Magnetosphere {
    double ro_sw, pr_sw, vx_sw, bz_imf;
    double radius, a0;
    double ro_floor, pr_floor;
    bool mask_cfl = true;
  };
  void set_magnetosphere_boundary(const Magnetosphere &m) {
    const double p[9] = {m.ro_sw,  m.pr_sw,    m.vx_sw,    m.bz_imf,         m.radius,
                         m.a0,     m.ro_floor, m.pr_floor, m.mask_cfl ? 1.0 : 0.0};
    check(miso_b200_set_boundary(h_, MISO_B200_BOUNDARY_MAGNETOSPHERE, p, 9), h_,
          "miso_b200_set_boundary");
  }
  // the state the boundary blends toward near the sphere (the initial
  // condition, typically)
  template <class Fields>
  void set_blend_state(const Fields &qq) {
    const Real *src[9] = {qq.ro.data(), qq.vx.data(), qq.vy.data(), qq.vz.data(), qq.bx.data(),
                          qq.by.data(), qq.bz.data(), qq.ei.data(), qq.ph.data()};
    const double *q[9];
    stage_in(src, q);
    check(miso_b200_set_blend_state(h_, q), h_, "miso_b200_set_blend_state");
  }

  // the checks behind update(): see the header comment
  template <class EOS>
  void check_eos(const EOS &eos) const {
    if ((double)eos.gm != gm_ && (Real)eos.gm != (Real)gm_)
      throw Error(MISO_B200_ERR_ARG, "the EOS's gm differs from Physics::gm");
  }
  template <class BC>
  void set_boundary(const BC &bc) {
    static_assert(is_boundary_descriptor<BC>::value,
                  "miso_b200::Integrator takes the miso_b200::Boundary descriptor; reference "
                  "boundary functors run through include/miso_b200_backend.hpp");
    for (int a = 0; a < 3; ++a)
      if (bc.periodic[a] != bc_.periodic[a])
        throw Error(MISO_B200_ERR_ARG, "the boundary's periodicity differs from the integrator's");
    bool same = true;
    for (int a = 0; a < 3; ++a)
      for (int s = 0; s < 2; ++s)
        for (int f = 0; f < 9; ++f) same = same && bc.sign[a][s][f] == bc_.sign[a][s][f];
    if (same) return;
    check(miso_b200_set_mirror_signs(h_, &bc.sign[0][0][0]), h_, "miso_b200_set_mirror_signs");
    bc_ = bc;
  }
  template <class Src>
  void set_source(const Src &src) {
    if constexpr (std::is_same<Src, NoSource>::value) {
      if (src_on_) {
        check(miso_b200_set_source(h_, MISO_B200_SOURCE_NONE, nullptr, 0), h_,
              "miso_b200_set_source");
        src_on_ = false;
      }
    } else if constexpr (std::is_same<Src, PointGravity<Real>>::value) {
      const double g = (double)src.g;
      if (!src_on_ || g != src_g_) {
        check(miso_b200_set_source(h_, MISO_B200_SOURCE_POINT_GRAVITY, &g, 1), h_,
              "miso_b200_set_source");
        src_on_ = true;
        src_g_ = g;
      }
    } else {
      static_assert(sizeof(Src) == 0,
                    "miso_b200::Integrator takes NoSource or PointGravity<Real> as the source");
    }
  }

  // nsteps of ModelBase::update() with dt kept on the device (resident state)
  void run(int nsteps, bool graph = true) {
    check(miso_b200_run(h_, nsteps, graph ? 1 : 0), h_, "miso_b200_run");
  }
  void sync() { check(miso_b200_sync(h_), h_, "miso_b200_sync"); }
  miso_b200_handle *handle() { return h_; }

 private:
  // double fields pass straight through (host or device pointers); float
  // host fields are widened / narrowed through host staging arrays
  void stage_in(const Real *const src[9], const double *q[9]) {
    if (std::is_same<Real, double>::value) {
      for (int f = 0; f < 9; ++f) q[f] = reinterpret_cast<const double *>(src[f]);
      return;
    }
    host_only(src);
    stage_.resize(9 * cells_);
    for (int f = 0; f < 9; ++f) {
      double *d = stage_.data() + (size_t)f * cells_;
      for (size_t c = 0; c < cells_; ++c) d[c] = (double)src[f][c];
      q[f] = d;
    }
  }
  void stage_out_ptrs(Real *const dst[9], double *q[9]) {
    if (std::is_same<Real, double>::value) {
      for (int f = 0; f < 9; ++f) q[f] = reinterpret_cast<double *>(dst[f]);
      return;
    }
    host_only(dst);
    stage_.resize(9 * cells_);
    for (int f = 0; f < 9; ++f) q[f] = stage_.data() + (size_t)f * cells_;
  }
  void stage_out(Real *const dst[9]) {
    if (std::is_same<Real, double>::value) return;
    for (int f = 0; f < 9; ++f) {
      const double *s = stage_.data() + (size_t)f * cells_;
      for (size_t c = 0; c < cells_; ++c) dst[f][c] = (Real)s[c];
    }
  }

  // float fields are converted on the host: device arrays are refused
  template <class P>
  void host_only(P const p[9]) {
    for (int f = 0; f < 9; ++f) {
      int kind = 0;
      check(miso_b200_pointer_kind(p[f], &kind), h_, "miso_b200_pointer_kind");
      if (kind == 1)
        throw Error(MISO_B200_ERR_ARG,
                    "Real = float fields must be host arrays (device float fields are not "
                    "converted)");
    }
  }

  miso_b200_handle *h_ = nullptr;
  size_t cells_ = 0;
  bool resident_ = false;
  std::vector<double> stage_;
  double gm_ = 0.0;
  Boundary bc_;
  const void *pushed_ = nullptr;  // fields whose state cfl() left on the device
  bool src_on_ = false;
  double src_g_ = 0.0;
};

}  // namespace miso_b200

#endif  // MISO_B200_HPP
