// miso_b200_backend.hpp -- the B200 backend of MISO's own model framework.
//
// Include it (after, or instead of, the MISO headers it pulls in) and use
//
//     using Backend = miso::backend::B200;
//     struct Model : miso::mhd::ModelBase<Model, Real, Backend> { ... };
//
// and the reference's unmodified mhd::MHD and mhd::ModelBase
// (miso/include/miso/mhd.hpp:15-50, mhd_model_base.hpp:41-120) run the time
// step on libmiso_b200.so.  This header adds, next to backend::Host and
// backend::CUDA (miso/include/miso/backend.hpp:9-13):
//
//   backend::B200                       the tag
//   Grid<Real, backend::B200>           the host grid (grid.hpp:147-450), whose
//                                       views read a copy of its coordinate
//                                       arrays in memory host and device share
//   mhd::Fields<Real, backend::B200>    the state, held on the device by the
//                                       integrator it is bound to
//   mhd::ExecContext<Real, backend::B200>
//   mhd::Integrator<Real, backend::B200>  constructed as
//       Integrator(Config &, Grid<Real, B200> &, ExecContext<Real, B200> &)
//     with the reference integrator's members
//       Real cfl(const Fields &, const EOS &)               cuda.cuh:450-478
//       void update(Real dt, const EOS &, const BC &, const Src &, Fields &)
//                                                            cuda.cuh:481-487
//       void apply_boundary_condition(const BC &, Fields &)  cuda.cuh:396-401
//   boundary_condition::symmetric(backend::B200, ...) and
//   for_each(backend::B200, ...), so boundary functors written against the
//   reference's helpers compile for this backend.
//
// Precision.  Real = double runs the FP64 form, bit for bit the reference's
// own double-precision host path; the config key `b200.precision:
// fp32_split` selects the split form instead.  Real = float runs the FP32
// split form (FP32 arithmetic, compensated hi/lo state on the device).
//
// The equation of state must be eos::IdealEOS<Real> (its gm equal to the
// config's eos.gm).  The source: mhd::EmptySourceTerm<Real> and
// miso_b200::PointGravity<Real> run on the device; any other functor of the
// reference's Source concept (vx, vy, vz, ei of (FieldsView<const Real>, i,
// j, k), mhd_model_base.hpp:131-155) is evaluated, in the FP64 form, on host
// copies of every stage's argument state (miso_b200_set_source_callback):
// exact, and slow (with b200.precision: fp32_split, the split form hands it
// the argument state as FP64 primitives).
// Where the model's translation unit is compiled by nvcc
// and the functor type is declared device-callable --
//
//     template <> struct miso_b200::device_source<MySource> : std::true_type {};
//
// (its four methods __host__ __device__, the object trivially copyable, and
// whatever it reads device-accessible: the state, and views of the B200 grid,
// whose coordinate arrays live in shared memory) -- the functor is evaluated
// on the device instead: before every stage one kernel of this header, run
// on the library's stream, fills the four terms of every interior cell from
// the stage's argument state, as the reference's CUDA integrator evaluates
// it inside its kernels (mhd_integrator_cuda.cuh:341-392).  Real = float
// (the split form on FP32 views) refuses such functors with an exception.
//
// Boundary functors (bc.apply(FieldsView<Real>, GridView<const Real>)):
//   * mhd::EmptyBoundaryCondition<Real>: every non-degenerate axis must be
//     periodic (domain.periodic), else the integrator throws -- the
//     reference would leave those ghosts unfilled.
//   * any other functor is run once on a host copy of the state while its
//     boundary_condition::symmetric calls are recorded.  If the recorded
//     calls mirror every non-periodic face for all 9 fields, nothing else
//     was touched, and the functor's result equals that of the library's
//     own face fill (compared bit for bit), the library's device fill runs
//     with the recorded signs from then on (the functor object is assumed
//     to keep doing the same).
//   * otherwise, in the FP64 form, the functor itself runs after every pass
//     on host copies of the fields (miso_b200_set_boundary_callback): exact,
//     and slow (a host round trip per pass).  In the split form such a
//     functor is refused with an exception.
//
// Single rank: a decomposition over several MPI ranks is refused (use the
// halo interface of the C ABI, miso_b200_set_halo / miso_b200_set_halo3).
// Errors are thrown as
// miso_b200::Error (std::runtime_error).
#ifndef MISO_B200_BACKEND_HPP
#define MISO_B200_BACKEND_HPP

#include <cstring>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <typeinfo>
#include <vector>

#include <miso/array3d.hpp>
#include <miso/backend.hpp>
#include <miso/boundary_condition.hpp>
#include <miso/config.hpp>
#include <miso/eos.hpp>
#include <miso/execution.hpp>
#include <miso/grid.hpp>
#include <miso/mhd_core.hpp>
#include <miso/mhd_fields.hpp>
#include <miso/mhd_integrator.hpp>
#include <miso/mhd_model_base.hpp>
#include <miso/types.hpp>

#include "miso_b200.h"

namespace miso {
namespace backend {
/// Tag of the B200 backend (libmiso_b200.so).
struct B200 {};
}  // namespace backend
}  // namespace miso

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

// The magnetosphere demo's point gravity (demo/mhd3d_magnetosphere/src/
// src.hpp:17-44) as a source the device forms itself: force per volume
// -ro g x / |x|^3 about the coordinate origin, no heating.
template <typename Real>
struct PointGravity {
  Real g;
};

// A Source functor type the model declares device-callable: specialise to
// std::true_type (in a translation unit compiled by nvcc).
template <typename Source>
struct device_source : std::false_type {};

namespace detail {

inline void check(int rc, miso_b200_handle *h, const char *what) {
  if (rc != MISO_B200_OK)
    throw Error(rc, std::string(what) + ": " + miso_b200_last_error(h));
}

template <typename T>
struct always_false : std::false_type {};

// What boundary_condition::symmetric(backend::B200, ...) and
// for_each(backend::B200, ...) do on the calling thread: run as the host
// backend does, and, while a functor is being examined, record the mirror
// calls (field, axis, side, sign) and note anything else.
struct BcRecorder {
  bool recording = false;
  const void *fields[9] = {};
  struct Op {
    int field, axis, side;
    double sign;
  };
  std::vector<Op> ops;
  bool opaque = false;  // a call that is not a mirror of one of the 9 fields
};
inline BcRecorder &recorder() {
  static thread_local BcRecorder r;
  return r;
}

}  // namespace detail
}  // namespace miso_b200

namespace miso {

/// Non-owning 3-D array over memory the B200 backend hands to a boundary
/// functor (host copies of the device state); it makes the reference's
/// Array3DView for it.
template <typename T>
class Array3D<T, backend::B200> {
 public:
  Array3D(T *data, int n0, int n1, int n2) noexcept : data_(data), shape_{n0, n1, n2} {}
  Array3DView<T> view() const noexcept { return Array3DView<T>(data_, shape_[0], shape_[1], shape_[2]); }
  T *data() const noexcept { return data_; }

 private:
  T *data_;
  int shape_[3];
};

/// The B200 backend's for_each runs on the host (boundary functors call it
/// on host copies); a functor that calls it is not a plain set of mirrors.
template <class F>
inline void for_each(backend::B200, Range1D range, F f) {
  miso_b200::detail::recorder().opaque |= miso_b200::detail::recorder().recording;
  for_each(backend::Host{}, range, f);
}
template <class F>
inline void for_each(backend::B200, Range3D range, F f) {
  miso_b200::detail::recorder().opaque |= miso_b200::detail::recorder().recording;
  for_each(backend::Host{}, range, f);
}

namespace boundary_condition {
/// boundary_condition::symmetric for the B200 backend: the host mirror of
/// boundary_condition.hpp:109-136 on the array it is given, recorded while
/// the integrator examines a functor.
template <typename Real>
void symmetric(backend::B200, Array3DView<Real> arr, GridView<const Real> grid, Sign sign,
               Direction direction, Side side) {
  auto &r = miso_b200::detail::recorder();
  if (r.recording) {
    int f = -1;
    for (int n = 0; n < 9; ++n)
      if (r.fields[n] == (const void *)arr.data()) f = n;
    if (f < 0) {
      r.opaque = true;
    } else {
      const int axis = direction == Direction::X ? 0 : direction == Direction::Y ? 1 : 2;
      r.ops.push_back({f, axis, side == Side::INNER ? 0 : 1, sign == Sign::Pos ? 1.0 : -1.0});
    }
  }
  symmetric(backend::Host{}, arr, grid, sign, direction, side);
}
}  // namespace boundary_condition

/// The grid of the B200 backend is the host grid (its spacings are copied
/// into the library's descriptor).  Its views read a copy of the nine
/// coordinate and spacing arrays in memory that host and device share
/// (miso_b200_alloc_shared), so that a functor holding a view of the grid --
/// a source term that reads the cell centres -- runs on either side.
template <typename Real>
struct Grid<Real, backend::B200> : Grid<Real, backend::Host> {
  using HostGrid = Grid<Real, backend::Host>;
  explicit Grid(const HostGrid &grid) : HostGrid(grid) { mirror(); }
  Grid(const Grid &o) : HostGrid(o) { mirror(); }
  Grid &operator=(const Grid &o) {
    HostGrid::operator=(o);
    mirror();
    return *this;
  }

  GridView<Real> view() noexcept { return make_view<Real>(); }
  GridView<const Real> view() const noexcept { return make_view<const Real>(); }
  GridView<const Real> const_view() const noexcept { return view(); }

 private:
  std::shared_ptr<Real> shared_;
  Real *arr_[9] = {};  // x, y, z, dx, dy, dz, dxi, dyi, dzi

  void mirror() {
    const std::vector<Real> *src[9] = {&this->x,  &this->y,  &this->z,   &this->dx, &this->dy,
                                       &this->dz, &this->dxi, &this->dyi, &this->dzi};
    size_t n = 0;
    for (auto *v : src) n += v->size();
    void *p = nullptr;
    const int rc = miso_b200_alloc_shared(n * sizeof(Real), &p);
    if (rc != MISO_B200_OK)
      throw miso_b200::Error(rc, "miso_b200_alloc_shared: no memory for the grid's coordinates");
    shared_.reset(static_cast<Real *>(p), [](Real *q) { miso_b200_free_shared(q); });
    Real *at = shared_.get();
    for (int a = 0; a < 9; ++a) {
      arr_[a] = at;
      std::memcpy(at, src[a]->data(), src[a]->size() * sizeof(Real));
      at += src[a]->size();
    }
  }
  template <typename T>
  GridView<T> make_view() const noexcept {
    return GridView<T>(this->i_total, this->j_total, this->k_total, this->is, this->js, this->ks,
                       this->i_margin, this->j_margin, this->k_margin, this->min_dxyz, arr_[0],
                       arr_[1], arr_[2], arr_[3], arr_[4], arr_[5], arr_[6], arr_[7], arr_[8]);
  }
};

namespace mhd {

template <typename Real>
struct ExecContext<Real, backend::B200> {
  mpi::Shape &mpi_shape;
  ExecContext(mpi::Shape &mpi_shape_, const Grid<Real, backend::Host> &) : mpi_shape(mpi_shape_) {}
};

}  // namespace mhd
}  // namespace miso

namespace miso_b200 {
namespace detail {

// The state behind a Fields<Real, backend::B200>: on the device of the
// integrator it is bound to, and a host mirror for copies in and out.
template <typename Real>
struct FieldsState {
  int dims[3];
  size_t cells;
  miso_b200_handle *h = nullptr;
  std::unique_ptr<miso::mhd::Fields<Real, miso::backend::Host>> mirror;
  bool host_newer = false;  // the mirror holds a state the device has not seen
  std::vector<double> stage;  // Real = float: FP64 staging of the C ABI

  FieldsState(int i, int j, int k) : dims{i, j, k}, cells((size_t)i * j * k) {}

  miso::mhd::Fields<Real, miso::backend::Host> &host() {
    if (!mirror) mirror.reset(new miso::mhd::Fields<Real, miso::backend::Host>(dims[0], dims[1], dims[2]));
    return *mirror;
  }
  static void ptrs(const miso::mhd::Fields<Real, miso::backend::Host> &q, const Real *p[9]) {
    const Real *a[9] = {q.ro.data(), q.vx.data(), q.vy.data(), q.vz.data(), q.bx.data(),
                        q.by.data(), q.bz.data(), q.ei.data(), q.ph.data()};
    for (int f = 0; f < 9; ++f) p[f] = a[f];
  }
  void upload(const miso::mhd::Fields<Real, miso::backend::Host> &src) {
    const Real *p[9];
    ptrs(src, p);
    const double *q[9];
    if (std::is_same<Real, double>::value) {
      for (int f = 0; f < 9; ++f) q[f] = reinterpret_cast<const double *>(p[f]);
    } else {
      stage.resize(9 * cells);
      for (int f = 0; f < 9; ++f) {
        double *d = stage.data() + (size_t)f * cells;
        for (size_t c = 0; c < cells; ++c) d[c] = (double)p[f][c];
        q[f] = d;
      }
    }
    check(miso_b200_upload(h, q), h, "miso_b200_upload");
  }
  void download() {
    auto &m = host();
    const Real *p[9];
    ptrs(m, p);
    double *q[9];
    if (std::is_same<Real, double>::value) {
      for (int f = 0; f < 9; ++f) q[f] = reinterpret_cast<double *>(const_cast<Real *>(p[f]));
      check(miso_b200_download(h, q), h, "miso_b200_download");
      return;
    }
    stage.resize(9 * cells);
    for (int f = 0; f < 9; ++f) q[f] = stage.data() + (size_t)f * cells;
    check(miso_b200_download(h, q), h, "miso_b200_download");
    for (int f = 0; f < 9; ++f) {
      Real *d = const_cast<Real *>(p[f]);
      const double *s = stage.data() + (size_t)f * cells;
      for (size_t c = 0; c < cells; ++c) d[c] = (Real)s[c];
    }
  }
};

}  // namespace detail
}  // namespace miso_b200

namespace miso {
namespace mhd {

/// The MHD state of the B200 backend.  Once an integrator has used it, the
/// state lives on that integrator's device; copy_from() uploads, and the
/// conversion to const Fields<Real, backend::Host>& (what Checkpoint::save
/// and qq_h.copy_from(qq) use) downloads into a host mirror.
template <typename Real>
struct Fields<Real, backend::B200> {
  std::shared_ptr<miso_b200::detail::FieldsState<Real>> st;

  Fields(const int i_total, const int j_total, const int k_total)
      : st(std::make_shared<miso_b200::detail::FieldsState<Real>>(i_total, j_total, k_total)) {}

  template <typename GridType>
  explicit Fields(const GridType &grid) : Fields(grid.i_total, grid.j_total, grid.k_total) {}

  void copy_from(const Fields<Real, backend::Host> &other) {
    if (other.ro.size() != (int)st->cells) throw miso_b200::Error(MISO_B200_ERR_ARG, "copy_from: size mismatch");
    if (st->h) {
      st->upload(other);
      return;
    }
    st->host().copy_from(other);
    st->host_newer = true;
  }
  void copy_from(const Fields<Real, backend::B200> &other) { copy_from(other.host()); }

  /// The state on the host (downloaded from the device when bound).
  const Fields<Real, backend::Host> &host() const {
    if (st->h) {
      st->download();
      st->host_newer = false;
    }
    return st->host();
  }
  operator const Fields<Real, backend::Host> &() const { return host(); }

  Fields(const Fields &) = delete;
  Fields &operator=(const Fields &) = delete;
  Fields(Fields &&) = default;
  Fields &operator=(Fields &&) = default;
};

}  // namespace mhd
}  // namespace miso

#if defined(__CUDACC__)
namespace miso_b200 {
namespace detail {

// The four terms of a device-callable Source functor at every interior cell
// of the stage's argument state qq (FP64 arrays of the field layout):
// s[0..2] the forces per volume src.vx / vy / vz, s[3] the heating src.ei,
// as the reference's stage kernels call them per cell
// (mhd_integrator_cuda.cuh:341-392 on mhd_integrator_host.hpp:134, 151,
// 168, 241).
template <typename Real, typename Source>
__global__ void __launch_bounds__(256)
source_terms_kernel(const Source src, const miso::mhd::FieldsView<const Real> qq, double *s0,
                    double *s1, double *s2, double *s3, int n1, int n2, int m0, int m1, int m2,
                    int ni, int nj, int nk) {
  const long long total = (long long)ni * nj * nk;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t % nk) + m2;
    const long long r = t / nk;
    const int j = (int)(r % nj) + m1;
    const int i = (int)(r / nj) + m0;
    const long long c = ((long long)i * n1 + j) * n2 + k;
    s0[c] = (double)src.vx(qq, i, j, k);
    s1[c] = (double)src.vy(qq, i, j, k);
    s2[c] = (double)src.vz(qq, i, j, k);
    s3[c] = (double)src.ei(qq, i, j, k);
  }
}

}  // namespace detail
}  // namespace miso_b200
#endif

namespace miso {
namespace mhd {

/// The reference integrator's interface (mhd_integrator_cuda.cuh:291-501)
/// over libmiso_b200.so.
template <typename Real>
struct Integrator<Real, backend::B200> {
  static_assert(std::is_same<Real, double>::value || std::is_same<Real, float>::value,
                "Real must be float or double");

  Grid<Real, backend::B200> &grid;
  ExecContext<Real, backend::B200> &exec_ctx;
  Real cfl_number;

  Integrator(Config &config, Grid<Real, backend::B200> &grid_,
             ExecContext<Real, backend::B200> &exec_ctx_)
      : grid(grid_), exec_ctx(exec_ctx_) {
    const mpi::Shape &sh = exec_ctx.mpi_shape;
    if (sh.x_procs * sh.y_procs * sh.z_procs != 1)
      throw miso_b200::Error(MISO_B200_ERR_ARG,
                             "the B200 backend runs one grid per process (mpi x/y/z_procs = 1)");
    miso_b200_grid_desc gd{};
    gd.i_size = grid.i_size;
    gd.j_size = grid.j_size;
    gd.k_size = grid.k_size;
    gd.margin = grid.i_margin > grid.j_margin ? grid.i_margin : grid.j_margin;
    if (grid.k_margin > gd.margin) gd.margin = grid.k_margin;
    gd.x_min = grid.x_min;
    gd.x_max = grid.x_max;
    gd.y_min = grid.y_min;
    gd.y_max = grid.y_max;
    gd.z_min = grid.z_min;
    gd.z_max = grid.z_max;
    gd.periodic[0] = config["domain"]["periodic"]["x"].as<bool>() ? 1 : 0;
    gd.periodic[1] = config["domain"]["periodic"]["y"].as<bool>() ? 1 : 0;
    gd.periodic[2] = config["domain"]["periodic"]["z"].as<bool>() ? 1 : 0;
    for (int a = 0; a < 3; ++a)
      for (int s = 0; s < 2; ++s)
        for (int f = 0; f < 9; ++f) gd.sign[a][s][f] = 1.0;
    for (int a = 0; a < 3; ++a) periodic_[a] = gd.periodic[a];
    sizes_[0] = grid.i_size;
    sizes_[1] = grid.j_size;
    sizes_[2] = grid.k_size;
    miso_b200_params pp{};
    pp.gm = config["eos"]["gm"].as<double>();
    pp.cfl_number = config["mhd"]["cfl_number"].as<double>();
    pp.ep = config["mhd"]["artificial_viscosity"]["ep"].as<double>();
    pp.fh = config["mhd"]["artificial_viscosity"]["fh"].as<double>();
    pp.cs_fac = config["mhd"]["artificial_viscosity"]["cs_fac"].as<double>();
    pp.ca_fac = config["mhd"]["artificial_viscosity"]["ca_fac"].as<double>();
    pp.vv_fac = config["mhd"]["artificial_viscosity"]["vv_fac"].as<double>();
    pp.precision = std::is_same<Real, double>::value ? MISO_B200_FP64 : MISO_B200_FP32_SPLIT;
    const YAML::Node &root = config.yaml_obj;
    if (std::is_same<Real, double>::value && root["b200"] && root["b200"]["precision"]) {
      const std::string p = root["b200"]["precision"].template as<std::string>();
      if (p == "fp32_split")
        pp.precision = MISO_B200_FP32_SPLIT;
      else if (p != "fp64")
        throw miso_b200::Error(MISO_B200_ERR_ARG, "b200.precision must be fp64 or fp32_split");
    }
    gm_ = pp.gm;
    precision_ = pp.precision;
    cfl_number = config["mhd"]["cfl_number"].as<Real>();
    miso_b200::detail::check(miso_b200_create(&gd, &pp, nullptr, &h_), nullptr,
                             "miso_b200_create");
  }
  ~Integrator() {
    if (h_) miso_b200_destroy(h_);
  }

  template <typename BoundaryCondition>
  void apply_boundary_condition(const BoundaryCondition &bc, Fields<Real, backend::B200> &qq) {
    bind(qq);
    configure_boundary(bc, qq);
    miso_b200::detail::check(miso_b200_fill_ghosts(h_), h_, "miso_b200_fill_ghosts");
  }

  template <typename EOS>
  Real cfl(const Fields<Real, backend::B200> &qq, const EOS &eos) {
    bind(qq);
    check_eos(eos);
    double dt = 0.0;
    miso_b200::detail::check(miso_b200_cfl(h_, &dt), h_, "miso_b200_cfl");
    return (Real)dt;
  }

  template <typename EOS, typename BoundaryCondition, typename Source>
  void update(Real dt, const EOS &eos, const BoundaryCondition &bc, const Source &src,
              Fields<Real, backend::B200> &qq) {
    bind(qq);
    check_eos(eos);
    configure_boundary(bc, qq);
    configure_source(src);
    miso_b200::detail::check(miso_b200_update(h_, (double)dt), h_, "miso_b200_update");
  }

  /// How the last boundary functor runs: 0 the library's periodic / mirror
  /// fill, 1 the functor itself on host copies after every pass.
  int boundary_path() const { return bc_path_; }
  miso_b200_handle *handle() const { return h_; }

  Integrator(const Integrator &) = delete;
  Integrator &operator=(const Integrator &) = delete;
  Integrator(Integrator &&) = delete;
  Integrator &operator=(Integrator &&) = delete;

 private:
  miso_b200_handle *h_ = nullptr;
  double gm_ = 0.0;
  int precision_ = MISO_B200_FP64;
  int periodic_[3] = {0, 0, 0};
  int sizes_[3] = {1, 1, 1};
  const std::type_info *bc_type_ = nullptr;
  const void *bc_obj_ = nullptr;
  int bc_path_ = 0;
  std::function<void(FieldsView<Real>)> bc_fn_;
  int src_kind_ = MISO_B200_SOURCE_NONE;  // or kSourceFunctor
  double src_g_ = 0.0;
  static constexpr int kSourceFunctor = -1;  // a caller's functor through the callback
  const void *src_obj_ = nullptr;
  std::function<void(const double *const *, double *const *)> src_fn_;

  void bind(const Fields<Real, backend::B200> &qq) {
    auto &st = *qq.st;
    if (st.h == h_) return;
    if (st.h) throw miso_b200::Error(MISO_B200_ERR_STATE, "the fields belong to another integrator");
    if (st.dims[0] != grid.i_total || st.dims[1] != grid.j_total || st.dims[2] != grid.k_total)
      throw miso_b200::Error(MISO_B200_ERR_ARG, "the fields do not match the integrator's grid");
    st.h = h_;
    if (st.host_newer) {
      st.upload(st.host());
      st.host_newer = false;
    }
  }

  template <typename EOS>
  void check_eos(const EOS &eos) {
    static_assert(std::is_same<EOS, eos::IdealEOS<Real>>::value,
                  "the B200 backend implements eos::IdealEOS<Real> only");
    if (eos.gm != (Real)gm_)
      throw miso_b200::Error(MISO_B200_ERR_ARG, "the EOS's gm differs from the config's eos.gm");
  }

  // leave the functor path (before a built-in source is set)
  void drop_source_functor() {
    if (src_kind_ != kSourceFunctor) return;
    miso_b200::detail::check(miso_b200_set_source_callback(h_, nullptr, nullptr, 0), h_,
                             "miso_b200_set_source_callback");
    src_kind_ = MISO_B200_SOURCE_NONE;
    src_obj_ = nullptr;
  }

  template <typename Source>
  void configure_source(const Source &src) {
    if constexpr (std::is_same<Source, EmptySourceTerm<Real>>::value) {
      drop_source_functor();
      if (src_kind_ != MISO_B200_SOURCE_NONE) {
        miso_b200::detail::check(miso_b200_set_source(h_, MISO_B200_SOURCE_NONE, nullptr, 0), h_,
                                 "miso_b200_set_source");
        src_kind_ = MISO_B200_SOURCE_NONE;
      }
    } else if constexpr (std::is_same<Source, miso_b200::PointGravity<Real>>::value) {
      drop_source_functor();
      const double g = (double)src.g;
      if (src_kind_ != MISO_B200_SOURCE_POINT_GRAVITY || src_g_ != g) {
        miso_b200::detail::check(
            miso_b200_set_source(h_, MISO_B200_SOURCE_POINT_GRAVITY, &g, 1), h_,
            "miso_b200_set_source");
        src_kind_ = MISO_B200_SOURCE_POINT_GRAVITY;
        src_g_ = g;
      }
    } else {
      // any other functor of the Source concept: its four terms on the
      // device (a functor declared device-callable) or on host copies of
      // every stage's argument state (the object must outlive the steps, as
      // the model's own `src` member does)
      if (!std::is_same<Real, double>::value)
        throw miso_b200::Error(MISO_B200_ERR_STATE,
                               std::string("source functor ") + typeid(Source).name() +
                                   " runs with Real = double only (the FP64 form, or the split "
                                   "form by b200.precision)");
      if (src_kind_ == kSourceFunctor && src_obj_ == (const void *)&src) return;
      if (src_kind_ != MISO_B200_SOURCE_NONE && src_kind_ != kSourceFunctor) {
        miso_b200::detail::check(miso_b200_set_source(h_, MISO_B200_SOURCE_NONE, nullptr, 0), h_,
                                 "miso_b200_set_source");
      }
      if constexpr (miso_b200::device_source<Source>::value) {
#if defined(__CUDACC__)
        static_assert(std::is_trivially_copyable<Source>::value,
                      "a device source functor is copied into a kernel: it must be trivially "
                      "copyable");
        src_obj_ = (const void *)&src;
        miso_b200::detail::check(
            miso_b200_set_source_callback(h_, &Integrator::src_device_trampoline<Source>, this,
                                          0),
            h_, "miso_b200_set_source_callback");
        src_kind_ = kSourceFunctor;
        return;
#else
        static_assert(miso_b200::detail::always_false<Source>::value,
                      "a device source functor needs its translation unit compiled by nvcc");
#endif
      }
      const Source *sp = &src;
      src_fn_ = [this, sp](const double *const *q, double *const *s) {
        const int n0 = grid.i_total, n1 = grid.j_total, n2 = grid.k_total;
        auto v = [&](int f) {
          return Array3D<const Real, backend::B200>(reinterpret_cast<const Real *>(q[f]), n0, n1,
                                                    n2)
              .view();
        };
        const FieldsView<const Real> qq(v(0), v(1), v(2), v(3), v(4), v(5), v(6), v(7), v(8));
        for (int i = grid.i_margin; i < n0 - grid.i_margin; ++i)
          for (int j = grid.j_margin; j < n1 - grid.j_margin; ++j)
            for (int k = grid.k_margin; k < n2 - grid.k_margin; ++k) {
              const long c = ((long)i * n1 + j) * n2 + k;
              s[0][c] = (double)sp->vx(qq, i, j, k);
              s[1][c] = (double)sp->vy(qq, i, j, k);
              s[2][c] = (double)sp->vz(qq, i, j, k);
              s[3][c] = (double)sp->ei(qq, i, j, k);
            }
      };
      miso_b200::detail::check(
          miso_b200_set_source_callback(h_, &Integrator::src_trampoline, this, 1), h_,
          "miso_b200_set_source_callback");
      src_kind_ = kSourceFunctor;
      src_obj_ = (const void *)&src;
    }
  }

#if defined(__CUDACC__)
  // before every stage: the device-callable functor's terms by one kernel
  // on the library's stream, from the stage's argument state (device arrays)
  template <typename Source>
  static int src_device_trampoline(void *user, const double *const q[9], double *const s[4],
                                   void *stream) {
    auto *self = static_cast<Integrator *>(user);
    const Grid<Real, backend::B200> &g = self->grid;
    const int n0 = g.i_total, n1 = g.j_total, n2 = g.k_total;
    auto v = [&](int f) {
      return Array3D<const Real, backend::B200>(reinterpret_cast<const Real *>(q[f]), n0, n1, n2)
          .view();
    };
    const FieldsView<const Real> qq(v(0), v(1), v(2), v(3), v(4), v(5), v(6), v(7), v(8));
    const int ni = n0 - 2 * g.i_margin, nj = n1 - 2 * g.j_margin, nk = n2 - 2 * g.k_margin;
    const long long total = (long long)ni * nj * nk;
    long long blocks = (total + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    if (blocks < 1) blocks = 1;
    cudaGetLastError();
    miso_b200::detail::source_terms_kernel<Real, Source>
        <<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(
            *static_cast<const Source *>(self->src_obj_), qq, s[0], s[1], s[2], s[3], n1, n2,
            g.i_margin, g.j_margin, g.k_margin, ni, nj, nk);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
  }
#endif

  static int src_trampoline(void *user, const double *const q[9], double *const s[4], void *) {
    auto *self = static_cast<Integrator *>(user);
    try {
      self->src_fn_(q, s);
      return 0;
    } catch (...) {
      return 1;
    }
  }

  static int bc_trampoline(void *user, double *const q[9], void *) {
    if constexpr (!std::is_same<Real, double>::value) {
      return 1;  // the callback path is the FP64 form's (Real = double)
    }
    auto *self = static_cast<Integrator *>(user);
    try {
      const int n0 = self->grid.i_total, n1 = self->grid.j_total, n2 = self->grid.k_total;
      Real *p[9];
      for (int f = 0; f < 9; ++f) p[f] = reinterpret_cast<Real *>(q[f]);
      const Array3D<Real, backend::B200> a0(p[0], n0, n1, n2), a1(p[1], n0, n1, n2),
          a2(p[2], n0, n1, n2), a3(p[3], n0, n1, n2), a4(p[4], n0, n1, n2), a5(p[5], n0, n1, n2),
          a6(p[6], n0, n1, n2), a7(p[7], n0, n1, n2), a8(p[8], n0, n1, n2);
      self->bc_fn_(FieldsView<Real>(a0.view(), a1.view(), a2.view(), a3.view(), a4.view(),
                                    a5.view(), a6.view(), a7.view(), a8.view()));
      return 0;
    } catch (...) {
      return 1;
    }
  }

  // The faces descriptor's fill on a host copy (axes x, y, z; both sides;
  // all fields): what the device does for the mirror faces.
  void descriptor_fill(Fields<Real, backend::Host> &c, const double (&sign)[3][2][9]) const {
    Array3DView<Real> v[9] = {c.ro.view(), c.vx.view(), c.vy.view(), c.vz.view(), c.bx.view(),
                              c.by.view(), c.bz.view(), c.ei.view(), c.ph.view()};
    const Direction dirs[3] = {Direction::X, Direction::Y, Direction::Z};
    const Side sides[2] = {Side::INNER, Side::OUTER};
    for (int a = 0; a < 3; ++a) {
      if (sizes_[a] <= 1 || periodic_[a]) continue;
      for (int s = 0; s < 2; ++s)
        for (int f = 0; f < 9; ++f)
          boundary_condition::symmetric(backend::Host{}, v[f], grid.const_view(),
                                        sign[a][s][f] < 0 ? Sign::Neg : Sign::Pos, dirs[a],
                                        sides[s]);
    }
  }

  template <typename BoundaryCondition>
  void configure_boundary(const BoundaryCondition &bc, Fields<Real, backend::B200> &qq) {
    if (bc_type_ == &typeid(BoundaryCondition) && bc_obj_ == (const void *)&bc) return;
    if constexpr (std::is_same<BoundaryCondition, EmptyBoundaryCondition<Real>>::value) {
      for (int a = 0; a < 3; ++a)
        if (sizes_[a] > 1 && !periodic_[a])
          throw miso_b200::Error(MISO_B200_ERR_ARG,
                                 "EmptyBoundaryCondition leaves the ghosts of a non-periodic "
                                 "axis unfilled; set domain.periodic or pass a boundary functor");
      set_path(0, nullptr);
    } else {
      // examine the functor on a host copy of the state
      auto &st = *qq.st;
      if (st.h && !st.host_newer) st.download();
      Fields<Real, backend::Host> &m = st.host();
      Fields<Real, backend::Host> c(grid.i_total, grid.j_total, grid.k_total);
      c.copy_from(m);
      auto &r = miso_b200::detail::recorder();
      const void *fp[9] = {m.ro.data(), m.vx.data(), m.vy.data(), m.vz.data(), m.bx.data(),
                           m.by.data(), m.bz.data(), m.ei.data(), m.ph.data()};
      for (int f = 0; f < 9; ++f) r.fields[f] = fp[f];
      r.ops.clear();
      r.opaque = false;
      r.recording = true;
      try {
        bc.apply(m.view(), grid.const_view());
      } catch (...) {
        r.recording = false;
        throw;
      }
      r.recording = false;
      bool plain = !r.opaque;
      double sign[3][2][9];
      int seen[3][2][9] = {};
      for (int a = 0; a < 3; ++a)
        for (int s = 0; s < 2; ++s)
          for (int f = 0; f < 9; ++f) sign[a][s][f] = 1.0;
      for (const auto &op : r.ops) {
        if (sizes_[op.axis] <= 1) continue;  // a degenerate axis has no ghosts: no effect
        if (seen[op.axis][op.side][op.field]++ || periodic_[op.axis]) plain = false;
        sign[op.axis][op.side][op.field] = op.sign;
      }
      for (int a = 0; a < 3; ++a)
        for (int s = 0; s < 2; ++s)
          for (int f = 0; f < 9; ++f)
            if (sizes_[a] > 1 && !periodic_[a] && !seen[a][s][f]) plain = false;
      if (plain) {
        descriptor_fill(c, sign);
        const Real *x[9] = {m.ro.data(), m.vx.data(), m.vy.data(), m.vz.data(), m.bx.data(),
                            m.by.data(), m.bz.data(), m.ei.data(), m.ph.data()};
        const Real *y[9] = {c.ro.data(), c.vx.data(), c.vy.data(), c.vz.data(), c.bx.data(),
                            c.by.data(), c.bz.data(), c.ei.data(), c.ph.data()};
        for (int f = 0; f < 9 && plain; ++f)
          plain = std::memcmp(x[f], y[f], sizeof(Real) * st.cells) == 0;
      }
      // the examined copy now differs from the device state
      st.host_newer = false;
      if (plain) {
        miso_b200::detail::check(miso_b200_set_mirror_signs(h_, &sign[0][0][0]), h_,
                                 "miso_b200_set_mirror_signs");
        set_path(0, nullptr);
      } else {
        if (precision_ != MISO_B200_FP64)
          throw miso_b200::Error(
              MISO_B200_ERR_STATE,
              std::string("boundary functor ") + typeid(BoundaryCondition).name() +
                  " is not a set of mirror faces; only the FP64 form (Real = double) runs "
                  "such a functor");
        const BoundaryCondition *b = &bc;
        bc_fn_ = [this, b](FieldsView<Real> v) { b->apply(v, grid.const_view()); };
        set_path(1, &Integrator::bc_trampoline);
      }
    }
    bc_type_ = &typeid(BoundaryCondition);
    bc_obj_ = (const void *)&bc;
  }

  void set_path(int path, miso_b200_boundary_fn fn) {
    if (path == bc_path_ && path == 0) return;
    miso_b200::detail::check(miso_b200_set_boundary_callback(h_, fn, fn ? this : nullptr, 1), h_,
                             "miso_b200_set_boundary_callback");
    bc_path_ = path;
  }
};

}  // namespace mhd
}  // namespace miso

#endif  // MISO_B200_BACKEND_HPP
