// A MISO model run through the reference's own, unmodified mhd::ModelBase
// (miso/include/miso/mhd_model_base.hpp:41-120) with Backend =
// miso::backend::B200 -- the time step on libmiso_b200.so.  Built by
// tests/cpp/Makefile against the reference's headers where they lie; run by
// tests/test_cpp_modelbase.py.
//
//   modelbase_demo <config.yaml> <initial.bin> <bc> <mode> [const:vx,vy,vz,ei | grav:g]
//
// initial.bin: the 9 primitive arrays (ro .. ph, ghosts included) as raw
// Real values -- the initial condition functor copies them in, so the host
// and the checker start from the same bits.  bc: "empty"
// (mhd::EmptyBoundaryCondition, periodic config), "mirror" (the demos'
// functor: boundary_condition::symmetric with Sign::Pos on every physical
// face and field, demo/mhd1d_shock_tube/src/main.cpp:85-162), "loop" (the
// same mirror written as plain loops, which the backend cannot reduce to
// mirror faces and so runs as a host functor after every pass).  mode:
// "run" (ModelBase::run: initial condition, the time loop to time.tend with
// snapshots every time.dt_output) or "update:N" (N calls of
// ModelBase::update, then one snapshot).  The optional last argument gives
// the model a source functor of its own: four constants as the Source
// concept's vx, vy, vz, ei, which the backend evaluates on host copies of
// every stage's argument state, or the point gravity of constant g, which
// it evaluates on the device where nvcc built the program.  It prints the boundary path the backend
// chose and exits 0, or prints the exception and exits 3.
#include <miso/boundary_condition.hpp>
#include <miso/mhd_model_base.hpp>

#include "miso_b200_backend.hpp"

#include <cstdio>
#include <fstream>
#include <string>
#include <utility>

using namespace miso;

#ifdef MISO_B200_DEMO_FLOAT
using Real = float;
#else
using Real = double;
#endif
using Backend = backend::B200;

struct FileInitialCondition {
  std::string path;
  void apply(mhd::FieldsView<Real> qq, GridView<const Real> grid) const {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open " + path);
    const size_t n = (size_t)grid.i_total * grid.j_total * grid.k_total;
    Array3DView<Real> *f[9] = {&qq.ro, &qq.vx, &qq.vy, &qq.vz, &qq.bx,
                               &qq.by, &qq.bz, &qq.ei, &qq.ph};
    for (auto *a : f) in.read(reinterpret_cast<char *>(a->data()), sizeof(Real) * n);
    if (!in) throw std::runtime_error("short initial state in " + path);
  }
};

// The demos' outflow boundary: the reference's mirror helper on every
// physical face, all 9 fields, Sign::Pos.
struct MirrorBoundaryCondition {
  mpi::Shape &mpi_shape;
  void apply(mhd::FieldsView<Real> qq, GridView<const Real> grid) const {
    namespace bc = miso::boundary_condition;
    Backend btag{};
    Array3DView<Real> *f[9] = {&qq.ro, &qq.vx, &qq.vy, &qq.vz, &qq.bx,
                               &qq.by, &qq.bz, &qq.ei, &qq.ph};
    const Direction dirs[3] = {Direction::X, Direction::Y, Direction::Z};
    const Side sides[2] = {Side::INNER, Side::OUTER};
    for (Direction d : dirs)
      for (Side s : sides)
        if (bc::is_physical_boundary(d, s, mpi_shape))
          for (auto *a : f) bc::symmetric(btag, *a, grid, Sign::Pos, d, s);
  }
};

// The same mirror as plain loops over the ghost layers of each physical
// face (x, then y, then z; full transverse range).
struct LoopBoundaryCondition {
  mpi::Shape &mpi_shape;
  void apply(mhd::FieldsView<Real> qq, GridView<const Real> grid) const {
    namespace bc = miso::boundary_condition;
    Array3DView<Real> *f[9] = {&qq.ro, &qq.vx, &qq.vy, &qq.vz, &qq.bx,
                               &qq.by, &qq.bz, &qq.ei, &qq.ph};
    const int tot[3] = {grid.i_total, grid.j_total, grid.k_total};
    const int mar[3] = {grid.i_margin, grid.j_margin, grid.k_margin};
    const Direction dirs[3] = {Direction::X, Direction::Y, Direction::Z};
    for (int a = 0; a < 3; ++a)
      for (int s = 0; s < 2; ++s) {
        if (!bc::is_physical_boundary(dirs[a], s ? Side::OUTER : Side::INNER, mpi_shape)) continue;
        for (int g = 0; g < mar[a]; ++g) {
          const int gh = s ? tot[a] - mar[a] + g : g;
          const int tg = s ? tot[a] - mar[a] - g - 1 : 2 * mar[a] - g - 1;
          for (int i = 0; i < (a == 0 ? 1 : tot[0]); ++i)
            for (int j = 0; j < (a == 1 ? 1 : tot[1]); ++j)
              for (int k = 0; k < (a == 2 ? 1 : tot[2]); ++k)
                for (auto *arr : f) {
                  const int ig = a == 0 ? gh : i, jg = a == 1 ? gh : j, kg = a == 2 ? gh : k;
                  const int it = a == 0 ? tg : i, jt = a == 1 ? tg : j, kt = a == 2 ? tg : k;
                  (*arr)(ig, jg, kg) = (*arr)(it, jt, kt);
                }
        }
      }
  }
};

// A source functor of the model's own: four constants (force per volume
// along x, y, z and the energy term), in the reference's Source concept
// (mhd_model_base.hpp:131-155).
struct ConstSource {
  Real c[4] = {0, 0, 0, 0};
  Real vx(mhd::FieldsView<const Real>, int, int, int) const { return c[0]; }
  Real vy(mhd::FieldsView<const Real>, int, int, int) const { return c[1]; }
  Real vz(mhd::FieldsView<const Real>, int, int, int) const { return c[2]; }
  Real ei(mhd::FieldsView<const Real>, int, int, int) const { return c[3]; }
};

// The magnetosphere demo's point gravity written as a model's own Source
// functor: force per volume -ro g x / |x|^3 about the coordinate origin, no
// heating.  It keeps a view of the grid for the cell centres.  Built by nvcc,
// the model declares it device-callable, and the backend evaluates it on the
// device before every stage; built by the host compiler, on host copies.
struct GravitySource {
  GridView<const Real> grid;
  Real g;
  __host__ __device__ Real r3(int i, int j, int k) const {
    return util::pow3(util::sqrt(grid.x[i] * grid.x[i] + grid.y[j] * grid.y[j] +
                                 grid.z[k] * grid.z[k]));
  }
  __host__ __device__ Real vx(mhd::FieldsView<const Real> qq, int i, int j, int k) const {
    return -qq.ro(i, j, k) * g * grid.x[i] / r3(i, j, k);
  }
  __host__ __device__ Real vy(mhd::FieldsView<const Real> qq, int i, int j, int k) const {
    return -qq.ro(i, j, k) * g * grid.y[j] / r3(i, j, k);
  }
  __host__ __device__ Real vz(mhd::FieldsView<const Real> qq, int i, int j, int k) const {
    return -qq.ro(i, j, k) * g * grid.z[k] / r3(i, j, k);
  }
  __host__ __device__ Real ei(mhd::FieldsView<const Real>, int, int, int) const { return 0; }
};
#if defined(__CUDACC__)
template <>
struct miso_b200::device_source<GravitySource> : std::true_type {};
#endif

template <class BC> struct MakeBC {
  static BC make(mpi::Shape &s) { return BC{s}; }
};
template <> struct MakeBC<mhd::EmptyBoundaryCondition<Real>> {
  static mhd::EmptyBoundaryCondition<Real> make(mpi::Shape &) { return {}; }
};

// the source object from the model's grid (the gravity keeps its view)
template <class Src> struct MakeSrc {
  static Src make(const Src &s, Grid<Real, Backend> &) { return s; }
};
struct GravitySpec {
  Real g;
};
template <> struct MakeSrc<GravitySpec> {
  static GravitySource make(const GravitySpec &s, Grid<Real, Backend> &grid) {
    return GravitySource{grid.const_view(), s.g};
  }
};

template <class BC, class Spec>
struct Model : public mhd::ModelBase<Model<BC, Spec>, Real, Backend> {
  using Base = mhd::ModelBase<Model<BC, Spec>, Real, Backend>;
  using Src = decltype(MakeSrc<Spec>::make(std::declval<const Spec &>(),
                                           std::declval<Grid<Real, Backend> &>()));
  eos::IdealEOS<Real> eos;
  FileInitialCondition ic;
  BC bc;
  Src src;
  Model(Config &config, const std::string &init, const Spec &s)
      : Base(config), eos(config), ic{init}, bc(MakeBC<BC>::make(this->mpi_shape)),
        src(MakeSrc<Spec>::make(s, this->mhd.grid)) {}
};

template <class BC, class Spec>
int drive(Config &config, const std::string &init, const std::string &mode, const Spec &s) {
  Model<BC, Spec> model(config, init, s);
  if (mode == "run") {
    model.run();
  } else {
    const int n = std::stoi(mode.substr(mode.find(':') + 1));
    model.mhd.apply_initial_condition(model.ic, model.bc);
    for (int s = 0; s < n; ++s) model.update();
    model.save_state();
  }
  std::printf("boundary_path %d steps %d time %.17g\n", model.mhd.integrator.boundary_path(),
              model.time.n_step, (double)model.time.time);
  return 0;
}

int main(int argc, char **argv) {
  if (argc < 5) {
    std::fprintf(stderr, "usage: %s config.yaml initial.bin empty|mirror|loop run|update:N\n",
                 argv[0]);
    return 2;
  }
  Env env(argc, argv);
  Config config(argv[1]);
  const std::string init = argv[2], bc = argv[3], mode = argv[4];
  const std::string source = argc > 5 ? argv[5] : "none";
  try {
    if (source.rfind("const:", 0) == 0) {
      ConstSource cs;
      std::string rest = source.substr(6);
      for (int t = 0; t < 4; ++t) {
        const size_t cut = rest.find(',');
        cs.c[t] = (Real)std::stod(rest.substr(0, cut));
        rest = cut == std::string::npos ? "" : rest.substr(cut + 1);
      }
      if (bc == "empty") return drive<mhd::EmptyBoundaryCondition<Real>>(config, init, mode, cs);
      if (bc == "mirror") return drive<MirrorBoundaryCondition>(config, init, mode, cs);
      if (bc == "loop") return drive<LoopBoundaryCondition>(config, init, mode, cs);
    } else if (source.rfind("grav:", 0) == 0) {
      const GravitySpec gs{(Real)std::stod(source.substr(5))};
      if (bc == "empty") return drive<mhd::EmptyBoundaryCondition<Real>>(config, init, mode, gs);
      if (bc == "mirror") return drive<MirrorBoundaryCondition>(config, init, mode, gs);
      if (bc == "loop") return drive<LoopBoundaryCondition>(config, init, mode, gs);
    } else {
      const mhd::EmptySourceTerm<Real> none{};
      if (bc == "empty") return drive<mhd::EmptyBoundaryCondition<Real>>(config, init, mode, none);
      if (bc == "mirror") return drive<MirrorBoundaryCondition>(config, init, mode, none);
      if (bc == "loop") return drive<LoopBoundaryCondition>(config, init, mode, none);
    }
  } catch (const std::exception &e) {
    std::printf("error: %s\n", e.what());
    return 3;
  }
  std::fprintf(stderr, "unknown boundary %s\n", bc.c_str());
  return 2;
}
