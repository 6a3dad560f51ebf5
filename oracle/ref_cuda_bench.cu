/*
 * ref_cuda_bench.cu -- times the reference's OWN CUDA integrator
 * (miso::mhd::Integrator<Real, backend::CUDA>, mhd_integrator_cuda.cuh:
 * 291-501, with its artificial viscosity and halo exchanger) on one grid,
 * compiled by nvcc for sm_100a from the MISO headers where they lie.  It is
 * the measured baseline of the reference's GPU path; nothing in the product
 * loads it.  Built by oracle/Makefile (target refcuda) into
 * oracle/_ref/miso_ref_cuda_f64 and _f32 (REF_REAL = double / float: the
 * reference's reduction kernel declares its dynamic shared array per type,
 * so one translation unit holds one Real type).
 *
 *   miso_ref_cuda_f64 <in.bin> <warmup> <steps> [out.bin]
 *
 * in.bin: int32 i_size, j_size, k_size, margin, periodic[3];
 *         float64 x_min, x_max, y_min, y_max, z_min, z_max, gm, cfl_number,
 *                 ep, fh, cs_fac, ca_fac, vv_fac;
 *         float64 sign[3][2][9];
 *         float64 fields[9][i_total * j_total * k_total]
 *
 * Each step is ModelBase::update() (mhd_model_base.hpp:57-62): dt =
 * integrator.cfl(qq, eos), then integrator.update(dt, eos, bc, src, qq).
 * The timed steps are bracketed by CUDA events on the default stream the
 * reference launches on.  Prints one JSON line; with out.bin, writes the
 * final 9 fields as float64.
 */
#include <miso/boundary_condition.hpp>
#include <miso/eos.hpp>
#include <miso/mhd_integrator.hpp>
#include <miso/mhd_model_base.hpp>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <unistd.h>
#include <vector>

using namespace miso;

#ifndef REF_REAL
#define REF_REAL double
#endif

namespace {

struct Desc {
  int size[3], margin, periodic[3];
  double lim[6], gm, cfl, ep, fh, cs_fac, ca_fac, vv_fac;
  double sign[3][2][9];
};

// the demos' "outflow" boundary (demo/mhd1d_shock_tube/src/main.cpp:85-162):
// boundary_condition::symmetric on every physical face, per-field sign
template <typename Real>
struct DescBC {
  mpi::Shape &shape;
  const Desc &d;
  DescBC(mpi::Shape &s, const Desc &dd) : shape(s), d(dd) {}
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
            bc::symmetric(backend::CUDA{}, *f[v], grid,
                          d.sign[a][s][v] < 0 ? Sign::Neg : Sign::Pos, dirs[a], sides[s]);
  }
};

std::string write_config(const Desc &d) {
  char tmpl[] = "/tmp/miso_ref_cuda_cfgXXXXXX";
  const int fd = mkstemp(tmpl);
  if (fd < 0) throw std::runtime_error("mkstemp failed");
  close(fd);
  std::ostringstream y;
  y.precision(17);
  y << "io:\n  enabled: false\n  continue: false\n  save_dir: ./\n";
  y << "grid:\n  i_size: " << d.size[0] << "\n  j_size: " << d.size[1] << "\n  k_size: "
    << d.size[2] << "\n  margin: " << d.margin << "\n  x_min: " << d.lim[0]
    << "\n  x_max: " << d.lim[1] << "\n  y_min: " << d.lim[2] << "\n  y_max: " << d.lim[3]
    << "\n  z_min: " << d.lim[4] << "\n  z_max: " << d.lim[5] << "\n";
  y << "mpi:\n  x_procs: 1\n  y_procs: 1\n  z_procs: 1\n";
  y << "domain:\n  periodic:\n    x: " << (d.periodic[0] ? "true" : "false")
    << "\n    y: " << (d.periodic[1] ? "true" : "false")
    << "\n    z: " << (d.periodic[2] ? "true" : "false") << "\n";
  y << "mhd:\n  cfl_number: " << d.cfl << "\n  artificial_viscosity:\n    ep: " << d.ep
    << "\n    fh: " << d.fh << "\n    cs_fac: " << d.cs_fac << "\n    ca_fac: " << d.ca_fac
    << "\n    vv_fac: " << d.vv_fac << "\n";
  y << "eos:\n  gm: " << d.gm << "\n";
  std::ofstream f(tmpl);
  f << y.str();
  return tmpl;
}

template <typename Real>
int run(const Desc &d, const std::vector<double> &fields, int warm, int steps,
        const char *out_path) {
  const std::string cfg_path = write_config(d);
  Config config(cfg_path);
  mpi::Shape shape(config);
  Grid<Real, backend::Host> grid_h(d.size[0], d.size[1], d.size[2], d.margin, (Real)d.lim[0],
                                   (Real)d.lim[1], (Real)d.lim[2], (Real)d.lim[3],
                                   (Real)d.lim[4], (Real)d.lim[5]);
  mhd::ExecContext<Real, backend::CUDA> ctx(shape, grid_h);
  Grid<Real, backend::CUDA> grid(grid_h);
  mhd::Integrator<Real, backend::CUDA> integ(config, grid, ctx);
  eos::IdealEOS<Real> eos((Real)d.gm);
  DescBC<Real> bc(shape, d);
  mhd::EmptySourceTerm<Real> src;
  mhd::Fields<Real, backend::CUDA> qq(grid_h);
  mhd::Fields<Real, backend::Host> qq_h(grid_h);
  Array3D<Real, backend::Host> *hf[9] = {&qq_h.ro, &qq_h.vx, &qq_h.vy, &qq_h.vz, &qq_h.bx,
                                         &qq_h.by, &qq_h.bz, &qq_h.ei, &qq_h.ph};
  const size_t cells = (size_t)hf[0]->size();
  for (int v = 0; v < 9; ++v)
    for (size_t c = 0; c < cells; ++c) hf[v]->data()[c] = (Real)fields[v * cells + c];
  qq.copy_from(qq_h);
  integ.apply_boundary_condition(bc, qq);
  for (int n = 0; n < warm; ++n) {
    const Real dt = integ.cfl(qq, eos);
    integ.update(dt, eos, bc, src, qq);
  }
  cudaDeviceSynchronize();
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  for (int n = 0; n < steps; ++n) {
    const Real dt = integ.cfl(qq, eos);
    integ.update(dt, eos, bc, src, qq);
  }
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  const cudaError_t err = cudaGetLastError();
  const double interior = (double)d.size[0] * d.size[1] * d.size[2];
  std::printf("{\"impl\": \"reference-cuda\", \"real_bytes\": %d, \"steps\": %d, "
              "\"warmup\": %d, \"ms_per_step\": %.6f, \"gcell_updates_per_s\": %.6f, "
              "\"cuda_error\": \"%s\"}\n",
              (int)sizeof(Real), steps, warm, ms / steps,
              interior * steps / (ms * 1e-3) / 1e9, cudaGetErrorString(err));
  if (out_path) {
    qq_h.copy_from(qq);
    std::ofstream o(out_path, std::ios::binary);
    std::vector<double> buf(cells);
    for (int v = 0; v < 9; ++v) {
      for (size_t c = 0; c < cells; ++c) buf[c] = (double)hf[v]->data()[c];
      o.write(reinterpret_cast<const char *>(buf.data()), sizeof(double) * cells);
    }
  }
  std::remove(cfg_path.c_str());
  return err == cudaSuccess ? 0 : 3;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s in.bin warmup steps [out.bin]\n", argv[0]);
    return 1;
  }
  std::ifstream in(argv[1], std::ios::binary);
  if (!in) return 1;
  Desc d{};
  int hdr[7];
  in.read(reinterpret_cast<char *>(hdr), sizeof hdr);
  for (int a = 0; a < 3; ++a) d.size[a] = hdr[a];
  d.margin = hdr[3];
  for (int a = 0; a < 3; ++a) d.periodic[a] = hdr[4 + a];
  double p[13];
  in.read(reinterpret_cast<char *>(p), sizeof p);
  for (int a = 0; a < 6; ++a) d.lim[a] = p[a];
  d.gm = p[6];
  d.cfl = p[7];
  d.ep = p[8];
  d.fh = p[9];
  d.cs_fac = p[10];
  d.ca_fac = p[11];
  d.vv_fac = p[12];
  in.read(reinterpret_cast<char *>(d.sign), sizeof d.sign);
  size_t cells = 1;
  for (int a = 0; a < 3; ++a) cells *= (size_t)(d.size[a] + (d.size[a] > 1 ? 2 * d.margin : 0));
  std::vector<double> fields(9 * cells);
  in.read(reinterpret_cast<char *>(fields.data()), sizeof(double) * fields.size());
  if (!in) {
    std::fprintf(stderr, "short input file\n");
    return 1;
  }
  const int warm = std::atoi(argv[2]), steps = std::atoi(argv[3]);
  const char *out = argc > 4 ? argv[4] : nullptr;
  try {
    Env env;
    return run<REF_REAL>(d, fields, warm, steps, out);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "miso_ref_cuda: %s\n", e.what());
    return 2;
  }
}
