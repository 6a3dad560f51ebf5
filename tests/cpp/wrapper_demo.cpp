// Drives miso_b200::Integrator (include/miso_b200.hpp) through the
// reference's integrator interface -- cfl(qq, eos) then
// update(dt, eos, bc, src, qq), as mhd::ModelBase::update does
// (mhd_model_base.hpp:57-62) -- on fields read from a file, and writes the
// result back.  Field and grid types here are small stand-ins with the
// member names of the reference's mhd::Fields and Grid.
//
//   wrapper_demo <in.bin> <out.bin> <nsteps> <resident 0|1> <float 0|1>
//
// in.bin: int32 i_size, j_size, k_size, margin, periodic[3];
//         float64 x_min, x_max, y_min, y_max, z_min, z_max, gm, cfl_number;
//         float64 fields[9][i_total*j_total*k_total]
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "miso_b200.hpp"

template <class Real>
struct Arr {
  std::vector<Real> v;
  Real *data() { return v.data(); }
  const Real *data() const { return v.data(); }
};

template <class Real>
struct Fields {
  Arr<Real> ro, vx, vy, vz, bx, by, bz, ei, ph;
  Arr<Real> *all[9] = {&ro, &vx, &vy, &vz, &bx, &by, &bz, &ei, &ph};
};

struct Grid {
  int i_size, j_size, k_size, i_margin, j_margin, k_margin;
  double x_min, x_max, y_min, y_max, z_min, z_max;
};

struct IdealEOS {
  double gm;
};

template <class Real>
static int run(FILE *in, FILE *out, int nsteps, bool resident) {
  int hdr[7];
  double dd[8];
  if (fread(hdr, sizeof(int), 7, in) != 7 || fread(dd, sizeof(double), 8, in) != 8) return 2;
  Grid g;
  g.i_size = hdr[0];
  g.j_size = hdr[1];
  g.k_size = hdr[2];
  g.i_margin = hdr[0] > 1 ? hdr[3] : 0;
  g.j_margin = hdr[1] > 1 ? hdr[3] : 0;
  g.k_margin = hdr[2] > 1 ? hdr[3] : 0;
  g.x_min = dd[0];
  g.x_max = dd[1];
  g.y_min = dd[2];
  g.y_max = dd[3];
  g.z_min = dd[4];
  g.z_max = dd[5];
  const size_t cells = (size_t)(g.i_size + 2 * g.i_margin) * (g.j_size + 2 * g.j_margin) *
                       (g.k_size + 2 * g.k_margin);
  miso_b200::Physics ph;
  ph.gm = dd[6];
  ph.cfl_number = dd[7];
  miso_b200::Boundary bc;
  for (int a = 0; a < 3; ++a) bc.periodic[a] = hdr[4 + a];
  Fields<Real> qq;
  std::vector<double> buf(cells);
  for (auto *a : qq.all) {
    if (fread(buf.data(), sizeof(double), cells, in) != cells) return 3;
    a->v.assign(buf.begin(), buf.end());
  }
  try {
    miso_b200::Integrator<Real> integ(g, ph, bc, MISO_B200_FP64);
    IdealEOS eos{ph.gm};
    const miso_b200::Boundary &nobc = bc;
    miso_b200::NoSource src;
    integ.apply_boundary_condition(nobc, qq);
    if (resident) {
      integ.set_resident(true);
      integ.push(qq);
    }
    for (int s = 0; s < nsteps; ++s) {
      const Real dt = integ.cfl(qq, eos);
      integ.update(dt, eos, nobc, src, qq);
    }
    if (resident) integ.pull(qq);
  } catch (const miso_b200::Error &e) {
    std::fprintf(stderr, "miso_b200 error %d: %s\n", e.code(), e.what());
    return 4;
  }
  for (auto *a : qq.all) {
    for (size_t c = 0; c < cells; ++c) buf[c] = (double)a->v[c];
    fwrite(buf.data(), sizeof(double), cells, out);
  }
  return 0;
}

int main(int argc, char **argv) {
  if (argc < 6) return 1;
  FILE *in = std::fopen(argv[1], "rb");
  FILE *out = std::fopen(argv[2], "wb");
  if (!in || !out) return 1;
  const int nsteps = std::atoi(argv[3]);
  const bool resident = std::atoi(argv[4]) != 0;
  const int rc = std::atoi(argv[5]) ? run<float>(in, out, nsteps, resident)
                                    : run<double>(in, out, nsteps, resident);
  std::fclose(in);
  std::fclose(out);
  return rc;
}
