"""The C++ drop-in (include/miso_b200.hpp): miso_b200::Integrator<Real>
driven through the reference's integrator interface, cfl(qq, eos) then
update(dt, eos, bc, src, qq) (mhd_model_base.hpp:57-62).

CPU: the header compiles against the reference's own mhd::Fields and Grid
types (float and double), its source and boundary calls included, and the
demo program builds and links.
GPU: the demo's FP64 result equals the oracle bit for bit, in the default
(copy in / copy out per call) and the resident mode.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, interior, rel_l1
from oracle.oracle import REFERENCE_INCLUDE

REF_INCLUDE = REFERENCE_INCLUDE
DEMO = os.path.join(ROOT, "tests", "cpp", "wrapper_demo.cpp")
LIBDIR = os.path.join(ROOT, "miso_b200", "lib")

CHECK_TU = r"""
#include <miso/mhd_fields.hpp>
#include <miso/grid.hpp>
#include "miso_b200.hpp"
struct E { double gm = 5.0 / 3.0; };
template <class Real> void drive() {
  miso::Grid<Real, miso::backend::Host> g(16, 16, 1, 2, 0, 1, 0, 1, 0, 1);
  miso::mhd::Fields<Real, miso::backend::Host> qq(g);
  const auto B = miso_b200::Boundary::all_mirror();
  miso_b200::Integrator<Real> integ(g, miso_b200::Physics(), B);
  Real dt = integ.cfl(qq, E());
  integ.update(dt, E(), B, miso_b200::NoSource(), qq);
  integ.update(dt, E(), B, miso_b200::PointGravity<Real>{Real(1e-3)}, qq);
  integ.apply_boundary_condition(B, qq);
  integ.set_resident(true);
  integ.push(qq);
  integ.pull(qq);
  integ.set_point_gravity(1.35e-6);
  typename miso_b200::Integrator<Real>::Magnetosphere m{5e-4, 3.56e-8, 0.05, -1.5e-4,
                                                        3.5, 100.0, 1e-8, 1e-10, true};
  integ.set_magnetosphere_boundary(m);
  integ.set_blend_state(qq);
}
template void drive<double>();
template void drive<float>();
"""


def _gxx():
    g = shutil.which("g++")
    if not g:
        pytest.skip("g++ not available")
    return g


@pytest.mark.skipif(not os.path.isdir(REF_INCLUDE), reason="reference headers not present")
def test_header_compiles_against_reference_types(tmp_path):
    src = tmp_path / "check.cpp"
    src.write_text(CHECK_TU)
    r = subprocess.run([_gxx(), "-std=c++17", "-fsyntax-only", "-Wall",
                        "-I" + os.path.join(ROOT, "oracle", "ref_shim"), "-I" + REF_INCLUDE,
                        "-I" + os.path.join(ROOT, "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.skipif(not os.path.isdir(REF_INCLUDE), reason="reference headers not present")
@pytest.mark.parametrize("call,message", [
    ("integ.update(Real(1), E(), Functor(), miso_b200::NoSource(), qq);", "Boundary descriptor"),
    ("integ.update(Real(1), E(), miso_b200::Boundary(), Src(), qq);", "NoSource or PointGravity"),
], ids=["functor", "source"])
def test_header_refuses_unsupported_arguments(tmp_path, call, message):
    """Boundary functors and source terms the standalone header cannot run
    are compile-time errors (they were silently ignored before)."""
    src = tmp_path / "bad.cpp"
    src.write_text(r"""
#include <miso/mhd_fields.hpp>
#include <miso/grid.hpp>
#include "miso_b200.hpp"
struct E { double gm = 5.0 / 3.0; };
struct Functor {};
struct Src {};
using Real = double;
void drive() {
  miso::Grid<Real, miso::backend::Host> g(16, 16, 1, 2, 0, 1, 0, 1, 0, 1);
  miso::mhd::Fields<Real, miso::backend::Host> qq(g);
  miso_b200::Integrator<Real> integ(g, miso_b200::Physics(), miso_b200::Boundary());
  """ + call + "\n}\n")
    r = subprocess.run([_gxx(), "-std=c++17", "-fsyntax-only",
                        "-I" + os.path.join(ROOT, "oracle", "ref_shim"), "-I" + REF_INCLUDE,
                        "-I" + os.path.join(ROOT, "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode != 0
    assert message in r.stderr


def _build_demo(out_dir):
    lib = os.path.join(LIBDIR, "libmiso_b200.so")
    if not os.path.exists(lib):
        pytest.skip("libmiso_b200.so not built")
    exe = os.path.join(str(out_dir), "wrapper_demo")
    r = subprocess.run([_gxx(), "-std=c++17", "-O2", "-Wall", "-Wextra",
                        "-I" + os.path.join(ROOT, "include"), DEMO, "-L" + LIBDIR, "-lmiso_b200",
                        "-Wl,-rpath," + LIBDIR, "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_demo_builds(tmp_path):
    assert os.path.exists(_build_demo(tmp_path))


def _write_input(path, prob):
    g = prob.grid
    cfg = prob.config
    per = [int(bool(x)) for x in cfg["domain"]["periodic"].values()] \
        if isinstance(cfg["domain"]["periodic"], dict) else [int(x) for x in cfg["domain"]["periodic"]]
    with open(path, "wb") as f:
        np.array([g.i_size, g.j_size, g.k_size, g.margin] + per, dtype=np.int32).tofile(f)
        np.array([g.x_min, g.x_max, g.y_min, g.y_max, g.z_min, g.z_max,
                  cfg["eos"]["gm"], cfg["mhd"]["cfl_number"]], dtype=np.float64).tofile(f)
        np.ascontiguousarray(prob.q, dtype=np.float64).tofile(f)


@pytest.mark.gpu
@pytest.mark.parametrize("resident", [0, 1])
def test_demo_fp64_matches_oracle(tmp_path, oracle, resident):
    from miso_b200 import problems as P
    exe = _build_demo(tmp_path)
    prob = P.orszag_tang(32)
    nsteps = 8
    _write_input(tmp_path / "in.bin", prob)
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), str(nsteps),
                        str(resident), "0"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = np.fromfile(tmp_path / "out.bin", dtype=np.float64).reshape(prob.q.shape)
    ref = prob.q.copy()
    oracle.run(prob, ref, nsteps)
    a, b = interior(prob, out), interior(prob, ref)
    assert int(np.sum(a != b)) == 0


@pytest.mark.gpu
def test_demo_float_fields(tmp_path, oracle):
    """Real = float fields (the demos' precision) go through host staging;
    the result stays within FP32 rounding of the FP64 oracle."""
    from miso_b200 import problems as P
    exe = _build_demo(tmp_path)
    prob = P.orszag_tang(32)
    nsteps = 8
    _write_input(tmp_path / "in.bin", prob)
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), str(nsteps),
                        "0", "1"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = np.fromfile(tmp_path / "out.bin", dtype=np.float64).reshape(prob.q.shape)
    ref = prob.q.copy()
    oracle.run(prob, ref, nsteps)
    assert rel_l1(interior(prob, out)[0], interior(prob, ref)[0]) < 1e-5
