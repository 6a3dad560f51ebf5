"""The reference's own mhd::ModelBase on the B200 backend
(include/miso_b200_backend.hpp): tests/cpp/modelbase_demo.cpp defines MISO
models with Backend = miso::backend::B200 and runs them through the
unmodified ModelBase::run / ModelBase::update
(miso/include/miso/mhd_model_base.hpp:57-116); the snapshots the
reference's Checkpoint writes are compared with the oracle.

CPU: the programs build against the reference's headers (with the host
compiler, and with nvcc for device source functors), and an equation of
state the backend does not implement is a compile-time error.
GPU: Orszag-Tang (periodic, EmptyBoundaryCondition), Brio-Wu and a 3-D
blast (the demos' mirror functor, reduced to the library's face fill; the
same mirror as plain loops, run as a host functor after every pass) equal
the oracle bit for bit in the FP64 form; so do models with source functors
of their own (constants on host copies; the point gravity on host copies
and, built by nvcc, on the device); Real = float runs the split form;
functors and configurations the backend cannot run fail with a message.
"""
import glob
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, interior, rel_l1
from miso_b200 import problems as P
from oracle.oracle import REFERENCE_INCLUDE, REFERENCE_ROOT

CPP = os.path.join(ROOT, "tests", "cpp")
BIN = os.path.join(CPP, "_bin")
HAVE_REF = os.path.isdir(REFERENCE_INCLUDE)


def _binary(name):
    exe = os.path.join(BIN, name)
    if HAVE_REF and shutil.which("make"):
        r = subprocess.run(["make", "-s", "-C", CPP, "MISO_REFERENCE=" + REFERENCE_ROOT],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
    if not os.path.exists(exe):
        pytest.skip("the ModelBase programs are built where the MISO headers are present")
    return exe


def test_modelbase_programs_build():
    assert os.path.exists(_binary("modelbase_fp64"))
    assert os.path.exists(_binary("modelbase_f32"))
    assert os.path.exists(_binary("modelbase_fp64_cuda"))  # nvcc: device source functors


BAD_TU = r"""
#include <miso/mhd_model_base.hpp>
#include "miso_b200_backend.hpp"
using namespace miso;
using Real = double;
struct IC { void apply(mhd::FieldsView<Real>, GridView<const Real>) const {} };
struct MySource {
  Real vx(mhd::FieldsView<const Real>, int, int, int) const { return 0; }
  Real vy(mhd::FieldsView<const Real>, int, int, int) const { return 0; }
  Real vz(mhd::FieldsView<const Real>, int, int, int) const { return 0; }
  Real ei(mhd::FieldsView<const Real>, int, int, int) const { return 0; }
};
struct MyEOS { Real gm = 1.4; };
struct Model : mhd::ModelBase<Model, Real, backend::B200> {
  EOS_TYPE eos;
  IC ic;
  mhd::EmptyBoundaryCondition<Real> bc;
  SRC_TYPE src;
  Model(Config &c) : ModelBase(c), eos(EOS_INIT), ic(), bc(), src() {}
};
void go(Config &c) { Model m(c); m.run(); }
"""


def _syntax(tmp_path, eos, eos_init, src):
    tu = tmp_path / "tu.cpp"
    tu.write_text(BAD_TU)
    return subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-w",
                           f"-DEOS_TYPE={eos}", f"-DEOS_INIT={eos_init}", f"-DSRC_TYPE={src}",
                           "-I" + os.path.join(ROOT, "oracle", "ref_shim"),
                           "-I" + REFERENCE_INCLUDE, "-I" + os.path.join(ROOT, "include"),
                           str(tu)], capture_output=True, text=True)


@pytest.mark.skipif(not HAVE_REF, reason="needs the MISO headers")
def test_unsupported_eos_fails_to_compile(tmp_path):
    r = _syntax(tmp_path, "MyEOS", "", "mhd::EmptySourceTerm<Real>")
    assert r.returncode != 0
    assert "eos::IdealEOS<Real> only" in r.stderr


@pytest.mark.skipif(not HAVE_REF, reason="needs the MISO headers")
def test_user_source_functor_compiles(tmp_path):
    """A source functor of the model's own (the Source concept) compiles for
    the backend: it runs on host copies of each stage's argument state."""
    r = _syntax(tmp_path, "eos::IdealEOS<Real>", "c", "MySource")
    assert r.returncode == 0, r.stderr


# ---------------------------------------------------------------------------
def _yaml(prob, tend, dt_output, extra=""):
    g, cfg = prob.grid, prob.config
    per = cfg["domain"]["periodic"]
    av = cfg["mhd"]["artificial_viscosity"]

    def b(x):
        return "true" if x else "false"
    return f"""io:
  enabled: true
  save_dir: data/
  continue: false
mpi:
  x_procs: 1
  y_procs: 1
  z_procs: 1
domain:
  periodic:
    x: {b(per['x'])}
    y: {b(per['y'])}
    z: {b(per['z'])}
grid:
  margin: {g.margin}
  i_size: {g.i_size}
  j_size: {g.j_size}
  k_size: {g.k_size}
  x_min: {g.x_min!r}
  x_max: {g.x_max!r}
  y_min: {g.y_min!r}
  y_max: {g.y_max!r}
  z_min: {g.z_min!r}
  z_max: {g.z_max!r}
time:
  tend: {tend!r}
  dt_output: {dt_output!r}
eos:
  gm: {cfg['eos']['gm']!r}
mhd:
  cfl_number: {cfg['mhd']['cfl_number']!r}
  artificial_viscosity:
    ep: {av['ep']!r}
    fh: {av['fh']!r}
    cs_fac: {av['cs_fac']!r}
    ca_fac: {av['ca_fac']!r}
    vv_fac: {av['vv_fac']!r}
{extra}"""


def _run(exe, tmp_path, prob, bc, mode, tend=1.0, dt_output=1.0, real=np.float64, extra="",
         source=None):
    (tmp_path / "config.yaml").write_text(_yaml(prob, tend, dt_output, extra))
    np.ascontiguousarray(prob.q, dtype=real).tofile(tmp_path / "initial.bin")
    args = [exe, str(tmp_path / "config.yaml"), str(tmp_path / "initial.bin"), bc, mode]
    if source:
        args.append(source)
    r = subprocess.run(args, capture_output=True, text=True, timeout=600, cwd=str(tmp_path))
    return r


def _snapshot(tmp_path, prob, n_output, real=np.float64):
    files = glob.glob(str(tmp_path / "data" / "mhd" / f"mhd.{n_output:08d}.*.bin"))
    assert len(files) == 1, files
    raw = open(files[0], "rb").read()
    assert np.frombuffer(raw[:4], dtype=np.uint32)[0] == np.dtype(real).itemsize
    return np.frombuffer(raw[4:], dtype=real).reshape(prob.q.shape).astype(np.float64)


def _path_of(stdout):
    for line in stdout.splitlines():
        if line.startswith("boundary_path"):
            return int(line.split()[1])
    raise AssertionError(stdout)


CASES = [
    ("ot32_empty", lambda: P.orszag_tang(32), "empty", 0, 12),
    ("bw128_mirror", lambda: P.brio_wu(128, scale=[1.1, 0.9, 1.0, 1.2, 0.8, 1.05]), "mirror", 0, 40),
    ("bw128_loop", lambda: P.brio_wu(128, scale=[1.1, 0.9, 1.0, 1.2, 0.8, 1.05]), "loop", 1, 40),
    ("blast12_mirror", lambda: P.blast(12, seed=5), "mirror", 0, 5),
    ("blast12_loop", lambda: P.blast(12, seed=5), "loop", 1, 3),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,make,bc,path,nsteps", CASES, ids=[c[0] for c in CASES])
def test_modelbase_run_fp64_bit_exact(tmp_path, oracle, name, make, bc, path, nsteps):
    """ModelBase::run to time.tend = the time after `nsteps` oracle steps:
    the final snapshot equals the oracle bit for bit on the interior."""
    exe = _binary("modelbase_fp64")
    prob = make()
    ref = prob.q.copy()
    dts = oracle.run(prob, ref, nsteps)
    t = 0.0
    for dt in dts:  # Time::update: time += dt, in Real
        t += float(dt)
    r = _run(exe, tmp_path, prob, bc, "run", tend=t, dt_output=t)
    assert r.returncode == 0, r.stdout + r.stderr
    assert _path_of(r.stdout) == path
    assert f"steps {nsteps} " in r.stdout, r.stdout
    out = _snapshot(tmp_path, prob, 1)
    a, b = interior(prob, out), interior(prob, ref)
    assert int(np.sum(a != b)) == 0, float(np.max(np.abs(a - b)))


@pytest.mark.gpu
def test_modelbase_update_loop_fp64_bit_exact(tmp_path, oracle):
    """ModelBase::update called N times (cfl -> update -> time += dt), then
    ModelBase::save_state."""
    exe = _binary("modelbase_fp64")
    prob = P.turbulence(12, seed=3)
    ref = prob.q.copy()
    oracle.run(prob, ref, 4)
    r = _run(exe, tmp_path, prob, "empty", "update:4")
    assert r.returncode == 0, r.stdout + r.stderr
    out = _snapshot(tmp_path, prob, 0)
    assert int(np.sum(interior(prob, out) != interior(prob, ref))) == 0


@pytest.mark.gpu
def test_modelbase_float_runs_split_form(tmp_path, oracle):
    """Real = float (the demos' precision) runs the split form: within FP32
    rounding of the FP64 oracle."""
    exe = _binary("modelbase_f32")
    prob = P.orszag_tang(32)
    ref = prob.q.copy()
    oracle.run(prob, ref, 8)
    r = _run(exe, tmp_path, prob, "empty", "update:8", real=np.float32)
    assert r.returncode == 0, r.stdout + r.stderr
    out = _snapshot(tmp_path, prob, 0, real=np.float32)
    assert rel_l1(interior(prob, out)[P.RO], interior(prob, ref)[P.RO]) < 1e-5


@pytest.mark.gpu
def test_modelbase_double_split_form_by_config(tmp_path, oracle):
    exe = _binary("modelbase_fp64")
    prob = P.blast(16, seed=1)
    ref = prob.q.copy()
    oracle.run(prob, ref, 6)
    r = _run(exe, tmp_path, prob, "mirror", "update:6", extra="b200:\n  precision: fp32_split\n")
    assert r.returncode == 0, r.stdout + r.stderr
    assert _path_of(r.stdout) == 0
    out = _snapshot(tmp_path, prob, 0)
    assert rel_l1(interior(prob, out)[P.RO], interior(prob, ref)[P.RO]) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("exe_name", ["modelbase_fp64", "modelbase_fp64_cuda"],
                         ids=["host_functor", "device_functor"])
def test_modelbase_gravity_functor_split_form_by_config(tmp_path, oracle, exe_name):
    """Real = double with b200.precision fp32_split: the model's own gravity
    functor (on host copies, or on the device from nvcc's build) is handed
    each stage's argument state as FP64 primitives and the split form adds
    its terms, within 1e-6 in ro and 1e-4 in the momentum (relative L1) of
    the oracle's gravity."""
    exe = _binary(exe_name)
    base = P.blast(12, seed=5)
    prob = P.with_point_gravity(base, 0.3)
    ref = prob.q.copy()
    oracle.run(prob, ref, 4)
    r = _run(exe, tmp_path, base, "mirror", "update:4", source="grav:0.3",
             extra="b200:\n  precision: fp32_split\n")
    assert r.returncode == 0, r.stdout + r.stderr
    a, b = interior(base, _snapshot(tmp_path, base, 0)), interior(base, ref)
    assert rel_l1(a[P.RO], b[P.RO]) < 1e-6
    assert rel_l1(a[P.RO] * a[P.VX:P.VZ + 1], b[P.RO] * b[P.VX:P.VZ + 1]) < 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("exe_name,make,bc,message", [
    ("modelbase_f32", lambda: P.brio_wu(64), "loop", "not a set of mirror faces"),
    ("modelbase_fp64", lambda: P.brio_wu(64), "empty", "EmptyBoundaryCondition leaves"),
], ids=["split_form_host_functor", "empty_bc_on_mirror_axis"])
def test_modelbase_refusals_fail_loudly(tmp_path, exe_name, make, bc, message):
    exe = _binary(exe_name)
    prob = make()
    real = np.float32 if exe_name.endswith("f32") else np.float64
    r = _run(exe, tmp_path, prob, bc, "update:1", real=real)
    assert r.returncode == 3, r.stdout + r.stderr
    assert message in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["update:4", "run"])
def test_modelbase_user_source_fp64_bit_exact(tmp_path, oracle, mode):
    """The model's own source functor (four constants, src.ei included)
    through ModelBase::update / ::run: every interior value equals the
    oracle's constant source, which equals the reference's
    (tests/test_oracle_vs_reference.py), bit for bit."""
    import copy
    exe = _binary("modelbase_fp64")
    vals = [1e-3, -2e-3, 5e-4, 2e-4]
    base = P.blast(12, seed=5)
    prob = copy.deepcopy(base)
    prob.config["source"] = {"kind": "constant", "values": vals}
    ref = prob.q.copy()
    dts = oracle.run(prob, ref, 4)
    t = 0.0
    for dt in dts:
        t += float(dt)
    src = "const:" + ",".join(repr(v) for v in vals)
    if mode == "run":
        r = _run(exe, tmp_path, base, "mirror", "run", tend=t, dt_output=t, source=src)
        n_out = 1
    else:
        r = _run(exe, tmp_path, base, "mirror", mode, source=src)
        n_out = 0
    assert r.returncode == 0, r.stdout + r.stderr
    out = _snapshot(tmp_path, base, n_out)
    a, b = interior(base, out), interior(base, ref)
    assert int(np.sum(a != b)) == 0, float(np.max(np.abs(a - b)))


@pytest.mark.gpu
@pytest.mark.parametrize("exe_name", ["modelbase_fp64", "modelbase_fp64_cuda"],
                         ids=["host_functor", "device_functor"])
def test_modelbase_gravity_source_bit_exact(tmp_path, oracle, exe_name):
    """The point gravity as the model's own Source functor, holding a view
    of the B200 grid for the cell centres: evaluated on host copies (the
    host compiler's build) or on the device by the backend's kernel (nvcc's
    build, the functor declared device-callable), every interior value after
    ModelBase::update x 4 equals the oracle's built-in gravity -- which
    equals the reference's own magnetosphere source -- bit for bit."""
    exe = _binary(exe_name)
    base = P.blast(12, seed=5)
    prob = P.with_point_gravity(base, 0.3)
    ref = prob.q.copy()
    oracle.run(prob, ref, 4)
    r = _run(exe, tmp_path, base, "mirror", "update:4", source="grav:0.3")
    assert r.returncode == 0, r.stdout + r.stderr
    out = _snapshot(tmp_path, base, 0)
    a, b = interior(base, out), interior(base, ref)
    assert int(np.sum(a != b)) == 0, float(np.max(np.abs(a - b)))


@pytest.mark.gpu
def test_modelbase_user_source_refused_with_float(tmp_path):
    exe = _binary("modelbase_f32")
    prob = P.blast(12, seed=5)
    r = _run(exe, tmp_path, prob, "mirror", "update:1", real=np.float32,
             source="const:0,0,0,0")
    assert r.returncode == 3, r.stdout + r.stderr
    assert "Real = double only" in r.stdout
