"""A source functor of the caller's own on the FP64 form
(miso_b200_set_source_callback): the reference's Source concept
(src.vx, src.vy, src.vz, src.ei evaluated on each stage's argument state,
mhd_model_base.hpp:131-155), added where update_sc4 adds them
(mhd_integrator_host.hpp:134, 151, 168, 241).  With the reference's host dt
sequence every interior value and every dt must equal the oracle's, whose
constant source is pinned to the reference build and whose callback source
to its built-in point gravity (tests/test_oracle_vs_reference.py)."""
import copy
import ctypes

import numpy as np
import pytest

from conftest import interior
from miso_b200 import _lib
from miso_b200 import problems as P
from miso_b200.integrator import Integrator

pytestmark = pytest.mark.gpu

VALS = [1e-3, -2e-3, 5e-4, 2e-4]


def _gravity(grid, gconst):
    X, Y, Z = np.meshgrid(grid.x, grid.y, grid.z, indexing="ij")
    rr = np.sqrt(X * X + Y * Y + Z * Z)
    r3 = rr * rr * rr  # util::pow3
    return X, Y, Z, r3, gconst


def _host_dt_run(integ, nsteps):
    dts = []
    for _ in range(nsteps):
        dt = integ.cfl()
        integ.update(dt)
        dts.append(dt)
    return np.array(dts)


@pytest.mark.parametrize("make,nsteps", [
    (lambda: P.with_point_gravity(P.blast(12, seed=5), 0.3), 6),
    (lambda: P.with_point_gravity(P.orszag_tang(32), 2.0), 10)], ids=["blast12", "ot32"])
def test_host_callback_gravity_bit_exact(make, nsteps, oracle):
    prob = make()
    X, Y, Z, r3, gc = _gravity(prob.grid, prob.config["source"]["g"])

    def grav(q, s):
        s[0][...] = -q[P.RO] * gc * X / r3
        s[1][...] = -q[P.RO] * gc * Y / r3
        s[2][...] = -q[P.RO] * gc * Z / r3
        s[3][...] = 0.0
    ref = prob.q.copy()
    dts_o = oracle.run(prob, ref, nsteps)  # the built-in gravity
    cfg = copy.deepcopy({k: v for k, v in prob.config.items() if k != "source"})
    cfg["source"] = {"kind": "callback", "fn": grav}
    integ = Integrator(cfg, prob.grid, sign=prob.sign, precision="fp64")
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    dts = _host_dt_run(integ, nsteps)
    out = integ.download()
    integ.close()
    assert np.array_equal(dts, dts_o)
    assert np.array_equal(interior(prob, out), interior(prob, ref))


def test_host_callback_constant_terms_bit_exact(oracle):
    """All four terms, src.ei included, against the oracle's constants."""
    base = P.blast(12, seed=5)
    prob = copy.deepcopy(base)
    prob.config["source"] = {"kind": "constant", "values": VALS}
    ref = prob.q.copy()
    dts_o = oracle.run(prob, ref, 5)

    def const(q, s):
        for t in range(4):
            s[t][...] = VALS[t]
    cfg = copy.deepcopy(base.config)
    integ = Integrator(cfg, base.grid, sign=base.sign, precision="fp64")
    integ.set_source_callback(const)
    integ.upload(base.q)
    integ.apply_boundary_condition()
    dts = _host_dt_run(integ, 5)
    out = integ.download()
    integ.close()
    assert np.array_equal(dts, dts_o)
    assert np.array_equal(interior(prob, out), interior(prob, ref))


def test_device_callback_gravity_bit_exact(oracle):
    """on_host=False: the callback gets device addresses and the handle's
    stream (here it reads the density back and writes the terms with the
    CUDA runtime's own copies on that stream)."""
    from cuda.bindings import runtime as rt
    prob = P.with_point_gravity(P.blast(12, seed=7), 0.3)
    X, Y, Z, r3, gc = _gravity(prob.grid, 0.3)
    shape = tuple(prob.grid.shape)
    nbytes = int(np.prod(shape)) * 8

    def dev(q, s, stream):
        ro = np.empty(shape)
        rt.cudaMemcpyAsync(ro.ctypes.data, q[P.RO], nbytes,
                           rt.cudaMemcpyKind.cudaMemcpyDeviceToHost, stream)
        rt.cudaStreamSynchronize(stream)
        terms = [-ro * gc * X / r3, -ro * gc * Y / r3, -ro * gc * Z / r3, np.zeros(shape)]
        for t in range(4):
            rt.cudaMemcpyAsync(s[t], terms[t].ctypes.data, nbytes,
                               rt.cudaMemcpyKind.cudaMemcpyHostToDevice, stream)
        rt.cudaStreamSynchronize(stream)  # the host arrays end with this call
    ref = prob.q.copy()
    dts_o = oracle.run(prob, ref, 4)
    cfg = copy.deepcopy({k: v for k, v in prob.config.items() if k != "source"})
    integ = Integrator(cfg, prob.grid, sign=prob.sign, precision="fp64")
    integ.set_source_callback(dev, on_host=False)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    dts = _host_dt_run(integ, 4)
    out = integ.download()
    integ.close()
    assert np.array_equal(dts, dts_o)
    assert np.array_equal(interior(prob, out), interior(prob, ref))


def test_source_callback_refusals_and_errors():
    prob = P.blast(12, seed=5)

    def zero(q, s):
        for t in range(4):
            s[t][...] = 0.0
    with Integrator(prob.config, prob.grid, precision="fp32_split") as sp:
        with pytest.raises(_lib.MisoError) as e:
            sp.set_source_callback(zero)
        assert e.value.code == _lib.ERR_STATE
    integ = Integrator(prob.config, prob.grid, precision="fp64")
    integ.set_source_callback(zero)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    with pytest.raises(_lib.MisoError) as e:
        integ.run(2, graph=True)  # a host callback between stages: no graph
    assert e.value.code == _lib.ERR_STATE
    # the built-in source is refused while a callback is set
    par = (ctypes.c_double * 1)(0.3)
    assert integ._lib.miso_b200_set_source(integ._h, 1, par, 1) == _lib.ERR_STATE

    def broken(q, s):
        raise RuntimeError("no terms today")
    integ.set_source_callback(broken)
    with pytest.raises(_lib.MisoError) as e:
        integ.update(integ.cfl())
    assert e.value.code == _lib.ERR_CALLBACK
    # a zero source gives the no-source step bit for bit
    integ.set_source_callback(zero)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    a = _host_dt_run(integ, 3)
    qa = integ.download()
    integ.set_source_callback(None)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    b = _host_dt_run(integ, 3)
    qb = integ.download()
    integ.close()
    assert np.array_equal(a, b) and np.array_equal(qa, qb)
