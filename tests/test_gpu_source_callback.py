"""A source functor of the caller's own (miso_b200_set_source_callback): the
reference's Source concept (src.vx, src.vy, src.vz, src.ei evaluated on
each stage's argument state, mhd_model_base.hpp:131-155), added where
update_sc4 adds them (mhd_integrator_host.hpp:134, 151, 168, 241).  FP64
form: with the reference's host dt sequence every interior value and every
dt must equal the oracle's, whose constant source is pinned to the
reference build and whose callback source to its built-in point gravity
(tests/test_oracle_vs_reference.py).  Split form: within the stated
tolerances of the FP64 form stepped with the same dt sequence."""
import copy
import ctypes

import numpy as np
import pytest

from conftest import interior, rel_l1
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


def _split_same_dts(prob, cfg, dts, fn=None, on_host=True):
    integ = Integrator(cfg, prob.grid, sign=prob.sign, precision="fp32_split")
    if fn is not None:
        integ.set_source_callback(fn, on_host=on_host)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    for dt in dts:
        integ.update(dt)
    out = integ.download()
    integ.close()
    return out


def _device_gravity(grid, gconst):
    """A device callback: the gravity from the device arrays with torch, on
    the library's stream."""
    import torch
    X, Y, Z, r3, _ = _gravity(grid, gconst)
    shape = tuple(grid.shape)
    n = int(np.prod(shape))
    dev = {k: torch.as_tensor(v, device="cuda") for k, v in (("x", X), ("y", Y), ("z", Z),
                                                             ("r3", r3))}

    def view(ptr):
        class _V:
            __cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False),
                                        "version": 3}
        return torch.as_tensor(_V(), device="cuda").view(shape)

    def fn(q, s, stream):
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            a = -view(q[P.RO]) * gconst / dev["r3"]
            view(s[0]).copy_(a * dev["x"])
            view(s[1]).copy_(a * dev["y"])
            view(s[2]).copy_(a * dev["z"])
            view(s[3]).zero_()
    return fn


@pytest.mark.parametrize("make,nsteps,on_host", [
    (lambda: P.with_point_gravity(P.blast(24, seed=5), 0.3), 10, True),
    (lambda: P.with_point_gravity(P.orszag_tang(64), 2.0), 20, False)],
    ids=["blast24_host", "ot64_device"])
def test_split_form_callback_gravity(make, nsteps, on_host):
    """The split form with the gravity as a caller's callback -- the stage's
    argument state handed over as FP64 primitives (hi + lo for U^n), the
    terms read by the pipelined RK stage (3-D) or the per-cell one (2-D) --
    follows the FP64 form with the built-in gravity stepped with the same dt
    sequence: relative L1 of ro <= 1e-6 and of the momentum <= 1e-4, while
    dropping the source moves the momentum by more than 100x that."""
    prob = make()
    g = prob.config["source"]["g"]
    ref = Integrator(prob.config, prob.grid, sign=prob.sign, precision="fp64")
    ref.upload(prob.q)
    ref.apply_boundary_condition()
    dts = _host_dt_run(ref, nsteps)
    b = interior(prob, ref.download())
    ref.close()
    cfg = copy.deepcopy({k: v for k, v in prob.config.items() if k != "source"})
    if on_host:
        X, Y, Z, r3, gc = _gravity(prob.grid, g)

        def fn(q, s):
            s[0][...] = -q[P.RO] * gc * X / r3
            s[1][...] = -q[P.RO] * gc * Y / r3
            s[2][...] = -q[P.RO] * gc * Z / r3
            s[3][...] = 0.0
    else:
        fn = _device_gravity(prob.grid, g)
    a = interior(prob, _split_same_dts(prob, cfg, dts, fn, on_host))
    assert rel_l1(a[P.RO], b[P.RO]) <= 1e-6
    ma, mb = a[P.RO] * a[P.VX:P.VZ + 1], b[P.RO] * b[P.VX:P.VZ + 1]
    assert rel_l1(ma, mb) <= 1e-4
    c = interior(prob, _split_same_dts(prob, cfg, dts))
    assert rel_l1(c[P.RO] * c[P.VX:P.VZ + 1], mb) > 100 * rel_l1(ma, mb)


def test_split_form_callback_constant_terms():
    """All four terms, src.ei (added outside the dt factor) included: the
    split form follows the FP64 form with the same callback and dt sequence
    to relative L1 <= 1e-6 in ro and in the pressure."""
    prob = P.blast(16, seed=2)

    def const(q, s):
        for t in range(4):
            s[t][...] = VALS[t]
    ref = Integrator(prob.config, prob.grid, sign=prob.sign, precision="fp64")
    ref.set_source_callback(const)
    ref.upload(prob.q)
    ref.apply_boundary_condition()
    dts = _host_dt_run(ref, 6)
    b = interior(prob, ref.download())
    ref.close()
    a = interior(prob, _split_same_dts(prob, prob.config, dts, const))
    gm = prob.config["eos"]["gm"]
    assert rel_l1(a[P.RO], b[P.RO]) <= 1e-6
    pa, pb = (gm - 1) * a[P.RO] * a[P.EI], (gm - 1) * b[P.RO] * b[P.EI]
    assert rel_l1(pa, pb) <= 1e-6
    # the heating acts: without the source the pressure differs by far more
    c = interior(prob, _split_same_dts(prob, prob.config, dts))
    assert rel_l1((gm - 1) * c[P.RO] * c[P.EI], pb) > 100 * rel_l1(pa, pb)


def test_source_callback_refusals_and_errors():
    prob = P.blast(12, seed=5)

    def zero(q, s):
        for t in range(4):
            s[t][...] = 0.0
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
