"""Boundary paths of the C ABI beyond the built-in faces.

* miso_b200_set_boundary_callback: the caller's own boundary functor runs
  after every pass on host copies of the FP64 state, then the library fills
  the periodic faces -- the reference's bc.apply followed by its halo
  exchange (mhd_integrator_host.hpp:250-255).  A mirror written in numpy
  through this path equals the oracle bit for bit, corners included.
* miso_b200_set_mirror_signs: signs set after create act as signs given at
  create.
* miso_b200_pointer_kind tells device from host memory.
"""
import numpy as np
import pytest

from conftest import interior
from miso_b200 import _lib
from miso_b200 import problems as P
from miso_b200.integrator import Integrator

pytestmark = pytest.mark.gpu


def _aniso():
    from miso_b200.config import make_config
    from miso_b200.grid import Grid
    g = Grid(10, 7, 13, 2, 0.0, 1.0, 0.0, 0.7, 0.0, 1.3)
    base = P.turbulence(13, seed=7)
    q = np.ascontiguousarray(base.q[:, :g.i_total, :g.j_total, :g.k_total])
    cfg = make_config(5.0 / 3.0, periodic=(True, False, True), cfl_number=0.3, ep=1.3, fh=0.8,
                      cs_fac=0.9, ca_fac=1.1, vv_fac=0.7)
    sign = np.ones((3, 2, 9))
    sign[1, 0, P.VY] = -1.0
    sign[1, 1, P.BY] = -1.0
    return P.Problem("aniso", g, cfg, q, sign)


def numpy_mirror(prob):
    """boundary_condition::symmetric on every non-periodic face, x then y
    then z, full transverse range (boundary_condition.hpp:77-136)."""
    g = prob.grid
    per = prob.config["domain"]["periodic"]
    periodic = (per["x"], per["y"], per["z"])
    sign = np.ones((3, 2, 9)) if prob.sign is None else np.asarray(prob.sign)
    sizes = (g.i_size, g.j_size, g.k_size)

    def fill(q):
        for a in range(3):
            if sizes[a] <= 1 or periodic[a]:
                continue
            m, t = g.margin, q.shape[1 + a]
            for gh in range(m):
                for side, (dst, src) in enumerate(((gh, 2 * m - gh - 1),
                                                   (t - m + gh, t - m - gh - 1))):
                    for f in range(9):
                        d = [f, slice(None), slice(None), slice(None)]
                        s = list(d)
                        d[1 + a], s[1 + a] = dst, src
                        q[tuple(d)] = sign[a, side, f] * q[tuple(s)]
    return fill


def _run(prob, nsteps, callback=None, signs_after=False):
    sign = None if signs_after else prob.sign
    integ = Integrator(prob.config, prob.grid, sign=sign, precision="fp64")
    if signs_after and prob.sign is not None:
        integ.set_mirror_signs(prob.sign)
    if callback:
        integ.set_boundary_callback(callback)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    for _ in range(nsteps):
        integ.update(integ.cfl())
    out = integ.download()
    integ.close()
    return out


CASES = [("bw128", lambda: P.brio_wu(128, scale=[1.1, 0.9, 1.0, 1.2, 0.8, 1.05]), 30),
         ("blast12", lambda: P.blast(12, seed=5), 4),
         ("aniso", _aniso, 3)]


@pytest.mark.parametrize("name,make,nsteps", CASES, ids=[c[0] for c in CASES])
def test_boundary_callback_equals_oracle(name, make, nsteps, oracle):
    prob = make()
    ref = prob.q.copy()
    oracle.run(prob, ref, nsteps)
    out = _run(prob, nsteps, callback=numpy_mirror(prob))
    a, b = interior(prob, out), interior(prob, ref)
    assert int(np.sum(a != b)) == 0


def test_mirror_signs_set_after_create(oracle):
    prob = _aniso()
    ref = prob.q.copy()
    oracle.run(prob, ref, 3)
    out = _run(prob, 3, signs_after=True)
    assert int(np.sum(interior(prob, out) != interior(prob, ref))) == 0


def test_boundary_callback_errors_and_graph_refusal():
    prob = P.brio_wu(64)
    integ = Integrator(prob.config, prob.grid, precision="fp64")
    integ.upload(prob.q)

    def failing(q):
        raise RuntimeError("boundary failed")
    integ.set_boundary_callback(failing)
    with pytest.raises(_lib.MisoError) as exc:
        integ.apply_boundary_condition()
    assert exc.value.code == _lib.ERR_CALLBACK
    integ.set_boundary_callback(numpy_mirror(prob))
    with pytest.raises(_lib.MisoError) as exc:
        integ.run(2, graph=True)
    assert exc.value.code == _lib.ERR_STATE
    integ.set_boundary_callback(None)
    integ.apply_boundary_condition()
    integ.run(2, graph=True)
    integ.sync()
    integ.close()
    split = Integrator(prob.config, prob.grid, precision="fp32_split")
    with pytest.raises(_lib.MisoError) as exc:
        split.set_boundary_callback(numpy_mirror(prob))
    assert exc.value.code == _lib.ERR_STATE
    split.close()


def test_pointer_kind():
    import ctypes
    import torch
    lib = _lib.load()
    kind = ctypes.c_int(-1)
    dev = torch.zeros(16, device="cuda")
    assert lib.miso_b200_pointer_kind(ctypes.c_void_p(dev.data_ptr()), ctypes.byref(kind)) == 0
    assert kind.value == 1
    host = np.zeros(16)
    assert lib.miso_b200_pointer_kind(ctypes.c_void_p(host.ctypes.data), ctypes.byref(kind)) == 0
    assert kind.value == 0
    pinned = torch.zeros(16).pin_memory()
    assert lib.miso_b200_pointer_kind(ctypes.c_void_p(pinned.data_ptr()),
                                      ctypes.byref(kind)) == 0
    assert kind.value == 0
