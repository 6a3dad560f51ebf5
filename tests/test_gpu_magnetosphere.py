"""The magnetosphere demo's boundary and masked CFL on the FP64 form,
through the C ABI, against the oracle (itself pinned bit for bit to the
reference build running a restatement of the demo's boundary functor):
every time step and every interior value equal, with the state blended
toward the initial condition or toward zeros."""
import numpy as np
import pytest

from conftest import interior
from miso_b200 import _lib
from miso_b200 import problems as P
from miso_b200.integrator import Integrator

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,blend,steps", [(16, True, 6), (16, False, 4), (20, True, 4)],
                         ids=["n16_blend_ic", "n16_blend_zero", "n20_blend_ic"])
def test_fp64_bit_exact_with_oracle(n, blend, steps, oracle):
    prob = P.magnetosphere(n, extent=12.0, blend_to_initial=blend)
    ref = prob.q.copy()
    dts_o = oracle.run(prob, ref, steps)
    integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision="fp64",
                       blend=prob.blend)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    dts = []
    for _ in range(steps):
        dt = integ.cfl()
        integ.update(dt)
        dts.append(dt)
    out = integ.download()
    integ.close()
    assert np.array_equal(np.array(dts), dts_o), (dts[:3], dts_o[:3])
    a, b = interior(prob, out), interior(prob, ref)
    assert np.array_equal(a, b), float(np.max(np.abs(a - b)))


def test_masked_cfl_and_boundary_act(oracle):
    """The boundary changes the state (the blend and the inflow) and the
    mask changes the step, on the device as in the oracle."""
    prob = P.magnetosphere(16, extent=12.0)
    q = prob.q.copy()
    oracle.fill_ghosts(prob, q)
    integ = Integrator(prob.config, prob.grid, precision="fp64", blend=prob.blend)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    assert integ.cfl() == oracle.cfl(prob, q)
    assert np.array_equal(interior(prob, integ.download()), interior(prob, q))
    integ.close()
    plain = P.magnetosphere(16, extent=12.0)
    plain.config["boundary"]["cfl_mask"] = False
    integ = Integrator(plain.config, plain.grid, precision="fp64", blend=plain.blend)
    integ.upload(plain.q)
    integ.apply_boundary_condition()
    dt_plain = integ.cfl()
    integ.close()
    assert dt_plain == oracle.cfl(plain, q) and dt_plain != oracle.cfl(prob, q)


def test_refusals():
    prob = P.magnetosphere(16, extent=12.0)
    with pytest.raises(_lib.MisoError) as e:
        Integrator(prob.config, prob.grid, precision="fp32_split")
    assert e.value.code == _lib.ERR_STATE
    per = P.turbulence(16, seed=1)
    per.config["boundary"] = dict(prob.config["boundary"])
    for key in ("solar_wind", "magnetosphere", "floor"):
        per.config[key] = prob.config[key]
    with pytest.raises(_lib.MisoError) as e:
        Integrator(per.config, per.grid, precision="fp64")
    assert e.value.code == _lib.ERR_ARG
