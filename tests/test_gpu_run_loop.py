"""The time loop of ModelBase::run kept on the device (miso_b200_run_until):
steps while the device-held time is below t_end, checked after every step
as the reference's loop checks it (mhd_model_base.hpp:108-111); with a
graph the whole loop is one launch of a conditional WHILE node (two steps
per body, the second under an IF node, where a step swaps the split form's
hi / lo sets)."""
import numpy as np
import pytest

from conftest import interior, rel_l1
from miso_b200 import problems as P
from miso_b200.integrator import Integrator

pytestmark = pytest.mark.gpu


def _fresh(prob, precision, yvar=None):
    integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision=precision)
    if yvar is not None:
        integ.set_variant(2, yvar)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    return integ


@pytest.mark.parametrize("make,precision,nsteps,yvar", [
    (lambda: P.orszag_tang(64), "fp64", 7, None),          # one step per body
    # the separate y and z sweeps: three swaps a step, two steps per body
    (lambda: P.turbulence(32, seed=2), "fp32_split", 5, 0),   # odd count
    (lambda: P.turbulence(32, seed=2), "fp32_split", 6, 0),
    # the fused y and z sweeps (the default): two swaps, one step per body
    (lambda: P.turbulence(32, seed=2), "fp32_split", 5, None),
    (lambda: P.orszag_tang(64), "fp32_split", 5, None),
], ids=["ot64_fp64_7", "turb32_split_sep_5", "turb32_split_sep_6", "turb32_split_5",
        "ot64_split_5"])
def test_graph_loop_equals_host_launched_steps(make, precision, nsteps, yvar):
    """t_end = the time after `nsteps` host-launched steps: the graph loop
    stops after the same step, with the same time and the same bits."""
    prob = make()
    a = _fresh(prob, precision, yvar)
    t, n = a.run_until(0.0, 1e30, max_steps=nsteps, graph=False)
    assert n == nsteps
    ref = a.download()
    a.close()
    b = _fresh(prob, precision, yvar)
    t2, n2 = b.run_until(0.0, t, graph=True)
    assert n2 == nsteps and t2 == t
    out = b.download()
    # a second call continues from there
    t3, n3 = b.run_until(t2, t2 + 1e-12, graph=True)
    assert n3 == 1 and t3 > t2
    b.close()
    assert np.array_equal(out, ref)


def test_graph_loop_fp64_against_oracle(oracle):
    prob = P.orszag_tang(64)
    ref = prob.q.copy()
    dts = oracle.run(prob, ref, 12)
    t_end = 0.0
    for dt in dts:
        t_end += float(dt)
    integ = _fresh(prob, "fp64")
    t, n = integ.run_until(0.0, t_end, graph=True)
    out = integ.download()
    integ.close()
    assert n == 12
    # dt kept on the device: the damping factor from the device exp
    assert rel_l1(interior(prob, out), interior(prob, ref)) <= 1e-12


def test_model_run_device_loop(tmp_path):
    """Model.run(device_loop=True): the same snapshots (steps and times) as
    the host loop, the states equal to FP64 rounding."""
    from miso_b200.model import Model
    prob = P.orszag_tang(48)
    cfg = dict(prob.config)
    cfg["time"] = {"tend": 0.2, "dt_output": 0.05}
    outs = []
    for loop, sub in ((False, "host"), (True, "device")):
        cfg["io"] = {"enabled": True, "continue": False, "save_dir": str(tmp_path / sub) + "/"}
        m = Model(cfg, prob.grid, prob.q, precision="fp64")
        m.run(device_loop=loop)
        outs.append((m.n_step, m.n_output, m.time, m.state()))
        m.close()
    (s1, o1, t1, q1), (s2, o2, t2, q2) = outs
    assert (s1, o1) == (s2, o2)
    assert abs(t1 - t2) <= 1e-12 * t1
    assert rel_l1(interior(prob, q2), interior(prob, q1)) <= 1e-12
