"""The y and z viscosity sweeps fused into one pass (y sweep variant 3).

The fused pass runs the y sweep down each k column of a plane and the z
sweep along each finished row, with the separate sweeps' per-cell
arithmetic, so it must give the same bits as the y line sweep followed by
the z sweep: every value of the state, every dt, and the monitors (whose
FP64 sums only change order).
"""
import numpy as np
import pytest

from miso_b200 import problems as P
from miso_b200.integrator import Integrator

pytestmark = pytest.mark.gpu

SHAPES = [
    # one k block with both periodic wraps
    ("turb40", lambda: P.turbulence(40, seed=5), None),
    # mirror faces on every axis
    ("blast20", lambda: P.blast(20, seed=4), None),
    # two k blocks, the second ragged (156 = 112 + 44), periodic
    ("turb156", lambda: P.turbulence(156, seed=2), None),
    # 116 = 112 + 4: a second k block of four cells, mirror faces
    ("blast116", lambda: P.blast(116, seed=1), None),
    # unequal axes, and rows cut into chunks of 16 (items start mid-axis)
    ("turb_24x68x44_chunk16", lambda: P.turbulence(24, seed=8, shape=(24, 68, 44)), 16),
]


def _run(prob, fused, steps=3, chunk=None, graph=True, mon=False):
    integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision="fp32_split")
    integ.set_variant(2, 3 if fused else 0)
    integ.set_variant(3, 0)
    if chunk:
        integ.set_chunks(64, chunk)
    if mon:
        integ.set_monitor_fusion(True)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    dts = []
    if graph:
        integ.run(steps, graph=True)
        integ.sync()
    else:
        for _ in range(steps):
            dt = integ.cfl()
            integ.update(dt)
            dts.append(dt)
    dts.append(integ.cfl())
    m = integ.monitors()
    out = integ.download()
    integ.close()
    return out, dts, m


@pytest.mark.parametrize("name,make,chunk", SHAPES, ids=[s[0] for s in SHAPES])
def test_fused_equals_separate_sweeps(name, make, chunk):
    prob = make()
    a, dta, _ = _run(prob, False, chunk=chunk)
    b, dtb, _ = _run(prob, True, chunk=chunk)
    assert dta == dtb
    assert np.array_equal(a, b), f"{int(np.sum(a != b))} values differ"


def test_fused_host_dt_and_monitors():
    """The reference's host-dt sequence (cfl -> update) with the monitors
    folded into the fused pass: same dt sequence and state as the separate
    sweeps, monitors within FP64 summation order of the unfused ones."""
    prob = P.turbulence(48, seed=3)
    a, dta, ma = _run(prob, False, steps=4, graph=False)
    b, dtb, mb = _run(prob, True, steps=4, graph=False, mon=True)
    assert dta == dtb
    assert np.array_equal(a, b)
    # sums whose terms cancel (the momenta of a periodic box) are held to
    # 1e-12 of the mass, the scale of their terms
    for key in ("mass", "mom_x", "mom_y", "mom_z", "energy", "ph2", "divb_l1", "divb_max"):
        tol = 1e-12 * max(abs(ma[key]), abs(ma["mass"]) if key.startswith("mom") else 0.0)
        assert abs(mb[key] - ma[key]) <= tol, (key, ma[key], mb[key])


def test_fused_run_until():
    """With the fused pass a step swaps the hi / lo sets twice, so the
    device-held time loop is a one-step body; it equals host-launched
    steps."""
    prob = P.turbulence(32, seed=4)
    outs = []
    for use_graph in (True, False):
        integ = Integrator(prob.config, prob.grid, precision="fp32_split")
        integ.set_variant(2, 3)
        integ.upload(prob.q)
        integ.apply_boundary_condition()
        t, n = integ.run_until(0.0, 1.0, max_steps=7, graph=use_graph)
        outs.append((t, n, integ.download()))
        integ.close()
    assert outs[0][0] == outs[1][0] and outs[0][1] == outs[1][1] == 7
    assert np.array_equal(outs[0][2], outs[1][2])


def _single(prob, yvar, nsteps):
    integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision="fp32_split")
    integ.set_variant(2, yvar)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    integ.run(nsteps, graph=False)
    out = integ.download()
    integ.close()
    return out


@pytest.mark.parametrize("yvar", [3, 0], ids=["fused", "separate"])
def test_batch_views_keep_their_own_sets(yvar):
    """A batch's 3-D instances run through views; with the fused pass a
    view's step swaps its hi / lo sets twice while the batch's other
    instances swap three times, so each view keeps its own set.  Eager and
    graph-replayed steps, an upload of one view's state between them, and
    the downloads must all find each view's state: every view equals its
    grid stepped alone, bit for bit."""
    from conftest import interior
    from miso_b200.batch import Batch
    probs = [P.turbulence(32, seed=1), P.orszag_tang(32), P.blast(24, seed=2)]
    with Batch(probs, precision="fp32_split") as b:
        if b.views() != 2:
            pytest.skip("the 3-D instances do not run through views here")
        b.set_variant(2, yvar)
        b.upload_all()
        b.run(1, graph=False)
        b.run(4, graph=True)
        b.run(1, graph=False)
        b.upload(0, probs[0].q)  # instance 0 starts again
        b.run(3, graph=True)
        b.sync()
        outs = [b.download(i) for i in range(len(probs))]
    for i, n in ((0, 3), (2, 9)):
        ref = _single(probs[i], yvar, n)
        assert np.array_equal(interior(probs[i], outs[i]), interior(probs[i], ref)), i
