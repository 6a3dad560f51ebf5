"""The run loop (miso_b200.model.Model, the reference's ModelBase::run):
output scheduling, the snapshot files, and a resumed run."""
import os

import numpy as np
import pytest

from miso_b200 import problems as P
from miso_b200.checkpoint import Output
from miso_b200.integrator import MHD
from miso_b200.model import Model

pytestmark = pytest.mark.gpu


def _cfg(prob, tmp, tend, dt_output, cont=False):
    cfg = dict(prob.config)
    cfg["time"] = {"tend": tend, "dt_output": dt_output}
    cfg["io"] = {"enabled": True, "continue": cont, "save_dir": str(tmp) + "/",
                 "n_output_digits": 8}
    return cfg


def _manual(prob, tend):
    """The same loop by hand: cfl, update until time >= tend."""
    m = MHD(prob.config, prob.grid, sign=prob.sign, precision="fp64")
    m.apply_initial_condition(prob.q)
    t, times = 0.0, []
    while t < tend:
        t += m.step()
        times.append(t)
    out = m.integrator.download()
    m.integrator.close()
    return out, times


def test_run_writes_snapshots_on_schedule(tmp_path):
    prob = P.orszag_tang(32)
    tend, dto = 0.05, 0.02
    model = Model(_cfg(prob, tmp_path, tend, dto), prob.grid, prob.q, sign=prob.sign)
    model.run()
    final = model.state()
    model.close()
    ref, times = _manual(prob, tend)
    assert np.array_equal(final, ref)
    # snapshots at t = 0 and at the first step reaching each multiple of dt_output
    want = [0.0]
    n = 1
    for t in times:
        if t >= dto * n:
            want.append(t)
            n += 1
    out = Output(str(tmp_path) + "/", prob.config, prob.grid)
    got = [out.load_time(k)[0] for k in range(len(want))]
    assert got == want
    assert not os.path.exists(out.mhd_path(len(want)))
    with open(os.path.join(out.time_dir, "n_output.txt")) as f:
        assert int(f.readline()) == len(want) - 1
    # snapshot 0 holds the initial state
    inner = (slice(None),) + prob.grid.interior
    assert np.array_equal(out.load(0)[inner], prob.q[inner])


def test_resumed_run_equals_uninterrupted(tmp_path):
    prob = P.orszag_tang(32)
    a = Model(_cfg(prob, tmp_path / "a", 0.03, 0.01), prob.grid, prob.q, sign=prob.sign)
    a.run()
    a.close()
    b = Model(_cfg(prob, tmp_path / "a", 0.06, 0.01, cont=True), prob.grid, prob.q,
              sign=prob.sign)
    b.run()
    resumed = b.state()
    b.close()
    c = Model(_cfg(prob, tmp_path / "c", 0.06, 0.01), prob.grid, prob.q, sign=prob.sign)
    c.run()
    straight = c.state()
    c.close()
    assert np.array_equal(resumed, straight)


@pytest.mark.parametrize("make,dims,precision", [
    (lambda: P.orszag_tang(32), (2, 2, 1), "fp64"),
    (lambda: P.turbulence(16, seed=3), (1, 2, 2), "fp64"),
    (lambda: P.turbulence(16, seed=3), (2, 1, 2), "fp32_split")],
    ids=["ot32_2x2x1_fp64", "turb16_1x2x2_fp64", "turb16_2x1x2_split"])
def test_decomposed_run_equals_single_grid(tmp_path, make, dims, precision):
    """ModelBase::run of a grid decomposed over ranks (here threads on one
    GPU): the same snapshot times as the single grid, and every snapshot,
    assembled from the ranks' files by coords.csv, equals the single grid's
    interior bit for bit."""
    from miso_b200.model import run_local_models
    prob = make()
    tend, dto = 0.03, 0.01
    one = Model(_cfg(prob, tmp_path / "one", tend, dto), prob.grid, prob.q, sign=prob.sign,
                precision=precision)
    one.run()
    one.close()
    models = run_local_models(_cfg(prob, tmp_path / "many", tend, dto), prob.grid, prob.q, dims,
                              sign=prob.sign, precision=precision)
    assert len({(m.time, m.n_step, m.n_output) for m in models}) == 1
    assert (models[0].time, models[0].n_step, models[0].n_output) == \
        (one.time, one.n_step, one.n_output)
    a = Output(str(tmp_path / "one") + "/", prob.config, prob.grid)
    b = Output(str(tmp_path / "many") + "/", prob.config, prob.grid, dims=dims)
    inner = (slice(None),) + prob.grid.interior
    for n in range(one.n_output):
        assert a.load_time(n) == b.load_time(n)
        assert np.array_equal(b.load_global(n), a.load(n)[inner]), n
