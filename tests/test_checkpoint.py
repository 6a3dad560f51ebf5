"""Snapshots in the reference's on-disk layout (miso_b200/checkpoint.py).

CPU: a run directory written here is read back by the reference's own
post-processing reader, pymiso (pymiso/src/pymiso/data.py:103-166), when it
is present; our restart reader round-trips float64 and float32 files.
GPU: the asynchronous snapshot writes the same bytes as the synchronous one
while stepping goes on, and a run restarted from a snapshot continues bit for
bit like the uninterrupted FP64 run.
"""
import os
import sys
import types

import numpy as np
import pytest

from miso_b200 import problems as P
from miso_b200.checkpoint import Output
from oracle.oracle import REFERENCE_ROOT

PYMISO_SRC = os.path.join(REFERENCE_ROOT, "pymiso", "src")


class _FakeHandle:
    def __init__(self, q):
        self.q = q

    def download(self):
        return self.q.copy()


def _box_module():
    """A minimal stand-in for python-box (attribute access on nested dicts),
    which pymiso imports and this image does not ship."""
    class Box(dict):
        def __init__(self, d=None):
            super().__init__()
            for k, v in (d or {}).items():
                self[k] = Box(v) if isinstance(v, dict) else v

        def __getattr__(self, k):
            try:
                return self[k]
            except KeyError as e:
                raise AttributeError(k) from e

        def __setattr__(self, k, v):
            self[k] = v

    mod = types.ModuleType("box")
    mod.Box = Box
    return mod


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_round_trip(tmp_path, real):
    prob = P.orszag_tang(24)
    out = Output(str(tmp_path / "data"), prob.config, prob.grid, real=real)
    out.write_setup()
    out.save(_FakeHandle(prob.q), time=0.125, n_output=3, n_step=17)
    q = out.load(3)
    assert np.array_equal(q, prob.q.astype(real).astype(np.float64))
    assert out.load_time(3) == (0.125, 3, 17)
    # the header is the element size as uint32, then 9 whole arrays
    size = os.path.getsize(out.mhd_path(3))
    assert size == 4 + 9 * prob.q[0].size * np.dtype(real).itemsize


@pytest.mark.skipif(not os.path.isdir(PYMISO_SRC), reason="pymiso sources not present")
@pytest.mark.parametrize("make", [lambda: P.orszag_tang(24), lambda: P.turbulence(8, seed=1),
                                  lambda: P.brio_wu(40)], ids=["ot2d", "turb3d", "bw1d"])
def test_pymiso_reads_output(tmp_path, monkeypatch, make):
    prob = make()
    save_dir = str(tmp_path / "data")
    out = Output(save_dir, prob.config, prob.grid)
    out.write_setup()
    out.save(_FakeHandle(prob.q), time=0.5, n_output=2, n_step=40)
    monkeypatch.setitem(sys.modules, "box", _box_module())
    monkeypatch.syspath_prepend(PYMISO_SRC)
    for name in [m for m in sys.modules if m == "pymiso" or m.startswith("pymiso.")]:
        monkeypatch.delitem(sys.modules, name)
    import pymiso
    d = pymiso.Data(save_dir)
    d.load(2)
    assert d.time.time == 0.5 and d.time.load_n_step == 40
    inner = prob.q[(slice(None),) + prob.grid.interior]
    for v, name in enumerate(("ro", "vx", "vy", "vz", "bx", "by", "bz", "ei", "ph")):
        assert np.array_equal(getattr(d, name), np.squeeze(inner[v])), name
    g = prob.grid
    assert np.array_equal(d.grid.x, g.x[g.i_margin:g.i_total - g.i_margin])
    assert np.array_equal(d.grid.z, g.z[g.k_margin:g.k_total - g.k_margin])


@pytest.mark.gpu
def test_async_snapshot_and_restart(tmp_path):
    from miso_b200.integrator import Integrator
    prob = P.orszag_tang(48)
    out = Output(str(tmp_path / "data"), prob.config, prob.grid)
    out.write_setup()
    integ = Integrator(prob.config, prob.grid, precision="fp64")
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    t = 0.0
    for _ in range(5):
        dt = integ.cfl()
        integ.update(dt)
        t += dt
    out.save(integ, t, 1, 5)
    out.save_async(integ, t, 2, 5)  # same state, written while stepping goes on
    for _ in range(5):
        integ.update(integ.cfl())
    out.wait()
    with open(out.mhd_path(1), "rb") as f1, open(out.mhd_path(2), "rb") as f2:
        assert f1.read() == f2.read()
    full = integ.download()
    integ.close()
    # restart from snapshot 1 and take the same 5 steps
    again = Integrator(prob.config, prob.grid, precision="fp64")
    again.upload(out.load(1))
    for _ in range(5):
        again.update(again.cfl())
    assert np.array_equal(again.download(), full)
    again.close()


@pytest.mark.skipif(not os.path.isdir(PYMISO_SRC), reason="pymiso sources not present")
@pytest.mark.parametrize("make,dims", [(lambda: P.orszag_tang(24), (2, 3, 1)),
                                       (lambda: P.turbulence(8, seed=2), (2, 2, 2))],
                         ids=["ot2d_2x3", "turb3d_2x2x2"])
def test_pymiso_reads_decomposed_output(tmp_path, monkeypatch, make, dims):
    """A run directory of a grid in boxes (one mhd file per rank, every
    rank's coordinates in coords.csv, the global grid in grid.bin and
    config.yaml) is read by pymiso as the global field, and by our own
    load_global alike."""
    from miso_b200.shard import split_grid3, split_state
    prob = make()
    save_dir = str(tmp_path / "data")
    per = prob.config["domain"]["periodic"]
    specs = split_grid3(prob.grid, dims, (per["x"], per["y"], per["z"]))
    outs = [Output(save_dir, prob.config, prob.grid, rank=s.rank, dims=dims, box=s.grid)
            for s in specs]
    for o in outs:
        o.write_setup()
    for o, s in zip(outs, specs):
        o.save(_FakeHandle(split_state(prob.q, prob.grid, s)), time=0.25, n_output=1, n_step=9)
    inner = prob.q[(slice(None),) + prob.grid.interior]
    assert np.array_equal(outs[0].load_global(1), inner)
    monkeypatch.setitem(sys.modules, "box", _box_module())
    monkeypatch.syspath_prepend(PYMISO_SRC)
    for name in [m for m in sys.modules if m == "pymiso" or m.startswith("pymiso.")]:
        monkeypatch.delitem(sys.modules, name)
    import pymiso
    d = pymiso.Data(save_dir)
    d.load(1)
    assert d.time.time == 0.25
    for v, name in enumerate(("ro", "vx", "vy", "vz", "bx", "by", "bz", "ei", "ph")):
        assert np.array_equal(getattr(d, name), np.squeeze(inner[v])), name
