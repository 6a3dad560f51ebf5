"""The workloads as they are stated, and the 3-D kernels with real tiling,
against the oracle (the C restatement pinned bit for bit to the reference's
own host integrator, mhd_integrator_host.hpp:258-350).

* 3-D grids of unequal, non-tile-multiple sizes (70 x 44 x 72): the split
  form's Runge-Kutta stage runs 6 (j) x 3 (k) tiles of 8 x 32 with ragged
  last tiles and 3 chunks of 32 planes along i (the last one 6 planes); the
  x / y sweeps run 3 chunks of 32 planes; the z sweep 3 segments per row.
  Periodic (turbulence) and mirror (blast) faces; FP64 bit for bit, split
  form within the single-grid tolerances.
* Brio-Wu x 4096 (sizes U{512..8192}, each left / right value scaled by
  U[0.8, 1.2]) and Orszag-Tang x 32 (sizes U{128..1024}^2), each as one
  batch, 10 steps in FP64 and in split form; 16 instances -- the smallest,
  the largest and 14 seeded others -- against the oracle (run in a spawned
  process pool).
"""
import numpy as np
import pytest

from conftest import interior, rel_l1
from miso_b200 import problems as P
from miso_b200.batch import Batch
from miso_b200.integrator import Integrator
from oracle_pool import run_many

pytestmark = pytest.mark.gpu

SHAPE = (70, 44, 72)


def _pressure(q, gm):
    return (gm - 1.0) * q[P.RO] * q[P.EI]


def _errors(a, b, gm):
    return (rel_l1(a[P.RO], b[P.RO]), rel_l1(_pressure(a, gm), _pressure(b, gm)),
            rel_l1(a[P.BX:P.BZ + 1], b[P.BX:P.BZ + 1]))


def _run(prob, nsteps, precision, chunks=None):
    integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision=precision)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    if chunks:
        integ.set_chunks(*chunks)
    dts = []
    for _ in range(nsteps):
        dt = integ.cfl()
        integ.update(dt)
        dts.append(dt)
    out = integ.download()
    integ.close()
    return out, np.array(dts)


MAKERS = {"turbulence": lambda: P.turbulence(SHAPE[0], seed=21, shape=SHAPE),
          "blast": lambda: P.blast(SHAPE[0], seed=22, shape=SHAPE)}


@pytest.mark.parametrize("kind", sorted(MAKERS))
def test_fp64_ragged_3d_bit_exact(kind, oracle):
    prob = MAKERS[kind]()
    nsteps = 4
    ref = prob.q.copy()
    dts_o = oracle.run(prob, ref, nsteps)
    out, dts = _run(prob, nsteps, "fp64")
    assert np.array_equal(dts, dts_o)
    a, b = interior(prob, out), interior(prob, ref)
    assert int(np.sum(a != b)) == 0


@pytest.mark.parametrize("kind", sorted(MAKERS))
def test_split_ragged_3d_multi_tile_vs_oracle(kind, oracle):
    """Default kernels (pipelined RK stage with the deferred last update,
    line x / y sweeps, shuffle z sweep) on many ragged tiles and chunks:
    relative L1 of rho <= 1e-6, of p and B <= 1e-5 after 20 steps."""
    prob = MAKERS[kind]()
    nsteps = 20
    ref = prob.q.copy()
    oracle.run(prob, ref, nsteps)
    integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision="fp32_split")
    assert integ.get_variant(0) == 3 and integ.get_variant(1) == 0
    integ.close()
    out, _ = _run(prob, nsteps, "fp32_split", chunks=(32, 32))
    e_ro, e_p, e_b = _errors(interior(prob, out), interior(prob, ref), prob.config["eos"]["gm"])
    print(f"{kind} {SHAPE}: L1 rho {e_ro:.2e} p {e_p:.2e} B {e_b:.2e}")
    assert e_ro <= 1e-6
    assert e_p <= 1e-5
    assert e_b <= 1e-5


def _sample(sizes, count=16, seed=7):
    """Indices of the smallest and the largest instance and count - 2 others."""
    order = np.argsort(sizes, kind="stable")
    pick = [int(order[0]), int(order[-1])]
    rng = np.random.default_rng(seed)
    rest = [i for i in rng.permutation(len(sizes)) if i not in pick]
    return pick + [int(i) for i in rest[:count - 2]]


def _batch_case(name):
    if name == "brio_wu_4096":
        rng = np.random.default_rng(0)
        sizes = rng.integers(512, 8192 + 1, size=4096)
        scales = rng.uniform(0.8, 1.2, size=(4096, 6))
        probs = P.brio_wu_batch(4096, 512, 8192, seed=0)
        jobs = [("brio_wu", {"n": int(n), "axis": 0, "scale": [float(x) for x in sc]})
                for n, sc in zip(sizes, scales)]
    else:
        rng = np.random.default_rng(0)
        sizes = rng.integers(128, 1024 + 1, size=32)
        probs = P.orszag_tang_batch(32, 128, 1024, seed=0)
        jobs = [("orszag_tang", {"n": int(n)}) for n in sizes]
    for p, n in zip(probs, sizes):  # the jobs rebuild exactly these instances
        assert max(p.grid.i_size, p.grid.j_size) == n
    return probs, jobs, sizes


@pytest.mark.slow
@pytest.mark.parametrize("name", ["brio_wu_4096", "orszag_tang_32"])
def test_batch_stated_config_vs_oracle(name):
    probs, jobs, sizes = _batch_case(name)
    nsteps = 10
    picks = _sample(sizes)
    assert sizes[picks[0]] == sizes.min() and sizes[picks[1]] == sizes.max()
    refs = run_many([jobs[i][:2] + (nsteps,) for i in picks])
    for precision in ("fp64", "fp32_split"):
        with Batch(probs, precision) as b:
            b.upload_all()
            b.run(nsteps, graph=True)
            b.sync()
            for i, (ref, dts) in zip(picks, refs):
                p = probs[i]
                a = interior(p, b.download(i))
                if precision == "fp64":
                    # same per-cell arithmetic as the single grid; the
                    # damping factor comes from the device exp (<= 1 ulp)
                    assert rel_l1(a, ref) <= 1e-12, (name, i, int(sizes[i]))
                else:
                    e_ro, e_p, e_b = _errors(a, ref, p.config["eos"]["gm"])
                    tol = 1e-5 if name.startswith("brio") else 1e-6
                    assert e_ro <= tol, (name, i, int(sizes[i]), e_ro)
                    assert e_p <= 1e-5 and e_b <= 1e-5, (name, i, e_p, e_b)


def test_blast384_sharp_matches_reference_record():
    """The blast configuration as stated (384^3, sharp pressure edge, seed
    0) in the FP64 form: its time step and its FP64 sum of ei over the
    interior equal the reference host integrator's at every one of steps
    1-21, bit for bit (tests/golden/blast384_sharp_reference.json, made by
    tests/golden/make_blast384_record.py), and, like the reference's, its
    step 22 leaves non-finite values, which the next CFL pass reports."""
    import json
    import os

    from miso_b200 import _lib
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                        "blast384_sharp_reference.json")
    rec = json.load(open(path))["steps"]
    assert len(rec) == 22 and not np.isfinite(rec[21]["sum_ei"])
    prob = P.blast(384, seed=0)
    g = prob.grid
    integ = Integrator(prob.config, g, sign=prob.sign, precision="fp64")
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    out = np.empty((9,) + tuple(g.shape))
    for r in rec:
        dt = integ.cfl()
        assert dt == r["dt"], r["step"]
        integ.update(dt)
        integ.download(out=out)
        total = float(np.sum(out[P.EI][g.interior], dtype=np.float64))
        if np.isfinite(r["sum_ei"]):
            assert total == r["sum_ei"], r["step"]
        else:
            assert not np.isfinite(total)
    with pytest.raises(_lib.MisoError) as e:
        integ.cfl()
    assert e.value.code == _lib.ERR_NONFINITE
    integ.close()
