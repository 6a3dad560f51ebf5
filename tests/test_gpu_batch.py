"""Batched solver: a mix of 1-D, 2-D and 3-D instances of uneven sizes and
parameters in one work list, against the oracle instance by instance."""
import numpy as np
import pytest

from conftest import interior, rel_l1
from miso_b200 import problems as P
from miso_b200.batch import Batch

pytestmark = pytest.mark.gpu


def mixed():
    return [P.brio_wu(96, scale=[1.1, 0.9, 1.0, 1.2, 0.8, 1.05]), P.orszag_tang(24),
            P.brio_wu(150, axis=1), P.turbulence(10, seed=5), P.sod(70, axis=2),
            P.blast(12, seed=9), P.orszag_tang(36)]


def test_batch_fp64_matches_oracle(oracle):
    probs = mixed()
    nsteps = 6
    with Batch(probs, "fp64") as b:
        b.upload_all()
        b.run(nsteps, graph=True)
        b.sync()
        for i, p in enumerate(probs):
            ref = p.q.copy()
            oracle.run(p, ref, nsteps)
            out = b.download(i)
            # same per-cell arithmetic as the single-grid path; the damping
            # factor exp(-dt/tau) comes from the device exp (<= 1 ulp)
            assert rel_l1(interior(p, out), interior(p, ref)) <= 1e-12, p.name


def test_batch_fp64_equals_single_grids():
    """Every FP64 batch instance evolves bit for bit as its grid on its own
    handle with the device-held dt (both take the damping factor from the
    device exp): the row sweeps of the 1-D / 2-D instances (shuffles along
    the unit-stride axis, a march along the other) and the closed-form
    degenerate sweeps give the per-cell sweep's bits."""
    from miso_b200.integrator import Integrator
    probs = mixed()
    nsteps = 6
    with Batch(probs, "fp64") as b:
        b.upload_all()
        b.run(nsteps, graph=True)
        b.sync()
        dts = b.dt()
        outs = [b.download(i) for i in range(len(probs))]
    for i, p in enumerate(probs):
        integ = Integrator(p.config, p.grid, sign=p.sign, precision="fp64")
        integ.upload(p.q)
        integ.apply_boundary_condition()
        integ.run(nsteps, graph=False)
        ref = integ.download()
        dt = integ.last_dt()
        integ.close()
        assert dt == dts[i], (p.name, dt, dts[i])
        a, r = interior(p, outs[i]), interior(p, ref)
        assert np.array_equal(a, r), (p.name, int(np.sum(a != r)))


def test_batch_rows_deferred_update_bit_identical():
    """RK variant 3 (the default) defers the 1-D / 2-D instances' last
    Runge-Kutta update into the step's first sweep, which forms U^{n+1} and
    its speed from hi, lo and the stage's right-hand side with the stage's
    own arithmetic: every instance off the pipelined path (rows and the
    block-tile 3-D grid) gives the bits of variant 2."""
    probs = mixed()
    outs = []
    for variant in (3, 2):
        with Batch(probs, "fp32_split") as b:
            b.set_variant(0, variant)
            b.upload_all()
            b.run(3, graph=False)
            b.run(4, graph=True)
            b.sync()
            outs.append(([b.download(i) for i in range(len(probs))], b.dt()))
    for i, p in enumerate(probs):
        g = p.grid
        if g.i_size > 1 and g.j_size > 1 and g.k_size > 1 and (g.k_size + 4) % 4 == 0:
            continue  # a view on the pipelined kernels: variants 2 and 3 round differently
        assert outs[0][1][i] == outs[1][1][i], p.name
        assert np.array_equal(interior(p, outs[0][0][i]), interior(p, outs[1][0][i])), p.name


def test_batch_whole_gpu_view_on_batch_stream():
    """A 3-D instance large enough to fill the GPU (256^3) steps on the
    batch's own stream, in turn with the 2-D instances' kernels, not beside
    them: it still equals its grid stepped alone, bit for bit, through
    eager and graph-replayed steps and a download."""
    from miso_b200.integrator import Integrator
    probs = [P.turbulence(256, seed=4), P.orszag_tang(64)]
    with Batch(probs, "fp32_split") as b:
        assert b.views() == 1
        b.upload_all()
        b.run(1, graph=False)
        b.run(2, graph=True)
        b.sync()
        big = b.download(0)
    p = probs[0]
    integ = Integrator(p.config, p.grid, precision="fp32_split")
    integ.upload(p.q)
    integ.apply_boundary_condition()
    integ.run(3, graph=False)
    ref = integ.download()
    integ.close()
    assert np.array_equal(interior(p, big), interior(p, ref))


def test_batch_per_instance_dt(oracle):
    probs = mixed()
    with Batch(probs, "fp64") as b:
        b.upload_all()
        b.run(1, graph=False)
        dts = b.dt()
    for p, dt in zip(probs, dts):
        q = p.q.copy()
        oracle.fill_ghosts(p, q)
        assert dt == oracle.cfl(p, q), p.name


def test_batch_split_matches_oracle(oracle):
    probs = mixed()
    nsteps = 10
    with Batch(probs, "fp32_split") as b:
        b.upload_all()
        b.run(nsteps, graph=True)
        b.sync()
        for i, p in enumerate(probs):
            ref = p.q.copy()
            oracle.run(p, ref, nsteps)
            out = b.download(i)
            a, r = interior(p, out), interior(p, ref)
            assert rel_l1(a[P.RO], r[P.RO]) <= 1e-5, p.name


def test_batch_graph_equals_eager():
    probs = mixed()[:4]
    outs = []
    for graph in (True, False):
        with Batch(probs, "fp32_split") as b:
            b.upload_all()
            b.run(5, graph=graph)
            outs.append([b.download(i) for i in range(len(probs))])
    for a, c in zip(*outs):
        assert np.array_equal(a, c)


def test_batch_split_fused_cfl_equals_cfl_pass():
    """The FP32 batch folds each step's CFL minima into its last viscosity
    sweep; after a ghost fill (which drops them) the next step runs the
    separate CFL pass.  Both give the same time steps and states, bit for
    bit."""
    probs = mixed()
    with Batch(probs, "fp32_split") as b1, Batch(probs, "fp32_split") as b2:
        for b in (b1, b2):
            b.upload_all()
        b1.run(4, graph=True)
        b2.run(3, graph=True)
        b2.fill_ghosts()
        b2.run(1, graph=False)
        assert np.array_equal(b1.dt(), b2.dt())
        for i in range(len(probs)):
            assert np.array_equal(b1.download(i), b2.download(i)), probs[i].name


def three_d_mix():
    return [P.turbulence(32, seed=2), P.blast(24, seed=4),
            P.turbulence(40, seed=6, shape=(40, 36, 44)), P.brio_wu(200), P.orszag_tang(48),
            P.blast(16, seed=8)]


def test_batch_3d_instances_equal_single_grids():
    """3-D split instances run through views on the pipelined kernels, each
    on its own stream inside the step's graph: every instance evolves bit
    for bit as the same grid on its own handle (same kernels, same device
    dt), the 1-D / 2-D instances beside them as before."""
    from miso_b200.integrator import Integrator
    probs = three_d_mix()
    nsteps = 6
    with Batch(probs, "fp32_split") as b:
        b.upload_all()
        b.run(nsteps, graph=True)
        b.sync()
        dts = b.dt()
        outs = [b.download(i) for i in range(len(probs))]
    for i, p in enumerate(probs):
        if p.grid.k_size == 1:
            continue
        integ = Integrator(p.config, p.grid, sign=p.sign, precision="fp32_split")
        integ.upload(p.q)
        integ.apply_boundary_condition()
        integ.run(nsteps, graph=False)
        ref = integ.download()
        dt = integ.last_dt()
        integ.close()
        assert dt == dts[i], (p.name, dt, dts[i])
        assert np.array_equal(interior(p, outs[i]), interior(p, ref)), p.name


def test_batch_3d_instances_vs_oracle(oracle):
    probs = three_d_mix()
    nsteps = 6
    with Batch(probs, "fp32_split") as b:
        b.upload_all()
        b.run(nsteps, graph=True)
        b.sync()
        for i, p in enumerate(probs):
            ref = p.q.copy()
            oracle.run(p, ref, nsteps)
            a, r = interior(p, b.download(i)), interior(p, ref)
            assert rel_l1(a[P.RO], r[P.RO]) <= 1e-6, p.name


def test_batch_autotune_picks_and_caches(tmp_path, monkeypatch):
    """The batch tuner times the work-item lengths of the 3-D instances on
    whole graph-replayed steps, applies the fastest and caches it per batch
    composition; the chunk lengths leave every instance's result unchanged
    (each item is computed the same wherever it is cut); the variants agree
    to FP32 rounding."""
    import torch
    from miso_b200.autotune import BATCH_CHUNKS, BATCH_VARIANTS, autotune_batch
    monkeypatch.setenv("MISO_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    probs = [P.turbulence(32, seed=1), P.blast(24, seed=2), P.orszag_tang(40)]
    stream = torch.cuda.Stream()
    outs = []
    for tune in (False, True):
        with Batch(probs, "fp32_split", stream=stream.cuda_stream) as b:
            assert b.views() == 2
            b.upload_all()
            if tune:
                c = autotune_batch(b, steps=1)
                assert (c["rk_chunk"], c["av_chunk"]) in BATCH_CHUNKS
                assert len(c["ms_per_step"]) == len(BATCH_CHUNKS) * len(BATCH_VARIANTS)
                # cached: the second call returns the same choice at once
                assert autotune_batch(b) == c
                b.upload_all()
            b.run(4, graph=True)
            b.sync()
            outs.append([b.download(i) for i in range(len(probs))])
    for p, a, c in zip(probs, *outs):
        assert rel_l1(interior(p, a)[P.RO], interior(p, c)[P.RO]) <= 1e-5
