"""A grid decomposed into shards -- along i through miso_b200_set_halo, along
any of i, j and k through miso_b200_set_halo3 -- with the face halos
exchanged between passes, advances exactly like the single grid: the
shards here share one GPU (one host thread each, device copies for the
halo), and the gathered interior and every time step must be the single
grid's bit for bit -- the per-cell arithmetic does not depend on where a
shard ends, and the CFL minimum is exact."""
import numpy as np
import pytest

from miso_b200 import problems as P
from miso_b200.integrator import Integrator
from miso_b200.shard import run_local_shards

pytestmark = pytest.mark.gpu


def single(prob, steps, precision, variants=None):
    integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision=precision,
                       blend=prob.blend)
    for cls, var in (variants or {}).items():
        integ.set_variant(cls, var)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    dts = []
    for _ in range(steps):
        dt = integ.cfl()
        integ.update(dt)
        dts.append(dt)
    out = integ.download()[(slice(None),) + prob.grid.interior]
    integ.close()
    return out, dts


CASES = [
    ("turb32_split_x2", lambda: P.turbulence(32, seed=3), "fp32_split", 2, None),
    ("turb32_split_x4", lambda: P.turbulence(32, seed=3), "fp32_split", 4, None),
    ("blast32_split_x2", lambda: P.blast(32, seed=1), "fp32_split", 2, None),
    ("turb32_fp64_x2", lambda: P.turbulence(32, seed=3), "fp64", 2, None),
    ("blast24_fp64_x3", lambda: P.blast(24, seed=2), "fp64", 3, None),
    ("ot64_fp64_x2", lambda: P.orszag_tang(64), "fp64", 2, None),
    ("ot64_split_x2", lambda: P.orszag_tang(64), "fp32_split", 2, None),
    # sweep variants that read i ghosts directly (flat) or march across the face
    ("turb32_split_flat_x2", lambda: P.turbulence(32, seed=3), "fp32_split", 2,
     {0: 1, 1: 1, 2: 1, 3: 1}),
    ("blast32_split_march_x2", lambda: P.blast(32, seed=1), "fp32_split", 2,
     {0: 0, 1: 2, 2: 2}),
    # the magnetosphere demo's boundary: inflow on the first shard only, the
    # blend on every shard's cells before the exchange
    ("magneto16_fp64_x2", lambda: P.magnetosphere(16, extent=12.0), "fp64", 2, None),
]


@pytest.mark.parametrize("make,count", [(lambda: P.turbulence(40, seed=3), 2),
                                        (lambda: P.blast(36, seed=1), 3),
                                        (lambda: P.turbulence(32, seed=4), 4)],
                         ids=["turb40_x2", "blast36_x3", "turb32_x4"])
def test_overlapped_exchange_equals_single_grid(make, count):
    """The exchange on its own stream while each next pass finishes the
    planes that need no ghost, the boundary plane groups after it: the same
    bits as the single grid (and so as the blocking exchange)."""
    prob = make()
    steps = 4
    ref, dts = single(prob, steps, "fp32_split")
    got, sdts = run_local_shards(prob, count, steps, "fp32_split", overlap=True)
    assert sdts == dts
    assert np.array_equal(got, ref)


def test_overlap_refused_off_the_pipelined_path():
    from miso_b200 import _lib
    prob = P.turbulence(24, seed=1)
    with Integrator(prob.config, prob.grid, precision="fp32_split") as integ:
        with pytest.raises(_lib.MisoError) as e:
            integ.set_halo_overlap(1)  # no halo exchange set
        assert e.value.code == _lib.ERR_STATE


@pytest.mark.parametrize("name,make,precision,count,variants", CASES,
                         ids=[c[0] for c in CASES])
def test_shards_equal_single_grid(name, make, precision, count, variants):
    prob = make()
    steps = 3
    ref, dts = single(prob, steps, precision, variants)
    got, sdts = run_local_shards(prob, count, steps, precision, variants)
    assert sdts == dts
    assert got.shape == ref.shape
    assert np.array_equal(got, ref), float(np.max(np.abs(got - ref)))


def test_shard_refuses_device_dt_steps():
    from miso_b200 import _lib
    from miso_b200.shard import LocalHalo, split_grid, split_state
    prob = P.turbulence(16, seed=0)
    spec = split_grid(prob.grid, 2, True)[0]
    integ = Integrator(prob.config, spec.grid, precision="fp32_split")
    LocalHalo(2, True).attach(integ, spec)
    integ.upload(split_state(prob.q, prob.grid, spec))
    with pytest.raises(_lib.MisoError) as e:
        integ.run(1, graph=False)
    assert e.value.code == _lib.ERR_STATE
    integ.close()


def test_dist_halo_one_rank_nccl_equals_single_grid():
    """The torch.distributed transport on the GPU: one NCCL rank whose two
    i faces are shared with itself (the periodic wrap through the exchange
    callback, dt through an NCCL all-reduce) steps like the single grid."""
    import datetime
    import socket

    import torch.distributed as dist

    from miso_b200.shard import DistHalo, ShardSpec

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        prob = P.turbulence(32, seed=4)
        ref, dts = single(prob, 3, "fp32_split")
        integ = Integrator(prob.config, prob.grid, precision="fp32_split")
        DistHalo(periodic_x=True, device="cuda").attach(
            integ, ShardSpec(0, 1, 0, 32, prob.grid, True, True))
        integ.upload(prob.q)
        integ.apply_boundary_condition()
        got_dts = []
        for _ in range(3):
            dt = integ.cfl()
            integ.update(dt)
            got_dts.append(dt)
        got = integ.download()[(slice(None),) + prob.grid.interior]
        integ.close()
        assert got_dts == dts
        assert np.array_equal(got, ref)
    finally:
        dist.destroy_process_group()


# decompositions along j and k (shards per axis), both forms
CASES3 = [
    ("turb32_fp64_2x2x1", lambda: P.turbulence(32, seed=3), "fp64", (2, 2, 1), None),
    ("blast24_fp64_1x2x2", lambda: P.blast(24, seed=2), "fp64", (1, 2, 2), None),
    ("ot64_fp64_1x2x1", lambda: P.orszag_tang(64), "fp64", (1, 2, 1), None),
    ("magneto16_fp64_1x2x2", lambda: P.magnetosphere(16, extent=12.0), "fp64", (1, 2, 2), None),
    ("turb32_split_2x2x2", lambda: P.turbulence(32, seed=3), "fp32_split", (2, 2, 2), None),
    ("blast32_split_1x2x2", lambda: P.blast(32, seed=1), "fp32_split", (1, 2, 2), None),
    ("ot64_split_2x2x1", lambda: P.orszag_tang(64), "fp32_split", (2, 2, 1), None),
    # j only: the fused y and z pass reads the exchanged j ghosts
    ("turb40_split_1x2x1", lambda: P.turbulence(40, seed=5), "fp32_split", (1, 2, 1), None),
    # k only, periodic: separate y and z sweeps, no wrap copies at a shared face;
    # 240 = 2 x (112 + 8): a second, ragged k block on each shard
    ("turb_16x16x240_split_1x1x2", lambda: P.turbulence(16, seed=2, shape=(16, 16, 240)),
     "fp32_split", (1, 1, 2), None),
    ("blast_20x20x36_split_1x1x3", lambda: P.blast(20, seed=6, shape=(20, 20, 36)),
     "fp32_split", (1, 1, 3), None),
    # sweep variants that read ghosts directly (flat), march across a face,
    # or stream k rows (z line)
    ("turb32_split_flat_1x2x2", lambda: P.turbulence(32, seed=3), "fp32_split", (1, 2, 2),
     {0: 1, 1: 1, 2: 1, 3: 1}),
    ("blast32_split_march_2x2x2", lambda: P.blast(32, seed=1), "fp32_split", (2, 2, 2),
     {0: 0, 1: 2, 2: 2, 3: 2}),
    ("turb32_split_zline_1x1x2", lambda: P.turbulence(32, seed=4), "fp32_split", (1, 1, 2),
     {2: 0, 3: 2}),
    # the thinnest shards: 2 * margin = 4 interior rows / columns each
    ("turb16_split_1x4x1", lambda: P.turbulence(16, seed=7), "fp32_split", (1, 4, 1), None),
    ("turb16_split_1x1x4", lambda: P.turbulence(16, seed=7), "fp32_split", (1, 1, 4), None),
    ("blast16_fp64_2x2x4", lambda: P.blast(16, seed=3), "fp64", (2, 2, 4), None),
]


@pytest.mark.parametrize("name,make,precision,dims,variants", CASES3,
                         ids=[c[0] for c in CASES3])
def test_shards_along_j_and_k_equal_single_grid(name, make, precision, dims, variants):
    prob = make()
    steps = 3
    ref, dts = single(prob, steps, precision, variants)
    count = dims[0] * dims[1] * dims[2]
    got, sdts = run_local_shards(prob, count, steps, precision, variants, dims=dims)
    assert sdts == dts
    assert got.shape == ref.shape
    assert np.array_equal(got, ref), float(np.max(np.abs(got - ref)))


def test_halo3_refusals():
    """A shared face on a degenerate axis and the overlapped exchange with a
    shared j or k face are refused; a decomposition along i through the
    per-axis call keeps the overlap."""
    import ctypes

    from miso_b200 import _lib
    from miso_b200.shard import LocalHalo, split_grid3
    ot = P.orszag_tang(32)
    with Integrator(ot.config, ot.grid, precision="fp64") as integ:
        fn = _lib.HALO3_EXCHANGE_FN(lambda *a: 0)
        ops = _lib.Halo3Ops(fn, _lib.HALO_MIN_FN(0), None)
        ext = (ctypes.c_int * 6)(0, 0, 0, 0, 1, 1)  # k has one cell
        assert integ._lib.miso_b200_set_halo3(integ._h, ext, ctypes.byref(ops)) == _lib.ERR_ARG
    prob = P.turbulence(32, seed=1)
    spec = split_grid3(prob.grid, (1, 2, 1), (True, True, True))[0]
    with Integrator(prob.config, spec.grid, precision="fp32_split") as integ:
        LocalHalo(2, True, dims=(1, 2, 1), periodic=(True, True, True)).attach(integ, spec)
        with pytest.raises(_lib.MisoError) as e:
            integ.set_halo_overlap(1)
        assert e.value.code == _lib.ERR_STATE


@pytest.mark.parametrize("precision", ["fp64", "fp32_split"])
def test_dist_halo_one_rank_all_faces_equals_single_grid(precision):
    """One NCCL rank whose six faces are all shared with itself: the j and k
    faces go through the library's packing, the callback's wrap copy and
    the unpacking, the i faces in place, dt through an NCCL all-reduce; the
    periodic box steps like the single grid, bit for bit."""
    import datetime
    import socket

    import torch.distributed as dist

    from miso_b200.shard import DistHalo, ShardSpec

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        prob = P.turbulence(24, seed=6, shape=(24, 20, 28))
        ref, dts = single(prob, 3, precision)
        integ = Integrator(prob.config, prob.grid, precision=precision)
        spec = ShardSpec(0, 1, 0, 24, prob.grid, True, True, dims=(1, 1, 1), coord=(0, 0, 0),
                         lo=(0, 0, 0), hi=(24, 20, 28), ext=((True, True),) * 3)
        DistHalo(periodic_x=True, device="cuda", periodic=(True, True, True)).attach(integ, spec)
        integ.upload(prob.q)
        integ.apply_boundary_condition()
        got_dts = []
        for _ in range(3):
            dt = integ.cfl()
            integ.update(dt)
            got_dts.append(dt)
        got = integ.download()[(slice(None),) + prob.grid.interior]
        integ.close()
        assert got_dts == dts
        assert np.array_equal(got, ref)
    finally:
        dist.destroy_process_group()


def test_halo3_callback_error_stops_the_step():
    """An exchange callback that fails on the k faces stops the step with
    MISO_B200_ERR_HALO (the error is reported, nothing aborts); the i and j
    exchanges before it went through the same callback."""
    import ctypes

    from miso_b200 import _lib
    prob = P.turbulence(16, seed=2)
    calls = []

    def exchange(user, axis, n, nbytes, ext_lo, ext_hi, slo, shi, rlo, rhi, stream):
        calls.append(axis)
        return 1 if axis == 2 else 0
    with Integrator(prob.config, prob.grid, precision="fp32_split") as integ:
        fn = _lib.HALO3_EXCHANGE_FN(exchange)
        ops = _lib.Halo3Ops(fn, _lib.HALO_MIN_FN(0), None)
        ext = (ctypes.c_int * 6)(1, 1, 1, 1, 1, 1)
        assert integ._lib.miso_b200_set_halo3(integ._h, ext, ctypes.byref(ops)) == _lib.OK
        integ.upload(prob.q)
        with pytest.raises(_lib.MisoError) as e:
            integ.apply_boundary_condition()
        assert e.value.code == _lib.ERR_HALO
        assert calls == [0, 1, 2]
        # back to a single grid
        assert integ._lib.miso_b200_set_halo3(integ._h, None, None) == _lib.OK
        integ.upload(prob.q)
        integ.apply_boundary_condition()
        integ.update(integ.cfl())
