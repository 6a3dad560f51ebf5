"""Host logic of the decomposition (miso_b200/shard.py) on CPU: shard
extents and spacings, cutting and gathering states, and the torch.distributed
halo transport run as two and three gloo ranks on host buffers laid out as
the library lays out an array (ghost planes, then interior planes)."""
import ctypes
import json
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from miso_b200 import problems as P  # noqa: E402
from miso_b200.shard import gather, split_grid, split_state  # noqa: E402


def test_split_grid_extents_and_spacing():
    prob = P.turbulence(16, seed=0)
    specs = split_grid(prob.grid, 4, periodic_x=True)
    assert [(s.i0, s.i1) for s in specs] == [(0, 4), (4, 8), (8, 12), (12, 16)]
    for s in specs:
        assert s.grid.dx[0] == prob.grid.dx[0]
        assert s.ext_lo and s.ext_hi
    specs = split_grid(P.blast(16).grid, 2, periodic_x=False)
    assert (specs[0].ext_lo, specs[0].ext_hi, specs[1].ext_lo, specs[1].ext_hi) == \
        (False, True, True, False)
    with pytest.raises(ValueError):
        split_grid(prob.grid, 5, True)  # 16 planes cannot give 5 shards of >= 4


def test_split_state_and_gather_round_trip():
    prob = P.turbulence(16, seed=1)
    specs = split_grid(prob.grid, 2, True)
    parts = [split_state(prob.q, prob.grid, s) for s in specs]
    m = prob.grid.i_margin
    # a shard's ghost planes are the global state's neighbouring planes
    assert np.array_equal(parts[0][:, -m:], prob.q[:, 8 + m:8 + 2 * m])
    assert np.array_equal(parts[1][:, :m], prob.q[:, 8:8 + m])
    assert np.array_equal(gather(parts, specs, prob.grid),
                          prob.q[(slice(None),) + prob.grid.interior])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


N_INT, M, PLANE, NARR = 5, 2, 6, 3


def _rank(rank, world, port, periodic, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    import datetime
    import torch.distributed as dist
    from miso_b200.shard import DistHalo
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    halo = DistHalo(periodic, device="cpu")
    t0 = N_INT + 2 * M
    arrs = []
    for a in range(NARR):
        x = np.full((t0, PLANE), -1.0, dtype=np.float32)
        for i in range(N_INT):  # interior plane i of array a on this rank
            x[M + i] = 1000 * rank + 100 * a + i
        arrs.append(x)
    el = 4
    nbytes = M * PLANE * el
    base = [x.ctypes.data for x in arrs]
    slo = [b + M * PLANE * el for b in base]
    shi = [b + N_INT * PLANE * el for b in base]
    rlo = list(base)
    rhi = [b + (N_INT + M) * PLANE * el for b in base]
    ext_lo = periodic or rank > 0
    ext_hi = periodic or rank < world - 1
    halo.exchange(rank, slo, shi, rlo, rhi, nbytes, ext_lo, ext_hi, 0)
    dt = halo.min_all(rank, 0.5 + rank)
    res = {"ghost_lo": [x[:M, 0].tolist() for x in arrs],
           "ghost_hi": [x[N_INT + M:, 0].tolist() for x in arrs], "dt": dt}
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump(res, f)
    dist.destroy_process_group()


@pytest.mark.parametrize("world,periodic", [(2, True), (3, True), (3, False), (1, True)])
def test_dist_halo_pairs_faces(tmp_path, world, periodic):
    import torch.multiprocessing as tmp
    tmp.start_processes(_rank, args=(world, _free_port(), periodic, str(tmp_path)),
                        nprocs=world, join=True, start_method="spawn")
    for r in range(world):
        d = json.load(open(tmp_path / f"r{r}.json"))
        assert d["dt"] == 0.5
        lo = (r - 1) % world if (periodic or r > 0) else None
        hi = (r + 1) % world if (periodic or r < world - 1) else None
        for a in range(NARR):
            # low ghosts = the low neighbour's top interior planes
            want_lo = [-1.0] * M if lo is None else \
                [1000 * lo + 100 * a + i for i in range(N_INT - M, N_INT)]
            want_hi = [-1.0] * M if hi is None else [1000 * hi + 100 * a + i for i in range(M)]
            assert d["ghost_lo"][a] == want_lo, (r, a)
            assert d["ghost_hi"][a] == want_hi, (r, a)


def _rank3(rank, world, port, dims, periodic, out_dir):
    """One rank of a decomposition over i, j and k: along each axis with
    more than one shard it sends face buffers marked with its rank, the
    axis and the side, as the library calls the exchange once per axis."""
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    import datetime
    import torch.distributed as dist
    from miso_b200.shard import DistHalo, _rank_coord
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    halo = DistHalo(periodic[0], device="cpu", dims=dims, periodic=periodic)
    coord = _rank_coord(rank, dims)
    res = {}
    for axis in range(3):
        if dims[axis] == 1:
            continue
        ext_lo = periodic[axis] or coord[axis] > 0
        ext_hi = periodic[axis] or coord[axis] < dims[axis] - 1
        bufs = {k: [np.full(4, -1.0, dtype=np.float32) for _ in range(NARR)]
                for k in ("slo", "shi", "rlo", "rhi")}
        for a in range(NARR):
            bufs["slo"][a][:] = 1000 * rank + 100 * axis + 10 * a
            bufs["shi"][a][:] = 1000 * rank + 100 * axis + 10 * a + 1
        ptr = {k: [x.ctypes.data for x in v] for k, v in bufs.items()}
        halo.exchange(rank, ptr["slo"], ptr["shi"], ptr["rlo"], ptr["rhi"], 16, ext_lo, ext_hi,
                      0, axis=axis)
        res[str(axis)] = {"lo": [float(x[0]) for x in bufs["rlo"]],
                          "hi": [float(x[0]) for x in bufs["rhi"]]}
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump(res, f)
    dist.destroy_process_group()


@pytest.mark.parametrize("dims,periodic", [((1, 2, 2), (False, True, True)),
                                           ((2, 2, 1), (True, False, False)),
                                           ((1, 1, 3), (False, False, True))],
                         ids=["j2k2_periodic", "i2j2_mixed", "k3_periodic"])
def test_dist_halo_pairs_faces_per_axis(tmp_path, dims, periodic):
    """The per-axis exchange of a decomposition along j and k: along each
    axis a rank's low ghosts come from the high face of its low neighbour
    (the rank one coordinate below, across the wrap on a periodic axis) and
    its high ghosts from the low face of its high neighbour; two shards on a
    periodic axis are each other's low and high neighbour."""
    import torch.multiprocessing as tmp
    from miso_b200.shard import _neighbour, _rank_coord
    world = dims[0] * dims[1] * dims[2]
    tmp.start_processes(_rank3, args=(world, _free_port(), dims, periodic, str(tmp_path)),
                        nprocs=world, join=True, start_method="spawn")
    for r in range(world):
        d = json.load(open(tmp_path / f"r{r}.json"))
        coord = _rank_coord(r, dims)
        assert sorted(d) == [str(a) for a in range(3) if dims[a] > 1]
        for axis in range(3):
            if dims[axis] == 1:
                continue
            lo = _neighbour(coord, dims, periodic, axis, -1)
            hi = _neighbour(coord, dims, periodic, axis, +1)
            for a in range(NARR):
                want_lo = -1.0 if lo is None else 1000 * lo + 100 * axis + 10 * a + 1
                want_hi = -1.0 if hi is None else 1000 * hi + 100 * axis + 10 * a
                assert d[str(axis)]["lo"][a] == want_lo, (r, axis, a)
                assert d[str(axis)]["hi"][a] == want_hi, (r, axis, a)


def test_split_grid3_boxes_and_round_trip():
    """The Cartesian decomposition's boxes: ranks in row-major coordinate
    order, the reference's spacing on every shard, shared faces where a
    neighbour or a periodic wrap lies, and cutting then gathering a state
    gives it back."""
    from miso_b200.shard import split_grid3
    prob = P.turbulence(16, seed=1)
    specs = split_grid3(prob.grid, (2, 2, 2), (True, True, True))
    assert [s.coord for s in specs][:4] == [(0, 0, 0), (0, 0, 1), (0, 1, 0), (0, 1, 1)]
    for s in specs:
        assert (s.grid.dx[0], s.grid.dy[0], s.grid.dz[0]) == \
            (prob.grid.dx[0], prob.grid.dy[0], prob.grid.dz[0])
        assert s.ext == ((True, True),) * 3
    parts = [split_state(prob.q, prob.grid, s) for s in specs]
    assert np.array_equal(gather(parts, specs, prob.grid),
                          prob.q[(slice(None),) + prob.grid.interior])
    blast = P.blast(20, seed=2)  # mirror faces; 20 = 6 + 7 + 7 along k
    specs = split_grid3(blast.grid, (1, 2, 3), (False, False, False))
    assert [(s.lo[2], s.hi[2]) for s in specs[:3]] == [(0, 6), (6, 13), (13, 20)]
    assert specs[0].ext == ((False, False), (False, True), (False, True))
    assert specs[4].ext == ((False, False), (True, False), (True, True))
    parts = [split_state(blast.q, blast.grid, s) for s in specs]
    assert np.array_equal(gather(parts, specs, blast.grid),
                          blast.q[(slice(None),) + blast.grid.interior])
    with pytest.raises(ValueError):
        split_grid3(prob.grid, (1, 5, 1), (True, True, True))


def test_bench_box_dims():
    """bench.py --decomp box: N ranks as shards per axis whose product is N,
    the counts as even as N's prime factors allow, z first."""
    from bench import box_dims
    assert [box_dims(n) for n in (1, 2, 4, 8, 12)] == \
        [(1, 1, 1), (1, 1, 2), (1, 2, 2), (2, 2, 2), (2, 2, 3)]
    for n in range(1, 33):
        d = box_dims(n)
        assert d[0] * d[1] * d[2] == n
