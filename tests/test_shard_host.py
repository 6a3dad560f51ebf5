"""Host logic of the i decomposition (miso_b200/shard.py) on CPU: shard
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
