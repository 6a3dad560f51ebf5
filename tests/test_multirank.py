"""Host logic of bench.py's multi-rank path, as world-size-2 gloo ranks on
CPU: the process group comes up from the torchrun environment, the timing
reduction gives every rank the maximum over ranks, barriers pass, the
reference arm prints from rank 0 only, and the batched workloads give each
rank its own instance list."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import bench
    import torch.distributed as dist
    r, w, local = bench.dist_init(backend="gloo", timeout_s=60)
    bench.barrier(w)
    worst = bench.max_over_ranks(1.5 + r, w)
    bench.barrier(w)
    from miso_b200 import problems as P
    sizes = [int(p.grid.i_size) for p in P.brio_wu_batch(6, seed=r)]
    with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
        json.dump({"rank": r, "world": w, "local": local, "max": worst, "sizes": sizes}, f)
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_max_and_split_work(tmp_path):
    import torch.multiprocessing as tmp
    port = _free_port()
    tmp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                        start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    for r, d in enumerate(res):
        assert d["rank"] == r and d["world"] == 2 and d["local"] == r
        assert d["max"] == 2.5  # max over ranks of 1.5 + rank, on every rank
    # each rank advances its own seeded instance list (weak scaling)
    assert res[0]["sizes"] != res[1]["sizes"]


def test_reference_arm_prints_on_rank0_only(tmp_path):
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0"], env=env, capture_output=True,
                         text=True, timeout=120)
    assert out.returncode == 0
    assert out.stdout.strip() == ""
