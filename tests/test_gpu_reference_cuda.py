"""The reference's own CUDA integrator (oracle/_ref/miso_ref_cuda_f64 / _f32,
built from mhd_integrator_cuda.cuh by oracle/Makefile) on the B200: its FP64
result against this library's FP64 result on the same initial data, and its
throughput beside this library's on the same grid (printed as JSON lines;
the reference's GPU path is a measured baseline, not a target).

The reference's CUDA kernels are compiled with nvcc's default fused
multiply-add, so they agree with the host path (and with this library's
FP64 form, which is bit-exact with the host path) to round-off, not bit for
bit: relative L1 <= 1e-9 is required.
"""
import json
import os
import subprocess
import time

import numpy as np
import pytest

from conftest import ROOT, interior, rel_l1
from miso_b200 import problems as P

pytestmark = pytest.mark.gpu

BIN = {8: os.path.join(ROOT, "oracle", "_ref", "miso_ref_cuda_f64"),
       4: os.path.join(ROOT, "oracle", "_ref", "miso_ref_cuda_f32")}


def _need(real):
    if not os.path.exists(BIN[real]):
        pytest.skip("reference CUDA build (oracle/_ref) not present")


def write_input(path, prob):
    g, cfg = prob.grid, prob.config
    av = cfg["mhd"]["artificial_viscosity"]
    per = [int(bool(cfg["domain"]["periodic"][a])) for a in ("x", "y", "z")]
    with open(path, "wb") as f:
        np.array([g.i_size, g.j_size, g.k_size, g.margin] + per, dtype=np.int32).tofile(f)
        np.array([g.x_min, g.x_max, g.y_min, g.y_max, g.z_min, g.z_max, cfg["eos"]["gm"],
                  cfg["mhd"]["cfl_number"], av["ep"], av["fh"], av["cs_fac"], av["ca_fac"],
                  av["vv_fac"]], dtype=np.float64).tofile(f)
        np.ascontiguousarray(prob.sign, dtype=np.float64).tofile(f)
        np.ascontiguousarray(prob.q, dtype=np.float64).tofile(f)


def run_reference(tmp_path, prob, real, warm, steps, want_out=True):
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    write_input(inp, prob)
    args = [BIN[real], str(inp), str(warm), str(steps)] + ([str(out)] if want_out else [])
    r = subprocess.run(args, capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0, r.stderr[-2000:]
    rec = json.loads(r.stdout.strip().splitlines()[-1])
    q = np.fromfile(out, dtype=np.float64).reshape(prob.q.shape) if want_out else None
    return rec, q


def run_ours(prob, precision, steps):
    from miso_b200.integrator import Integrator
    integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision=precision)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    for _ in range(steps):
        integ.update(integ.cfl())
    q = integ.download()
    integ.close()
    return q


@pytest.mark.parametrize("make,steps", [(lambda: P.orszag_tang(64), 20),
                                        (lambda: P.turbulence(24, seed=2), 10),
                                        (lambda: P.brio_wu(128), 40)],
                         ids=["ot64", "turb24", "bw128"])
def test_reference_cuda_matches_fp64(tmp_path, make, steps):
    _need(8)
    prob = make()
    rec, q_ref = run_reference(tmp_path, prob, 8, 0, steps)
    assert rec["cuda_error"] == "no error"
    q = run_ours(prob, "fp64", steps)
    a, b = interior(prob, q), interior(prob, q_ref)
    for f in range(9):
        den = float(np.sum(np.abs(b[f])))
        if den > 1e-8 * float(np.sum(np.abs(b[P.RO]))):
            assert rel_l1(a[f], b[f]) <= 1e-9, (P.FIELDS[f], rel_l1(a[f], b[f]))


def _ours_throughput(prob, precision, warm, steps):
    import torch
    from miso_b200.integrator import Integrator
    integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision=precision)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    integ.run(warm, graph=False)
    integ.sync()
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(steps):
        integ.update(integ.cfl())  # the reference's own per-step host round trip
    integ.sync()
    el = time.perf_counter() - t
    integ.close()
    return prob.grid.n_interior * steps / el / 1e9


@pytest.mark.slow
@pytest.mark.parametrize("n", [256, 512])
def test_reference_cuda_throughput(tmp_path, n):
    """Reference CUDA path (FP64 and FP32) vs this library (FP64 and FP32
    split), 3-D turbulence n^3, same cfl -> update(dt) loop; prints one JSON
    line per run."""
    _need(8)
    _need(4)
    prob = P.turbulence(n, seed=0)
    warm, steps = 2, 5
    for real, prec in ((8, "fp64"), (4, "fp32_split")):
        rec, _ = run_reference(tmp_path, prob, real, warm, steps, want_out=False)
        assert rec["cuda_error"] == "no error"
        ours = _ours_throughput(prob, prec, warm, steps)
        print(json.dumps({"workload": f"turbulence {n}^3", "reference_cuda_real_bytes": real,
                          "reference_cuda_gcell_s": rec["gcell_updates_per_s"],
                          "reference_cuda_ms_per_step": rec["ms_per_step"],
                          "miso_b200_precision": prec, "miso_b200_gcell_s": ours,
                          "speedup": ours / rec["gcell_updates_per_s"]}), flush=True)
