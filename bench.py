#!/usr/bin/env python
"""Throughput benchmark of the MISO MHD time step on B200.

Workload (default): 3-D decaying MHD turbulence, 512^3 interior cells,
periodic, gamma = 5/3, rho = 1, p = 1/gamma, seeded solenoidal v and B with
1 <= |k| <= 4, E(k) ~ k^-2, Mach 0.5, beta 1 -- advanced in the FP32
split-precision form.  One "step" is one full time step of the reference's
ModelBase::update(): CFL reduction, 4 Runge-Kutta stages, 3 artificial-
viscosity sweeps and the ghost fills.  The metric is cell-updates per second
(interior cells x steps / device seconds).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun each rank advances its own grid (independent replicas, weak
scaling; the time is the maximum over ranks).  ``--impl reference`` times
the reference's own CPU integrator (oracle/_ref, built from the MISO
sources) on the host cores instead.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import datetime
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gcell-updates/s/GPU (FP32-split vs FP64) and % HBM roofline at stated L1 err vs FP64"
UNIT = "Gcell-updates/s"
# algorithmic bytes per interior cell per step (canonical 7-pass structure:
# 9 fields, perfect stencil reuse, derived quantities never stored)
ALG_BYTES = {"fp32_split": 912.0, "fp64": 1248.0}
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--n", type=int, default=512, help="interior cells per axis")
    ap.add_argument("--precision", choices=["fp32_split", "fp64"], default="fp32_split")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched workloads reported beside the headline")
    ap.add_argument("--cpu-n", type=int, default=64, help="reference CPU sample grid size per core")
    ap.add_argument("--workload", choices=["turbulence", "brio_wu_batch", "ot_batch",
                                           "turbulence_blast_batch", "turbulence512_ot_batch"],
                    default="turbulence",
                    help="turbulence: one 3-D grid (the headline); the batch workloads run "
                         "many instances through the batched solver")
    ap.add_argument("--count", type=int, default=0, help="instances of a batch workload")
    ap.add_argument("--decomp", choices=["replicas", "slab", "box"], default="replicas",
                    help="turbulence under torchrun: independent n^3 grids per rank "
                         "(replicas), one (n*N) x n x n periodic grid cut into N slabs "
                         "along x (slab), or one periodic grid of N n^3 boxes cut along "
                         "x, y and z (box: N's prime factors shared out over z, y, x), with "
                         "the face halos exchanged over NCCL after every pass")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# peaks, clocks
# ---------------------------------------------------------------------------
def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            v = float(json.load(f)["hbm_gbs"])
        return v, "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi sampling around the timed region: samples every 100 ms,
    each with its timestamp, and keeps those taken between ``mark()`` and
    ``stop()`` (all of them if none falls inside, as for a region shorter
    than the interval)."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.t0 = self.t1 = None
        self.tmp = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.tmp, stderr=subprocess.DEVNULL)
            time.sleep(0.5)  # nvidia-smi's start-up, outside the timed region
        except Exception:
            self.proc = None
        self.mark()

    def mark(self):
        """The timed region starts now."""
        self.t0 = datetime.datetime.now()

    def stop(self):
        self.t1 = datetime.datetime.now()
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)  # the sample that closes the region
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.tmp.flush()
        with open(self.tmp.name) as f:
            rows = [[x.strip() for x in r.strip().split(",")] for r in f if r.strip()]
        os.unlink(self.tmp.name)

        def when(r):
            try:
                return datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f")
            except (ValueError, IndexError):
                return None

        inside = [r for r in rows if when(r) and self.t0 <= when(r) <= self.t1]
        use = inside or rows
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in use:
            try:
                sm.append(float(r[2]))
                smax.append(float(r[3]))
            except (ValueError, IndexError):
                continue
            for nm, val in zip(names, r[6:10]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "samples_in_region": len(inside), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# reference CPU path (oracle/_ref, else the oracle restatement)
# ---------------------------------------------------------------------------
def _cpu_worker(args):
    n, steps, warm, seed = args
    from oracle import oracle as om
    from miso_b200 import problems as P
    lib = om.Reference() if om.reference_available() else om.Oracle()
    prob = P.turbulence(n, seed=seed)
    q = prob.q.copy()
    lib.fill_ghosts(prob, q)
    if warm:
        lib.run(prob, q, warm, fill_first=False)
    t = time.perf_counter()
    lib.run(prob, q, steps, fill_first=False)
    return time.perf_counter() - t


def cpu_reference(n: int, steps: int, warm: int, procs: int):
    """Reference host integrator on `procs` host cores, one independent
    `n`^3 sample per core (the reference is single-threaded per rank)."""
    from oracle import oracle as om
    kind = "reference" if om.reference_available() else "port"
    if procs == 1:
        el = [_cpu_worker((n, steps, warm, 0))]
    else:
        with mp.get_context("spawn").Pool(procs) as pool:
            el = pool.map(_cpu_worker, [(n, steps, warm, r) for r in range(procs)])
    value = procs * n ** 3 * steps / max(el) / 1e9
    return {"value": value, "unit": UNIT, "cores": procs, "kind": kind,
            "sample": f"turbulence {n}^3 FP64, {steps} steps per core after {warm} warm-up, "
                      f"{procs} independent process(es)"}


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def dist_init(backend: str = "nccl", timeout_s: float = 300.0):
    """Rank, world size and local rank from the torchrun environment; joins
    the process group when there is more than one rank (NCCL on the GPU
    box; the multi-rank host logic is tested with gloo on CPU)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local


def max_over_ranks(x: float, world: int) -> float:
    """The maximum of a per-rank time over all ranks (every rank gets it)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_b200(args):
    import numpy as np
    import torch

    from miso_b200 import problems as P
    from miso_b200.integrator import Integrator

    rank, world, local = dist_init()
    torch.cuda.set_device(local)
    n, K, W = args.n, args.steps, args.warmup
    prob = P.turbulence(n, seed=0)
    cells = prob.grid.n_interior
    stream = torch.cuda.Stream()

    def timed_run(integ, steps, graph):
        """Device time of `steps` steps on the library's stream (CUDA events)."""
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        integ.run(steps, graph=graph)
        e1.record(stream)
        torch.cuda.synchronize()
        integ.sync()
        barrier(world)
        return max_over_ranks(e0.elapsed_time(e1), world)

    # ---- split (or chosen) precision: warm-up, timed region, breakdown
    integ = Integrator(prob.config, prob.grid, precision=args.precision,
                       stream=stream.cuda_stream)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    integ.run(W, graph=False)
    integ.sync()
    from miso_b200.autotune import autotune
    tuning = autotune(integ) if args.precision == "fp32_split" else {}
    integ.run(1, graph=False)
    integ.sync()
    # per-kernel breakdown: the same K steps launched one by one, each
    # kernel bracketed by CUDA events on the library stream
    integ.set_timing(True)
    ms_events = timed_run(integ, K, graph=False)
    report = integ.timing_report()
    integ.set_timing(False)

    # the timed region: K steps of the production path, run() replaying the
    # step captured in a CUDA graph (dt stays on the device); a graph holds
    # one or two steps, so K is rounded up to an even count
    Kg = K if K % 2 == 0 else K + 1
    integ.run(2, graph=True)  # capture outside the timed region
    integ.sync()
    sampler = ClockSampler(local)
    l0 = integ.launch_count()
    sampler.start()
    ms = timed_run(integ, Kg, graph=True)
    clocks = sampler.stop()
    launches = integ.launch_count() - l0
    value = world * cells * Kg / (ms / 1e3) / 1e9

    # ---- e2e through the reference-facing API: cfl() -> host dt -> update(dt)
    # -> monitors() (the step's result read back), every step; the monitors'
    # sums ride on each step's last sweep (set_monitor_fusion), so the
    # monitors call adds only the div B reduction
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    fused = False
    if args.precision == "fp32_split":
        try:
            integ.set_monitor_fusion(True)
            fused = True
        except Exception:
            fused = False
    integ.update(integ.cfl())  # one step that leaves the fused sums
    integ.monitors()
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(K):
        dt = integ.cfl()
        integ.update(dt)
        integ.monitors()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    # the monitors' read-back: the last sweep's per-block sums (6 doubles per
    # block of the fused y and z pass, 3 CTAs per SM, or of the z sweep, 8
    # per SM) and the div B march's (8 doubles per block, 2 per SM); the
    # unfused monitor kernel's (8 doubles per block, 4 per SM)
    zparts = (3 if tuning.get("av_y") == 3 else 8) * sms
    d2h_mon = (6 * zparts + 8 * 2 * sms) * 8 if fused else 8 * 4 * sms * 8
    e2e = {"value": world * cells * K / e2e_s / 1e9, "unit": UNIT,
           "h2d_bytes_per_step": 96, "d2h_bytes_per_step": 96 + d2h_mon,
           "monitors_fused": fused,
           "path": "Integrator.cfl() -> update(dt) -> monitors() per step, host dt"}
    if fused:
        integ.set_monitor_fusion(False)
    # ---- the reference's own ModelBase::update (mhd_model_base.hpp:57-62):
    # cfl() -> host dt -> update(dt), no monitors
    integ.update(integ.cfl())
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(K):
        integ.update(integ.cfl())
    torch.cuda.synchronize()
    eu_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e_update = {"value": world * cells * K / eu_s / 1e9, "unit": UNIT,
                  "h2d_bytes_per_step": 96, "d2h_bytes_per_step": 96,
                  "path": "Integrator.cfl() -> update(dt) per step (ModelBase::update), host dt"}

    # ---- the same step with the whole FP64 primitive state crossing PCIe
    # both ways every step (pinned host fields, upload -> cfl -> update ->
    # download): what a caller holding its fields on the host pays per step
    host_fields = None
    try:
        hb = torch.empty((9,) + tuple(prob.grid.shape), dtype=torch.float64, pin_memory=True)
        hbn = hb.numpy()
        integ.download(out=hbn)
        Kh = 2
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(Kh):
            integ.upload(hbn)
            dt = integ.cfl()
            integ.update(dt)
            integ.download(out=hbn)
        torch.cuda.synchronize()
        hs = max_over_ranks(time.perf_counter() - t0, world)
        fb = hbn.nbytes
        host_fields = {"value": world * cells * Kh / hs / 1e9, "unit": UNIT, "steps": Kh,
                       "h2d_bytes_per_step": fb + 96, "d2h_bytes_per_step": fb + 8,
                       "path": "upload(host fp64) -> cfl() -> update(dt) -> download() per step"}
        del hb, hbn
    except Exception as exc:  # pinned host memory may be short on a small host
        host_fields = {"value": None, "unit": UNIT, "skipped": f"{type(exc).__name__}: {exc}"}
    integ.close()

    # ---- FP64 comparison on the same workload (same steps)
    fp64 = None
    if not args.no_fp64 and args.precision != "fp64":
        i64 = Integrator(prob.config, prob.grid, precision="fp64", stream=stream.cuda_stream)
        i64.upload(prob.q)
        i64.apply_boundary_condition()
        i64.run(W, graph=False)
        i64.run(2, graph=True)  # graph capture outside the timed region
        i64.sync()
        ms64 = timed_run(i64, Kg, graph=True)
        v64 = world * cells * Kg / (ms64 / 1e3) / 1e9
        st64 = i64.download()
        i64.close()
        n64 = W + 2 + Kg
        # the same steps in the split form from the same initial state, with
        # the tuned kernel variants (the timed integrator above also
        # advanced through the tuner's steps)
        isp = Integrator(prob.config, prob.grid, precision=args.precision,
                         stream=stream.cuda_stream)
        if tuning:
            from miso_b200.autotune import apply as apply_tuning
            apply_tuning(isp, tuning)
        isp.upload(prob.q)
        isp.apply_boundary_condition()
        isp.run(n64, graph=False)
        isp.sync()
        state_split = isp.download()
        isp.close()
        inner = (slice(None),) + prob.grid.interior
        a, b = state_split[inner], st64[inner]
        gm = prob.config["eos"]["gm"]

        def l1(x, y):
            return float(np.sum(np.abs(x - y)) / np.sum(np.abs(y)))
        fp64 = {"value": v64, "ms_per_step": ms64 / Kg,
                "split_speedup": value / v64,
                "l1_vs_fp64_after_steps": n64,
                "l1_rho": l1(a[P.RO], b[P.RO]),
                "l1_p": l1(a[P.RO] * a[P.EI] * (gm - 1), b[P.RO] * b[P.EI] * (gm - 1)),
                "l1_B": l1(a[P.BX:P.BZ + 1], b[P.BX:P.BZ + 1])}

    # ---- roofline of the dominant kernel
    roofline = roofline_of(report, args.precision, value / world)

    # ---- the batched workloads beside the headline (same box, same run)
    batch = None
    if not args.no_batch:
        single = {"fp32_split": value / world,
                  "fp64": fp64["value"] / world if fp64 else None}
        batch = batch_figures(stream, K, W, single, local, world, rank, prob)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_reference(96, 4, 0, 1)
        except Exception as exc:  # the checker may be absent on a stripped box
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "unavailable",
                   "sample": f"{type(exc).__name__}: {exc}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": Kg,
            "warmup": W, "ms_per_step": ms / Kg, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.precision == "fp32_split" else "f64",
            "data": "synthetic (seeded solenoidal Fourier modes)",
            "config": {"workload": f"3D decaying MHD turbulence {n}^3 periodic, "
                                   f"{args.precision}, gamma 5/3, Mach 0.5, beta 1",
                       "precision": args.precision, "cells_per_gpu": cells,
                       "l2": "inputs larger than L2 (state > 1 GB)",
                       "parallelism": f"replicas x{world}"},
            "timed_path": "Integrator.run(K, graph=True): CUDA-graph replay, dt on the device",
            "ms_per_step_events": ms_events / K,
            "tuning": tuning,
            "gpu_launches": launches,
            "kernels": {k: {"launches": v["launches"], "ms_per_step": v["ms"] / K,
                            "GBps": v["bytes"] / (v["ms"] / 1e3) / 1e9 if v["ms"] else None}
                        for k, v in report.items()},
            "roofline": roofline, "e2e": e2e, "e2e_model_update": e2e_update,
            "e2e_host_fields": host_fields, "fp64": fp64, "cpu_baseline": cpu,
            "clocks": clocks, "batch": batch,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def roofline_of(report: dict, precision: str, value_per_gpu: float) -> dict:
    """Roofline of the dominant kernel of a per-kernel timing report."""
    peak, peak_src = hbm_peak()
    dname, d = max(report.items(), key=lambda kv: kv[1]["ms"])
    achieved = (d["bytes"] / d["launches"]) / (d["ms"] / d["launches"] / 1e3) / 1e9
    traffic = step_dram = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            with open(tpath) as f:
                tj = json.load(f)
            traffic = tj.get(f"{precision}:{dname}")
            step_dram = tj.get(f"{precision}:step_per_cell")
        except Exception:
            traffic = step_dram = None
    out = {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": peak,
           "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_src,
           "traffic": traffic, "step_frac": value_per_gpu * ALG_BYTES[precision] / peak,
           "alg_bytes_per_cell_step": ALG_BYTES[precision]}
    if step_dram:
        # the step fuses passes of the canonical structure (the last RK
        # update rides on the x sweep), so its DRAM bytes per cell, measured
        # by ncu, go beside the canonical fraction
        out["step_dram_bytes_per_cell"] = step_dram
        out["step_dram_frac"] = value_per_gpu * step_dram / peak
    return out


def box_dims(world):
    """Shards per axis (x, y, z) for N ranks: N's prime factors, largest
    first, each to the axis that has the fewest shards so far (z, then y,
    then x on a tie)."""
    f, n, p = [], world, 2
    while n > 1:
        while n % p == 0:
            f.append(p)
            n //= p
        p += 1
    dims = [1, 1, 1]
    for q in sorted(f, reverse=True):
        a = min((2, 1, 0), key=lambda ax: dims[ax])
        dims[a] *= q
    return tuple(dims)


def run_slab(args):
    """One periodic grid of (n * N) x n x n cells over N GPUs, cut into N
    slabs along x (miso_b200.shard): every pass's i ghost planes travel to
    the neighbouring ranks by NCCL point-to-point copies, dt is reduced by
    an all-reduce of the minimum, and a step is the reference's host-dt
    sequence cfl() -> update(dt).  Every slab holds the unit cube's
    turbulence field (its Fourier modes have period 1 in x, so the stacked
    field is the periodic field of the long box).  Weak scaling: n^3 cells
    per GPU.  With --decomp box the N cubes are stacked along x, y and z
    (box_dims) and the j and k faces travel too, packed by the library."""
    import torch

    from miso_b200 import problems as P
    from miso_b200.integrator import Integrator
    from miso_b200.shard import DistHalo, ShardSpec

    rank, world, local = dist_init()
    torch.cuda.set_device(local)
    n, K, W = args.n, args.steps, args.warmup
    prob = P.turbulence(n, seed=0)
    cells = prob.grid.n_interior
    stream = torch.cuda.Stream()
    integ = Integrator(prob.config, prob.grid, precision=args.precision,
                       stream=stream.cuda_stream)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    tuning = {}
    if args.precision == "fp32_split":
        from miso_b200.autotune import autotune
        tuning = autotune(integ)  # the tuner steps with run(): before the halo is attached
        integ.upload(prob.q)
    box = args.decomp == "box"
    dims = box_dims(world) if box else (world, 1, 1)
    if world > 1:
        coord = (rank // (dims[1] * dims[2]), (rank // dims[2]) % dims[1], rank % dims[2])
        ext = tuple((dims[a] > 1, dims[a] > 1) for a in range(3))
        spec = ShardSpec(rank, world, 0, n, prob.grid, ext[0][0], ext[0][1], dims=dims,
                         coord=coord, lo=tuple(c * n for c in coord),
                         hi=tuple((c + 1) * n for c in coord), ext=ext)
        DistHalo(periodic_x=True, device="cuda", dims=dims,
                 periodic=(True, True, True)).attach(integ, spec)
    integ.apply_boundary_condition()

    def steps(k):
        for _ in range(k):
            integ.update(integ.cfl())

    steps(W)
    integ.sync()
    integ.set_timing(True)
    steps(2)
    integ.sync()
    report = integ.timing_report()
    integ.set_timing(False)
    barrier(world)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    l0 = integ.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    sampler.start()
    e0.record(stream)
    steps(K)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = integ.launch_count() - l0
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    value = world * cells * K / (ms / 1e3) / 1e9
    # e2e: the same host-dt steps with the step's monitors read back
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(K):
        integ.update(integ.cfl())
        integ.monitors()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    e2e = {"value": world * cells * K / e2e_s / 1e9, "unit": UNIT,
           "h2d_bytes_per_step": 96, "d2h_bytes_per_step": 8 + 8 * 8 * 2 * sms,
           "path": "Integrator.cfl() (dt all-reduced) -> update(dt) -> monitors() per step"}
    integ.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.precision == "fp32_split" else "f64",
            "data": "synthetic (seeded solenoidal Fourier modes)",
            "config": {"workload": (f"3D decaying MHD turbulence ({n}*{dims[0]})x({n}*{dims[1]})"
                                    f"x({n}*{dims[2]}) periodic, one grid in "
                                    f"{dims[0]}x{dims[1]}x{dims[2]} boxes, {args.precision}"
                                    if box else
                                    f"3D decaying MHD turbulence ({n}*{world})x{n}x{n} periodic, "
                                    f"one grid in {world} slabs along x, {args.precision}"),
                       "precision": args.precision, "cells_per_gpu": cells,
                       "l2": "inputs larger than L2 (state > 1 GB)",
                       "parallelism": (f"box {dims[0]}x{dims[1]}x{dims[2]}" if box
                                       else f"slab x{world}") + " (NCCL halo exchange)"},
            "timed_path": "Integrator.cfl() -> update(dt) per step, dt all-reduced over ranks",
            "tuning": tuning, "gpu_launches": launches,
            "kernels": {k: {"launches": v["launches"], "ms_per_step": v["ms"] / 2}
                        for k, v in report.items()},
            "roofline": roofline_of(report, args.precision, value / world), "e2e": e2e,
            "cpu_baseline": None, "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def time_batch(probs, precision, stream, K, W, local, world):
    """Device time of K graph-replayed steps of one batch (CUDA events on the
    batch's stream, max over ranks), with the clocks sampled meanwhile."""
    import torch

    from miso_b200.autotune import autotune_batch
    from miso_b200.batch import Batch
    with Batch(probs, precision, stream=stream.cuda_stream) as b:
        b.upload_all()
        b.run(W, graph=True)
        b.sync()
        tuning = autotune_batch(b) if b.views() else {}
        # a captured step graph holds two steps where a step swaps the hi / lo
        # sets: two graph steps here leave the graph matching the state, so
        # nothing is captured inside the timed region
        b.run(2, graph=True)
        b.sync()
        K = K + (K & 1)
        info = b.info()
        cells, l0 = info["interior_cells"], info["launches"]
        sampler = ClockSampler(local)
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        sampler.start()
        e0.record(stream)
        b.run(K, graph=True)
        e1.record(stream)
        torch.cuda.synchronize()
        clocks = sampler.stop()
        b.sync()
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        launches = b.info()["launches"] - l0
    return {"value": world * cells * K / (ms / 1e3) / 1e9, "ms_per_step": ms / K,
            "interior_cells": cells, "instances": len(probs), "gpu_launches": launches,
            "tuning": tuning, "clocks": clocks}


def batch_figures(stream, K, W, single, local, world, rank, big=None):
    """Brio-Wu x4096 (sizes U{512..8192}, left / right values scaled by
    U[0.8, 1.2]) and Orszag-Tang x32 (sizes U{128..1024}^2), each in the
    split form and in FP64; in the split form also 3-D grids of uneven
    sizes (24 turbulence 64^3 + 16 blast 48^3) and the headline's grid
    (`big`, 512^3 turbulence) in one batch with the 32 Orszag-Tang grids.
    Gcell-updates/s and the fraction of the single-grid value per GPU of the
    same form (`single`)."""
    from miso_b200 import problems as P
    out = {}
    mixes = [("turbulence64_x24_blast48_x16",
              lambda: [P.turbulence(64, seed=rank * 64 + s) for s in range(24)] +
              [P.blast(48, seed=rank * 64 + s) for s in range(16)])]
    if big is not None:
        mixes.append(("turbulence512_with_orszag_tang_x32",
                      lambda: [big] + P.orszag_tang_batch(32, 128, 1024, seed=rank)))
    for name, make in mixes:
        probs = make()
        r = time_batch(probs, "fp32_split", stream, K, W, local, world)
        r["frac_of_single_grid"] = r["value"] / world / single["fp32_split"]
        out[name] = {"fp32_split": r}
        del probs
    for name, make in (("brio_wu_x4096", lambda: P.brio_wu_batch(4096, 512, 8192, seed=rank)),
                       ("orszag_tang_x32", lambda: P.orszag_tang_batch(32, 128, 1024, seed=rank))):
        probs = make()
        entry = {}
        for precision in ("fp32_split", "fp64"):
            r = time_batch(probs, precision, stream, K, W, local, world)
            if single.get(precision):
                r["frac_of_single_grid"] = r["value"] / world / single[precision]
            entry[precision] = r
        out[name] = entry
        del probs
    return out


def run_batch(args):
    """Batched workloads: Brio-Wu x4096 (sizes U{512..8192}, values scaled
    U[0.8, 1.2]) or 32 Orszag-Tang grids of sizes U{128..1024}^2."""
    import torch

    from miso_b200 import problems as P
    from miso_b200.batch import Batch

    rank, world, local = dist_init()
    torch.cuda.set_device(local)
    if args.workload == "brio_wu_batch":
        probs = P.brio_wu_batch(args.count or 4096, seed=rank)
    elif args.workload == "ot_batch":
        probs = P.orszag_tang_batch(args.count or 32, seed=rank)
    elif args.workload == "turbulence_blast_batch":
        # 3-D grids of uneven sizes: 24 turbulence 64^3 + 16 blast 48^3
        probs = ([P.turbulence(64, seed=rank * 64 + s) for s in range(24)] +
                 [P.blast(48, seed=rank * 64 + s) for s in range(16)])
    else:
        # the 512^3 turbulence grid in one batch with 32 Orszag-Tang grids
        probs = [P.turbulence(args.n, seed=rank)] + P.orszag_tang_batch(32, seed=rank)
    K, W = args.steps, args.warmup
    stream = torch.cuda.Stream()
    with Batch(probs, args.precision, stream=stream.cuda_stream) as b:
        b.upload_all()
        b.run(W, graph=True)
        b.sync()
        from miso_b200.autotune import autotune_batch
        tuning = autotune_batch(b) if b.views() else {}
        b.run(2, graph=True)  # the captured graph matches the state's hi / lo set
        b.sync()
        K = K + (K & 1)
        cells = b.info()["interior_cells"]
        l0 = b.info()["launches"]
        sampler = ClockSampler(local)
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        sampler.start()
        e0.record(stream)
        b.run(K, graph=True)
        e1.record(stream)
        torch.cuda.synchronize()
        clocks = sampler.stop()
        b.sync()
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        launches = b.info()["launches"] - l0
    value = world * cells * K / (ms / 1e3) / 1e9
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.precision == "fp32_split" else "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": args.workload, "instances": len(probs),
                       "interior_cells": cells, "precision": args.precision,
                       "launch": "one persistent launch per pass, CUDA graph per step"},
            "gpu_launches": launches, "tuning": tuning, "clocks": clocks}), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    procs = os.cpu_count() or 1
    n = args.cpu_n
    res = cpu_reference(n, args.steps, args.warmup, procs)
    line = {"impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded solenoidal Fourier modes)",
            "config": {"workload": f"3D decaying MHD turbulence {args.n}^3 periodic "
                                   f"(CPU sample {n}^3 per core)",
                       "precision": "fp64 (reference host path)"},
            "cpu_baseline": res,
            "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload != "turbulence":
        run_batch(args)
    elif args.decomp in ("slab", "box"):
        run_slab(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
