"""Autotuner for the 3-D FP32-split kernels.

For one grid shape it times, on the device and on the live state, every
kernel variant of each kernel class -- the Runge-Kutta stage and the x, y
and z viscosity sweeps, each as a tiled kernel (TMA plane tiles, streaming
lines, warp-shuffle rows) or a flat one (one thread per cell), and for the
Runge-Kutta stage also the pipelined plane kernel -- and a few
work-item lengths along the march axis, and keeps the fastest of each.
Where the pipelined RK stage and the line x sweep win, it also times the
pipelined stage with its last update deferred into the x sweep (RK variant
3), which moves work from one class to the other, on the whole step, and
then the y and z sweeps fused into one pass (y variant 3), also on the whole
step.
Results are cached in a JSON file keyed by precision, grid shape and SM
count ($MISO_B200_TUNE_CACHE, default ~/.cache/miso_b200/tune.json), so a
later run of the same shape skips the search.

Timing runs whole steps, so the state advances by the steps tuned; tune
before the run it is meant for (bench.py tunes during its warm-up).
"""
from __future__ import annotations

import json
import os

CLASSES = {"rk_stage": 0, "av_x": 1, "av_y": 2, "av_z": 3}
# variants per class: 0 tiled, 1 flat, 2 pipelined (RK: planes with packed
# differences; x / y sweeps: one warp per line segment marching along the
# axis; z sweep: rows streamed by TMA); RK 3: variant 2 with the last stage's update deferred into the x
# sweep (compared on the whole step, not per class); y 3: the y and z sweeps
# fused into one pass (the z variant then unused; also on the whole step)
VARIANTS = {"rk_stage": (0, 1, 2, 3), "av_x": (0, 1, 2), "av_y": (0, 1, 2, 3), "av_z": (0, 1, 2)}
PER_CLASS = {"rk_stage": (0, 1, 2), "av_x": (0, 1, 2), "av_y": (0, 1, 2), "av_z": (0, 1, 2)}
CHUNKS = (32, 64, 128)


def cache_path() -> str:
    return os.environ.get("MISO_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "miso_b200",
                                       "tune.json"))


def _key(integ) -> str:
    import torch
    g = integ.grid
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    src = (integ.config.get("source") or {}).get("kind", "none")
    tag = "" if src == "none" else f":{src}"
    return f"{integ.precision}:{g.i_size}x{g.j_size}x{g.k_size}:sm{sms}{tag}"


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save(cache):
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    except OSError:
        pass


def _times(integ, steps):
    integ.run(1, graph=False)
    integ.sync()
    integ.set_timing(True)
    integ.run(steps, graph=False)
    rep = integ.timing_report()
    integ.set_timing(False)
    return {k: v["ms"] / v["launches"] for k, v in rep.items()}


def _step_ms(t: dict) -> float:
    return (t.get("rk_stage", 0) * 4 + t.get("av_x", 0) + t.get("av_y", 0) +
            t.get("av_z", 0) + t.get("av_yz", 0))


def _try_variant(integ, kc: int, var: int) -> bool:
    """Set a variant; False where the handle refuses it (a source term
    pins the RK stage to variants 2 and 3)."""
    from . import _lib
    try:
        integ.set_variant(kc, var)
        return True
    except _lib.MisoError as exc:
        if exc.code == _lib.ERR_STATE:
            return False
        raise


def apply(integ, choice: dict):
    for name, kc in CLASSES.items():
        integ.set_variant(kc, int(choice[name]))
    integ.set_chunks(int(choice["rk_chunk"]), int(choice["av_chunk"]))


def autotune(integ, steps: int = 2, use_cache: bool = True) -> dict:
    """Pick and apply the fastest kernel variants for `integ` (a 3-D
    FP32-split Integrator); returns the choice with the per-class times."""
    if integ.get_variant(0) < 0:
        return {}  # grid served by the per-cell kernels only
    cache = _load() if use_cache else {}
    key = _key(integ)
    if key in cache:
        apply(integ, cache[key])
        return dict(cache[key], cached=True)
    best = {}
    for var in range(max(len(v) for v in PER_CLASS.values())):
        live = {name for name, kc in CLASSES.items()
                if var in PER_CLASS[name] and _try_variant(integ, kc, var)}
        for name, ms in _times(integ, steps).items():
            if name in live and (name not in best or ms < best[name][1]):
                best[name] = (var, ms)
    choice = {name: v for name, (v, _) in best.items()}
    for name, kc in CLASSES.items():
        integ.set_variant(kc, choice[name])
    if choice["rk_stage"] == 2 and choice["av_x"] == 0 and 1 not in (choice["av_y"],
                                                                      choice["av_z"]):
        # the deferred last stage: cheaper RK stages, a dearer x sweep
        t2 = _times(integ, steps)
        integ.set_variant(0, 3)
        t3 = _times(integ, steps)
        if _step_ms(t3) < _step_ms(t2):
            choice["rk_stage"] = 3
            best["rk_stage"] = (3, t3["rk_stage"])
            best["av_x"] = (0, t3["av_x"])
        else:
            integ.set_variant(0, 2)
    if choice["av_y"] != 1 and choice["av_z"] != 1:
        # the y and z sweeps in one pass: one write and one read of the state
        # fewer, both sweeps' arithmetic in one kernel
        t_sep = _times(integ, steps)
        integ.set_variant(2, 3)
        t_fused = _times(integ, steps)
        if _step_ms(t_fused) < _step_ms(t_sep):
            choice["av_y"] = 3
            best["av_y"] = (3, t_fused["av_yz"])
            best.pop("av_z", None)
        else:
            integ.set_variant(2, choice["av_y"])
    # work-item lengths for the winning variants
    chunk_best = None
    for rk_chunk in CHUNKS:
        for av_chunk in CHUNKS:
            integ.set_chunks(rk_chunk, av_chunk)
            t = _times(integ, 1)
            total = _step_ms(t)
            if chunk_best is None or total < chunk_best[0]:
                chunk_best = (total, rk_chunk, av_chunk)
    choice["rk_chunk"], choice["av_chunk"] = chunk_best[1], chunk_best[2]
    choice["ms"] = {name: ms for name, (_, ms) in best.items()}
    apply(integ, choice)
    cache[key] = choice
    if use_cache:
        _save(cache)
    return choice


# ---------------------------------------------------------------------------
# Batched solver: work-item lengths of the 3-D instances' pipelined kernels
# ---------------------------------------------------------------------------
BATCH_CHUNKS = ((64, 128), (32, 64), (16, 32), (16, 16), (8, 16))
# (RK stage, x sweep, y sweep) variants tried with each chunk pair: the
# default (deferred last stage, line x sweep, the y and z sweeps in one
# pass); the same with the separate sweeps; the warp-march x / y sweeps,
# whose 32-cell segments fit grids narrower than a line's 128-cell k block
BATCH_VARIANTS = ((3, 0, 3), (3, 0, 0), (2, 2, 2), (3, 0, 2))


def _batch_key(batch) -> str:
    import torch
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    shapes = {}
    for p in batch.problems:
        g = p.grid
        k = f"{g.i_size}x{g.j_size}x{g.k_size}"
        shapes[k] = shapes.get(k, 0) + 1
    comp = ",".join(f"{n}*{k}" for k, n in sorted(shapes.items()))
    return f"batch:{batch.precision}:{comp}:sm{sms}"


def _apply_batch(batch, c: dict):
    vr, vx, vy = c.get("variants", (3, 0, 3))
    batch.set_variant(1, vx)
    batch.set_variant(2, vy)
    batch.set_variant(0, vr)
    batch.set_chunks(c["rk_chunk"], c["av_chunk"])


def autotune_batch(batch, steps: int = 4, use_cache: bool = True) -> dict:
    """Pick and apply the work-item lengths (Runge-Kutta, x / y sweep
    chunks) of a batch's 3-D instances by timing whole graph-replayed steps
    of the batch itself (CUDA events); cached per batch composition (the
    count of each grid shape), precision and SM count.  Short items keep
    more small grids in flight at once; long ones spend less on halo
    planes.  The state advances by the steps timed."""
    import torch
    if batch.views() == 0:
        return {}
    steps += steps & 1  # whole replays of a two-step graph: no eager step timed
    key = _batch_key(batch)
    cache = _load() if use_cache else {}
    if key in cache:
        c = cache[key]
        _apply_batch(batch, c)
        return c
    import time
    # events on the batch's own stream when the caller gave it one, else the
    # host's clock around the synchronised steps
    stream = torch.cuda.ExternalStream(batch.stream) if batch.stream else None
    best = None
    times = {}
    for (vr, vx, vy), (rk_chunk, av_chunk) in [(v, c) for v in BATCH_VARIANTS
                                               for c in BATCH_CHUNKS]:
        batch.set_variant(1, vx)
        batch.set_variant(2, vy)
        batch.set_variant(0, vr)
        batch.set_chunks(rk_chunk, av_chunk)
        batch.run(2, graph=True)  # capture (and warm) outside the timing
        batch.sync()
        torch.cuda.synchronize()
        if stream is not None:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            batch.run(steps, graph=True)
            e1.record(stream)
            batch.sync()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
        else:
            t0 = time.perf_counter()
            batch.run(steps, graph=True)
            batch.sync()
            ms = (time.perf_counter() - t0) * 1e3 / steps
        times[f"{vr}{vx}{vy}:{rk_chunk}/{av_chunk}"] = ms
        if best is None or ms < best[0]:
            best = (ms, rk_chunk, av_chunk, (vr, vx, vy))
    choice = {"rk_chunk": best[1], "av_chunk": best[2], "variants": list(best[3]),
              "ms_per_step": times}
    _apply_batch(batch, choice)
    cache[key] = choice
    if use_cache:
        _save(cache)
    return choice
