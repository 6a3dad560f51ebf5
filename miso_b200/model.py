"""The reference's run loop for one grid: ModelBase (mhd_model_base.hpp:41-116).

``Model.run()`` is ModelBase::run: apply the initial condition, resume from
the last snapshot when ``io.continue`` is set and one exists, write the run's
set-up files, then step (cfl, update, time += dt: ModelBase::update and
Time::update, time.hpp:64-67) until ``time.tend``, writing a snapshot after
every step at which ``time >= time.dt_output * n_output`` (save_if_needed,
mhd_model_base.hpp:81-87).  Snapshots go to the reference's run-directory
layout through :class:`miso_b200.checkpoint.Output`; they are taken with
``save_async``, so the device-to-host copy of a snapshot overlaps the steps
that follow it.

Configuration keys, as the reference reads them: ``time.tend``,
``time.dt_output``, ``io.enabled``, ``io.continue``, ``io.save_dir``.

A model of a decomposed grid (``shard``, a ShardSpec of miso_b200.shard,
with ``halo``, its LocalHalo or DistHalo) steps its own box of the global
grid -- the halos exchanged after every pass and dt reduced over all ranks,
as the reference's ModelBase does with MPI -- and writes its snapshots in
the reference's multi-rank layout (one mhd file per rank, coords.csv);
``run_local_models`` runs such a decomposition as threads on one GPU.

``run(device_loop=True)`` keeps the steps between two outputs on the device:
one ``Integrator.run_until`` call -- a CUDA graph whose WHILE node runs
steps until the device-held time reaches the next output time or
``time.tend`` -- per output interval.  The steps are the same; dt stays on
the device (the GLM damping factor from the device exp, as
``Integrator.run``), so the FP64 form then agrees with the host loop to
rounding, not bit for bit.
"""
from __future__ import annotations

import os

import numpy as np

from .checkpoint import Output
from .grid import Grid
from .integrator import MHD


class Model:
    """One grid's model: fields, integrator, time and output."""

    def __init__(self, config: dict, grid: Grid, initial_state: np.ndarray, sign=None,
                 precision: str = "fp64", blend=None, shard=None, halo=None, stream=None):
        t = config.get("time") or {}
        if "tend" not in t or "dt_output" not in t:
            raise KeyError("config needs time.tend and time.dt_output")
        self.tend = float(t["tend"])
        self.dt_output = float(t["dt_output"])
        if not (self.tend > 0 and self.dt_output > 0):
            raise ValueError("time.tend and time.dt_output must be > 0")
        io = config.get("io") or {}
        self.io_enabled = bool(io.get("enabled", True))
        self.resume = bool(io.get("continue", False))
        self.config = config
        self.grid = grid
        self.shard = shard
        box = grid
        if shard is not None:
            from .shard import split_state
            if halo is None:
                raise ValueError("a shard needs its halo exchange")
            box = shard.grid
            initial_state = split_state(initial_state, grid, shard)
            if blend is not None:
                blend = split_state(blend, grid, shard)
        self.q0 = initial_state
        self.mhd = MHD(config, box, sign=sign, precision=precision, blend=blend, stream=stream)
        if shard is not None:
            halo.attach(self.mhd.integrator, shard)
        self.output = (Output(io.get("save_dir", "data/"), config, grid,
                              rank=shard.rank if shard is not None else 0,
                              dims=shard.dims if shard is not None else (1, 1, 1), box=box)
                       if self.io_enabled else None)
        # Time::initialize (time.hpp:37-41)
        self.time = 0.0
        self.n_step = 0
        self.n_output = 0

    # -- ModelBase -------------------------------------------------------------
    def update(self) -> float:
        """ModelBase::update: cfl, update, time += dt."""
        dt = self.mhd.cfl()
        self.mhd.update(dt)
        self.time += dt
        self.n_step += 1
        return dt

    def save_state(self):
        if self.output is not None:
            self.output.save_async(self.mhd.integrator, self.time, self.n_output, self.n_step)

    def load_state(self):
        """Time::load and Checkpoint::load of the snapshot named in
        time/n_output.txt (the state is uploaded with its ghost cells, as
        the reference reads them back)."""
        with open(os.path.join(self.output.time_dir, "n_output.txt")) as f:
            n = int(f.readline())
        self.time, self.n_output, self.n_step = self.output.load_time(n)
        self.mhd.integrator.upload(self.output.load(self.n_output))

    def save_if_needed(self):
        if self.time >= self.dt_output * self.n_output:
            self.save_state()
            self.n_output += 1

    def run(self, device_loop: bool = False):
        """ModelBase::run (mhd_model_base.hpp:88-116).  A shard steps from
        the host (its dt is reduced over the ranks)."""
        if device_loop and self.shard is not None:
            raise ValueError("a shard steps from the host: device_loop=False")
        self.mhd.apply_initial_condition(self.q0)
        if (self.resume and self.output is not None and
                os.path.exists(os.path.join(self.output.time_dir, "n_output.txt"))):
            self.load_state()
        if self.output is not None:
            self.output.write_setup()
        self.save_if_needed()
        while self.time < self.tend:
            if device_loop:
                # the steps up to the next output (or the end) in one launch;
                # the loop stops after the step that reaches it, as here
                t_next = min(self.tend, self.dt_output * self.n_output)
                self.time, n = self.mhd.integrator.run_until(self.time, t_next)
                self.n_step += n
            else:
                self.update()
            self.save_if_needed()
        if self.output is not None:
            self.output.wait()

    def state(self) -> np.ndarray:
        return self.mhd.integrator.download()

    def close(self):
        if self.output is not None:
            self.output.wait()
        self.mhd.integrator.close()


def run_local_models(config: dict, grid: Grid, initial_state: np.ndarray, dims, sign=None,
                     precision: str = "fp64", blend=None, stream=None):
    """ModelBase::run of one grid decomposed into dims[0] x dims[1] x dims[2]
    boxes, each a Model on the current GPU driven by its own host thread
    (all on one CUDA stream, the halos moved by device copies: LocalHalo).
    The snapshots land in the reference's multi-rank layout under
    ``io.save_dir``.  Returns the models (closed)."""
    import threading

    import torch

    from .shard import LocalHalo, split_grid3
    per = config["domain"]["periodic"]
    periodic = (bool(per["x"]), bool(per["y"]), bool(per["z"]))
    specs = split_grid3(grid, dims, periodic)
    count = len(specs)
    halo = LocalHalo(count, periodic[0], dims=dims, periodic=periodic)
    keep = None
    if stream is None:
        keep = torch.cuda.Stream()
        stream = keep.cuda_stream
    models = [Model(config, grid, initial_state, sign=sign, precision=precision, blend=blend,
                    shard=s, halo=halo, stream=stream) for s in specs]
    errors = []

    def drive(r):
        try:
            models[r].run()
        except Exception as exc:
            errors.append(exc)
            halo._bar.abort()

    threads = [threading.Thread(target=drive, args=(r,)) for r in range(count)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for m in models:
        m.close()
    if errors:
        raise errors[0]
    return models
