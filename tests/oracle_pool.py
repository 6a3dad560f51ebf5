"""Runs the oracle on many problems at once, in spawned worker processes.

TEST INFRASTRUCTURE ONLY.  Each job names a problem constructor of
miso_b200.problems with its keyword arguments, so a worker builds the
initial state itself; it returns the interior of the state after `nsteps`
oracle steps and the time steps taken.  The pool is started with `spawn`,
so no worker inherits a CUDA context from the test process.
"""
from __future__ import annotations

import multiprocessing as mp
import os
from concurrent.futures import ProcessPoolExecutor


def _run_one(job):
    kind, kwargs, nsteps = job
    from miso_b200 import problems as P
    from oracle.oracle import Oracle
    prob = getattr(P, kind)(**kwargs)
    q = prob.q.copy()
    dts = Oracle().run(prob, q, nsteps)
    return q[(slice(None),) + prob.grid.interior], dts


def run_many(jobs, workers: int | None = None):
    """[(interior after nsteps, dts)] for [(constructor, kwargs, nsteps)]."""
    workers = workers or max(1, min(len(jobs), os.cpu_count() or 1))
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_run_one, jobs))
