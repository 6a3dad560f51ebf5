"""Many independent grids advanced together (miso_b200_batch_* in the C ABI).

A :class:`Batch` holds any mix of 1-D, 2-D and 3-D problems of uneven sizes
and parameters.  Every pass of a step is one persistent launch over a tile
list of all instances, each instance keeps its own CFL time step, and
``run(n, graph=True)`` replays one captured step.  Each instance follows the
same update as a single :class:`~miso_b200.integrator.Integrator`.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .integrator import _field_ptrs, make_descs


class Batch:
    def __init__(self, problems, precision: str = "fp64", stream: int | None = None):
        lib = _lib.load()
        n = len(problems)
        grids = (_lib.GridDesc * n)()
        params = (_lib.Params * n)()
        for i, p in enumerate(problems):
            gd, pp = make_descs(p.config, p.grid, p.sign, precision)
            grids[i], params[i] = gd, pp
        h = ctypes.c_void_p()
        _lib.check(lib.miso_b200_batch_create(n, grids, params, ctypes.c_void_p(stream or 0),
                                              ctypes.byref(h)), None)
        self._h, self._lib = h, lib
        self.stream = stream  # the cudaStream_t handle given, or None (the library's own)
        self.problems = list(problems)
        self.precision = precision

    def _check(self, code):
        if code != _lib.OK:
            msg = self._lib.miso_b200_batch_last_error(self._h)
            raise _lib.MisoError(code, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.miso_b200_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def upload(self, index: int, q):
        self._check(self._lib.miso_b200_batch_upload(self._h, index, _field_ptrs(q)))

    def upload_all(self):
        for i, p in enumerate(self.problems):
            self.upload(i, p.q)
        self.fill_ghosts()

    def download(self, index: int) -> np.ndarray:
        out = np.empty((9,) + self.problems[index].grid.shape, dtype=np.float64)
        self._check(self._lib.miso_b200_batch_download(self._h, index, _field_ptrs(out)))
        return out

    def fill_ghosts(self):
        self._check(self._lib.miso_b200_batch_fill_ghosts(self._h))

    def run(self, nsteps: int, graph: bool = True):
        self._check(self._lib.miso_b200_batch_run(self._h, int(nsteps), int(bool(graph))))

    def sync(self):
        self._check(self._lib.miso_b200_batch_sync(self._h))

    def dt(self) -> np.ndarray:
        out = np.empty(len(self.problems))
        self._check(self._lib.miso_b200_batch_dt(self._h, out.ctypes.data_as(_lib._dp)))
        return out

    def set_chunks(self, rk_chunk: int, av_chunk: int):
        """Planes per work item of the 3-D instances' pipelined kernels."""
        self._check(self._lib.miso_b200_batch_set_chunks(self._h, int(rk_chunk), int(av_chunk)))

    def set_variant(self, kernel_class: int, variant: int):
        """Kernel variant of the 3-D instances' pipelined path."""
        self._check(self._lib.miso_b200_batch_set_variant(self._h, int(kernel_class),
                                                          int(variant)))

    def views(self) -> int:
        """Instances that run the single grid's pipelined kernels."""
        n = ctypes.c_int()
        self._check(self._lib.miso_b200_batch_views(self._h, ctypes.byref(n)))
        return n.value

    def info(self) -> dict:
        cells, tiles, launches = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_longlong()
        self._check(self._lib.miso_b200_batch_info(self._h, ctypes.byref(cells),
                                                   ctypes.byref(tiles), ctypes.byref(launches)))
        return {"interior_cells": cells.value, "tiles": tiles.value, "launches": launches.value}
