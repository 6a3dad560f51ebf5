"""Snapshots in the reference's on-disk layout, readable by pymiso unchanged.

A run directory holds (relative to ``save_dir``)::

    config.yaml              Config::save (config.hpp:127-141): the run's
                             configuration with data_type.Endian added
    grid.bin                 Grid::save (grid.hpp:385-422): uint32 element
                             size, then the x, y, z cell-centre coordinates
                             including the margins
    mpi/coords.csv           the Cartesian rank coordinates (mpi_util.hpp:
                             111-126): "rank,x,y,z"
    time/time.<n>.txt        Time::save (time.hpp:68-87): time, n_output,
    time/n_output.txt        n_step; and the latest n_output
    mhd/mhd.<n>.<rank>.bin   Checkpoint::save (mhd_checkpoint.hpp:35-62):
                             uint32 element size, then ro, vx, vy, vz, bx, by,
                             bz, ei, ph over the whole (i_total, j_total,
                             k_total) box, ghosts included

``<n>`` and ``<rank>`` are zero-filled to ``io.n_output_digits`` digits.
A grid decomposed over ranks (``dims`` shards per axis, ranks in
MPI_Cart_create's row-major order) writes the same directory: config.yaml
with the global grid and ``mpi.x_procs / y_procs / z_procs``, grid.bin with
the global coordinates (Grid::save, grid.hpp:385-422) and coords.csv with
every rank's coordinates (written by rank 0), and one mhd file per rank
holding its own box with its ghost layers.
Values are written in the run's Real type (float64 or float32) in the
machine's byte order, as the reference does.  ``Output.save`` copies the
state off the device and writes it; ``Output.save_async`` enqueues the copy
into pinned host memory behind the step that produced the state and writes
the file from a background thread while the simulation goes on.
"""
from __future__ import annotations

import copy
import ctypes
import os
import sys
import threading

import numpy as np
import yaml

from .grid import Grid

FIELDS = ("ro", "vx", "vy", "vz", "bx", "by", "bz", "ei", "ph")


def _zfill(n: int, digits: int) -> str:
    return str(int(n)).zfill(digits)


class Output:
    """One run directory in the reference's layout, as written by one rank:
    ``grid`` is the global grid; a rank of a decomposed grid gives its
    ``rank``, the shards per axis ``dims`` and its own ``box`` (the local
    grid of its snapshots)."""

    def __init__(self, save_dir: str, config: dict, grid: Grid, real=np.float64, rank: int = 0,
                 dims=(1, 1, 1), box: Grid | None = None):
        self.save_dir = save_dir
        self.grid = grid
        self.box = box if box is not None else grid
        self.rank = int(rank)
        self.dims = tuple(int(d) for d in dims)
        self.real = np.dtype(real)
        if self.real not in (np.dtype(np.float64), np.dtype(np.float32)):
            raise ValueError("Real must be float64 or float32")
        cfg = copy.deepcopy(config)
        io = cfg.setdefault("io", {})
        io.setdefault("enabled", True)
        io.setdefault("save_dir", "data/")
        io.setdefault("time_save_dir", "time/")
        io.setdefault("mpi_save_dir", "mpi/")
        io.setdefault("mhd_save_dir", "mhd/")
        io.setdefault("rt_save_dir", "rt/")
        io.setdefault("n_output_digits", 8)
        cfg["grid"] = {"i_size": grid.i_size, "j_size": grid.j_size, "k_size": grid.k_size,
                       "margin": grid.margin, "x_min": grid.x_min, "x_max": grid.x_max,
                       "y_min": grid.y_min, "y_max": grid.y_max, "z_min": grid.z_min,
                       "z_max": grid.z_max}
        cfg["mpi"] = {"x_procs": self.dims[0], "y_procs": self.dims[1],
                      "z_procs": self.dims[2]}
        cfg.setdefault("time", {})
        cfg["data_type"] = {"Endian": "little" if sys.byteorder == "little" else "big"}
        self.config = cfg
        self.digits = int(io["n_output_digits"])
        self.mhd_dir = os.path.join(save_dir, io["mhd_save_dir"])
        self.time_dir = os.path.join(save_dir, io["time_save_dir"])
        self.mpi_dir = os.path.join(save_dir, io["mpi_save_dir"])
        self._threads = []

    # -- run set-up files --------------------------------------------------
    def write_setup(self):
        """config.yaml, grid.bin and mpi/coords.csv (written once per run,
        by rank 0)."""
        for d in (self.save_dir, self.mhd_dir, self.time_dir, self.mpi_dir):
            os.makedirs(d, exist_ok=True)
        if self.rank != 0:
            return
        with open(os.path.join(self.save_dir, "config.yaml"), "w") as f:
            yaml.safe_dump(_plain(self.config), f, sort_keys=False)
        g = self.grid
        with open(os.path.join(self.save_dir, "grid.bin"), "wb") as f:
            np.array([self.real.itemsize], dtype=np.uint32).tofile(f)
            for s in (g.x, g.y, g.z):
                np.asarray(s, dtype=self.real).tofile(f)
        dx, dy, dz = self.dims
        with open(os.path.join(self.mpi_dir, "coords.csv"), "w") as f:
            f.write("rank,x,y,z\n")
            for r in range(dx * dy * dz):
                f.write(f"{r},{r // (dy * dz)},{(r // dz) % dy},{r % dz}\n")

    # -- snapshots -----------------------------------------------------------
    def mhd_path(self, n_output: int, rank: int | None = None) -> str:
        rank = self.rank if rank is None else rank
        return os.path.join(self.mhd_dir, f"mhd.{_zfill(n_output, self.digits)}."
                                          f"{_zfill(rank, self.digits)}.bin")

    def _write_time(self, time: float, n_output: int, n_step: int):
        if self.rank != 0:
            return  # Time::save writes from the root rank
        with open(os.path.join(self.time_dir, f"time.{_zfill(n_output, self.digits)}.txt"),
                  "w") as f:
            f.write(f"{repr(float(time))}\n{int(n_output)}\n{int(n_step)}\n")
        with open(os.path.join(self.time_dir, "n_output.txt"), "w") as f:
            f.write(f"{int(n_output)}\n")

    def _write_mhd(self, q: np.ndarray, n_output: int):
        with open(self.mhd_path(n_output), "wb") as f:
            np.array([self.real.itemsize], dtype=np.uint32).tofile(f)
            for v in range(9):
                np.ascontiguousarray(q[v], dtype=self.real).tofile(f)

    def save(self, integ, time: float, n_output: int, n_step: int):
        """Snapshot the handle's current state (synchronous)."""
        self._write_mhd(integ.download(), n_output)
        self._write_time(time, n_output, n_step)

    def save_async(self, integ, time: float, n_output: int, n_step: int):
        """Snapshot without stalling the stepping: the device-to-host copy is
        enqueued behind the step that produced the state (into pinned
        memory), and a background thread writes the files once it lands."""
        import torch
        from . import _lib
        from .integrator import _field_ptrs
        buf = torch.empty((9,) + tuple(self.box.shape), dtype=torch.float64, pin_memory=True)
        ev = torch.cuda.Event()
        ev.record()  # creates the event; the library re-records it on its stream
        rc = integ._lib.miso_b200_download_async(integ._h, _field_ptrs(buf),
                                                 ctypes.c_void_p(ev.cuda_event))
        _lib.check(rc, integ._h)

        def work():
            ev.synchronize()
            self._write_mhd(buf.numpy(), n_output)
            self._write_time(time, n_output, n_step)

        th = threading.Thread(target=work, daemon=True)
        th.start()
        self._threads.append(th)
        return th

    def wait(self):
        """Wait for every pending asynchronous snapshot."""
        for th in self._threads:
            th.join()
        self._threads.clear()

    # -- restart ---------------------------------------------------------------
    def load(self, n_output: int, rank: int | None = None, shape=None) -> np.ndarray:
        """The 9 primitive fields of this rank's (or ``rank``'s, with its
        box ``shape``) snapshot n_output as a (9, I, J, K) float64 array
        (Checkpoint::load, mhd_checkpoint.hpp:65-95)."""
        with open(self.mhd_path(n_output, rank), "rb") as f:
            elem = int(np.fromfile(f, dtype=np.uint32, count=1)[0])
            if elem not in (4, 8):
                raise ValueError(f"unexpected element size {elem}")
            dt = np.float64 if elem == 8 else np.float32
            shape = tuple(shape) if shape is not None else tuple(self.box.shape)
            data = np.fromfile(f, dtype=dt, count=9 * int(np.prod(shape)))
        return data.reshape((9,) + shape).astype(np.float64)

    def load_global(self, n_output: int) -> np.ndarray:
        """The global interior (9, nI, nJ, nK) of snapshot n_output of a
        decomposed run, assembled from every rank's file by the coordinates
        in coords.csv (boxes of equal size, as the reference cuts them,
        grid.hpp:279-313)."""
        g = self.grid
        sizes = (g.i_size, g.j_size, g.k_size)
        margins = (g.i_margin, g.j_margin, g.k_margin)
        local = [sizes[a] // self.dims[a] for a in range(3)]
        out = np.empty((9,) + tuple(sizes))
        with open(os.path.join(self.mpi_dir, "coords.csv")) as f:
            rows = [line.strip().split(",") for line in f.readlines()[1:] if line.strip()]
        for r, cx, cy, cz in ((int(a), int(b), int(c), int(d)) for a, b, c, d in rows):
            c = (cx, cy, cz)
            shape = tuple(local[a] + 2 * margins[a] for a in range(3))
            q = self.load(n_output, r, shape)
            inner = tuple(slice(margins[a], margins[a] + local[a]) for a in range(3))
            dst = tuple(slice(c[a] * local[a], (c[a] + 1) * local[a]) for a in range(3))
            out[(slice(None),) + dst] = q[(slice(None),) + inner]
        return out

    def load_time(self, n_output: int):
        with open(os.path.join(self.time_dir, f"time.{_zfill(n_output, self.digits)}.txt")) as f:
            return float(f.readline()), int(f.readline()), int(f.readline())


def _plain(obj):
    """Plain Python containers for yaml.safe_dump (numpy scalars, tuples)."""
    if isinstance(obj, dict):
        return {str(k): _plain(v) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return [_plain(v) for v in obj]
    if isinstance(obj, np.generic):
        return obj.item()
    return obj
