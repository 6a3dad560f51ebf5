"""A grid decomposed into shards, one Integrator per shard.

The reference runs one grid over many GPUs by Cartesian domain
decomposition (miso/include/miso/grid.hpp:279-313): every rank owns a box
of the global grid and, after each pass, swaps face halos with its
neighbours (HaloExchanger, mhd_halo_exchange.hpp:451-621); the CFL time
step is reduced over all ranks (mhd_integrator_cuda.cuh:476).  A
decomposition along i alone (``split_grid``) cuts slabs whose face halo is
``margin`` whole planes of each array, contiguous in memory: the library
hands the plane ranges to an exchange callback (``miso_b200_set_halo``) and
nothing is packed.  The full decomposition over i, j and k
(``split_grid3``, ranks in the row-major order of their coordinates, as
MPI_Cart_create numbers them, mpi_util.hpp:69-102) goes through
``miso_b200_set_halo3``, whose callback is called per axis; the library
packs the j and k faces into contiguous buffers around it.  Two
transports implement the callbacks:

* ``LocalHalo``: shards of one process on one GPU, each driven by its own
  host thread, all on one CUDA stream; the planes move by device copies.
  This is how a decomposition is checked against the single grid on one
  GPU.
* ``DistHalo``: one shard per rank of a ``torch.distributed`` process
  group -- NCCL point-to-point sends and receives on the library's stream
  across GPUs, or gloo on CPU buffers for testing the pairing logic.

A face of the global grid that is periodic joins the first and the last
shard; a mirror face stays a mirror face of the outermost shard.
"""
from __future__ import annotations

import ctypes
import dataclasses
import threading

import numpy as np

from .grid import Grid
from .integrator import Integrator

__all__ = ["ShardSpec", "split_grid", "split_grid3", "split_state", "gather", "LocalHalo",
           "DistHalo", "run_local_shards"]


@dataclasses.dataclass
class ShardSpec:
    """Shard r of a decomposed grid: interior planes [i0, i1) of the global
    grid and which i faces it shares with a neighbour; for a decomposition
    along j or k as well, its coordinate and the shard counts per axis
    (``coord``, ``dims``), its interior box [lo, hi) per axis and its shared
    faces ``ext[axis] = (low, high)`` (for a split along i alone these
    follow from the i fields)."""
    rank: int
    count: int
    i0: int
    i1: int
    grid: Grid
    ext_lo: bool
    ext_hi: bool
    dims: tuple = None
    coord: tuple = None
    lo: tuple = None
    hi: tuple = None
    ext: tuple = None

    def __post_init__(self):
        if self.dims is None:
            self.dims = (self.count, 1, 1)
            self.coord = (self.rank, 0, 0)
            self.lo = (self.i0, 0, 0)
            self.hi = (self.i1, self.grid.j_size, self.grid.k_size)
            self.ext = ((bool(self.ext_lo), bool(self.ext_hi)), (False, False), (False, False))

    @property
    def axes3(self) -> bool:
        """Whether a j or k face is shared (the exchange goes per axis)."""
        return self.dims[1] > 1 or self.dims[2] > 1 or any(self.ext[1]) or any(self.ext[2])


def _extent(x0: float, n: int, dx: float) -> float:
    """An upper bound x1 near x0 + n * dx with (x1 - x0) / n == dx in double
    precision -- the spacing the library derives from a range -- so that
    the shard steps with the global grid's spacing bit for bit.  Where no
    such x1 lies within a few ulps, x0 + n * dx (a spacing off in the last
    bit, so results agree to rounding only)."""
    first = x1 = x0 + n * dx
    for _ in range(64):
        if (x1 - x0) / n == dx:
            return x1
        x1 = float(np.nextafter(x1, np.inf if (x1 - x0) / n < dx else -np.inf))
    return first


def split_grid(grid: Grid, count: int, periodic_x: bool) -> list[ShardSpec]:
    """Split ``grid`` into ``count`` shards of (nearly) equal i extent.

    Shard r starts where shard r-1 ends, and its range is chosen so that
    the spacing the library computes from it, (x1 - x0) / n, equals the
    global grid's (x_max - x_min) / N exactly where a range within a few
    ulps gives it (all the sizes the tests use)."""
    n = grid.i_size
    if count < 1 or n < count * 2 * grid.margin:
        raise ValueError("each shard needs at least 2 * margin interior planes")
    dx = (grid.x_max - grid.x_min) / n
    cuts = [n * r // count for r in range(count + 1)]
    out = []
    x0 = grid.x_min
    for r in range(count):
        i0, i1 = cuts[r], cuts[r + 1]
        x1 = _extent(x0, i1 - i0, dx) if count > 1 else grid.x_max
        g = Grid(i1 - i0, grid.j_size, grid.k_size, grid.margin, x0, x1,
                 grid.y_min, grid.y_max, grid.z_min, grid.z_max)
        ext_lo = count > 1 and (r > 0 or periodic_x)
        ext_hi = count > 1 and (r < count - 1 or periodic_x)
        out.append(ShardSpec(r, count, i0, i1, g, ext_lo, ext_hi))
        x0 = x1
    return out


def split_grid3(grid: Grid, dims, periodic) -> list[ShardSpec]:
    """Split ``grid`` into dims[0] x dims[1] x dims[2] shards, (nearly)
    equal extents per axis, ranks in the row-major order of their
    coordinates (k fastest, MPI_Cart_create's order).  The reference
    requires each global size to divide by its count (grid.hpp:258-276);
    here the first shards of an axis take one cell less where it does not.
    Each range is chosen as ``split_grid`` chooses the i ranges, so that
    every shard steps with the global grid's spacings bit for bit."""
    sizes = (grid.i_size, grid.j_size, grid.k_size)
    margins = (grid.i_margin, grid.j_margin, grid.k_margin)
    bounds = ((grid.x_min, grid.x_max), (grid.y_min, grid.y_max), (grid.z_min, grid.z_max))
    dims = tuple(int(d) for d in dims)
    if len(dims) != 3 or min(dims) < 1:
        raise ValueError("dims needs three counts >= 1")
    axes = []
    for a in range(3):
        n, c = sizes[a], dims[a]
        if c > 1 and (margins[a] == 0 or n < c * 2 * margins[a]):
            raise ValueError(f"axis {a}: each shard needs at least 2 * margin interior cells")
        d = (bounds[a][1] - bounds[a][0]) / n
        cuts = [n * r // c for r in range(c + 1)]
        parts, x0 = [], bounds[a][0]
        for r in range(c):
            x1 = _extent(x0, cuts[r + 1] - cuts[r], d) if c > 1 else bounds[a][1]
            parts.append((cuts[r], cuts[r + 1], x0, x1))
            x0 = x1
        axes.append(parts)
    out = []
    count = dims[0] * dims[1] * dims[2]
    for rank in range(count):
        coord = (rank // (dims[1] * dims[2]), (rank // dims[2]) % dims[1], rank % dims[2])
        box = [axes[a][coord[a]] for a in range(3)]
        g = Grid(box[0][1] - box[0][0], box[1][1] - box[1][0], box[2][1] - box[2][0],
                 grid.margin, box[0][2], box[0][3], box[1][2], box[1][3], box[2][2], box[2][3])
        ext = tuple((dims[a] > 1 and (coord[a] > 0 or bool(periodic[a])),
                     dims[a] > 1 and (coord[a] < dims[a] - 1 or bool(periodic[a])))
                    for a in range(3))
        out.append(ShardSpec(rank, count, box[0][0], box[0][1], g, ext[0][0], ext[0][1],
                             dims=dims, coord=coord, lo=tuple(b[0] for b in box),
                             hi=tuple(b[1] for b in box), ext=ext))
    return out


def _box(grid: Grid, spec: ShardSpec):
    m = (grid.i_margin, grid.j_margin, grid.k_margin)
    return tuple(slice(spec.lo[a], spec.hi[a] + 2 * m[a]) for a in range(3))


def split_state(q: np.ndarray, grid: Grid, spec: ShardSpec) -> np.ndarray:
    """The shard's (9, I, J, K) state, ghosts included, cut from the global
    state (whose ghost layers hold the global boundary)."""
    return np.ascontiguousarray(q[(slice(None),) + _box(grid, spec)])


def gather(parts: list[np.ndarray], specs: list[ShardSpec], grid: Grid) -> np.ndarray:
    """The global interior (9, nI, nJ, nK) from the shards' states."""
    out = np.empty((parts[0].shape[0], grid.i_size, grid.j_size, grid.k_size),
                   dtype=parts[0].dtype)
    for q, s in zip(parts, specs):
        dst = tuple(slice(s.lo[a], s.hi[a]) for a in range(3))
        out[(slice(None),) + dst] = q[(slice(None),) + s.grid.interior]
    return out


def _cuda_tensor(ptr: int, nbytes: int):
    import torch

    class _View:
        __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1",
                                    "data": (ptr, False), "version": 3}
    return torch.as_tensor(_View(), device="cuda")


def _host_tensor(ptr: int, nbytes: int):
    import torch
    buf = (ctypes.c_char * nbytes).from_address(ptr)
    return torch.frombuffer(buf, dtype=torch.uint8)


class _Halo:
    """ctypes side of ``miso_b200_set_halo``: keeps the C callbacks alive."""

    def attach(self, integ: Integrator, spec: ShardSpec):
        from . import _lib
        self._spec = spec

        def exchange3(user, axis, n, nbytes, ext_lo, ext_hi, slo, shi, rlo, rhi, stream):
            try:
                self.exchange(spec.rank, [slo[a] for a in range(n)], [shi[a] for a in range(n)],
                              [rlo[a] for a in range(n)], [rhi[a] for a in range(n)],
                              int(nbytes), bool(ext_lo), bool(ext_hi), stream or 0, axis=axis)
                return 0
            except Exception as exc:  # reported to the library as MISO_B200_ERR_HALO
                self.error = exc
                return 1

        def exchange(user, n, nbytes, ext_lo, ext_hi, slo, shi, rlo, rhi, stream):
            return exchange3(user, 0, n, nbytes, ext_lo, ext_hi, slo, shi, rlo, rhi, stream)

        def min_all(user, value):
            try:
                value[0] = self.min_all(spec.rank, float(value[0]))
                return 0
            except Exception as exc:
                self.error = exc
                return 1

        self.error = None
        fn_m = _lib.HALO_MIN_FN(min_all)
        if spec.axes3:
            fn_x = _lib.HALO3_EXCHANGE_FN(exchange3)
            ops = _lib.Halo3Ops(fn_x, fn_m, None)
            ext = (ctypes.c_int * 6)(*[int(spec.ext[a][sd]) for a in range(3) for sd in range(2)])
            integ._halo_keep = (fn_x, fn_m, ops, ext, self)
            integ._check(integ._lib.miso_b200_set_halo3(integ._h, ext, ctypes.byref(ops)))
        else:
            fn_x = _lib.HALO_EXCHANGE_FN(exchange)
            ops = _lib.HaloOps(fn_x, fn_m, None)
            integ._halo_keep = (fn_x, fn_m, ops, self)
            integ._check(integ._lib.miso_b200_set_halo(integ._h, int(spec.ext_lo),
                                                       int(spec.ext_hi), ctypes.byref(ops)))


def _neighbour(coord, dims, periodic, axis, d):
    """Rank of the shard next to ``coord`` along ``axis`` (d = -1 / +1),
    across a periodic face by the wrap, None past a boundary."""
    c = list(coord)
    c[axis] += d
    if not 0 <= c[axis] < dims[axis]:
        if not periodic[axis]:
            return None
        c[axis] %= dims[axis]
    return (c[0] * dims[1] + c[1]) * dims[2] + c[2]


def _rank_coord(rank, dims):
    return (rank // (dims[1] * dims[2]), (rank // dims[2]) % dims[1], rank % dims[2])


class LocalHalo(_Halo):
    """Shards of one process on one GPU, each driven by its own host thread
    and all on one CUDA stream.  At an exchange every shard registers its
    planes and waits for the others; then each shard enqueues device copies
    of its neighbours' boundary planes into its own ghost planes, and all
    wait again before the next pass is enqueued.  The shared stream orders
    the copies after every shard's pass and before the next."""

    def __init__(self, count: int, periodic_x: bool, timeout: float = 120.0, dims=None,
                 periodic=None):
        self.count = count
        self.periodic_x = periodic_x
        self.dims = tuple(dims) if dims is not None else (count, 1, 1)
        self.periodic = tuple(periodic) if periodic is not None else (periodic_x, False, False)
        if self.dims[0] * self.dims[1] * self.dims[2] != count:
            raise ValueError("dims must multiply to count")
        self._bar = threading.Barrier(count, timeout=timeout)
        self._planes = [None] * count
        self._vals = [0.0] * count

    def attach(self, integ: Integrator, spec: ShardSpec):
        _Halo.attach(self, integ, spec)

    def _peer(self, r: int, d: int, axis: int = 0):
        return _neighbour(_rank_coord(r, self.dims), self.dims, self.periodic, axis, d)

    def exchange(self, r, slo, shi, rlo, rhi, nbytes, ext_lo, ext_hi, stream, axis=0):
        import torch
        self._planes[r] = (slo, shi, stream, axis)
        self._bar.wait()
        if any(p[2] != stream for p in self._planes):
            raise RuntimeError("in-process shards must share one CUDA stream")
        if any(p[3] != axis for p in self._planes):
            raise RuntimeError("the shards exchange along different axes at once")
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            for a in range(len(rlo)):
                if ext_lo:
                    src = self._planes[self._peer(r, -1, axis)][1][a]
                    _cuda_tensor(rlo[a], nbytes).copy_(_cuda_tensor(src, nbytes))
                if ext_hi:
                    src = self._planes[self._peer(r, +1, axis)][0][a]
                    _cuda_tensor(rhi[a], nbytes).copy_(_cuda_tensor(src, nbytes))
        self._bar.wait()

    def min_all(self, r, value):
        self._vals[r] = value
        self._bar.wait()
        out = min(self._vals)
        self._bar.wait()
        return out


class DistHalo(_Halo):
    """One shard per rank of a torch.distributed process group: the planes
    travel by point-to-point sends and receives (NCCL on the library's
    stream across GPUs; gloo on host buffers), the time step by an
    all-reduce of the minimum.  With one rank a periodic face is a copy."""

    def __init__(self, periodic_x: bool, device: str = "cuda", group=None, dims=None,
                 periodic=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.periodic_x = periodic_x
        self.device = device
        self.dims = tuple(dims) if dims is not None else (self.world, 1, 1)
        self.periodic = tuple(periodic) if periodic is not None else (periodic_x, False, False)
        if self.dims[0] * self.dims[1] * self.dims[2] != self.world:
            raise ValueError("dims must multiply to the world size")

    def _peer(self, d: int, axis: int = 0):
        return _neighbour(_rank_coord(self.rank, self.dims), self.dims, self.periodic, axis, d)

    def _t(self, ptr, nbytes):
        return _cuda_tensor(ptr, nbytes) if self.device == "cuda" else _host_tensor(ptr, nbytes)

    def exchange(self, r, slo, shi, rlo, rhi, nbytes, ext_lo, ext_hi, stream, axis=0):
        import torch
        dist = self.dist
        ctx = (torch.cuda.stream(torch.cuda.ExternalStream(stream))
               if self.device == "cuda" else _nullcontext())
        with ctx:
            lo, hi = self._peer(-1, axis), self._peer(+1, axis)
            if self.dims[axis] == 1:
                # one shard along the axis: a shared face can only be the
                # periodic wrap
                for a in range(len(rlo)):
                    if ext_lo:
                        self._t(rlo[a], nbytes).copy_(self._t(shi[a], nbytes))
                    if ext_hi:
                        self._t(rhi[a], nbytes).copy_(self._t(slo[a], nbytes))
                return
            # Messages between a pair of ranks match in the order they are
            # posted (NCCL has no tags), and with two ranks on a periodic
            # axis the low and the high neighbour are the same rank.  So per
            # array every rank posts the upward transfer (its high planes to
            # the high neighbour's low ghosts) before the downward one: the
            # k-th send from r to p then meets the k-th receive at p from r.
            ops = []
            up_send, up_recv = ext_hi and hi is not None, ext_lo and lo is not None
            for a in range(len(rlo)):
                if up_send:
                    ops.append(dist.P2POp(dist.isend, self._t(shi[a], nbytes), hi, self.group))
                if up_recv:
                    ops.append(dist.P2POp(dist.irecv, self._t(rlo[a], nbytes), lo, self.group))
                if up_recv:
                    ops.append(dist.P2POp(dist.isend, self._t(slo[a], nbytes), lo, self.group))
                if up_send:
                    ops.append(dist.P2POp(dist.irecv, self._t(rhi[a], nbytes), hi, self.group))
            for w in dist.batch_isend_irecv(ops) if ops else []:
                w.wait()

    def min_all(self, r, value):
        import torch
        t = torch.tensor([value], dtype=torch.float64,
                         device="cuda" if self.device == "cuda" else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN, group=self.group)
        return float(t.item())


class _nullcontext:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def run_local_shards(prob, count: int, steps: int, precision: str = "fp64", variants=None,
                     stream=None, overlap: bool = False,
                     dims=None) -> tuple[np.ndarray, list[float]]:
    """Advance ``prob`` by ``steps`` host-dt steps (cfl, then update) as
    ``count`` shards on the current GPU, one host thread per shard, all on
    one CUDA stream (``stream``, or a new one); return the gathered global
    interior and the time steps taken.  ``dims`` (shards per axis, product
    ``count``) decomposes along j and k too; by default the grid is cut
    along i.  With ``overlap`` the exchanges run on a second stream shared
    by the shards while each next pass finishes the planes that need no
    ghost (``Integrator.set_halo_overlap``; i faces only)."""
    import torch
    per = prob.config["domain"]["periodic"]
    periodic = (bool(per["x"]), bool(per["y"]), bool(per["z"]))
    periodic_x = periodic[0]
    if dims is None:
        specs = split_grid(prob.grid, count, periodic_x)
        halo = LocalHalo(count, periodic_x)
    else:
        specs = split_grid3(prob.grid, dims, periodic)
        halo = LocalHalo(count, periodic_x, dims=dims, periodic=periodic)
    # one stream for every shard (a null stream would give each handle its
    # own, and the halo copies would then race with the neighbours' passes)
    keep = None
    if stream is None:
        keep = torch.cuda.Stream()
        stream = keep.cuda_stream
    if not stream:
        raise ValueError("the shards need one explicit (non-null) CUDA stream")
    st = stream
    comm = torch.cuda.Stream() if overlap else None
    integs = []
    for s in specs:
        blend = getattr(prob, "blend", None)
        integ = Integrator(prob.config, s.grid, sign=prob.sign, precision=precision, stream=st,
                           blend=None if blend is None else split_state(blend, prob.grid, s))
        for cls, var in (variants or {}).items():
            integ.set_variant(cls, var)
        halo.attach(integ, s)
        if comm is not None:
            integ.set_halo_overlap(comm.cuda_stream)
        integ.upload(split_state(prob.q, prob.grid, s))
        integs.append(integ)
    dts = [[] for _ in specs]
    errors = []

    def drive(r):
        try:
            integs[r].apply_boundary_condition()
            for _ in range(steps):
                dt = integs[r].cfl()
                integs[r].update(dt)
                dts[r].append(dt)
            integs[r].sync()
        except Exception as exc:
            errors.append(exc)
            halo._bar.abort()

    threads = [threading.Thread(target=drive, args=(r,)) for r in range(count)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        for integ in integs:
            integ.close()
        raise errors[0]
    parts = [integ.download() for integ in integs]
    for integ in integs:
        integ.close()
    return gather(parts, specs, prob.grid), dts[0]
