"""Host-side mirror of the reference's integrator interface over the C ABI.

``Integrator`` stands where ``mhd::Integrator<Real, backend::CUDA>`` stands
in the reference (miso/include/miso/mhd_integrator_cuda.cuh:291-501):

* ``Integrator(config, grid)``            -- constructor (lines 328-339)
* ``cfl(qq=None, eos=None) -> dt``        -- Integrator::cfl (450-478)
* ``update(dt, eos, bc, src, qq=None)``   -- Integrator::update (481-487)
* ``apply_boundary_condition(bc, qq)``    -- (396-401)

and ``MHD`` mirrors ``mhd::MHD`` (miso/include/miso/mhd.hpp:15-50), which owns
the fields and forwards ``cfl``/``update``.  The equation of state, the
boundary condition and the source term are the built-in ones the reference's
MHD demos use: ideal gas with ``eos.gm``; periodic faces where
``domain.periodic`` says so and the symmetric mirror (per-field sign) on the
other faces; no source, or the magnetosphere demo's point gravity when
``source.kind`` is ``"point_gravity"`` (``source.g`` its acceleration).
With ``boundary.kind == "magnetosphere"`` (both forms) the magnetosphere
demo's boundary and masked CFL replace the plain faces, configured from the
demo's own ``solar_wind``, ``magnetosphere`` and ``floor`` sections; the
state it blends toward is the ``blend`` argument (zeros if None).
Every call goes through ``libmiso_b200.so``; nothing here computes on the
CPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .config import merge_defaults
from .grid import Grid

PRECISIONS = {"fp64": _lib.FP64, "fp32_split": _lib.FP32_SPLIT}


class IdealEOS:
    """Ideal-gas equation of state (miso/include/miso/eos.hpp:13-45)."""

    def __init__(self, gm: float):
        self.gm = float(gm)


class BuiltinBoundary:
    """Periodic / symmetric-mirror faces (the reference's HaloExchanger for
    periodic axes plus boundary_condition::symmetric on the others)."""

    def __init__(self, sign=None):
        self.sign = np.ones((3, 2, 9)) if sign is None else np.asarray(sign, dtype=np.float64)


class EmptySourceTerm:
    """No source terms (miso/include/miso/mhd_model_base.hpp:131-155)."""


def _field_ptrs(q):
    """9 pointers into a (9, I, J, K) float64 array (numpy, host) or a torch
    tensor (host or CUDA)."""
    arr = (ctypes.c_void_p * 9)()
    if isinstance(q, np.ndarray):
        if q.dtype != np.float64 or not q.flags.c_contiguous or q.shape[0] != 9:
            raise ValueError("fields must be a C-contiguous (9, I, J, K) float64 array")
        for f in range(9):
            arr[f] = q[f].ctypes.data
        return arr
    # torch tensor
    if q.dtype.__str__() != "torch.float64" or not q.is_contiguous() or q.shape[0] != 9:
        raise ValueError("fields must be a contiguous (9, I, J, K) float64 tensor")
    for f in range(9):
        arr[f] = q[f].data_ptr()
    return arr


def make_descs(config: dict, grid: Grid, sign=None, precision: str = "fp64"):
    """C-ABI grid descriptor and parameter block for a configuration."""
    cfg = merge_defaults(config)
    gd = _lib.GridDesc()
    gd.i_size, gd.j_size, gd.k_size, gd.margin = (grid.i_size, grid.j_size, grid.k_size,
                                                  grid.margin)
    gd.x_min, gd.x_max, gd.y_min, gd.y_max = grid.x_min, grid.x_max, grid.y_min, grid.y_max
    gd.z_min, gd.z_max = grid.z_min, grid.z_max
    per = cfg["domain"]["periodic"]
    gd.periodic[0], gd.periodic[1], gd.periodic[2] = (int(per["x"]), int(per["y"]),
                                                      int(per["z"]))
    sg = np.ones((3, 2, 9)) if sign is None else np.asarray(sign, dtype=np.float64)
    for n, v in enumerate(sg.reshape(-1)):
        gd.sign[n] = float(v)
    pp = _lib.Params()
    av = cfg["mhd"]["artificial_viscosity"]
    pp.gm = cfg["eos"]["gm"]
    pp.cfl_number = cfg["mhd"]["cfl_number"]
    pp.ep, pp.fh = av["ep"], av["fh"]
    pp.cs_fac, pp.ca_fac, pp.vv_fac = av["cs_fac"], av["ca_fac"], av["vv_fac"]
    pp.precision = PRECISIONS[precision]
    return gd, pp


def cfl_noalloc(config: dict, grid: Grid, q, stream: int | None = None) -> float:
    """CFL time step of caller-owned device fields (a CUDA (9, I, J, K)
    float64 tensor) through the allocation-free entry point
    miso_b200_cfl_noalloc: no handle, no device allocation.  Host arrays,
    CPU tensors and tensors of another shape are refused here, before the
    library is called; the library refuses non-device pointers itself."""
    shape = (9,) + tuple(grid.shape)
    if isinstance(q, np.ndarray) or not hasattr(q, "is_cuda") or not q.is_cuda:
        raise ValueError("cfl_noalloc needs the fields as a CUDA tensor (device memory)")
    if tuple(q.shape) != shape or str(q.dtype) != "torch.float64" or not q.is_contiguous():
        raise ValueError(f"cfl_noalloc needs a contiguous float64 tensor of shape {shape}, "
                         f"got {tuple(q.shape)} {q.dtype}")
    lib = _lib.load()
    gd, pp = make_descs(config, grid)
    dt = ctypes.c_double()
    _lib.check(lib.miso_b200_cfl_noalloc(ctypes.byref(gd), ctypes.byref(pp), _field_ptrs(q),
                                         ctypes.c_void_p(stream or 0), ctypes.byref(dt)), None)
    return dt.value


class Integrator:
    """One grid advanced on the current CUDA device."""

    def __init__(self, config: dict, grid: Grid, sign=None, precision: str = "fp64",
                 stream: int | None = None, blend=None):
        cfg = merge_defaults(config)
        self.config = cfg
        self.grid = grid
        self.precision = precision
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        self.eos = IdealEOS(cfg["eos"]["gm"])
        self.bc = BuiltinBoundary(sign)
        self.src = EmptySourceTerm()
        lib = _lib.load()
        gd, pp = make_descs(cfg, grid, sign=self.bc.sign, precision=precision)
        h = ctypes.c_void_p()
        _lib.check(lib.miso_b200_create(ctypes.byref(gd), ctypes.byref(pp),
                                        ctypes.c_void_p(stream or 0), ctypes.byref(h)), None)
        self._h = h
        self._lib = lib
        try:
            self._configure(cfg, blend)
        except Exception:
            self.close()
            raise

    def _configure(self, cfg: dict, blend):
        """The source and boundary descriptors of the configuration."""
        lib, h = self._lib, self._h
        src = cfg.get("source") or {}
        kind = src.get("kind", "none")
        if kind == "callback":
            self.set_source_callback(src["fn"])
        elif kind != "none":
            kinds = {"point_gravity": 1}
            if kind not in kinds:
                raise ValueError(f"unknown source kind {kind!r}")
            par = (ctypes.c_double * 1)(float(src["g"]))
            self._check(lib.miso_b200_set_source(h, kinds[kind], par, 1))
        bnd = cfg.get("boundary") or {}
        bkind = bnd.get("kind", "faces")
        if bkind == "magnetosphere":
            sw, ms, fl = cfg["solar_wind"], cfg["magnetosphere"], cfg["floor"]
            par = (ctypes.c_double * 9)(
                sw["mass_density"], sw["gas_pressure"], sw["x_velocity_field"],
                sw["z_magnetic_field"], ms["radius"], ms["a0"], fl["ro_floor"], fl["pr_floor"],
                1.0 if bnd.get("cfl_mask", True) else 0.0)
            self._check(lib.miso_b200_set_boundary(h, 1, par, 9))
            if blend is not None:
                self._check(lib.miso_b200_set_blend_state(h, _field_ptrs(blend)))
        elif bkind != "faces":
            raise ValueError(f"unknown boundary kind {bkind!r}")

    # -- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.miso_b200_destroy(self._h)
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

    def _check(self, code):
        _lib.check(code, self._h)

    # -- data movement --------------------------------------------------------
    def upload(self, q):
        """Copy the 9 primitive fields in (numpy host array or torch tensor)."""
        self._check(self._lib.miso_b200_upload(self._h, _field_ptrs(q)))

    def download(self, out=None) -> np.ndarray:
        """Copy the 9 primitive fields out as a (9, I, J, K) float64 array."""
        if out is None:
            out = np.empty((9,) + self.grid.shape, dtype=np.float64)
        self._check(self._lib.miso_b200_download(self._h, _field_ptrs(out)))
        return out

    # -- the reference's integrator interface ---------------------------------
    def apply_boundary_condition(self, bc=None, qq=None):
        self._check(self._lib.miso_b200_fill_ghosts(self._h))

    def cfl(self, qq=None, eos=None) -> float:
        dt = ctypes.c_double()
        self._check(self._lib.miso_b200_cfl(self._h, ctypes.byref(dt)))
        return dt.value

    def update(self, dt: float, eos=None, bc=None, src=None, qq=None):
        self._check(self._lib.miso_b200_update(self._h, float(dt)))

    # -- device-resident stepping --------------------------------------------
    def update_device(self):
        """One step with the dt of the last CFL pass, no host round trip."""
        self._check(self._lib.miso_b200_update_device(self._h))

    def run(self, nsteps: int, graph: bool = True):
        """nsteps of (cfl, update) with dt kept on the device."""
        self._check(self._lib.miso_b200_run(self._h, int(nsteps), int(bool(graph))))

    def sync(self):
        self._check(self._lib.miso_b200_sync(self._h))

    def last_dt(self) -> float:
        dt = ctypes.c_double()
        self._check(self._lib.miso_b200_last_dt(self._h, ctypes.byref(dt)))
        return dt.value

    def monitors(self) -> dict:
        out = (ctypes.c_double * 8)()
        self._check(self._lib.miso_b200_monitors(self._h, out))
        keys = ("mass", "mom_x", "mom_y", "mom_z", "energy", "divb_l1", "divb_max", "ph2")
        return dict(zip(keys, list(out)))

    def set_variant(self, kernel_class: int, variant: int):
        self._check(self._lib.miso_b200_set_variant(self._h, int(kernel_class), int(variant)))

    def set_chunks(self, rk_chunk: int, av_chunk: int):
        self._check(self._lib.miso_b200_set_chunks(self._h, int(rk_chunk), int(av_chunk)))

    def run_until(self, time: float, t_end: float, max_steps: int = 2**31 - 1,
                  graph: bool = True) -> tuple[float, int]:
        """Steps (cfl, update, time += dt) with dt and the time on the
        device while time < t_end (and fewer than max_steps); with ``graph``
        one CUDA graph launch (a conditional WHILE node) runs the loop.
        Returns the new time and the steps taken."""
        t = ctypes.c_double(time)
        n = ctypes.c_int()
        self._check(self._lib.miso_b200_run_until(self._h, ctypes.byref(t), float(t_end),
                                                  int(max_steps), int(bool(graph)),
                                                  ctypes.byref(n)))
        return t.value, n.value

    def set_halo_overlap(self, comm_stream: int | None):
        """Overlap each halo exchange with the next pass: the exchange runs
        on ``comm_stream`` (a cudaStream_t handle; shards of one process
        share one), the next pass finishes the planes that need no ghost
        first.  ``None`` turns it off."""
        self._check(self._lib.miso_b200_set_halo_overlap(self._h,
                                                         ctypes.c_void_p(comm_stream or 0)))

    def set_monitor_fusion(self, on: bool = True):
        """Fold the monitors' sums into every step's last sweep (3-D split
        grids): monitors() then only reduces |div B|."""
        self._check(self._lib.miso_b200_set_monitor_fusion(self._h, int(bool(on))))

    def set_wait_limit(self, cycles: int):
        """Bound (SM clock cycles) of the consumer waits for each plane's
        copy in the 3-D split kernels; 0 restores the default (~2 s)."""
        self._check(self._lib.miso_b200_set_wait_limit(self._h, int(cycles)))

    def set_mirror_signs(self, sign):
        """Mirror signs (3 axes, 2 sides, 9 fields) of the non-periodic faces."""
        s = np.ascontiguousarray(np.asarray(sign, dtype=np.float64).reshape(54))
        self._check(self._lib.miso_b200_set_mirror_signs(self._h,
                                                         s.ctypes.data_as(_lib._dp)))
        self.bc = BuiltinBoundary(s.reshape(3, 2, 9))

    def set_boundary_callback(self, fn):
        """A boundary functor of the caller's own (FP64 form): after every
        pass ``fn(q)`` gets the state just written as a (9, I, J, K) float64
        numpy array over host copies, fills the non-periodic faces in place
        (the periodic ones follow on the device), and returns None.
        ``fn=None`` returns to the built-in faces."""
        if fn is None:
            self._check(self._lib.miso_b200_set_boundary_callback(self._h, None, None, 0))
            self._bc_cb = None
            return
        shape = (9,) + tuple(self.grid.shape)
        cells = int(np.prod(shape[1:]))

        def trampoline(user, q, stream):
            try:
                base = ctypes.cast(q[0], ctypes.POINTER(ctypes.c_double))
                arr = np.ctypeslib.as_array(base, shape=(9 * cells,)).reshape(shape)
                # the 9 arrays are consecutive in the library's staging
                assert all(q[f] == q[0] + f * cells * 8 for f in range(9))
                fn(arr)
                return 0
            except Exception:
                return 1
        self._bc_cb = _lib.BOUNDARY_FN(trampoline)
        self._check(self._lib.miso_b200_set_boundary_callback(
            self._h, ctypes.cast(self._bc_cb, ctypes.c_void_p), None, 1))

    def set_source_callback(self, fn, on_host: bool = True):
        """A source functor of the caller's own (the reference's Source
        concept, mhd_model_base.hpp:131-155): before every Runge-Kutta stage
        ``fn(q, s)`` gets the stage's argument state ``q`` (the 9 primitive
        fields with ghosts, (9, I, J, K) float64) and fills ``s`` ((4, I, J,
        K): src.vx, src.vy, src.vz, src.ei of every interior cell) in place.
        With ``on_host`` both are numpy arrays over host copies; otherwise
        ``fn(q, s, stream)`` gets lists of device addresses (9 and 4) and the
        cudaStream_t of the handle.  In the split form ``q`` is the argument
        state converted to FP64 primitives (hi + lo for the step's first
        stage).  ``fn=None`` removes it."""
        if fn is None:
            self._check(self._lib.miso_b200_set_source_callback(self._h, None, None, 0))
            self._src_cb = None
            return
        shape = tuple(self.grid.shape)
        cells = int(np.prod(shape))

        def view(p, n):
            base = ctypes.cast(p, ctypes.POINTER(ctypes.c_double))
            return np.ctypeslib.as_array(base, shape=(n * cells,)).reshape((n,) + shape)

        def trampoline(user, q, s, stream):
            try:
                if on_host:
                    # the library stages q and then s as consecutive arrays
                    assert all(q[f] == q[0] + f * cells * 8 for f in range(9))
                    assert all(s[t] == s[0] + t * cells * 8 for t in range(4))
                    fn(view(q[0], 9), view(s[0], 4))
                else:
                    fn([q[f] for f in range(9)], [s[t] for t in range(4)], stream)
                return 0
            except Exception:
                return 1
        self._src_cb = _lib.SOURCE_FN(trampoline)
        self._check(self._lib.miso_b200_set_source_callback(
            self._h, ctypes.cast(self._src_cb, ctypes.c_void_p), None, int(bool(on_host))))

    def arm_timeout_test(self, cycles: int):
        """The next pipelined Runge-Kutta stage waits, with bound ``cycles``,
        on a barrier phase that nothing completes (a test of the timeout
        path; the step then reports MISO_B200_ERR_TIMEOUT)."""
        self._check(self._lib.miso_b200_arm_timeout_test(self._h, int(cycles)))

    def get_variant(self, kernel_class: int) -> int:
        v = ctypes.c_int()
        self._check(self._lib.miso_b200_get_variant(self._h, int(kernel_class), ctypes.byref(v)))
        return v.value

    def set_timing(self, enable: bool):
        self._check(self._lib.miso_b200_set_timing(self._h, int(bool(enable))))

    def timing_report(self) -> dict:
        import json
        buf = ctypes.create_string_buffer(1 << 16)
        self._check(self._lib.miso_b200_timing_report(self._h, buf, len(buf)))
        return json.loads(buf.value.decode())

    def device_bytes(self) -> int:
        b = ctypes.c_size_t()
        self._check(self._lib.miso_b200_device_bytes(self._h, ctypes.byref(b)))
        return b.value

    def launch_count(self) -> int:
        c = ctypes.c_longlong()
        self._check(self._lib.miso_b200_launch_count(self._h, ctypes.byref(c)))
        return c.value


class MHD:
    """Fields + integrator for one grid (miso/include/miso/mhd.hpp:15-50)."""

    def __init__(self, config: dict, grid: Grid, sign=None, precision: str = "fp64",
                 blend=None, stream=None):
        self.grid = grid
        self.integrator = Integrator(config, grid, sign=sign, precision=precision, blend=blend,
                                     stream=stream)

    def apply_initial_condition(self, q):
        """Upload initial fields and fill the ghosts (mhd.hpp:28-35)."""
        self.integrator.upload(q)
        self.integrator.apply_boundary_condition()

    def cfl(self, eos=None) -> float:
        return self.integrator.cfl()

    def update(self, dt, eos=None, bc=None, src=None):
        self.integrator.update(dt)

    def step(self) -> float:
        """ModelBase::update (mhd_model_base.hpp:57-62): cfl then update."""
        dt = self.cfl()
        self.update(dt)
        return dt
