"""ctypes bindings of the CPU checkers (TEST INFRASTRUCTURE ONLY).

* :class:`Oracle` loads ``oracle/_build/libmiso_oracle.so``, the C
  restatement of MISO's explicit MHD step (oracle/miso_oracle.c);
* :class:`Reference` loads ``oracle/_ref/libmiso_ref.so``, the reference's own
  host integrator compiled from its headers (oracle/ref_harness.cpp).

Both expose the same calls on a :class:`miso_b200.problems.Problem`-like
object (grid, config, sign) and a ``(9, I, J, K)`` float64 array.  Only the
tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use
this module; the product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libmiso_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmiso_ref.so")
REF_F32_SO = os.path.join(HERE, "_ref", "libmiso_ref_f32.so")

_dp = ctypes.POINTER(ctypes.c_double)

# The MISO checkout the reference build and the pymiso reader come from:
# $MISO_REFERENCE when set, else the default location.
REFERENCE_ROOT = os.environ.get("MISO_REFERENCE", "/root/reference")
REFERENCE_INCLUDE = os.path.join(REFERENCE_ROOT, "miso", "include")


class Desc(ctypes.Structure):
    _fields_ = [("i_size", ctypes.c_int), ("j_size", ctypes.c_int), ("k_size", ctypes.c_int),
                ("margin", ctypes.c_int),
                ("x_min", ctypes.c_double), ("x_max", ctypes.c_double),
                ("y_min", ctypes.c_double), ("y_max", ctypes.c_double),
                ("z_min", ctypes.c_double), ("z_max", ctypes.c_double),
                ("periodic", ctypes.c_int * 3),
                ("sign", ctypes.c_double * 54),
                ("gm", ctypes.c_double), ("cfl_number", ctypes.c_double),
                ("ep", ctypes.c_double), ("fh", ctypes.c_double),
                ("cs_fac", ctypes.c_double), ("ca_fac", ctypes.c_double),
                ("vv_fac", ctypes.c_double),
                ("source", ctypes.c_int), ("g_grav", ctypes.c_double),
                ("boundary", ctypes.c_int),
                ("sw_ro", ctypes.c_double), ("sw_pr", ctypes.c_double),
                ("sw_vx", ctypes.c_double), ("sw_bz", ctypes.c_double),
                ("r_inner", ctypes.c_double), ("a0", ctypes.c_double),
                ("ro_floor", ctypes.c_double), ("pr_floor", ctypes.c_double),
                ("blend", ctypes.c_void_p * 9), ("cfl_masked", ctypes.c_int),
                ("src_fn", ctypes.c_void_p), ("src_user", ctypes.c_void_p),
                ("src_const", ctypes.c_double * 4)]


# the oracle's source callback: (user, double *const q[9], double *const s[4])
SOURCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t),
                             ctypes.POINTER(ctypes.c_size_t))


def _source_trampoline(fn, shape):
    """A ctypes callback that hands ``fn`` the argument state (9, I, J, K)
    and the four source arrays (4, I, J, K) as numpy views."""
    cells = int(np.prod(shape))

    def view(p):
        return np.ctypeslib.as_array(ctypes.cast(p, _dp), shape=(cells,)).reshape(shape)

    def tramp(user, q, s):
        try:
            fn(np.stack([view(q[f]) for f in range(9)]), [view(s[t]) for t in range(4)])
            return 0
        except Exception:
            return 1
    return SOURCE_FN(tramp)


def make_desc(grid, config, sign=None, blend=None) -> Desc:
    """The descriptor of a run; ``blend`` (a (9, I, J, K) float64 array) is
    the state the magnetosphere boundary blends toward (zeros if None)."""
    d = Desc()
    d.i_size, d.j_size, d.k_size, d.margin = grid.i_size, grid.j_size, grid.k_size, grid.margin
    d.x_min, d.x_max = grid.x_min, grid.x_max
    d.y_min, d.y_max = grid.y_min, grid.y_max
    d.z_min, d.z_max = grid.z_min, grid.z_max
    p = config["domain"]["periodic"]
    d.periodic[0], d.periodic[1], d.periodic[2] = int(p["x"]), int(p["y"]), int(p["z"])
    s = np.ones((3, 2, 9)) if sign is None else np.asarray(sign, dtype=np.float64)
    for n, v in enumerate(s.reshape(-1)):
        d.sign[n] = float(v)
    d.gm = config["eos"]["gm"]
    d.cfl_number = config["mhd"]["cfl_number"]
    av = config["mhd"]["artificial_viscosity"]
    d.ep, d.fh = av["ep"], av["fh"]
    d.cs_fac, d.ca_fac, d.vv_fac = av["cs_fac"], av["ca_fac"], av["vv_fac"]
    src = config.get("source") or {}
    d.source = {"none": 0, "point_gravity": 1, "callback": 2,
                "constant": 3}[src.get("kind", "none")]
    d.g_grav = float(src.get("g", 0.0))
    if d.source == 3:
        for t, v in enumerate(src["values"]):
            d.src_const[t] = float(v)
    elif d.source == 2:
        # fn(q, s): q the stage's argument state (9, I, J, K), s a list of the
        # four (I, J, K) arrays to fill (src.vx, src.vy, src.vz, src.ei)
        cb = _source_trampoline(src["fn"], tuple(grid.shape))
        d.src_fn = ctypes.cast(cb, ctypes.c_void_p).value
        d._cb = cb  # the callback outlives the call
    bnd = config.get("boundary") or {}
    if bnd.get("kind", "faces") == "magnetosphere":
        sw, ms, fl = config["solar_wind"], config["magnetosphere"], config["floor"]
        d.boundary = 1
        d.sw_ro, d.sw_pr = sw["mass_density"], sw["gas_pressure"]
        d.sw_vx, d.sw_bz = sw["x_velocity_field"], sw["z_magnetic_field"]
        d.r_inner, d.a0 = ms["radius"], ms["a0"]
        d.ro_floor, d.pr_floor = fl["ro_floor"], fl["pr_floor"]
        d.cfl_masked = int(bool(bnd.get("cfl_mask", True)))
        if blend is not None:
            assert blend.dtype == np.float64 and blend.flags.c_contiguous and blend.shape[0] == 9
            for f in range(9):
                d.blend[f] = blend[f].ctypes.data
            d._keep = blend  # the arrays outlive the call
    return d


def _ptrs(q: np.ndarray):
    assert q.dtype == np.float64 and q.flags.c_contiguous and q.shape[0] == 9
    arr = (_dp * 9)()
    for f in range(9):
        arr[f] = q[f].ctypes.data_as(_dp)
    return arr


def build():
    """Compile the restatement (and the reference build where its sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if os.path.isdir(REFERENCE_INCLUDE):
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


class _Lib:
    prefix = ""
    path = ""

    def __init__(self):
        if not os.path.exists(self.path):
            raise FileNotFoundError(f"{self.path} is not built (run make -C oracle)")
        lib = ctypes.CDLL(self.path)
        P = self.prefix
        self._run = getattr(lib, P + "run")
        self._run.argtypes = [ctypes.POINTER(Desc), ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp]
        self._run.restype = ctypes.c_int
        self._cfl = getattr(lib, P + "cfl")
        self._cfl.argtypes = [ctypes.POINTER(Desc), ctypes.c_void_p]
        self._cfl.restype = ctypes.c_double
        self._stage = getattr(lib, P + "stage")
        self._stage.argtypes = [ctypes.POINTER(Desc), ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                ctypes.c_double]
        self._stage.restype = ctypes.c_int
        self._av = getattr(lib, P + "av")
        self._av.argtypes = [ctypes.POINTER(Desc), ctypes.c_void_p, ctypes.c_double]
        self._av.restype = ctypes.c_int
        self._fill = getattr(lib, P + "fill_ghosts")
        self._fill.argtypes = [ctypes.POINTER(Desc), ctypes.c_void_p]
        self._fill.restype = ctypes.c_int
        self._mind = getattr(lib, P + "min_dxyz")
        self._mind.argtypes = [ctypes.POINTER(Desc)]
        self._mind.restype = ctypes.c_double
        self.lib = lib

    def run(self, prob, q: np.ndarray, nsteps: int, fill_first: bool = True):
        """Advance ``q`` in place by ``nsteps`` (cfl + update); returns the dts."""
        d = make_desc(prob.grid, prob.config, prob.sign, getattr(prob, "blend", None))
        dts = np.zeros(max(nsteps, 1))
        rc = self._run(ctypes.byref(d), ctypes.cast(_ptrs(q), ctypes.c_void_p), nsteps,
                       int(fill_first), dts.ctypes.data_as(_dp))
        if rc:
            raise RuntimeError(f"{self.prefix}run failed: {rc}")
        return dts[:nsteps]

    def cfl(self, prob, q):
        d = make_desc(prob.grid, prob.config, prob.sign, getattr(prob, "blend", None))
        return self._cfl(ctypes.byref(d), ctypes.cast(_ptrs(q), ctypes.c_void_p))

    def stage(self, prob, orgn, argm, rslt, dt, ch2, tau):
        d = make_desc(prob.grid, prob.config, prob.sign, getattr(prob, "blend", None))
        rc = self._stage(ctypes.byref(d), ctypes.cast(_ptrs(orgn), ctypes.c_void_p),
                         ctypes.cast(_ptrs(argm), ctypes.c_void_p),
                         ctypes.cast(_ptrs(rslt), ctypes.c_void_p), dt, ch2, tau)
        if rc:
            raise RuntimeError(f"{self.prefix}stage failed: {rc}")

    def av(self, prob, q, dt):
        d = make_desc(prob.grid, prob.config, prob.sign, getattr(prob, "blend", None))
        rc = self._av(ctypes.byref(d), ctypes.cast(_ptrs(q), ctypes.c_void_p), dt)
        if rc:
            raise RuntimeError(f"{self.prefix}av failed: {rc}")

    def fill_ghosts(self, prob, q):
        d = make_desc(prob.grid, prob.config, prob.sign, getattr(prob, "blend", None))
        rc = self._fill(ctypes.byref(d), ctypes.cast(_ptrs(q), ctypes.c_void_p))
        if rc:
            raise RuntimeError(f"{self.prefix}fill_ghosts failed: {rc}")

    def min_dxyz(self, prob):
        d = make_desc(prob.grid, prob.config, prob.sign, getattr(prob, "blend", None))
        return self._mind(ctypes.byref(d))


class Oracle(_Lib):
    prefix = "miso_oracle_"
    path = ORACLE_SO


class Reference(_Lib):
    prefix = "miso_ref_"
    path = REF_SO

    def update(self, prob, q, dt):
        """One step of ``q`` in place with the given dt (Integrator::update)."""
        f = self.lib.miso_ref_update
        f.argtypes = [ctypes.POINTER(Desc), ctypes.c_void_p, ctypes.c_double]
        f.restype = ctypes.c_int
        d = make_desc(prob.grid, prob.config, prob.sign, getattr(prob, "blend", None))
        rc = f(ctypes.byref(d), ctypes.cast(_ptrs(q), ctypes.c_void_p), float(dt))
        if rc:
            raise RuntimeError(f"{self.prefix}update failed: {rc}")

    def symmetric_index(self, i, i_total, i_margin, outer):
        f = self.lib.miso_ref_symmetric_index
        f.argtypes = [ctypes.c_int] * 4 + [ctypes.POINTER(ctypes.c_int)] * 2
        g, t = ctypes.c_int(), ctypes.c_int()
        f(i, i_total, i_margin, int(outer), ctypes.byref(g), ctypes.byref(t))
        return g.value, t.value


class ReferenceF32(Reference):
    """The reference's integrator built with Real = float, as its demos are."""
    path = REF_F32_SO


def reference_available() -> bool:
    return os.path.exists(REF_SO)
