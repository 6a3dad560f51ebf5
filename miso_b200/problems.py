"""Seeded initial conditions for the benchmark and parity workloads.

Every generator returns a :class:`Problem`: the grid, the run configuration,
the boundary signs and the 9 primitive fields (ro, vx, vy, vz, bx, by, bz,
ei, ph) as one ``(9, i_total, j_total, k_total)`` float64 array in the
reference's layout, set on every cell including ghosts (the reference's
initial conditions loop over the full ``total`` box, e.g.
demo/mhd2d_vortex/src/main.cpp:21-38) -- the caller then fills the ghosts
from their images, as ``MHD::apply_initial_condition`` does (mhd.hpp:28-35).

Units are the reference's Gaussian ones (B^2/8pi, constants.hpp:8-16): a
Heaviside-Lorentz field B_HL is stored as sqrt(4 pi) * B_HL, which is what the
shock-tube demo does with its ``bm`` parameters
(demo/mhd1d_shock_tube/src/main.cpp:63-74).

No public data set is involved: all inputs are synthetic and seeded.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .config import make_config
from .grid import Grid

FIELDS = ("ro", "vx", "vy", "vz", "bx", "by", "bz", "ei", "ph")
RO, VX, VY, VZ, BX, BY, BZ, EI, PH = range(9)
SQRT4PI = math.sqrt(4.0 * math.pi)


@dataclasses.dataclass
class Problem:
    name: str
    grid: Grid
    config: dict
    q: np.ndarray                      # (9, I, J, K) float64, reference layout
    sign: np.ndarray = None            # (3, 2, 9) mirror signs on symmetric faces
    blend: np.ndarray = None           # state the magnetosphere boundary blends toward

    def __post_init__(self):
        if self.sign is None:
            self.sign = np.ones((3, 2, 9))

    @property
    def periodic(self):
        p = self.config["domain"]["periodic"]
        return (bool(p["x"]), bool(p["y"]), bool(p["z"]))


def _alloc(grid: Grid) -> np.ndarray:
    return np.zeros((9,) + grid.shape, dtype=np.float64)


def orszag_tang(n: int = 256, cfl: float = 0.4, gm: float = 5.0 / 3.0) -> Problem:
    """2-D Orszag-Tang vortex on [0, 2pi)^2, periodic.

    rho = 25/(36 pi), p = 5/(12 pi), v = (-sin y, sin x, 0),
    B_HL = (-sin y, sin 2x, 0)/sqrt(4 pi) -> B = (-sin y, sin 2x, 0).
    """
    g = Grid(n, n, 1, 2, 0.0, 2.0 * math.pi, 0.0, 2.0 * math.pi, 0.0, 1.0)
    q = _alloc(g)
    X = g.x[:, None, None]
    Y = g.y[None, :, None]
    ro = 25.0 / (36.0 * math.pi)
    pr = 5.0 / (12.0 * math.pi)
    q[RO] = ro
    q[EI] = pr / (gm - 1.0) / ro
    q[VX] = np.broadcast_to(-np.sin(Y), g.shape)
    q[VY] = np.broadcast_to(np.sin(X), g.shape)
    q[BX] = np.broadcast_to(-np.sin(Y), g.shape)
    q[BY] = np.broadcast_to(np.sin(2.0 * X), g.shape)
    cfgd = make_config(gm, periodic=(True, True, True), cfl_number=cfl)
    return Problem(f"orszag_tang_{n}", g, cfgd, q)


def brio_wu(n: int = 512, axis: int = 0, scale=None, gm: float = 2.0,
            cfl: float = 0.5) -> Problem:
    """1-D Brio-Wu shock tube along ``axis`` on [0, 1], mirror (outflow) faces.

    Left (rho, p, B_perp) = (1, 1, 1), right (0.125, 0.1, -1), B_par = 0.75,
    each of the six left/right values multiplied by ``scale[0..5]``
    (ordering rho_l, p_l, bp_l, rho_r, p_r, bp_r).  The parallel field is the
    axis component; the perpendicular one is the next axis, as in
    demo/mhd1d_shock_tube/src/main.cpp:44-59.
    """
    s = np.ones(6) if scale is None else np.asarray(scale, dtype=np.float64)
    sizes = [1, 1, 1]
    sizes[axis] = n
    g = Grid(*sizes, 2, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    q = _alloc(g)
    coord = (g.x, g.y, g.z)[axis]
    shape = [1, 1, 1]
    shape[axis] = -1
    left = (coord < 0.5).reshape(shape)
    rol, prl, bpl = 1.0 * s[0], 1.0 * s[1], 1.0 * s[2]
    ror, prr, bpr = 0.125 * s[3], 0.1 * s[4], -1.0 * s[5]
    bmain = (BX, BY, BZ)[axis]
    bperp = (BY, BZ, BX)[axis]
    q[RO] = np.where(left, rol, ror)
    q[EI] = np.where(left, prl / (gm - 1.0) / rol, prr / (gm - 1.0) / ror)
    q[bmain] = 0.75 * SQRT4PI
    q[bperp] = np.where(left, bpl * SQRT4PI, bpr * SQRT4PI)
    cfgd = make_config(gm, periodic=(False, False, False), cfl_number=cfl)
    return Problem(f"brio_wu_{n}_{'xyz'[axis]}", g, cfgd, q)


def brio_wu_batch(count: int = 4096, n_min: int = 512, n_max: int = 8192, seed: int = 0):
    """``count`` Brio-Wu instances, sizes U{n_min..n_max}, values scaled U[0.8, 1.2]."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(n_min, n_max + 1, size=count)
    scales = rng.uniform(0.8, 1.2, size=(count, 6))
    return [brio_wu(int(n), 0, sc) for n, sc in zip(sizes, scales)]


def _solenoidal_modes(rng, kmax: float = 4.0):
    """Integer wavevectors 1 <= |k| <= kmax, one of each +-k pair, amplitude
    |k|^-2 (shell energy ~ k^-2), random direction perpendicular to k, random
    phase."""
    r = int(math.floor(kmax))
    modes = []
    for kx in range(-r, r + 1):
        for ky in range(-r, r + 1):
            for kz in range(-r, r + 1):
                k2 = kx * kx + ky * ky + kz * kz
                if k2 == 0 or k2 > kmax * kmax:
                    continue
                if (kx, ky, kz) < (0, 0, 0) and (-kx, -ky, -kz) != (kx, ky, kz):
                    continue
                modes.append((kx, ky, kz))
    k = np.array(modes, dtype=np.float64)
    kn = np.linalg.norm(k, axis=1)
    e = rng.standard_normal((len(k), 3))
    e -= (np.sum(e * k, axis=1) / kn**2)[:, None] * k
    e /= np.linalg.norm(e, axis=1)[:, None]
    amp = kn ** -2.0
    phase = rng.uniform(0.0, 2.0 * math.pi, size=len(k))
    return k.astype(np.int64), (amp[:, None] * e), phase


def _modes_on_grid(g: Grid, k, vec, phase, L=(1.0, 1.0, 1.0), lo=(0.0, 0.0, 0.0)):
    """Sum_k vec_k cos(2 pi k.x / L + phase_k) on every cell, by separable
    contraction over the small set of integer wavenumbers."""
    r = int(np.abs(k).max())
    nk = 2 * r + 1
    out = np.empty((3,) + g.shape)
    ex = np.exp(1j * 2.0 * math.pi * np.outer((g.x - lo[0]) / L[0], np.arange(-r, r + 1)))
    ey = np.exp(1j * 2.0 * math.pi * np.outer((g.y - lo[1]) / L[1], np.arange(-r, r + 1)))
    ez = np.exp(1j * 2.0 * math.pi * np.outer((g.z - lo[2]) / L[2], np.arange(-r, r + 1)))
    for c in range(3):
        C = np.zeros((nk, nk, nk), dtype=np.complex128)
        for (kx, ky, kz), a, ph in zip(k, vec[:, c], phase):
            C[kx + r, ky + r, kz + r] += a * np.exp(1j * ph)
        t1 = np.tensordot(C, ez, axes=([2], [1]))             # (a, b, K)
        t2 = np.tensordot(t1, ey, axes=([1], [1]))            # (a, K, J)
        t2 = np.ascontiguousarray(np.transpose(t2, (0, 2, 1)))  # (a, J, K)
        flat = t2.reshape(nk, -1)
        out[c] = (ex.real @ flat.real - ex.imag @ flat.imag).reshape(g.shape)
    return out


def with_point_gravity(prob: Problem, g: float) -> Problem:
    """``prob`` with the magnetosphere demo's point gravity at the origin
    (demo/mhd3d_magnetosphere/src/src.hpp:17-44): force per volume
    -ro g x / |x|^3 in the momentum equations, no heating.  Sizes must keep
    every cell centre off the origin (even sizes on a centred box)."""
    cfg = dict(prob.config)
    cfg["source"] = {"kind": "point_gravity", "g": float(g)}
    return Problem(prob.name + "_grav", prob.grid, cfg, prob.q, prob.sign)


def magnetosphere(n: int = 128, extent: float = 44.8, radius: float = 3.5,
                  blend_to_initial: bool = True) -> Problem:
    """The magnetosphere demo (demo/mhd3d_magnetosphere: config.yaml and
    src/ic.hpp): a dipole planet at the origin of [-extent, extent]^3 in the
    solar wind, with the demo's boundary (mirror faces, the solar wind held
    in the x-inner ghosts, a blend toward a reference state near the sphere
    r = radius, floors), its CFL with that sphere masked and its point
    gravity.  ro = max(r^-3, 0.2 ro_sw), B the dipole r^-5 (-3xz, -3yz,
    x^2 + y^2 - 2z^2), p = max(p_earth r^-2, p_sw), v = 0, and the solar
    wind on x < x_min + 0.8.  The demo blends toward a field state that it
    allocates and never writes; here ``blend`` is the initial condition
    (zeros with ``blend_to_initial=False``).  Even n keeps cell centres off
    the origin."""
    g = Grid(n, n, n, 2, -extent, extent, -extent, extent, -extent, extent)
    gm = 5.0 / 3.0
    cfg = make_config(gm, periodic=(False, False, False), cfl_number=0.3, ep=1.2, fh=1.0,
                      cs_fac=1.0, ca_fac=0.8, vv_fac=1.0)
    sw = {"mass_density": 5.0e-4, "gas_pressure": 3.56e-8, "x_velocity_field": 0.05,
          "z_magnetic_field": -1.5e-4}
    ms = {"gas_pressure": 5.4e-7, "radius": float(radius), "a0": 100.0,
          "gravitational_acceleration": 1.35e-6}
    cfg["boundary"] = {"kind": "magnetosphere", "cfl_mask": True}
    cfg["solar_wind"] = sw
    cfg["magnetosphere"] = ms
    cfg["floor"] = {"ro_floor": 1.0e-8, "pr_floor": 1.0e-10}
    cfg["source"] = {"kind": "point_gravity", "g": ms["gravitational_acceleration"]}
    X, Y, Z = np.meshgrid(g.x, g.y, g.z, indexing="ij")
    rr = np.sqrt(X * X + Y * Y + Z * Z)
    q = _alloc(g)
    q[RO] = np.maximum(rr ** -3, 0.2 * sw["mass_density"])
    r5 = rr ** -5
    q[BX] = -r5 * 3.0 * X * Z
    q[BY] = -r5 * 3.0 * Y * Z
    q[BZ] = r5 * (X * X + Y * Y - 2.0 * Z * Z)
    pr = np.maximum(ms["gas_pressure"] * rr ** -2, sw["gas_pressure"])
    q[EI] = pr / (gm - 1.0) / q[RO]
    wind = X < g.x_min + 0.8
    q[RO][wind] = sw["mass_density"]
    q[EI][wind] = sw["gas_pressure"] / (gm - 1.0) / sw["mass_density"]
    q[VX][wind] = sw["x_velocity_field"]
    q[BZ][wind] = sw["z_magnetic_field"]
    blend = q.copy() if blend_to_initial else np.zeros_like(q)
    return Problem(f"magnetosphere_{n}", g, cfg, q, None, blend)


def turbulence(n: int = 256, seed: int = 0, mach: float = 0.5, beta: float = 1.0,
               gm: float = 5.0 / 3.0, cfl: float = 0.4, shape=None) -> Problem:
    """3-D decaying MHD turbulence on the periodic unit cube.

    rho = 1, p = 1/gamma (sound speed 1); v and B are independent random
    solenoidal Fourier sums with 1 <= |k| <= 4, E(k) ~ k^-2, scaled so that
    the rms speed is ``mach`` and 8 pi p / <B^2> = ``beta``.  ``shape``
    (i, j, k) gives a grid of unequal cell counts on the same cube.
    """
    ni, nj, nk = (n, n, n) if shape is None else shape
    g = Grid(ni, nj, nk, 2, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    rng = np.random.default_rng(seed)
    q = _alloc(g)
    pr = 1.0 / gm
    q[RO] = 1.0
    q[EI] = pr / (gm - 1.0)
    inner = g.interior
    for base, target in ((VX, None), (BX, None)):
        k, vec, ph = _solenoidal_modes(rng)
        f = _modes_on_grid(g, k, vec, ph)
        ms = float(np.mean(np.sum(f[(slice(None),) + inner] ** 2, axis=0)))
        want = mach * mach if base == VX else 8.0 * math.pi * pr / beta
        f *= math.sqrt(want / ms)
        q[base:base + 3] = f
        del f
    cfgd = make_config(gm, periodic=(True, True, True), cfl_number=cfl)
    return Problem(f"turbulence_{ni}x{nj}x{nk}" if shape else f"turbulence_{n}", g, cfgd, q)


def blast(n: int = 384, seed: int = 0, gm: float = 5.0 / 3.0, cfl: float = 0.4,
          smooth: float = 0.0, shape=None) -> Problem:
    """3-D magnetised blast wave on [-0.5, 0.5]^3 with mirror (outflow) faces.

    Ambient rho = 1, p = 0.1, B_HL = (1, 1, 0)/sqrt(2); inside r < 0.1,
    p = 10 and rho = 1 + 1% seeded uniform noise.  With smooth > 0 the
    sphere's edge is a tanh ramp `smooth` cells wide instead of a step
    (the 100:1 pressure step on fine grids drives the scheme's internal
    energy negative within the first steps).  ``shape`` (i, j, k) gives a
    grid of unequal cell counts on the same cube.
    """
    ni, nj, nk = (n, n, n) if shape is None else shape
    g = Grid(ni, nj, nk, 2, -0.5, 0.5, -0.5, 0.5, -0.5, 0.5)
    rng = np.random.default_rng(seed)
    q = _alloc(g)
    X = g.x[:, None, None]
    Y = g.y[None, :, None]
    Z = g.z[None, None, :]
    r2 = X * X + Y * Y + Z * Z
    inside = r2 < 0.01
    noise = 1.0 + 0.01 * rng.uniform(-1.0, 1.0, size=g.shape)
    if smooth > 0.0:
        w = 0.5 * (1.0 - np.tanh((np.sqrt(r2) - 0.1) / (smooth * g.dx[0])))
        q[RO] = 1.0 + (noise - 1.0) * w
        pr = 0.1 + 9.9 * w
    else:
        q[RO] = np.where(inside, noise, 1.0)
        pr = np.where(inside, 10.0, 0.1)
    q[EI] = pr / (gm - 1.0) / q[RO]
    q[BX] = SQRT4PI / math.sqrt(2.0)
    q[BY] = SQRT4PI / math.sqrt(2.0)
    cfgd = make_config(gm, periodic=(False, False, False), cfl_number=cfl)
    return Problem(f"blast_{ni}x{nj}x{nk}" if shape else f"blast_{n}", g, cfgd, q)


def orszag_tang_batch(count: int = 32, n_min: int = 128, n_max: int = 1024, seed: int = 0):
    """``count`` Orszag-Tang grids of random sizes U{n_min..n_max}^2."""
    rng = np.random.default_rng(seed)
    return [orszag_tang(int(n)) for n in rng.integers(n_min, n_max + 1, size=count)]


def sod(n: int = 128, axis: int = 0, gm: float = 1.4, cfl: float = 0.5) -> Problem:
    """Hydrodynamic Sod shock tube (B = 0) along ``axis`` on [0, 1], mirror
    faces: (rho, p) = (1, 1) for x < 0.5 and (0.125, 0.1) beyond, at rest --
    the configuration of the reference's shock-tube test
    (miso/tests/serial/test_hd1d_shock_tube/config/config_x.yaml)."""
    sizes = [1, 1, 1]
    sizes[axis] = n
    g = Grid(*sizes, 2, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    q = _alloc(g)
    coord = (g.x, g.y, g.z)[axis]
    shape = [1, 1, 1]
    shape[axis] = -1
    left = (coord < 0.5).reshape(shape)
    q[RO] = np.where(left, 1.0, 0.125)
    q[EI] = np.where(left, 1.0 / (gm - 1.0) / 1.0, 0.1 / (gm - 1.0) / 0.125)
    cfgd = make_config(gm, periodic=(False, False, False), cfl_number=cfl)
    return Problem(f"sod_{n}_{'xyz'[axis]}", g, cfgd, q)
