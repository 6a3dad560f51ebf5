"""Host-side logic: the grid and configuration mirrors and the problem
generators, checked against the oracle and the reference's rules."""
import math

import numpy as np
import pytest

from miso_b200 import problems as P
from miso_b200.config import DEFAULTS, make_config, merge_defaults
from miso_b200.grid import Grid
from oracle.oracle import make_desc


@pytest.mark.parametrize("shape", [(16, 16, 1), (32, 1, 1), (1, 1, 20), (7, 9, 11)])
def test_grid_matches_oracle_axes(oracle, shape):
    import ctypes
    g = Grid(*shape, 2, -0.3, 0.7, 0.0, 2.0, 1.0, 4.0)
    d = make_desc(g, make_config(1.4))
    for axis, (s, ds, dsi) in enumerate(((g.x, g.dx, g.dxi), (g.y, g.dy, g.dyi),
                                         (g.z, g.dz, g.dzi))):
        n = len(s)
        a, b, c = np.zeros(n), np.zeros(n), np.zeros(n)
        oracle._lib = getattr(oracle, "lib")
        f = oracle.lib.miso_oracle_axis
        f.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.POINTER(ctypes.c_double)] * 3
        assert f(ctypes.byref(d), axis, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                 b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                 c.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0
        assert np.array_equal(a, s) and np.array_equal(b, ds) and np.array_equal(c, dsi)
    prob = P.Problem("g", g, make_config(1.4), np.zeros((9,) + g.shape))
    assert g.min_dxyz == oracle.min_dxyz(prob)


def test_degenerate_axis_rules():
    g = Grid(64, 1, 1)
    assert g.shape == (68, 1, 1)
    assert (g.is_, g.js, g.ks) == (1, 0, 0)
    assert g.dy[0] == 1e30 and g.dyi[0] == 0.0
    assert g.ndim == 1


@pytest.mark.parametrize("bad", [dict(margin=0), dict(i_size=0), dict(x_min=1.0, x_max=0.5)])
def test_grid_argument_checks(bad):
    args = dict(i_size=8, j_size=8, k_size=8, margin=2, x_min=0.0, x_max=1.0)
    args.update(bad)
    with pytest.raises(ValueError):
        Grid(**args)


def test_config_defaults():
    cfg = merge_defaults({"eos": {"gm": 1.4}, "mhd": None})
    assert cfg["mhd"]["cfl_number"] == 0.5
    assert cfg["mhd"]["artificial_viscosity"] == DEFAULTS["mhd"]["artificial_viscosity"]
    cfg2 = make_config(2.0, cfl_number=0.3, ep=1.5)
    assert cfg2["mhd"]["cfl_number"] == 0.3
    assert cfg2["mhd"]["artificial_viscosity"]["ep"] == 1.5
    with pytest.raises(KeyError):
        make_config(2.0, eps=1.0)


def test_orszag_tang_initial_state():
    p = P.orszag_tang(32)
    gm = p.config["eos"]["gm"]
    pr = (gm - 1.0) * p.q[P.RO] * p.q[P.EI]
    np.testing.assert_allclose(pr, 5.0 / (12.0 * math.pi), rtol=1e-14)
    np.testing.assert_allclose(p.q[P.RO], 25.0 / (36.0 * math.pi))
    assert p.periodic == (True, True, True)


def test_turbulence_scales_and_divergence():
    p = P.turbulence(24, seed=5)
    inner = (slice(None),) + p.grid.interior
    v = p.q[P.VX:P.VZ + 1][inner]
    b = p.q[P.BX:P.BZ + 1][inner]
    assert abs(math.sqrt(np.mean(np.sum(v * v, axis=0))) - 0.5) < 1e-12
    gm = p.config["eos"]["gm"]
    assert abs(8 * math.pi * (1 / gm) / np.mean(np.sum(b * b, axis=0)) - 1.0) < 1e-12
    # spectral divergence of the analytic field vanishes; the 4th-order
    # difference of the sampled field is small compared with |grad B|
    dx = p.grid.dx[0]
    q = p.q
    def d4(a, ax):
        return (-np.roll(a, -2, ax) + 8 * np.roll(a, -1, ax) - 8 * np.roll(a, 1, ax)
                + np.roll(a, 2, ax)) / (12 * dx)
    bx, by, bz = (q[P.BX + c][p.grid.interior] for c in range(3))
    div = d4(bx, 0) + d4(by, 1) + d4(bz, 2)
    grad = np.abs(d4(bx, 0)) + np.abs(d4(by, 1)) + np.abs(d4(bz, 2))
    assert np.mean(np.abs(div[4:-4, 4:-4, 4:-4])) < 0.05 * np.mean(grad)


def test_brio_wu_batch_is_seeded():
    a = P.brio_wu_batch(6, 64, 96, seed=3)
    b = P.brio_wu_batch(6, 64, 96, seed=3)
    assert [x.grid.i_size for x in a] == [x.grid.i_size for x in b]
    assert all(64 <= x.grid.i_size <= 96 for x in a)
    assert all(np.array_equal(x.q, y.q) for x, y in zip(a, b))


def test_magnetosphere_initial_state():
    """The magnetosphere demo's initial condition (demo/mhd3d_magnetosphere/
    src/ic.hpp) at a few cells, the demo's configuration sections, and the
    blend state (the initial condition, or zeros)."""
    from miso_b200 import problems as P
    prob = P.magnetosphere(16, extent=12.0)
    g, q, cfg = prob.grid, prob.q, prob.config
    sw, ms = cfg["solar_wind"], cfg["magnetosphere"]
    gm = cfg["eos"]["gm"]
    for i, j, k in [(10, 9, 11), (3, 12, 7), (9, 9, 9)]:
        x, y, z = g.x[i], g.y[j], g.z[k]
        r = np.sqrt(x * x + y * y + z * z)
        assert np.isclose(q[P.RO][i, j, k], max(r ** -3, 0.2 * sw["mass_density"]), rtol=1e-14)
        assert np.isclose(q[P.BX][i, j, k], -3.0 * x * z * r ** -5, rtol=1e-12)
        assert np.isclose(q[P.BZ][i, j, k], (x * x + y * y - 2 * z * z) * r ** -5, rtol=1e-12,
                          atol=1e-300)
        pr = max(ms["gas_pressure"] * r ** -2, sw["gas_pressure"])
        assert np.isclose(q[P.EI][i, j, k], pr / (gm - 1.0) / q[P.RO][i, j, k], rtol=1e-13)
        assert q[P.VX][i, j, k] == 0.0 and q[P.PH][i, j, k] == 0.0
    # the solar wind on the first layer (x < x_min + 0.8)
    assert np.all(q[P.RO][0] == sw["mass_density"]) and np.all(q[P.VX][0] == sw["x_velocity_field"])
    assert cfg["boundary"] == {"kind": "magnetosphere", "cfl_mask": True}
    assert cfg["source"] == {"kind": "point_gravity", "g": ms["gravitational_acceleration"]}
    assert np.array_equal(prob.blend, q) and prob.blend is not q
    assert not np.any(P.magnetosphere(16, extent=12.0, blend_to_initial=False).blend)
