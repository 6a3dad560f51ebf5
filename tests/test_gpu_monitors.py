"""miso_b200_monitors against the same totals formed in numpy from the
downloaded state: mass, momentum, total energy, the L1 norm and maximum of
div B (4th-order central differences), and the integral of ph^2.  Grids
with 32 or more cells along k are summed by whole k rows, the others cell
by cell; both forms."""
import numpy as np
import pytest

from miso_b200 import problems as P
from miso_b200.integrator import Integrator

pytestmark = pytest.mark.gpu

PII8 = 1.0 / (8.0 * np.pi)


def totals(prob, q):
    g = prob.grid
    it = (slice(None),) + g.interior
    u = q[it]
    ro, vx, vy, vz = u[P.RO], u[P.VX], u[P.VY], u[P.VZ]
    bx, by, bz = u[P.BX], u[P.BY], u[P.BZ]
    sizes = (g.i_size, g.j_size, g.k_size)
    spacing = (g.dx[0], g.dy[0], g.dz[0])
    dv = float(np.prod([spacing[a] for a in range(3) if sizes[a] > 1]))
    et = ro * u[P.EI] + 0.5 * ro * (vx * vx + vy * vy + vz * vz) + PII8 * (bx * bx + by * by +
                                                                          bz * bz)
    divb = np.zeros_like(ro)
    margins = (g.i_margin, g.j_margin, g.k_margin)
    for a in range(3):
        if sizes[a] == 1:
            continue
        b = q[P.BX + a]

        def sh(o):
            sl = [slice(margins[d], margins[d] + sizes[d]) for d in range(3)]
            sl[a] = slice(margins[a] + o, margins[a] + o + sizes[a])
            return b[tuple(sl)]
        divb += (-sh(2) + 8.0 * sh(1) - 8.0 * sh(-1) + sh(-2)) / 12.0 / spacing[a]
    return {"mass": ro.sum() * dv, "mom_x": (ro * vx).sum() * dv, "mom_y": (ro * vy).sum() * dv,
            "mom_z": (ro * vz).sum() * dv, "energy": et.sum() * dv,
            "divb_l1": np.abs(divb).sum() * dv, "divb_max": np.abs(divb).max(),
            "ph2": (u[P.PH] ** 2).sum() * dv, "scale_mom": (ro * np.abs(vx) + ro * np.abs(vy) +
                                                         ro * np.abs(vz)).sum() * dv}


@pytest.mark.parametrize("precision", ["fp64", "fp32_split"])
@pytest.mark.parametrize("make", [lambda: P.turbulence(40, seed=3), lambda: P.blast(20, seed=5),
                                  lambda: P.orszag_tang(64)],
                         ids=["turb40_rows", "blast20_cells", "ot64_cells"])
def test_monitors_match_numpy(make, precision):
    prob = make()
    integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision=precision)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    for _ in range(3):
        integ.update(integ.cfl())
    m = integ.monitors()
    q = integ.download()
    integ.close()
    t = totals(prob, q)
    assert abs(m["mass"] - t["mass"]) <= 1e-13 * abs(t["mass"])
    assert abs(m["energy"] - t["energy"]) <= 1e-12 * abs(t["energy"])
    for k in ("mom_x", "mom_y", "mom_z"):
        assert abs(m[k] - t[k]) <= 1e-12 * t["scale_mom"], k
    assert abs(m["divb_l1"] - t["divb_l1"]) <= 1e-9 * t["divb_l1"] + 1e-300
    assert abs(m["divb_max"] - t["divb_max"]) <= 1e-9 * t["divb_max"] + 1e-300
    assert abs(m["ph2"] - t["ph2"]) <= 1e-9 * t["ph2"] + 1e-300


@pytest.mark.parametrize("make", [lambda: P.turbulence(40, seed=3), lambda: P.blast(36, seed=5)],
                         ids=["turb40", "blast36"])
@pytest.mark.parametrize("graph", [False, True], ids=["eager", "graph"])
def test_fused_monitors_match_numpy(make, graph):
    """Monitors folded into the step (the z sweep sums the new state, a div B
    kernel reads bx, by, bz): the same totals as numpy on the downloaded
    state, and the step itself is unchanged bit for bit."""
    prob = make()
    outs = []
    for fuse in (True, False):
        integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision="fp32_split")
        integ.upload(prob.q)
        integ.apply_boundary_condition()
        if fuse:
            integ.set_monitor_fusion(True)
        if graph:
            integ.run(4, graph=True)
        else:
            for _ in range(4):
                integ.update(integ.cfl())
        m = integ.monitors()
        q = integ.download()
        integ.close()
        outs.append(q)
        t = totals(prob, q)
        assert abs(m["mass"] - t["mass"]) <= 1e-13 * abs(t["mass"])
        assert abs(m["energy"] - t["energy"]) <= 1e-12 * abs(t["energy"])
        for k in ("mom_x", "mom_y", "mom_z"):
            assert abs(m[k] - t[k]) <= 1e-12 * t["scale_mom"], k
        assert abs(m["divb_l1"] - t["divb_l1"]) <= 1e-9 * t["divb_l1"] + 1e-300
        assert abs(m["divb_max"] - t["divb_max"]) <= 1e-9 * t["divb_max"] + 1e-300
        assert abs(m["ph2"] - t["ph2"]) <= 1e-9 * t["ph2"] + 1e-300
    assert np.array_equal(outs[0], outs[1])
