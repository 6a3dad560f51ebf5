"""FP32 split-precision form vs the FP64 oracle, through the C ABI.

The split form computes the right-hand side and the artificial viscosity in
FP32 and carries the conserved state as FP32 hi/lo pairs.  Tolerances
(relative L1 over the interior, against the FP64 oracle on the same initial
data and the same number of steps) are stated per case below; the mass and
momentum totals of periodic runs are checked against their initial values.
"""
import numpy as np
import pytest

from conftest import interior, rel_l1
from miso_b200 import problems as P
from miso_b200.integrator import Integrator

pytestmark = pytest.mark.gpu


def run_split(prob, nsteps, graph=False):
    integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision="fp32_split")
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    m0 = integ.monitors()
    if graph:
        integ.run(nsteps, graph=True)
    else:
        for _ in range(nsteps):
            integ.update(integ.cfl())
    integ.sync()
    m1 = integ.monitors()
    out = integ.download()
    integ.close()
    return out, m0, m1


def pressure(q, gm):
    return (gm - 1.0) * q[P.RO] * q[P.EI]


# (case, steps, tolerance on rel L1 of rho, of p, of B)
CASES = [
    ("ot64", lambda: P.orszag_tang(64), 100, 1e-6, 1e-5, 1e-5),
    ("turb16", lambda: P.turbulence(16, seed=1), 20, 1e-6, 1e-5, 1e-5),
    ("blast16", lambda: P.blast(16, seed=1), 20, 1e-6, 1e-5, 1e-5),
    ("bw_x", lambda: P.brio_wu(256), 200, 1e-5, 1e-5, 1e-5),
]


@pytest.mark.parametrize("name,make,nsteps,tol_ro,tol_p,tol_b", CASES,
                         ids=[c[0] for c in CASES])
def test_split_vs_fp64_oracle(name, make, nsteps, tol_ro, tol_p, tol_b, oracle):
    prob = make()
    ref = prob.q.copy()
    oracle.run(prob, ref, nsteps)
    out, m0, m1 = run_split(prob, nsteps)
    a, b = interior(prob, out), interior(prob, ref)
    gm = prob.config["eos"]["gm"]
    e_ro = rel_l1(a[P.RO], b[P.RO])
    e_p = rel_l1(pressure(a, gm), pressure(b, gm))
    e_b = rel_l1(a[P.BX:P.BZ + 1], b[P.BX:P.BZ + 1])
    print(f"{name}: L1 rho {e_ro:.2e} p {e_p:.2e} B {e_b:.2e}")
    assert e_ro <= tol_ro
    assert e_p <= tol_p
    assert e_b <= tol_b


def test_split_conservation_periodic():
    """Periodic turbulence: total mass and momentum drift at round-off level."""
    prob = P.turbulence(16, seed=4)
    out, m0, m1 = run_split(prob, 40, graph=True)
    print(m0, m1)
    assert abs(m1["mass"] - m0["mass"]) <= 1e-9 * abs(m0["mass"])
    scale = abs(m0["mass"])  # momentum scale: rho * v_rms * volume
    for k in ("mom_x", "mom_y", "mom_z"):
        assert abs(m1[k] - m0[k]) <= 1e-8 * scale
