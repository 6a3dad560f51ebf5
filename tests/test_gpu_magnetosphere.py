"""The magnetosphere demo's boundary and masked CFL on the FP64 form,
through the C ABI, against the oracle (itself pinned bit for bit to the
reference build running a restatement of the demo's boundary functor):
every time step and every interior value equal, with the state blended
toward the initial condition or toward zeros."""
import numpy as np
import pytest

from conftest import interior
from miso_b200 import _lib
from miso_b200 import problems as P
from miso_b200.integrator import Integrator

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,blend,steps", [(16, True, 6), (16, False, 4), (20, True, 4)],
                         ids=["n16_blend_ic", "n16_blend_zero", "n20_blend_ic"])
def test_fp64_bit_exact_with_oracle(n, blend, steps, oracle):
    prob = P.magnetosphere(n, extent=12.0, blend_to_initial=blend)
    ref = prob.q.copy()
    dts_o = oracle.run(prob, ref, steps)
    integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision="fp64",
                       blend=prob.blend)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    dts = []
    for _ in range(steps):
        dt = integ.cfl()
        integ.update(dt)
        dts.append(dt)
    out = integ.download()
    integ.close()
    assert np.array_equal(np.array(dts), dts_o), (dts[:3], dts_o[:3])
    a, b = interior(prob, out), interior(prob, ref)
    assert np.array_equal(a, b), float(np.max(np.abs(a - b)))


def test_masked_cfl_and_boundary_act(oracle):
    """The boundary changes the state (the blend and the inflow) and the
    mask changes the step, on the device as in the oracle."""
    prob = P.magnetosphere(16, extent=12.0)
    q = prob.q.copy()
    oracle.fill_ghosts(prob, q)
    integ = Integrator(prob.config, prob.grid, precision="fp64", blend=prob.blend)
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    assert integ.cfl() == oracle.cfl(prob, q)
    assert np.array_equal(interior(prob, integ.download()), interior(prob, q))
    integ.close()
    plain = P.magnetosphere(16, extent=12.0)
    plain.config["boundary"]["cfl_mask"] = False
    integ = Integrator(plain.config, plain.grid, precision="fp64", blend=plain.blend)
    integ.upload(plain.q)
    integ.apply_boundary_condition()
    dt_plain = integ.cfl()
    integ.close()
    assert dt_plain == oracle.cfl(plain, q) and dt_plain != oracle.cfl(prob, q)


@pytest.mark.parametrize("n,steps", [(24, 6), (32, 4)], ids=["n24", "n32"])
def test_split_form_follows_fp64(n, steps):
    """The FP32 split form with the magnetosphere boundary (its per-cell
    kernels, the boundary on the split state after every pass, the masked
    CFL) stepped with the FP64 form's dt sequence: relative L1 of rho
    <= 1e-7, of p <= 1e-5 and of B <= 1e-6; its own CFL within 1e-4 of
    FP64's (the time step is the minimum over cells, so it follows the few
    cells that set it, not the L1 average).

    The grids keep the FP64 solution off the floors.  On a coarser one
    (16 cells over [-12, 12]) a single step drives the cells just outside
    the inner sphere to the pressure floor (1e-10, beta near 1e-14), where
    the thermal energy is 1e-7 of the total: below what an FP32 word of the
    total energy resolves, so the split form's pressure there is rounding
    (relative L1 of p 3.6e-5 after one step, of rho 3.6e-6), while the same
    grid with a zero blend state stays at 5e-8 in rho."""
    prob = P.magnetosphere(n, extent=12.0)
    ref = Integrator(prob.config, prob.grid, sign=prob.sign, precision="fp64", blend=prob.blend)
    ref.upload(prob.q)
    ref.apply_boundary_condition()
    sp = Integrator(prob.config, prob.grid, sign=prob.sign, precision="fp32_split",
                    blend=prob.blend)
    sp.upload(prob.q)
    sp.apply_boundary_condition()
    for _ in range(steps):
        dt = ref.cfl()
        assert abs(sp.cfl() - dt) <= 1e-4 * dt
        ref.update(dt)
        sp.update(dt)
    a, b = interior(prob, sp.download()), interior(prob, ref.download())
    sp.close()
    ref.close()
    gm = prob.config["eos"]["gm"]

    def rl1(x, y):
        return float(np.sum(np.abs(x - y)) / np.sum(np.abs(y)))
    assert rl1(a[P.RO], b[P.RO]) <= 1e-7
    assert rl1(a[P.RO] * a[P.EI] * (gm - 1), b[P.RO] * b[P.EI] * (gm - 1)) <= 1e-5
    assert rl1(a[P.BX:P.BZ + 1], b[P.BX:P.BZ + 1]) <= 1e-6


def test_refusals():
    prob = P.magnetosphere(16, extent=12.0)
    per = P.turbulence(16, seed=1)
    per.config["boundary"] = dict(prob.config["boundary"])
    for key in ("solar_wind", "magnetosphere", "floor"):
        per.config[key] = prob.config[key]
    with pytest.raises(_lib.MisoError) as e:
        Integrator(per.config, per.grid, precision="fp64")
    assert e.value.code == _lib.ERR_ARG
