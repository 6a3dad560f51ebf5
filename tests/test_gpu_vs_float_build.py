"""The split form against the reference's own Real = float build (the type
its demos use), both measured against the Real = double build stepped with
the same dt sequence: the split form's error must be the smaller one."""
import pytest

from conftest import interior, rel_l1
from miso_b200 import problems as P
from miso_b200.integrator import Integrator

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make,nsteps", [(lambda: P.orszag_tang(64), 50),
                                         (lambda: P.turbulence(32, seed=2), 10),
                                         (lambda: P.blast(24, seed=3), 10)],
                         ids=["ot64", "turb32", "blast24"])
def test_split_form_beats_float_build(make, nsteps, reference):
    from oracle import oracle as om
    if not om.os.path.exists(om.REF_F32_SO):
        pytest.skip("Real = float reference build not available")
    f32 = om.ReferenceF32()
    prob = make()
    q64, q32 = prob.q.copy(), prob.q.copy()
    reference.fill_ghosts(prob, q64)
    f32.fill_ghosts(prob, q32)
    integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision="fp32_split")
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    for _ in range(nsteps):
        dt = reference.cfl(prob, q64)
        reference.update(prob, q64, dt)
        f32.update(prob, q32, dt)
        integ.update(dt)
    split = integ.download()
    integ.close()
    b = interior(prob, q64)
    e_split = rel_l1(interior(prob, split)[P.RO], b[P.RO])
    e_float = rel_l1(interior(prob, q32)[P.RO], b[P.RO])
    print(f"{prob.name}: rel L1 of ro vs the double build -- split {e_split:.3e}, "
          f"float build {e_float:.3e}")
    assert e_split < e_float
