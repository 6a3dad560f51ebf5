"""Accuracy of the FP32 split form against the FP64 form on the same
initial data and time steps (miso_b200/accuracy.py): relative L1 of density
at or below 1e-6 after 1000 steps of 3-D turbulence, and total mass kept to
round-off in both forms (momentum and energy drifts are reported)."""
import pytest

from miso_b200 import problems as P
from miso_b200.accuracy import compare

pytestmark = pytest.mark.gpu


def test_turbulence_64_200_steps():
    rec = compare(P.turbulence(64, seed=0), steps=200, every=200, emit=lambda s: None)
    assert rec["l1_rho"] <= 1e-6
    assert rec["l1_p"] <= 1e-5 and rec["l1_B"] <= 1e-5
    for form in ("drift_fp64", "drift_split"):
        assert abs(rec[form]["mass"]) <= 1e-9


@pytest.mark.slow
def test_turbulence_256_1000_steps():
    """The turbulence configuration at its stated size and step count."""
    rec = compare(P.turbulence(256, seed=0), steps=1000, every=1000, emit=lambda s: None)
    print(rec)
    assert rec["l1_rho"] <= 1e-6
