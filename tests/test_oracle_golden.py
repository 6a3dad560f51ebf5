"""The oracle against committed golden fixtures.

The fixtures (tests/golden/*.npz) were produced by the reference's own host
integrator through tests/golden/make_golden.py; the restatement must
reproduce every time step and every interior value exactly.  This pins the
oracle where the reference sources are not available.
"""
import os

import numpy as np
import pytest

from conftest import interior

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def cases():
    import sys
    sys.path.insert(0, GOLDEN)
    from make_golden import CASES
    return CASES


@pytest.mark.parametrize("name", sorted(cases()))
def test_oracle_reproduces_golden(name, oracle):
    make, nsteps = cases()[name]
    data = np.load(os.path.join(GOLDEN, name + ".npz"))
    prob = make()
    q = prob.q.copy()
    dts = oracle.run(prob, q, nsteps)
    assert np.array_equal(dts, data["dt"])
    assert np.array_equal(interior(prob, q), data["interior"])
