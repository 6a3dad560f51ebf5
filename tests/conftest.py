import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def oracle():
    """The C restatement (built on demand; it is small)."""
    from oracle import oracle as om
    if not os.path.exists(om.ORACLE_SO):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
    return om.Oracle()


@pytest.fixture(scope="session")
def reference():
    """The reference's own host integrator (oracle/_ref), when it was built."""
    from oracle import oracle as om
    if not om.reference_available():
        if os.path.isdir(om.REFERENCE_INCLUDE):
            subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
        else:
            pytest.skip("reference build (oracle/_ref) not available")
    return om.Reference()


def interior(prob, q):
    return q[(slice(None),) + prob.grid.interior]


def rel_l1(a, b):
    """sum |a-b| / sum |b| over all entries."""
    den = float(np.sum(np.abs(b)))
    return float(np.sum(np.abs(a - b))) / (den if den > 0 else 1.0)


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
