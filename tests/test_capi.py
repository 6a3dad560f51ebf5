"""The C ABI library: it loads, exports every entry point include/miso_b200.h
declares (and the Python binding knows each one), and rejects invalid
descriptors before touching the device.  No compute calls: these run
without a GPU."""
import ctypes
import os
import re

import pytest

from miso_b200 import _lib
from miso_b200.grid import Grid
from miso_b200 import problems as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "miso_b200.h")).read()
    return sorted(set(re.findall(r"\b(miso_b200_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no Python binding"


def test_binding_covers_only_declared_symbols():
    assert set(_lib.SIGNATURES) <= set(declared_symbols())


def test_version_string():
    assert _lib.load().miso_b200_version().startswith(b"miso_b200")


def _descs(grid, **over):
    from miso_b200.integrator import make_descs
    gd, pp = make_descs(P.turbulence(8).config, grid)
    for k, v in over.items():
        setattr(pp if hasattr(pp, k) else gd, k, v)
    return gd, pp


@pytest.mark.parametrize("field,value", [("margin", 1), ("i_size", 0), ("gm", 1.0),
                                         ("cfl_number", 0.0), ("precision", 7), ("ep", -1.0)])
def test_create_rejects_bad_descriptor(field, value):
    lib = _lib.load()
    gd, pp = _descs(Grid(8, 8, 8), **{field: value})
    h = ctypes.c_void_p()
    rc = lib.miso_b200_create(ctypes.byref(gd), ctypes.byref(pp), None, ctypes.byref(h))
    assert rc == _lib.ERR_ARG
    assert not h.value
    assert lib.miso_b200_last_error(None)


def test_null_arguments():
    lib = _lib.load()
    assert lib.miso_b200_create(None, None, None, None) == _lib.ERR_ARG
    assert lib.miso_b200_destroy(None) == _lib.ERR_ARG
    assert lib.miso_b200_sync(None) == _lib.ERR_ARG
    assert lib.miso_b200_update(None, 1e-3) == _lib.ERR_ARG
    assert lib.miso_b200_set_source(None, 1, None, 0) == _lib.ERR_ARG
    assert lib.miso_b200_set_halo(None, 1, 1, None) == _lib.ERR_ARG
    assert lib.miso_b200_set_halo3(None, None, None) == _lib.ERR_ARG


def test_cfl_noalloc_refuses_host_arrays_before_any_call():
    """The allocation-free CFL entry point takes device memory only: the
    Python binding refuses a numpy array, a CPU tensor and a tensor of the
    wrong shape before the library is called (no GPU needed)."""
    import numpy as np
    import torch
    from miso_b200.integrator import cfl_noalloc
    prob = P.orszag_tang(16)
    with pytest.raises(ValueError, match="CUDA tensor"):
        cfl_noalloc(prob.config, prob.grid, prob.q)
    with pytest.raises(ValueError, match="CUDA tensor"):
        cfl_noalloc(prob.config, prob.grid, torch.from_numpy(prob.q))
    small = np.zeros((9, 4, 4, 1))
    with pytest.raises(ValueError):
        cfl_noalloc(prob.config, prob.grid, small)
