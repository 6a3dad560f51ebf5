"""The allocation-free CFL entry point, miso_b200_cfl_noalloc.

Some callers of this library cannot let it allocate device memory: code
that runs while a stream is being captured into a CUDA graph, loops that
must not synchronise the device, and hosts that own every byte of device
memory through their own pool.  miso_b200_cfl_noalloc serves them: it
computes the CFL time step of 9 FP64 device arrays the caller owns, with no
handle and no cudaMalloc, using a fixed scratch array inside the library.

This file is collected last so that a run stopping at its first failure has
already run every other test; it passes alone in a fresh process as well.
"""
import ctypes

import pytest

from miso_b200 import _lib
from miso_b200 import problems as P
from miso_b200.integrator import Integrator, cfl_noalloc, make_descs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make", [lambda: P.orszag_tang(64), lambda: P.turbulence(16, seed=2),
                                  lambda: P.brio_wu(200)], ids=["ot64", "turb16", "bw200"])
def test_noalloc_cfl_matches_handle_cfl_two_calls(make):
    import torch
    prob = make()
    integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision="fp64")
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    dev = torch.empty((9,) + prob.grid.shape, dtype=torch.float64, device="cuda")
    for call in range(2):
        dt_handle = integ.cfl()
        dev.copy_(torch.from_numpy(integ.download()))
        torch.cuda.synchronize()
        dt_noalloc = cfl_noalloc(prob.config, prob.grid, dev)
        # the reduction is an exact float minimum: both paths agree bit for bit
        assert dt_noalloc == dt_handle, (call, dt_noalloc, dt_handle)
        integ.update(dt_handle)  # a new state for the second call
    integ.close()


def test_noalloc_rejects_oversized_grid():
    lib = _lib.load()
    from miso_b200.grid import Grid
    g = Grid(1024, 1024, 257, 2)
    gd, pp = make_descs(P.turbulence(8).config, g)
    ptrs = (ctypes.c_void_p * 9)(*([1] * 9))
    dt = ctypes.c_double()
    rc = lib.miso_b200_cfl_noalloc(ctypes.byref(gd), ctypes.byref(pp), ptrs, None,
                                   ctypes.byref(dt))
    assert rc == _lib.ERR_ARG
    assert b"too large" in lib.miso_b200_last_error(None)
