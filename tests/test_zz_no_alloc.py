"""The allocation-free CFL entry point, miso_b200_cfl_noalloc.

Some callers of this library cannot let it allocate device memory:
applications that give every byte of device memory to their own pool or
hold it to a fixed budget, and applications whose other streams must not be
stalled by the device-wide synchronisation that cudaMalloc / cudaFree can
cause.  miso_b200_cfl_noalloc serves them: it computes the CFL time step of
9 FP64 device arrays the caller owns, with no handle and no cudaMalloc,
using a fixed scratch array inside the library.

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


def test_noalloc_cfl_leaves_device_memory_alone():
    """After a first call (which may load the library's device code), more
    calls leave the device's free memory exactly where it was: nothing is
    allocated behind the caller's back."""
    import torch
    prob = P.turbulence(24, seed=3)
    dev = torch.from_numpy(prob.q).to("cuda")
    first = cfl_noalloc(prob.config, prob.grid, dev)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        assert cfl_noalloc(prob.config, prob.grid, dev) == first
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_refuses_host_and_short_arrays():
    """Through the C ABI directly: pointers to host memory and device arrays
    shorter than the grid are refused with MISO_B200_ERR_ARG before any
    launch."""
    import numpy as np
    import torch
    lib = _lib.load()
    prob = P.orszag_tang(32)
    gd, pp = make_descs(prob.config, prob.grid)
    dt = ctypes.c_double()
    host = np.ascontiguousarray(prob.q)
    ptrs = (ctypes.c_void_p * 9)(*[host[f].ctypes.data for f in range(9)])
    rc = lib.miso_b200_cfl_noalloc(ctypes.byref(gd), ctypes.byref(pp), ptrs, None,
                                   ctypes.byref(dt))
    assert rc == _lib.ERR_ARG
    assert b"not device memory" in lib.miso_b200_last_error(None)
    # the last field array placed so that it would end one cell past the end
    # of its device allocation (torch's segment): refused, nothing launched
    cells = int(np.prod(prob.grid.shape))
    buf = torch.zeros(9 * cells, dtype=torch.float64, device="cuda")
    seg = [s for s in torch.cuda.memory_snapshot()
           if s["address"] <= buf.data_ptr() < s["address"] + s["total_size"]]
    assert len(seg) == 1
    seg_end = seg[0]["address"] + seg[0]["total_size"]
    addrs = [buf.data_ptr() + f * cells * 8 for f in range(8)]
    addrs.append(seg_end - (cells - 1) * 8)
    assert addrs[8] >= buf.data_ptr()
    ptrs = (ctypes.c_void_p * 9)(*addrs)
    rc = lib.miso_b200_cfl_noalloc(ctypes.byref(gd), ctypes.byref(pp), ptrs, None,
                                   ctypes.byref(dt))
    assert rc == _lib.ERR_ARG
    assert b"shorter than the grid" in lib.miso_b200_last_error(None)
    # the same arrays laid out inside the allocation are accepted
    ptrs = (ctypes.c_void_p * 9)(*[buf.data_ptr() + f * cells * 8 for f in range(9)])
    buf.view(9, -1)[0].fill_(1.0)  # ro = 1
    buf.view(9, -1)[7].fill_(1.0)  # ei = 1
    torch.cuda.synchronize()
    rc = lib.miso_b200_cfl_noalloc(ctypes.byref(gd), ctypes.byref(pp), ptrs, None,
                                   ctypes.byref(dt))
    assert rc == _lib.OK and dt.value > 0.0


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
