"""ctypes binding of libmiso_b200.so (the C ABI of include/miso_b200.h).

The library is loaded from ``miso_b200/lib/`` (built in-tree by
``miso_b200.build``).  There is no fallback: if the shared library is
missing, importing the solver raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libmiso_b200.so")

OK = 0
ERR_ARG = -1
ERR_CUDA = -2
ERR_NONFINITE = -3
ERR_STATE = -4
ERR_NOMEM = -5
ERR_TIMEOUT = -6
ERR_HALO = -7
ERR_CALLBACK = -8

# int (*)(void *user, double *const q[9], void *stream)
BOUNDARY_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p,
                               ctypes.POINTER(ctypes.c_size_t), ctypes.c_void_p)
# miso_b200_source_fn: (user, const double *const q[9], double *const s[4], stream)
SOURCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t),
                             ctypes.POINTER(ctypes.c_size_t), ctypes.c_void_p)

FP64 = 0
FP32_SPLIT = 1

_dp = ctypes.POINTER(ctypes.c_double)


class GridDesc(ctypes.Structure):
    _fields_ = [("i_size", ctypes.c_int), ("j_size", ctypes.c_int), ("k_size", ctypes.c_int),
                ("margin", ctypes.c_int),
                ("x_min", ctypes.c_double), ("x_max", ctypes.c_double),
                ("y_min", ctypes.c_double), ("y_max", ctypes.c_double),
                ("z_min", ctypes.c_double), ("z_max", ctypes.c_double),
                ("periodic", ctypes.c_int * 3),
                ("sign", ctypes.c_double * 54)]


class Params(ctypes.Structure):
    _fields_ = [("gm", ctypes.c_double), ("cfl_number", ctypes.c_double),
                ("ep", ctypes.c_double), ("fh", ctypes.c_double),
                ("cs_fac", ctypes.c_double), ("ca_fac", ctypes.c_double),
                ("vv_fac", ctypes.c_double), ("precision", ctypes.c_int)]


_vpp = ctypes.POINTER(ctypes.c_void_p)
# int exchange(user, narrays, bytes, ext_lo, ext_hi, send_lo, send_hi, recv_lo, recv_hi, stream)
HALO_EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t,
                                    ctypes.c_int, ctypes.c_int, _vpp, _vpp, _vpp, _vpp,
                                    ctypes.c_void_p)
# int min_all(user, double *value)
HALO_MIN_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, _dp)


class HaloOps(ctypes.Structure):
    _fields_ = [("exchange", HALO_EXCHANGE_FN), ("min_all", HALO_MIN_FN),
                ("user", ctypes.c_void_p)]


# int exchange(user, axis, narrays, bytes, ext_lo, ext_hi, send_lo, send_hi, recv_lo, recv_hi,
#              stream)
HALO3_EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_size_t, ctypes.c_int, ctypes.c_int, _vpp, _vpp, _vpp,
                                     _vpp, ctypes.c_void_p)


class Halo3Ops(ctypes.Structure):
    _fields_ = [("exchange", HALO3_EXCHANGE_FN), ("min_all", HALO_MIN_FN),
                ("user", ctypes.c_void_p)]


# name -> (restype, argtypes); the exported set must match include/miso_b200.h
SIGNATURES = {
    "miso_b200_create": (ctypes.c_int, [ctypes.POINTER(GridDesc), ctypes.POINTER(Params),
                                        ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "miso_b200_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "miso_b200_upload": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "miso_b200_download": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "miso_b200_download_async": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                                ctypes.c_void_p]),
    "miso_b200_fill_ghosts": (ctypes.c_int, [ctypes.c_void_p]),
    "miso_b200_cfl": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "miso_b200_update": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "miso_b200_update_device": (ctypes.c_int, [ctypes.c_void_p]),
    "miso_b200_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "miso_b200_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "miso_b200_last_dt": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "miso_b200_monitors": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "miso_b200_fields_view": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "miso_b200_device_bytes": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t)]),
    "miso_b200_launch_count": (ctypes.c_int, [ctypes.c_void_p,
                                              ctypes.POINTER(ctypes.c_longlong)]),
    "miso_b200_set_source": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp, ctypes.c_int]),
    "miso_b200_set_boundary": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp, ctypes.c_int]),
    "miso_b200_set_blend_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "miso_b200_set_halo": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(HaloOps)]),
    "miso_b200_alloc_shared": (ctypes.c_int, [ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p)]),
    "miso_b200_free_shared": (ctypes.c_int, [ctypes.c_void_p]),
    "miso_b200_set_halo3": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(Halo3Ops)]),
    "miso_b200_set_variant": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "miso_b200_set_chunks": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "miso_b200_set_monitor_fusion": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "miso_b200_set_wait_limit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong]),
    "miso_b200_arm_timeout_test": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong]),
    "miso_b200_pointer_kind": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "miso_b200_batch_set_chunks": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "miso_b200_batch_set_variant": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "miso_b200_batch_views": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "miso_b200_run_until": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                           ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_int)]),
    "miso_b200_set_halo_overlap": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "miso_b200_set_mirror_signs": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    "miso_b200_set_boundary_callback": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p,
                                                       ctypes.c_void_p, ctypes.c_int]),
    "miso_b200_set_source_callback": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p,
                                                     ctypes.c_void_p, ctypes.c_int]),
    "miso_b200_get_variant": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_int)]),
    "miso_b200_set_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "miso_b200_timing_report": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "miso_b200_cfl_noalloc": (ctypes.c_int, [ctypes.POINTER(GridDesc), ctypes.POINTER(Params),
                                             ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p,
                                             _dp]),
    "miso_b200_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(GridDesc),
                                              ctypes.POINTER(Params), ctypes.c_void_p,
                                              ctypes.POINTER(ctypes.c_void_p)]),
    "miso_b200_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "miso_b200_batch_upload": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                              ctypes.POINTER(ctypes.c_void_p)]),
    "miso_b200_batch_download": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                                ctypes.POINTER(ctypes.c_void_p)]),
    "miso_b200_batch_fill_ghosts": (ctypes.c_int, [ctypes.c_void_p]),
    "miso_b200_batch_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "miso_b200_batch_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "miso_b200_batch_dt": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "miso_b200_batch_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong),
                                            ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_longlong)]),
    "miso_b200_batch_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "miso_b200_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "miso_b200_version": (ctypes.c_char_p, []),
}

_lib = None


def load():
    """Load the shared library once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m miso_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class MisoError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def check(code: int, handle=None):
    if code != OK:
        lib = load()
        msg = lib.miso_b200_last_error(handle)
        raise MisoError(code, msg.decode() if msg else "")
