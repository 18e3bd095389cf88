"""ctypes binding of the in-tree CUDA library ``libgatt_dns_b200.so``.

The product path is the CUDA library only: if it is missing or cannot be loaded this
module raises, it never falls back to a CPU implementation.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgatt_dns_b200.so")

_c_int, _c_double, _c_void_p = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
_pd = ctypes.POINTER(ctypes.c_double)
_pi = ctypes.POINTER(ctypes.c_int)
_pp = ctypes.POINTER(ctypes.c_void_p)

# name -> (restype, argtypes); every entry point include/gatt_dns.h declares
SIGNATURES = {
    "gatt_strerror": (ctypes.c_char_p, [_c_int]),
    "gatt_last_error": (ctypes.c_char_p, []),
    "gatt_create": (_c_int, [_pp, _c_int, _c_int, _c_int, _c_int]),
    "gatt_destroy": (None, [_c_void_p]),
    "gatt_set_stream": (_c_int, [_c_void_p, _c_void_p]),
    "gatt_set_physics": (_c_int, [_c_void_p, _c_double, _c_double, _c_double, _c_double, _c_double]),
    "gatt_set_matrices": (_c_int, [_c_void_p, _c_int, _c_int, _c_int, _c_int, _c_int, _pd, _pd, _pd, _pd, _pd,
                                   _c_int, _pi]),
    "gatt_set_filter": (_c_int, [_c_void_p, _c_int, _c_int, _c_int, _c_double]),
    "gatt_set_time_stepping": (_c_int, [_c_void_p, _c_int]),
    "gatt_set_neumann": (_c_int, [_c_void_p, _c_int, _pd, _c_int, _pd]),
    "gatt_set_bc": (_c_int, [_c_void_p, _c_int, _c_int, _c_int, _pi, _pd, _pi]),
    "gatt_set_corners": (_c_int, [_c_void_p, _c_int, _pi, _pi, _pi]),
    "gatt_add_disturbance": (_c_int, [_c_void_p, _c_int, _c_int, _pi, _pd, _c_int, _pd]),
    "gatt_clear_disturbances": (_c_int, [_c_void_p]),
    "gatt_add_forcing": (_c_int, [_c_void_p, _c_int, _pi, _c_int, _pd]),
    "gatt_clear_forcings": (_c_int, [_c_void_p]),
    "gatt_set_sfd": (_c_int, [_c_void_p, _c_int, _c_double, _c_double, _pd]),
    "gatt_upload": (_c_int, [_c_void_p, _c_int, _pd, _pd, _pd, _pd, _pd]),
    "gatt_download": (_c_int, [_c_void_p, _c_int, _pd, _pd, _pd, _pd, _pd]),
    "gatt_upload_mean": (_c_int, [_c_void_p, _c_int, _pd, _pd, _pd, _pd, _pd]),
    "gatt_download_mean": (_c_int, [_c_void_p, _c_int, _pd, _pd, _pd, _pd, _pd]),
    "gatt_upload_wnew": (_c_int, [_c_void_p, _c_int, _pd]),
    "gatt_download_wnew": (_c_int, [_c_void_p, _c_int, _pd]),
    "gatt_state_device_ptr": (_c_int, [_c_void_p, _c_int, _c_int, ctypes.POINTER(_pd)]),
    "gatt_apply_bc": (_c_int, [_c_void_p, _c_double]),
    "gatt_deriv_dir": (_c_int, [_c_void_p, _c_int, _c_int, _pd, _pd]),
    "gatt_rhs": (_c_int, [_c_void_p, _pd, _pd, _pd, _pd, _pd, _pd, _pd, _pd, _pd, _pd]),
    "gatt_filter": (_c_int, [_c_void_p, _c_double]),
    "gatt_step": (_c_int, [_c_void_p, _c_double, _c_double, _pd]),
    "gatt_run": (_c_int, [_c_void_p, _c_int, _c_double, _c_double, _pd]),
    "gatt_max_velocity": (_c_int, [_c_void_p, _pd]),
    "gatt_arnoldi": (_c_int, [_c_void_p, _c_int, _c_int, _c_double, _c_double, _c_double, _pd, _pd,
                              ctypes.c_void_p, _pd]),
    "gatt_arnoldi_vector": (_c_int, [_c_void_p, _c_int, _c_int, _pd]),
    "gatt_rhs_jvp": (_c_int, [_c_void_p, _pd, _pd, _pd]),
    "gatt_rhs_vjp": (_c_int, [_c_void_p, _pd, _pd, _pd]),
    "gatt_jvp": (_c_int, [_c_void_p, _c_int, _c_double, _c_double, _pd, _pd]),
    "gatt_vjp": (_c_int, [_c_void_p, _c_int, _c_double, _c_double, _c_int, _pd, _pd]),
    "gatt_selftest_pipeline_timeout": (_c_int, [_c_void_p]),
    "gatt_autotune": (_c_int, [_c_void_p, _c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), _pd]),
    "gatt_synchronize": (_c_int, [_c_void_p]),
    "gatt_kernel_launches": (ctypes.c_longlong, [_c_void_p]),
    "gatt_profile_kernels": (_c_int, [_c_void_p, _c_double, _c_double, _c_int, _pd, _pd]),
    "gatt_profile_name": (ctypes.c_char_p, [_c_int]),
    "gatt_max_change_noalloc": (_c_int, [_c_int, _c_int, ctypes.c_longlong, _pp, _pp, _pd, _c_void_p]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("CUDA library %s is missing: run `python -c 'import __graft_entry__ as g; g.build()'` "
                           "or `python -m gatt_dns_b200.build`" % path)
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class GattError(RuntimeError):
    def __init__(self, code, where):
        lib = load()
        msg = "%s failed: %s (%s)" % (where, lib.gatt_strerror(code).decode(), lib.gatt_last_error().decode())
        super().__init__(msg)
        self.code = code


def check(code, where):
    if code != 0:
        raise GattError(code, where)
    return code
