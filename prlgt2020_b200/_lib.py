"""ctypes binding of libnspt_b200.so (the C ABI in include/nspt_b200.h).

The library is built in-tree (``prlgt2020_b200/lib``) by ``build()``.  There is
no fallback: if the shared object is missing or does not load, every call
raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("NSPT_B200_LIB") or os.path.join(HERE, "lib", "libnspt_b200.so")
CSRC = os.path.join(HERE, "csrc")
HEADER = os.path.join(os.path.dirname(HERE), "include", "nspt_b200.h")

NSPT_OK = 0
NSPT_ERR_ARG = 1
NSPT_ERR_ORDER = 2
NSPT_ERR_NOMEM = 3
NSPT_ERR_CUDA = 4
NSPT_ERR_NODEVICE = 5
NSPT_ERR_STATE = 6
NSPT_ERR_IO = 7
NSPT_ERR_TIMEOUT = 8
NSPT_MAX_ORDER = 48

NSPT_TWIST_Y = 1 << 1
NSPT_TWIST_Z = 1 << 2
NSPT_TWIST_T = 1 << 3
NSPT_ZEROMODE = 1 << 4
NSPT_GF_FA = 1 << 5
NSPT_GF_LOCAL = 1 << 6
NSPT_ACTION_TLSYM = 1 << 7
NSPT_ACTION_IWA = 1 << 8
NSPT_ACTION_DBW2 = 1 << 9
NSPT_PRECISION_FF = 1 << 10
NSPT_UPDATE_ONTHEFLY = 1 << 11

# every entry point the header declares: name -> (restype, argtypes)
_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.c_int
SIGNATURES = {
    "nspt_create": (_I, [ctypes.POINTER(ctypes.c_int), _I, ctypes.c_uint, ctypes.c_double,
                         ctypes.POINTER(_P)]),
    "nspt_destroy": (_I, [_P]),
    "nspt_error_string": (ctypes.c_char_p, [_I]),
    "nspt_last_error": (ctypes.c_char_p, [_P]),
    "nspt_device_bytes": (ctypes.c_size_t, [_P]),
    "nspt_upload_links": (_I, [_P, ctypes.c_void_p, _I]),
    "nspt_download_links": (_I, [_P, ctypes.c_void_p, _I]),
    "nspt_cold_start": (_I, [_P]),
    "nspt_set_noise": (_I, [_P, _D]),
    "nspt_seed": (_I, [_P, ctypes.c_uint64, ctypes.c_uint64]),
    "nspt_get_seed": (_I, [_P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "nspt_step": (_I, [_P, ctypes.c_double, _I, _I]),
    "nspt_gauge_wilson": (_I, [_P, ctypes.c_double]),
    "nspt_zero_modes_subtraction": (_I, [_P]),
    "nspt_fa_gauge_fixing": (_I, [_P, ctypes.c_double]),
    "nspt_local_gauge_fixing": (_I, [_P, ctypes.c_double]),
    "nspt_set_gf_grid": (_I, [_P, ctypes.POINTER(ctypes.c_int)]),
    "nspt_set_local_gf_form": (_I, [_P, _I]),
    "nspt_twist_boundary": (_I, [_P]),
    "nspt_observables": (_I, [_P, _D, _D, _D]),
    "nspt_plaquette_measure": (_I, [_P, _D]),
    "nspt_rect_observables": (_I, [_P, _D]),
    "nspt_wilson_loops": (_I, [_P, _D]),
    "nspt_wl2x2": (_I, [_P, _D]),
    "nspt_set_timeout": (_I, [_P, ctypes.c_double]),
    "nspt_set_ff_scale": (_I, [_P, _I, _I]),
    "nspt_get_ff_scale": (_I, [_P, ctypes.POINTER(_I)]),
    "nspt_save_config": (_I, [_P, ctypes.c_char_p, _I]),
    "nspt_load_config": (_I, [_P, ctypes.c_char_p, _I, _D]),
    "nspt_load_lower_order": (_I, [_P, ctypes.c_char_p, _I, _D]),
    "nspt_last_step_ms": (ctypes.c_double, [_P]),
    "nspt_last_kernel_ms": (ctypes.c_double, [_P]),
    "nspt_measure_fp64_peak": (_I, [_D]),
    "nspt_batch_create": (_I, [_I, ctypes.POINTER(ctypes.c_int), _I, ctypes.c_uint, ctypes.c_double,
                               _D, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(_P)]),
    "nspt_batch_destroy": (_I, [_P]),
    "nspt_batch_context": (_I, [_P, _I, ctypes.POINTER(_P)]),
    "nspt_batch_step": (_I, [_P, _I, _I]),
    "nspt_batch_last_step_ms": (ctypes.c_double, [_P]),
    "nspt_batch_observables": (_I, [_P, _D]),
    "nspt_batch_tune": (_I, [_P, _I, ctypes.POINTER(_I)]),
    "nspt_batch_tune_shape": (_I, [_P, _I, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_float)]),
    "nspt_plaquette_measure_noalloc": (_I, [ctypes.c_void_p, _I, ctypes.POINTER(ctypes.c_int), _I,
                                           ctypes.c_uint, _D, ctypes.c_void_p]),
}

_lib = None


def build(verbose: bool = False) -> str:
    """Compile the CUDA engine for sm_100a into prlgt2020_b200/lib."""
    os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
    r = subprocess.run(["make", "-s", "-C", CSRC], capture_output=not verbose, text=True)
    if r.returncode != 0:
        raise RuntimeError("building libnspt_b200.so failed:\n%s%s" % (r.stdout or "", r.stderr or ""))
    return LIB_PATH


def header_symbols() -> list:
    """Function names declared in include/nspt_b200.h."""
    import re
    src = open(HEADER).read()
    return sorted(set(re.findall(r"\b(nspt_[a-z0-9_]+)\s*\(", src)))


def load():
    """Load the engine; raises if the shared object is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libnspt_b200.so not built (run prlgt2020_b200.build())")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class NsptError(RuntimeError):
    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        msg = "%s failed: %s" % (where, load().nspt_error_string(code).decode())
        if detail:
            msg += " (%s)" % detail
        super().__init__(msg)


def check(code: int, where: str, ctx=None):
    if code != NSPT_OK:
        detail = ""
        if ctx:
            d = load().nspt_last_error(ctx)
            detail = d.decode() if d else ""
        raise NsptError(code, where, detail)
