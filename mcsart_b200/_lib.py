"""ctypes binding of libmcsart.so (the C ABI declared in include/mcsart.h).

The library is loaded from ``mcsart_b200/lib/libmcsart.so`` inside this source
tree.  There is no fallback: if the library is missing or a call fails, an
exception is raised.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libmcsart.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "mcsart.h")

OK = 0
ERR_INVALID_ARGUMENT = -1
ERR_CUDA = -2
ERR_NO_DEVICE = -3
ERR_OUT_OF_MEMORY = -4
ERR_UNSUPPORTED = -5

F32, BF16, F16 = 0, 1, 2
INTERP_TEXTURE, INTERP_EXACT = 0, 1


class McsartError(RuntimeError):
    """A libmcsart call returned a non-zero status."""

    def __init__(self, code: int, func: str, message: str):
        super().__init__(f"{func} failed ({code}): {message}")
        self.code = code
        self.func = func


class Options(ctypes.Structure):
    _fields_ = [("storage", ctypes.c_int), ("interp", ctypes.c_int), ("use_graph", ctypes.c_int),
                ("fp_sum", ctypes.c_int), ("fp_groups", ctypes.c_int), ("subset", ctypes.c_int),
                ("dvf_inverse", ctypes.c_int), ("geom64", ctypes.c_int),
                ("autotune", ctypes.c_int)]


class Problem(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("na", ctypes.c_int), ("nb", ctypes.c_int), ("n_views", ctypes.c_int),
                ("SO", ctypes.c_float), ("SD", ctypes.c_float), ("da", ctypes.c_float),
                ("db", ctypes.c_float), ("ai", ctypes.c_float), ("bi", ctypes.c_float),
                ("lambda_", ctypes.c_float),
                ("h_angles", ctypes.c_void_p), ("h_volumes", ctypes.c_void_p),
                ("h_flows", ctypes.c_void_p), ("d_img", ctypes.c_void_p),
                ("d_proj", ctypes.c_void_p), ("d_fields", ctypes.c_void_p),
                ("d_resid", ctypes.c_void_p), ("d_norm", ctypes.c_void_p)]


_F = ctypes.c_float
_I = ctypes.c_int
_P = ctypes.c_void_p
_GEO = [_F, _F, _F, _F, _I, _F, _F, _I, _F, _I, _I, _I]  # angle, SO, SD, da, na, ai, db, nb, bi, nx, ny, nz

# name -> argtypes (after the context argument); every function returns int
SIGNATURES = {
    "mcsart_projection": [_P, _P] + _GEO,
    # first argument is a cudaStream_t here, not a context
    "mcsart_projection_noalloc": [_P, _P] + _GEO,
    "mcsart_backprojection": [_P, _P] + _GEO,
    "mcsart_backprojection_adjoint": [_P, _P] + _GEO,
    "mcsart_deform": [_P, _P, _I, _I, _I, _F, _F] + [_P] * 6,
    "mcsart_deform2": [_P, _P, _I, _I, _I, _F, _F] + [_P] * 6,
    "mcsart_invert_dvf": [_P] * 9 + [_F, _F, _I, _I, _I, _I],
    "mcsart_forward_dvf": [_P] * 9 + [_F, _F, _I, _I, _I],
    "mcsart_add": [_P, _P, _I, _I, _I, _F],
    "mcsart_add2": [_P, _P, _I, _I, _I, _P, _F, _I],
    "mcsart_initial": [_P, _I, _I, _I, _F],
    "mcsart_initial2": [_P, _I, _I, _I, _P, _F, _F],
    "mcsart_division": [_P, _P, _I, _I, _I],
    "mcsart_multiple": [_P, _I, _I, _I, _P, _F, _I],
    "mcsart_update_udvf": [_P] * 8 + [_F, _F, _I, _I, _I, _I],
    "mcsart_diff": [_P, _P, _I, _I, _I, _I],
    "mcsart_snrm2": [_I, _P, ctypes.POINTER(ctypes.c_float)],
    "mcsart_projection_views": [_P, _P, _P, _I, _F, _F, _F, _I, _F, _F, _I, _F, _I, _I, _I],
    "mcsart_projection_ex": [_P, _P, _I, _I, _I] + _GEO,
    "mcsart_backprojection_ex": [_P, _P, _I] + _GEO,
    "mcsart_deform_ex": [_P, _P, _I, _I, _I, _F, _F, _P, _I, _I],
    "mcsart_aumisart": [_P] * 6 + [_I] * 8 + [_P] + [_F] * 8 + [_P] * 4 + [_P] * 6,
    "mcsart_aumisart_fields": [_P] * 11 + [_I] * 8 + [_P] + [_F] * 8 + [_P] * 4 + [_P] * 6,
    "mcsart_aumisart_device": [ctypes.POINTER(Problem), _I, _P, ctypes.POINTER(Options)],
    "mcsart_batch_run": [ctypes.POINTER(Problem), _I, _I, _P, ctypes.POINTER(Options)],
    "mcsart_autotune": [ctypes.POINTER(Problem), ctypes.POINTER(Options)],
    "mcsart_tuning_get": [ctypes.POINTER(Problem), _I, ctypes.POINTER(ctypes.c_int)],
    "mcsart_tuning_save": [ctypes.c_char_p],
    "mcsart_tuning_load": [ctypes.c_char_p],
    "mcsart_set_stream": [_P],
    "mcsart_set_synchronous": [_I],
    "mcsart_set_interp": [_I],
    "mcsart_synchronize": [],
}

_lib = None


def load() -> ctypes.CDLL:
    """Load libmcsart.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} not found: build it with `python -m mcsart_b200.build` "
                      "(or __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = [_P] + args
        fn.restype = _I
    L.mcsart_version.restype = _I
    L.mcsart_last_error.restype = ctypes.c_char_p
    L.mcsart_create.argtypes = [ctypes.POINTER(_P), _I]
    L.mcsart_create.restype = _I
    L.mcsart_destroy.argtypes = [_P]
    L.mcsart_destroy.restype = _I
    L.mcsart_get_stream.argtypes = [_P]
    L.mcsart_get_stream.restype = _P
    L.mcsart_launch_count.argtypes = [_P]
    L.mcsart_launch_count.restype = ctypes.c_longlong
    for n in ("mcsart_profile_begin", "mcsart_profile_end", "mcsart_profile_count"):
        getattr(L, n).argtypes = [_P]
        getattr(L, n).restype = _I
    L.mcsart_profile_entry.argtypes = [_P, _I, ctypes.c_char_p, _I,
                                       ctypes.POINTER(ctypes.c_longlong),
                                       ctypes.POINTER(ctypes.c_double)]
    L.mcsart_profile_entry.restype = _I
    L.mcsart_default_options.argtypes = [ctypes.POINTER(Options)]
    L.mcsart_default_options.restype = None
    _lib = L
    return L


def check(code: int, func: str) -> None:
    if code != OK:
        msg = load().mcsart_last_error().decode(errors="replace")
        raise McsartError(code, func, msg)


def declared_functions() -> list[str]:
    """Names of the functions include/mcsart.h declares."""
    import re
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char \*|long long|void \*)\s*\*?"
                                 r"(mcsart_\w+)\s*\(", text, flags=re.M)))
