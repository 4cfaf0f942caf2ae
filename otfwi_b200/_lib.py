"""ctypes loader for the in-tree CUDA library (libotfwi.so).

The library must have been built (``otfwi_b200._build.build()`` or
``__graft_entry__.build()``). There is no CPU fallback: a missing or
unloadable library raises immediately.
"""
import ctypes
import os
from ctypes import POINTER, c_float, c_int, c_void_p, c_char_p

from ._build import LIB, DROPIN

_LIBS = {}

c_float_p = POINTER(c_float)
c_int_p = POINTER(c_int)
c_float_pp = POINTER(POINTER(c_float))
ADJ_CB = ctypes.CFUNCTYPE(None, c_float_p, c_float_p)


class OtfwiError(RuntimeError):
    """A call into the CUDA library reported a failure."""


def _declare(lib):
    lib.init_memory_sim.restype = None
    lib.init_memory_sim.argtypes = [c_int, c_int, c_int, c_float_p, c_float_p, c_float_p, c_float_p,
                                    c_int, c_int_p, c_int_p, c_int, c_int_p, c_int_p, c_float_p,
                                    c_float_p, c_float_pp]
    lib.init_memory_reg.restype = None
    lib.init_memory_reg.argtypes = [c_float_p, c_float_pp, c_int_p, c_int_p, c_int]
    lib.setCquad.restype = None
    lib.setCquad.argtypes = [c_float_p]
    lib.cuda_simulate.restype = None
    lib.cuda_simulate.argtypes = [c_int, c_int]
    lib.cuda_grad_ext.restype = None
    lib.cuda_grad_ext.argtypes = [c_float_p, c_void_p, c_int]
    lib.def_python_adj.restype = None
    lib.def_python_adj.argtypes = [c_void_p]
    lib.hilbert.restype = None
    lib.hilbert.argtypes = [c_float_p, c_float_p, c_float_p, c_int]
    if hasattr(lib, "otf_last_status"):
        lib.set_source.restype = None
        lib.set_source.argtypes = [c_int, c_int_p, c_int_p, c_float_p]
        lib.otf_last_status.restype = c_int
        lib.otf_last_status.argtypes = []
        lib.otf_last_error.restype = c_char_p
        lib.otf_last_error.argtypes = []
        lib.otf_clear_error.restype = None
        lib.otf_set_precision.restype = c_int
        lib.otf_set_precision.argtypes = [c_int]
        lib.otf_set_tile.restype = c_int
        lib.otf_set_tile.argtypes = [c_int]
        lib.otf_release.restype = None
    return lib


def load(path=None):
    """Load (once) the library at ``path`` (default: the in-tree libotfwi.so)."""
    path = os.path.abspath(path or LIB)
    if path in _LIBS:
        return _LIBS[path]
    if not os.path.exists(path):
        raise OtfwiError(f"CUDA library not built: {path} (run __graft_entry__.build())")
    lib = _declare(ctypes.CDLL(path))
    _LIBS[path] = lib
    return lib


def check(lib):
    """Raise OtfwiError if the last library call recorded a failure."""
    if hasattr(lib, "otf_last_status") and lib.otf_last_status() != 0:
        msg = lib.otf_last_error().decode(errors="replace")
        lib.otf_clear_error()
        raise OtfwiError(msg)


def exported_symbols_from_header(header_path):
    """Function names declared in include/otfwi.h (for the export check)."""
    import re
    text = open(header_path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", text)
    return sorted(set(n for n in names if n not in ("adj",)))


__all__ = ["load", "check", "OtfwiError", "ADJ_CB", "LIB", "DROPIN", "c_float_p", "c_int_p"]
