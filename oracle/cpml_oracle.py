"""ctypes binding of the CPML CPU oracle (oracle/cpml_oracle.c in liborc.so).

TEST INFRASTRUCTURE ONLY: the parity tests use it as the checker.
"""
import ctypes
import os
from ctypes import POINTER, c_double, c_float, c_int

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


def _load():
    L = ctypes.CDLL(os.path.join(_HERE, "liborc.so"))
    for suf, T in (("f32", c_float), ("f64", c_double)):
        f = getattr(L, f"orc_cpml_simulate_{suf}")
        f.restype = c_int
        f.argtypes = ([c_int] * 5 + [POINTER(c_int)] * 2 + [c_int] + [POINTER(c_int)] * 2 + [c_float] * 4 +
                      [POINTER(c_float)] * 18 + [c_int, POINTER(T)])
    f = L.orc_cpml_adjoint_f64
    f.restype = c_int
    f.argtypes = ([c_int] * 5 + [POINTER(c_int)] * 2 + [c_int] + [POINTER(c_int)] * 2 + [c_float] * 4 +
                  [POINTER(c_float)] * 18 + [c_int] + [POINTER(c_double)] * 3)
    return L


def simulate(inp, X, Z, T, idx_source=-1, ppe=1, mode="f32", dx=1.0, dt=1.0, qtpi=4.0 * np.pi):
    """Traces [n_rec, T] of the CPML scheme for the arrays ``inp`` built by
    otfwi_b200.cpml.CPMLSimulator (its ``inputs`` dict)."""
    L = _load()
    fp = lambda k: inp[k].ctypes.data_as(POINTER(c_float))
    ip = lambda k: inp[k].ctypes.data_as(POINTER(c_int))
    ns, nm = len(inp["ps_x"]), len(inp["pm_x"])
    dt_ = np.float32 if mode == "f32" else np.float64
    rec = np.zeros((nm, T), dt_)
    ct = c_float if mode == "f32" else c_double
    fn = getattr(L, f"orc_cpml_simulate_{mode}")
    rc = fn(X, Z, T, ns, ppe, ip("ps_x"), ip("ps_z"), nm, ip("pm_x"), ip("pm_z"), dx, dx, dt * dt, qtpi,
            fp("cq"), fp("kappa"), fp("rhx"), fp("rhz"),
            fp("K_x"), fp("a_x"), fp("b_x"), fp("K_xh"), fp("a_xh"), fp("b_xh"),
            fp("K_z"), fp("a_z"), fp("b_z"), fp("K_zh"), fp("a_zh"), fp("b_zh"),
            fp("src"), fp("init"), idx_source, rec.ctypes.data_as(POINTER(ct)))
    if rc != 0:
        raise RuntimeError("CPML oracle failed")
    return rec


def adjoint(inp, X, Z, T, g, idx_source=-1, ppe=1, dx=1.0, dt=1.0, qtpi=4.0 * np.pi):
    """(dL/dkappa [Z, X], traces [n_rec, T]) of the FP64 CPML forward for
    dL/dtraces = g [n_rec, T] (oracle/cpml_adjoint.c)."""
    L = _load()
    fp = lambda k: inp[k].ctypes.data_as(POINTER(c_float))
    ip = lambda k: inp[k].ctypes.data_as(POINTER(c_int))
    ns, nm = len(inp["ps_x"]), len(inp["pm_x"])
    gg = np.ascontiguousarray(np.asarray(g, np.float64))
    grad = np.zeros((Z, X))
    rec = np.zeros((nm, T))
    dp = lambda a: a.ctypes.data_as(POINTER(c_double))
    rc = L.orc_cpml_adjoint_f64(X, Z, T, ns, ppe, ip("ps_x"), ip("ps_z"), nm, ip("pm_x"), ip("pm_z"), dx, dx,
                                dt * dt, qtpi, fp("cq"), fp("kappa"), fp("rhx"), fp("rhz"),
                                fp("K_x"), fp("a_x"), fp("b_x"), fp("K_xh"), fp("a_xh"), fp("b_xh"),
                                fp("K_z"), fp("a_z"), fp("b_z"), fp("K_zh"), fp("a_zh"), fp("b_zh"),
                                fp("src"), fp("init"), idx_source, dp(gg), dp(grad), dp(rec))
    if rc != 0:
        raise RuntimeError("CPML adjoint oracle failed")
    return grad, rec
