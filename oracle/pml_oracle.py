"""ctypes binding of the CPU oracle (oracle/liborc.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg as the checker; the product never imports it.

``simulate`` restates cuda_simulate (regression_PML_single.cu:618-702) and
``grad`` restates cuda_grad_ext (regression_PML_single.cu:704-846), in mode
"f32" (the reference's own mixed FP32/FP64 arithmetic) or "f64" (FP64).
Inputs follow the reference ABI: cquad [Z, X] = (c dt/dx)^2, constvec
{dx, dz, dt}, damping d_x, d_z [Z, X], positions as integer x / z arrays.
"""
import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_float, c_int, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liborc.so")
_lib = None

_cbf = ctypes.CFUNCTYPE(None, POINTER(c_float), POINTER(c_float), c_void_p)
_cbd = ctypes.CFUNCTYPE(None, POINTER(c_double), POINTER(c_double), c_void_p)


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        subprocess.run(["make", "-C", HERE, "liborc.so"], check=True, capture_output=True)
    lib = ctypes.CDLL(LIB)
    fp, ip, dp = POINTER(c_float), POINTER(c_int), POINTER(c_double)
    common = [c_int, c_int, c_int, fp, fp, fp, fp, c_int, ip, ip, fp, c_int, c_int, ip, ip]
    lib.orc_simulate_f32.argtypes = common + [fp]
    lib.orc_simulate_f64.argtypes = common + [dp]
    lib.orc_grad_f32.argtypes = common + [c_int, ip, ip, _cbf, c_void_p, fp, fp]
    lib.orc_grad_f64.argtypes = common + [c_int, ip, ip, _cbd, c_void_p, dp, dp]
    lib.orc_exact_adjoint_f64.argtypes = common + [dp, dp, dp]
    lib.orc_forward_f64.argtypes = [c_int, c_int, c_int, dp, fp, fp, fp, c_int, ip, ip, fp, c_int, c_int,
                                    ip, ip, dp]
    lib.orc_frames_f32.argtypes = common + [c_int, POINTER(ctypes.c_ubyte), fp]
    for f in (lib.orc_simulate_f32, lib.orc_simulate_f64, lib.orc_grad_f32, lib.orc_grad_f64,
              lib.orc_num_threads, lib.orc_exact_adjoint_f64, lib.orc_forward_f64, lib.orc_frames_f32):
        f.restype = c_int
    _lib = lib
    return lib


def exact_adjoint(cquad, constvec, d_x, d_z, src_x, src_z, source, rec_x, rec_z, g, idx_source=-1):
    """(dL/d(c^2) [Z, X], traces [n_rec, T]) of the exact discrete adjoint
    (oracle/pml_adjoint.c) for dL/drec = g [n_rec, T], FP64."""
    lib = _load()
    Z, X = np.asarray(cquad).shape
    nsrc = len(np.atleast_1d(src_x))
    T = np.asarray(source).reshape(nsrc, -1).shape[1]
    arrs = _prep(cquad, constvec, d_x, d_z, src_x, src_z, source, rec_x, rec_z)
    nm = len(arrs[7])
    gg = np.ascontiguousarray(np.asarray(g, dtype=np.float64).reshape(nm, T))
    grad = np.zeros((Z, X))
    rec = np.zeros((nm, T))
    dp = POINTER(c_double)
    rc = lib.orc_exact_adjoint_f64(*_args(X, Z, T, arrs, idx_source), gg.ctypes.data_as(dp),
                                   grad.ctypes.data_as(dp), rec.ctypes.data_as(dp))
    if rc:
        raise RuntimeError("oracle exact adjoint failed")
    return grad, rec


def forward64(cquad64, constvec, d_x, d_z, src_x, src_z, source, rec_x, rec_z, idx_source=-1):
    """FP64 traces [n_rec, T] of the same map, with an FP64 c^2 (for finite
    differences)."""
    lib = _load()
    cq = np.ascontiguousarray(np.asarray(cquad64, dtype=np.float64))
    Z, X = cq.shape
    nsrc = len(np.atleast_1d(src_x))
    T = np.asarray(source).reshape(nsrc, -1).shape[1]
    arrs = _prep(cq, constvec, d_x, d_z, src_x, src_z, source, rec_x, rec_z)
    nm = len(arrs[7])
    rec = np.zeros((nm, T))
    a = _args(X, Z, T, arrs, idx_source)
    a[3] = cq.ctypes.data_as(POINTER(c_double))
    rc = lib.orc_forward_f64(*a, rec.ctypes.data_as(POINTER(c_double)))
    if rc:
        raise RuntimeError("oracle forward failed")
    return rec


def num_threads():
    return _load().orc_num_threads()


def _prep(cquad, constvec, d_x, d_z, sx, sz, src, mx, mz):
    f = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float32).ravel())
    i = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel())
    return f(cquad), f(constvec), f(d_x), f(d_z), i(sx), i(sz), f(src), i(mx), i(mz)


def _args(X, Z, T, arrs, idx_source):
    cq, cv, dx, dz, sx, sz, src, mx, mz = arrs
    fp = lambda a: a.ctypes.data_as(POINTER(c_float))
    ip = lambda a: a.ctypes.data_as(POINTER(c_int))
    return [X, Z, T, fp(cq), fp(cv), fp(dx), fp(dz), len(sx), ip(sx), ip(sz), fp(src),
            int(idx_source), len(mx), ip(mx), ip(mz)]


def simulate(cquad, constvec, d_x, d_z, src_x, src_z, source, rec_x, rec_z, idx_source=-1,
             mode="f32"):
    """Recorded traces [n_rec, T] (column 0 zero)."""
    lib = _load()
    Z, X = np.asarray(cquad).shape
    T = np.asarray(source).reshape(len(np.atleast_1d(src_x)), -1).shape[1]
    arrs = _prep(cquad, constvec, d_x, d_z, src_x, src_z, source, rec_x, rec_z)
    dt = np.float32 if mode == "f32" else np.float64
    rec = np.zeros((len(arrs[7]), T), dtype=dt)
    fn = lib.orc_simulate_f32 if mode == "f32" else lib.orc_simulate_f64
    ptr = rec.ctypes.data_as(POINTER(c_float if mode == "f32" else c_double))
    rc = fn(*_args(X, Z, T, arrs, idx_source), ptr)
    if rc:
        raise RuntimeError("oracle simulate failed")
    return rec


def frames(cquad, constvec, d_x, d_z, src_x, src_z, source, rec_x, rec_z, every=1, idx_source=-1):
    """Video frames of cuda_simulate(en_out = 1): (uint8 [(T-1)//every, Z, X],
    the FP32 total pressure of the same steps [(T-1)//every, Z, X])."""
    lib = _load()
    Z, X = np.asarray(cquad).shape
    T = np.asarray(source).reshape(len(np.atleast_1d(src_x)), -1).shape[1]
    arrs = _prep(cquad, constvec, d_x, d_z, src_x, src_z, source, rec_x, rec_z)
    n = (T - 1) // every
    fr = np.zeros((n, Z, X), np.uint8)
    pf = np.zeros((n, Z, X), np.float32)
    rc = lib.orc_frames_f32(*_args(X, Z, T, arrs, idx_source), int(every),
                            fr.ctypes.data_as(POINTER(ctypes.c_ubyte)), pf.ctypes.data_as(POINTER(c_float)))
    if rc:
        raise RuntimeError("oracle frames failed")
    return fr, pf


def grad(cquad, constvec, d_x, d_z, src_x, src_z, source, rec_x, rec_z, ring_x, ring_z, adj_fun,
         idx_source=-1, mode="f32"):
    """(gradient [Z, X], traces [n_rec, T], misfit). adj_fun(sim[n_rec,T] float64) ->
    (misfit, adjoint source [n_rec, T]) is called once, like the reference's callback."""
    lib = _load()
    Z, X = np.asarray(cquad).shape
    nsrc = len(np.atleast_1d(src_x))
    T = np.asarray(source).reshape(nsrc, -1).shape[1]
    arrs = _prep(cquad, constvec, d_x, d_z, src_x, src_z, source, rec_x, rec_z)
    nm = len(arrs[7])
    rx = np.ascontiguousarray(np.asarray(ring_x, dtype=np.int32))
    rz = np.ascontiguousarray(np.asarray(ring_z, dtype=np.int32))
    dt = np.float32 if mode == "f32" else np.float64
    ct = c_float if mode == "f32" else c_double
    g = np.zeros((Z, X), dtype=dt)
    rec = np.zeros((nm, T), dtype=dt)
    box = {}

    def cb(sim_p, adj_p, user):
        sim = np.ctypeslib.as_array(sim_p, shape=(nm * T,)).astype(np.float64).reshape(nm, T)
        mis, adj = adj_fun(sim)
        box["misfit"] = mis
        out = np.ctypeslib.as_array(adj_p, shape=(nm * T,))
        out[:] = np.asarray(adj, dtype=np.float64).ravel()

    cbo = (_cbf if mode == "f32" else _cbd)(cb)
    fn = lib.orc_grad_f32 if mode == "f32" else lib.orc_grad_f64
    rc = fn(*_args(X, Z, T, arrs, idx_source), len(rx), rx.ctypes.data_as(POINTER(c_int)),
            rz.ctypes.data_as(POINTER(c_int)), cbo, None, g.ctypes.data_as(POINTER(ct)),
            rec.ctypes.data_as(POINTER(ct)))
    if rc:
        raise RuntimeError("oracle grad failed")
    return g, rec, box.get("misfit")
