"""Drive any library with the reference simulator's C ABI through the call
sequence of the reference wrapper (cuda_interface_pml.py:114, 159, 164, 197,
218): init_memory_sim -> cuda_simulate per shot -> init_memory_reg ->
setCquad -> cuda_grad_ext per shot with an L2 adjoint source.

Used with the reference library (tests/golden/make_sim_golden.py) and with
libotfwi.so (the GPU parity tests), so both see identical calls.
"""
import ctypes

import numpy as np

from otfwi_b200._lib import ADJ_CB, c_float_p, c_float_pp, c_int_p

INPUT_KEYS = ("X", "Z", "T", "PML", "c_true", "c_start", "d_x", "d_z", "constvec", "src_x", "src_z",
              "source", "rec_x", "rec_z", "ring_x", "ring_z")


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32).ravel())


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel())


def _fp(a):
    return a.ctypes.data_as(c_float_p)


def _ip(a):
    return a.ctypes.data_as(c_int_p)


def l2_adjoint(sim, obs):
    """L2 residual with column 0 (never simulated) zeroed."""
    r = np.asarray(sim, dtype=np.float64) - obs
    r[:, 0] = 0.0
    return r


def run_abi(lib, X, Z, T, PML, c_true, c_start, d_x, d_z, constvec, src_x, src_z, source, rec_x,
            rec_z, ring_x, ring_z, check=None, **_):
    X, Z, T = int(X), int(Z), int(T)
    ns, nm = len(src_x), len(rec_x)
    k = dict(cq=_f32(np.asarray(c_true) ** 2), cv=_f32(constvec), dx=_f32(d_x), dz=_f32(d_z),
             sx=_i32(src_x), sz=_i32(src_z), mx=_i32(rec_x), mz=_i32(rec_z), src=_f32(source),
             init=_f32(np.zeros((Z, X, 2))), rx=_i32(ring_x), rz=_i32(ring_z))
    chk = check or (lambda: None)
    recptr = c_float_pp(c_float_p())
    lib.init_memory_sim(X, Z, T, _fp(k["cq"]), _fp(k["cv"]), _fp(k["dx"]), _fp(k["dz"]), ns, _ip(k["sx"]),
                        _ip(k["sz"]), nm, _ip(k["mx"]), _ip(k["mz"]), _fp(k["src"]), _fp(k["init"]), recptr)
    chk()
    res = {}

    def traces():
        return np.ctypeslib.as_array(recptr[0], shape=(nm * T,)).copy().reshape(nm, T)

    lib.cuda_simulate(0, -1)
    chk()
    res["traces_all"] = traces()
    for s in range(ns):
        lib.cuda_simulate(0, s)
        chk()
        res[f"traces_s{s}"] = traces()
    obs = np.stack([res[f"traces_s{s}"] for s in range(ns)])
    k["obs"] = _f32(obs)
    gradptr = c_float_pp(c_float_p())
    lib.init_memory_reg(_fp(k["obs"]), gradptr, _ip(k["rx"]), _ip(k["rz"]), len(k["rx"]))
    chk()
    k["cq0"] = _f32(np.asarray(c_start) ** 2)
    lib.setCquad(_fp(k["cq0"]))
    chk()
    box = {}

    def adj(sim_p, adj_p):
        sim = np.ctypeslib.as_array(sim_p, shape=(nm * T,)).astype(np.float64).reshape(nm, T)
        box["sim"] = sim.astype(np.float32)
        np.ctypeslib.as_array(adj_p, shape=(nm * T,))[:] = l2_adjoint(sim, obs[box["s"]]).ravel()

    cb = ADJ_CB(adj)
    for s in range(ns):
        box["s"] = s
        mse = (ctypes.c_float * 1)(0.0)
        lib.cuda_grad_ext(mse, ctypes.cast(cb, ctypes.c_void_p), s)
        chk()
        res[f"grad_s{s}"] = np.ctypeslib.as_array(gradptr[0], shape=(Z * X,)).copy().reshape(Z, X)
        res[f"sim_s{s}"] = box["sim"]
    return res
