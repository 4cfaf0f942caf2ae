"""Second-order CPML forward modelling through the reference's CPML C ABI.

The reference builds simulator/src/regression_CPML.cu into
bin/cuda_regression_CPML.so: a second-order pressure scheme with
convolutional-PML memory variables (init_memory_sim with 40 arguments,
setCquad, set_source, cuda_simulate2); no Python module of the reference
calls it, so its caller computes the CPML profiles itself. This module is
that caller: ``cpml_profiles`` builds the d, K, alpha, a, b profiles at the
integer and half points (the unsplit convolutional PML recursion
b = exp(-(d/K + alpha) dt), a = d (b - 1) / (K (d + K alpha))), and
``CPMLSimulator`` drives any library with this ABI -- this package's
lib/cuda_regression_CPML.so by default, which adds the exact discrete
adjoint (``CPMLSimulator.gradient``: dL/dkappa, no reference counterpart).
"""
import ctypes
import os
from ctypes import POINTER, c_float, c_int

import numpy as np

from . import _lib

CPML_LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "cuda_regression_CPML.so")


def cpml_profiles(n, pml, dx, dt, c_max, f0, R=1e-5, npower=2.0, k_max=1.0, alpha_max=None):
    """(d, K, alpha, a, b) at the integer points and at the half points (i +
    1/2) of an axis of n cells with absorbing layers of pml cells at both
    ends, each [n] float32. The damping grows as (distance into the layer /
    layer thickness)^npower from 0 to d0 = -(npower + 1) c_max ln(R) /
    (2 L); alpha falls linearly from alpha_max (pi f0 by default) to 0."""
    alpha_max = np.pi * f0 if alpha_max is None else alpha_max
    L = pml * dx
    d0 = -(npower + 1) * c_max * np.log(R) / (2.0 * L)
    out = []
    for shift in (0.0, 0.5):
        pos = (np.arange(n) + shift) * dx
        lo = pml * dx
        hi = (n - 1 - pml) * dx
        dist = np.maximum(np.maximum(lo - pos, pos - hi), 0.0) / L
        dist = np.minimum(dist, 1.0)
        inside = dist > 0
        d = np.where(inside, d0 * dist ** npower, 0.0)
        K = np.where(inside, 1.0 + (k_max - 1.0) * dist ** npower, 1.0)
        alpha = np.where(inside, alpha_max * (1.0 - dist), 0.0)
        b = np.exp(-(d / K + alpha) * dt)
        den = K * (d + K * alpha)
        a = np.where(np.abs(d) > 1e-30, d * (b - 1.0) / np.where(den == 0, 1.0, den), 0.0)
        out.append(tuple(np.asarray(v, np.float32) for v in (d, K, alpha, a, b)))
    return out[0], out[1]


def _declare(L):
    if getattr(L, "_cpml_declared", False):
        return L
    fp, ip = POINTER(c_float), POINTER(c_int)
    L.init_memory_sim.restype = None
    # 6 ints, 4 int*, 5 floats, 27 float* (c^2, kappa, 3 densities, 20 profiles, source, initial), float**
    L.init_memory_sim.argtypes = [c_int] * 6 + [ip] * 4 + [c_float] * 5 + [fp] * 27 + [POINTER(fp)]
    L.setCquad.restype = None
    L.setCquad.argtypes = [fp]
    L.set_source.restype = None
    L.set_source.argtypes = [c_int, ip, ip]
    L.cuda_simulate2.restype = None
    L.cuda_simulate2.argtypes = [c_int, c_int]
    if hasattr(L, "otf_cpml_gradient"):
        L.otf_cpml_gradient.restype = c_int
        L.otf_cpml_gradient.argtypes = [fp, fp, c_int, c_int]
    if hasattr(L, "otf_cpml_simulate_all"):
        L.otf_cpml_simulate_all.restype = c_int
        L.otf_cpml_simulate_all.argtypes = [fp]
    L._cpml_declared = True
    return L


class CPMLSimulator:
    """Second-order CPML modelling of one acquisition.

    X, Z, T grid and steps; c: velocity [Z, X]; rho: density [Z, X] (default
    1); src_mask / rec_mask: boolean [Z, X]; source: waveforms [n_src, T];
    dx, dt: spacing and step (the CFL number c dt / dx must stay below about
    0.55 for this stencil); ppe: pixels per element (1: ``simulate(idx)``
    fires source idx alone); k_max: the CPML stretching K at the outer edge.
    ``lib``: path of a library with the CPML ABI."""

    def __init__(self, X, Z, T, PML, c, src_mask, rec_mask, source, rho=None, dx=1.0, dt=1.0, f0=0.05,
                 qtpi=4.0 * np.pi, ppe=1, init=None, lib=None, k_max=1.0):
        self.lib_path = lib or CPML_LIB
        self.L = _declare(ctypes.CDLL(os.path.abspath(self.lib_path)))
        self.X, self.Z, self.T = X, Z, T
        c = np.asarray(c, np.float64)
        rho = np.ones((Z, X)) if rho is None else np.asarray(rho, np.float64)
        sz, sx = np.where(src_mask)
        mz, mx = np.where(rec_mask)
        self.n_src, self.n_rec = len(sx), len(mx)
        # half-point densities by arithmetic mean with the next cell (the last cell keeps its own)
        rhx = rho.copy()
        rhx[:, :-1] = 0.5 * (rho[:, :-1] + rho[:, 1:])
        rhz = rho.copy()
        rhz[:-1, :] = 0.5 * (rho[:-1, :] + rho[1:, :])
        (px, pxh) = cpml_profiles(X, PML, dx, dt, float(c.max()), f0, k_max=k_max)
        (pz, pzh) = cpml_profiles(Z, PML, dx, dt, float(c.max()), f0, k_max=k_max)
        f32 = lambda a: np.ascontiguousarray(np.asarray(a, np.float32).ravel())
        i32 = lambda a: np.ascontiguousarray(np.asarray(a, np.int32).ravel())
        self._keep = keep = {
            "ps_x": i32(sx), "ps_z": i32(sz), "pm_x": i32(mx), "pm_z": i32(mz),
            "cq": f32(c * c), "kappa": f32(rho * c * c), "rho": f32(rho), "rhx": f32(rhx), "rhz": f32(rhz),
            "src": f32(source), "init": f32(np.zeros((2, Z, X)) if init is None else init),
        }
        for name, prof in (("x", px), ("xh", pxh), ("z", pz), ("zh", pzh)):
            for k, v in zip(("d", "K", "alpha", "a", "b"), prof):
                keep[f"{k}_{name}"] = f32(v)
        fp = lambda a: a.ctypes.data_as(POINTER(c_float))
        ip = lambda a: a.ctypes.data_as(POINTER(c_int))
        rec = POINTER(c_float)()
        prof_args = []
        for name in ("x", "xh", "z", "zh"):
            prof_args += [fp(keep[f"{k}_{name}"]) for k in ("d", "K", "alpha", "a", "b")]
        self.L.init_memory_sim(X, Z, T, self.n_src, self.n_rec, ppe, ip(keep["ps_x"]), ip(keep["ps_z"]),
                               ip(keep["pm_x"]), ip(keep["pm_z"]), dx, dx, dt, dt * dt, qtpi, fp(keep["cq"]),
                               fp(keep["kappa"]), fp(keep["rho"]), fp(keep["rhx"]), fp(keep["rhz"]), *prof_args,
                               fp(keep["src"]), fp(keep["init"]), ctypes.byref(rec))
        self._check()
        self._rec = rec
        self.inputs = keep

    def _check(self):
        L = self.L
        if hasattr(L, "otf_last_status"):
            L.otf_last_status.restype = c_int
            L.otf_last_error.restype = ctypes.c_char_p
            if L.otf_last_status():
                msg = L.otf_last_error().decode()
                L.otf_clear_error()
                raise _lib.OtfwiError(msg)

    def simulate(self, idx_source=-1):
        """Traces [n_rec, T] (receiver order of np.where(rec_mask))."""
        self.L.cuda_simulate2(0, idx_source)
        self._check()
        n = self.n_rec * self.T
        return np.ctypeslib.as_array(self._rec, shape=(n,)).copy().reshape(self.n_rec, self.T)

    def simulate_all(self):
        """Traces [n_src, n_rec, T] of every source fired alone (the
        reference's per-source loop), all shots in one launch per step (this
        package's library only)."""
        if not hasattr(self.L, "otf_cpml_simulate_all"):
            raise _lib.OtfwiError("this CPML library has no batched forward")
        out = np.zeros((self.n_src, self.n_rec, self.T), np.float32)
        rc = self.L.otf_cpml_simulate_all(out.ctypes.data_as(POINTER(c_float)))
        self._check()
        if rc != 0:
            raise _lib.OtfwiError("otf_cpml_simulate_all failed")
        return out

    def gradient(self, g, idx_source=-1, checkpoint_every=None):
        """dL/dkappa [Z, X] for dL/dtraces = g [n_rec, T] (exact discrete
        adjoint of the forward; this package's library only)."""
        if not hasattr(self.L, "otf_cpml_gradient"):
            raise _lib.OtfwiError("this CPML library has no gradient")
        every = checkpoint_every or max(1, int(np.ceil(np.sqrt(self.T))))
        gg = np.ascontiguousarray(np.asarray(g, np.float32).reshape(self.n_rec, self.T))
        out = np.zeros((self.Z, self.X), np.float32)
        rc = self.L.otf_cpml_gradient(gg.ctypes.data_as(POINTER(c_float)), out.ctypes.data_as(POINTER(c_float)),
                                      int(every), int(idx_source))
        self._check()
        if rc != 0:
            raise _lib.OtfwiError("otf_cpml_gradient failed")
        return out
