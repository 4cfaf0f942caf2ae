"""Host-side mirror of the reference's ``cuda_interface_pml.Cuda_interface_PML``.

Same class name, constructor arguments, methods, attributes and call sequence
into the C ABI (cuda_interface_pml.py:33-249), so driver code written for the
reference (regression.py:34-49) runs against the B200 library unchanged.
The reference's own wrapper also runs unchanged against libotfwi.so (see
INTEGRATION.md); this mirror exists so the library can be driven where the
reference tree is absent, and it can drive any library with the reference's
ABI (``lib=`` path), which is how the parity tests run the reference library
itself in a separate process.

Differences from the reference wrapper: arrays are passed as numpy-backed
pointers instead of element-by-element ctypes copies; failures recorded by the
library raise ``OtfwiError`` (the reference's wrapper never checks); the
``_set_source`` method calls the ``set_source`` export this library provides.
"""
import ctypes

import numpy as np

from . import _lib


def pml_damping(X, Z, PML_size):
    """Quadratic damping profiles d_x, d_z [Z, X] (float64), cuda_interface_pml.py:116-132:
    d0 = 3*Vmax*ln(1/R)/(2*Lp^3) with R = 1e-5, Vmax = 0.5, Lp = PML_size;
    profile d0*x^2 on x = linspace(0, Lp, PML_size), reversed on the low sides."""
    R = 1e-5
    Vmax = 0.5
    Lp = PML_size * 1
    d0 = 3 * Vmax * np.log(1 / R) / (2 * Lp ** 3)
    x = np.linspace(0, Lp, PML_size)
    prof = d0 * x[:, np.newaxis] ** 2
    d_x = np.zeros((Z, X))
    d_z = np.zeros((Z, X))
    d_z[:PML_size, :] = prof[-1::-1]
    d_z[-PML_size:, :] = prof
    d_x[:, -PML_size:] = prof.T
    d_x[:, :PML_size] = prof[-1::-1].T
    return d_x, d_z


def ring_mask(X, Z, PML_size, pos_source, prec_deriv=8):
    """Boundary-ring mask for the time-reversed reconstruction,
    cuda_interface_pml.py:134-148: bands of width prec_deriv+1 just inside
    the PML on all four sides, plus every source cell."""
    m = prec_deriv + 1
    P = PML_size
    mask = np.full((Z, X), False)
    mask[P:P + m, P:-P] = True
    mask[-P - m:-P, P:-P] = True
    mask[P:-P, P:P + m] = True
    mask[P:-P, -P - m:-P] = True
    mask[pos_source] = True
    return mask


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32).ravel())


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel())


def _fp(a):
    return a.ctypes.data_as(_lib.c_float_p)


def _ip(a):
    return a.ctypes.data_as(_lib.c_int_p)


class Cuda_interface_PML:
    """cuda_interface_pml.py:33-249 re-stated over the B200 library."""

    def __init__(self, X, Z, T, PML_size, c, n_source, pos_source, n_sensor, pos_sensor, source,
                 initial=None, multishot=False, lib=None):
        self._lib = _lib.load(lib)
        self.pos_sensor = np.where(pos_sensor)
        self.pos_source = np.where(pos_source)
        self.X, self.Z, self.T = X, Z, T
        self.PML_size = PML_size
        self.cquad = (np.asarray(c) ** 2).astype(np.single)
        self.n_source = n_source
        self.pos_source_x = self.pos_source[1]
        self.pos_source_z = self.pos_source[0]
        self.n_sensor = n_sensor
        self.pos_sensor_x = self.pos_sensor[1]
        self.pos_sensor_z = self.pos_sensor[0]
        self.source = np.asarray(source).astype(np.single)
        self.d_x, self.d_z = self._calcPML()
        self.constvec = np.asarray([1, 1, 1]).astype(np.single)
        self._pos_revert = None
        self._pos_revert_x = None
        self._pos_revert_z = None
        self._tammaskrev = 0
        self.grad = np.zeros((Z, X)).astype(np.single)
        self.mse = np.zeros(1)
        self._cb = _lib.ADJ_CB(self.adj_wrapper)
        self.adj_wrapper_ptr = ctypes.cast(self._cb, ctypes.c_void_p)
        self._adj_fun = None
        self._multishot = multishot
        if multishot:
            self.recording = np.zeros((n_source, n_sensor, T)).astype(np.single)
        else:
            self.recording = np.zeros((n_sensor, T)).astype(np.single)
        self.idx_source = -1
        self.initial = np.zeros((Z, X, 2)) if initial is None else initial
        self.observed = None
        self.gradptr = None

        self._keep = [_f32(self.cquad), _f32(self.constvec), _f32(self.d_x), _f32(self.d_z),
                      _i32(self.pos_source_x), _i32(self.pos_source_z), _i32(self.pos_sensor_x),
                      _i32(self.pos_sensor_z), _f32(self.source), _f32(self.initial)]
        cq, cv, dx, dz, sx, sz, mx, mz, src, init = self._keep
        self.recptr = _lib.c_float_pp(_lib.c_float_p())
        self._lib.init_memory_sim(X, Z, T, _fp(cq), _fp(cv), _fp(dx), _fp(dz), int(n_source),
                                  _ip(sx), _ip(sz), int(n_sensor), _ip(mx), _ip(mz), _fp(src),
                                  _fp(init), self.recptr)
        _lib.check(self._lib)

    def _calcPML(self):
        return pml_damping(self.X, self.Z, self.PML_size)

    def init_regression(self, observed, adj_fun, prec_deriv=8):
        mask = ring_mask(self.X, self.Z, self.PML_size, self.pos_source, prec_deriv)
        self._pos_revert = np.where(mask)
        self._pos_revert_x = self._pos_revert[1]
        self._pos_revert_z = self._pos_revert[0]
        self._tammaskrev = int(np.sum(mask))
        self.observed = observed
        self._adj_fun = adj_fun
        self._keep_reg = [_f32(observed), _i32(self._pos_revert_x), _i32(self._pos_revert_z)]
        obs, rx, rz = self._keep_reg
        self.gradptr = _lib.c_float_pp(_lib.c_float_p())
        self._lib.init_memory_reg(_fp(obs), self.gradptr, _ip(rx), _ip(rz), self._tammaskrev)
        _lib.check(self._lib)

    def _set_c_quad(self, cquad):
        self.cquad = np.asarray(cquad).astype(np.single)
        buf = _f32(self.cquad)
        self._lib.setCquad(_fp(buf))
        _lib.check(self._lib)

    def _set_source(self, n_source, pos_source, source):
        self.pos_source = np.where(pos_source)
        self.source = np.asarray(source).astype(np.single)
        self.n_source = n_source
        self.pos_source_x = self.pos_source[1]
        self.pos_source_z = self.pos_source[0]
        sx, sz, src = _i32(self.pos_source_x), _i32(self.pos_source_z), _f32(self.source)
        self._lib.set_source(int(n_source), _ip(sx), _ip(sz), _fp(src))
        _lib.check(self._lib)

    def _rec_copy(self, out):
        ctypes.memmove(out.ctypes.data, self.recptr[0], self.n_sensor * self.T * 4)

    def simulate(self, output=False, c=None, idx_source=None):
        out_int = 1 if output else 0
        if c is not None:
            self._set_c_quad(np.asarray(c) ** 2)
        self.idx_source = -1 if idx_source is None else idx_source
        if not self._multishot:
            self._lib.cuda_simulate(out_int, int(self.idx_source))
            _lib.check(self._lib)
            self._rec_copy(self.recording)
        else:
            buffer = np.zeros((self.n_sensor, self.T)).astype(np.single)
            for s in range(self.n_source):
                self._lib.cuda_simulate(out_int, s)
                _lib.check(self._lib)
                self._rec_copy(buffer)
                self.recording[s, :, :] = buffer

    def calc_grad(self, c=None, idx_source=None):
        if c is not None:
            self._set_c_quad(np.asarray(c) ** 2)
        self.idx_source = -1 if idx_source is None else idx_source
        if not self._multishot:
            mse_f = (ctypes.c_float * 1)(*self.mse)
            self._lib.cuda_grad_ext(mse_f, self.adj_wrapper_ptr, int(self.idx_source))
            _lib.check(self._lib)
            ctypes.memmove(self.grad.ctypes.data, self.gradptr[0], self.Z * self.X * 4)
        else:
            self.mse[0] = 0
            mse_acc = 0
            grad_acc = np.zeros((self.Z, self.X)).astype(np.single)
            for s in range(self.n_source):
                self.idx_source = s
                mse_f = (ctypes.c_float * 1)(*self.mse)
                self._lib.cuda_grad_ext(mse_f, self.adj_wrapper_ptr, s)
                _lib.check(self._lib)
                ctypes.memmove(self.grad.ctypes.data, self.gradptr[0], self.Z * self.X * 4)
                grad_acc += self.grad
                mse_acc += self.mse[0]
            self.grad = grad_acc / self.n_source
            self.mse[0] = mse_acc / self.n_source

    def adj_wrapper(self, sim_c, adjoint_source_c):
        n = self.T * self.n_sensor
        # float64 copy of the float32 traces, as the reference's list slice does
        simulated = np.ctypeslib.as_array(sim_c, shape=(n,)).astype(np.float64).reshape(
            (self.n_sensor, self.T))
        if self._multishot:
            mse, source = self._adj_fun(simulated, self.observed[self.idx_source, :, :])
        else:
            mse, source = self._adj_fun(simulated, self.observed)
        out = np.ctypeslib.as_array(adjoint_source_c, shape=(n,))
        out[:] = np.asarray(source, dtype=np.float64).ravel()
        self.mse[0] = mse
