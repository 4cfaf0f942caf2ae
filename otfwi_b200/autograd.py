"""Differentiable wave propagation: a torch.autograd.Function over the
velocity model.

``PMLPropagator(...)(c)`` returns the traces of every shot [n_shots, n_rec,
T] for the nondimensional velocity model c [Z, X] (c = v dt/dx, the
reference's convention). Any loss built from the traces in torch
back-propagates into c through the library's exact discrete adjoint of the
forward map (otf_batch_backward_exact), with the wavefield kept only every
``checkpoint_every`` steps (default ceil(sqrt(T-1))) and each segment's
forward recomputed once during the backward sweep.
"""
import ctypes
import math


from . import _lib
from .batch import ShotBatch, _declare


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


class PMLPropagator:
    """Forward operator c -> traces for a fixed acquisition (one ShotBatch)."""

    def __init__(self, X, Z, T, PML_size, src_mask, rec_mask, source, shots=None, precision=1, tile=0,
                 checkpoint_every=None, constvec=(1.0, 1.0, 1.0)):
        self.batch = ShotBatch(X, Z, T, PML_size, src_mask, rec_mask, source, prec_deriv=4, shots=shots,
                               precision=precision, tile=tile, constvec=constvec)
        _declare(self.batch._lib)
        L = self.batch._lib
        L.otf_batch_forward_ckpt.restype = ctypes.c_int
        L.otf_batch_forward_ckpt.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        L.otf_batch_backward_exact.restype = ctypes.c_int
        L.otf_batch_backward_exact.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                               ctypes.c_void_p, ctypes.c_int]
        self.every = int(checkpoint_every or max(1, math.ceil(math.sqrt(T - 1))))
        self._version = 0

    @property
    def shape(self):
        b = self.batch
        return (b.n_shots, b.n_rec, b.T)

    def _forward(self, c):
        import torch
        b = self.batch
        b.set_model(cquad=(c.detach().float() ** 2).contiguous())
        out = torch.empty(self.shape, dtype=torch.float32, device=c.device)
        torch.cuda.current_stream().synchronize()
        b._ok(b._lib.otf_batch_forward_ckpt(b._h, self.every, _vp(out), 1))
        b.sync()
        self._version += 1
        return out

    def _backward(self, c, g):
        import torch
        b = self.batch
        grad_c2 = torch.empty((b.Z, b.X), dtype=torch.float32, device=c.device)
        g = g.detach().float().contiguous()
        torch.cuda.current_stream().synchronize()
        b._ok(b._lib.otf_batch_backward_exact(b._h, _vp(g), 1, _vp(grad_c2), 1))
        b.sync()
        return grad_c2

    def __call__(self, c):
        return _PMLFunction.apply(c, self)

    def gradient_c2(self, c, g):
        """dL/d(c^2) [Z, X] for dL/dtraces = g, at model c (runs the forward)."""
        self._forward(c)
        return self._backward(c, g)


class _PMLFunction:
    pass


def _make_function():
    import torch

    class PMLFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, c, prop):
            out = prop._forward(c)
            ctx.save_for_backward(c)
            ctx.prop = prop
            ctx.version = prop._version
            return out

        @staticmethod
        def backward(ctx, g):
            (c,) = ctx.saved_tensors
            prop = ctx.prop
            if prop._version != ctx.version:  # another forward reused the checkpoints
                prop._forward(c)
            grad_c2 = prop._backward(c, g)
            return (2.0 * c.detach().float() * grad_c2).to(c.dtype), None

    return PMLFunction


try:
    _PMLFunction = _make_function()
except ImportError:  # torch absent: the propagator is unusable anyway
    pass
