"""Batched multi-shot forward modelling and gradients on one GPU.

``ShotBatch`` wraps the library's batched C ABI (otf_batch_*). It takes the
same inputs as the reference wrapper (``Cuda_interface_PML``: grid, PML
damping, nondimensional velocity, source / receiver masks, source waveforms,
the boundary ring of ``init_regression``), but every shot of a shot table
advances in the same kernel launches, the misfit and its adjoint source are
computed on the device, and a gradient is one CUDA-graph replay.

Arrays may be numpy (host) or torch CUDA tensors (device); results come back
in the same kind as requested.
"""
import ctypes
from ctypes import POINTER, c_float, c_int, c_longlong, c_void_p

import numpy as np

from . import _lib
from .cuda_interface_pml import pml_damping, ring_mask

MISFITS = {"l2": 0, "wasserstein": 1, "wasserstein_softplus": 2, "wasserstein_quad": 3, "quad_envelope": 4,
           "wasserstein_pm": 5}


def _declare(lib):
    if getattr(lib, "_batch_declared", False):
        return lib
    fp, ip = POINTER(c_float), POINTER(c_int)
    lib.otf_batch_create.restype = c_void_p
    lib.otf_batch_create.argtypes = [c_int, c_int, c_int, fp, fp, fp, c_int, ip, ip, fp, c_int, ip, ip,
                                     c_int, ip, ip, c_int, c_int, c_int]
    lib.otf_batch_destroy.restype = None
    lib.otf_batch_destroy.argtypes = [c_void_p]
    for name, args in {
        "otf_batch_set_shots": [c_void_p, c_int, ip, ip],
        "otf_batch_set_model": [c_void_p, c_void_p, c_int],
        "otf_batch_set_observed": [c_void_p, c_void_p, c_int],
        "otf_batch_set_precision": [c_void_p, c_int],
        "otf_batch_set_tile": [c_void_p, c_int],
        "otf_batch_set_kernel": [c_void_p, c_int],
        "otf_batch_set_stream_rows": [c_void_p, c_int],
        "otf_batch_set_paired_lead": [c_void_p, c_int],
        "otf_batch_set_fused_rows": [c_void_p, c_int],
        "otf_batch_set_lanes": [c_void_p, c_int],
        "otf_batch_lanes": [c_void_p],
        "otf_batch_forward": [c_void_p, c_void_p, c_int],
        "otf_batch_forward_ring": [c_void_p, c_void_p, c_int],
        "otf_batch_gradient": [c_void_p, c_int, c_void_p, c_void_p, c_int],
        "otf_batch_misfit": [c_void_p, c_int, c_void_p, c_int],
        "otf_batch_adjoint": [c_void_p, c_void_p, c_int],
        "otf_batch_reverse": [c_void_p, c_void_p, c_int, c_void_p, c_float, c_int],
        "otf_batch_shot_grad": [c_void_p, c_int, c_void_p, c_int],
        "otf_batch_sync": [c_void_p],
        "otf_batch_objective": [c_void_p, c_int, c_void_p, c_int],
        "otf_batch_illumination": [c_void_p, c_int, c_void_p, c_int],
        "otf_batch_frames": [c_void_p, c_int, c_int, c_void_p],
        "otf_misfit": [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p,
                       c_longlong, c_void_p],
    }.items():
        f = getattr(lib, name)
        f.restype = c_int
        f.argtypes = args
    lib.otf_batch_stream.restype = c_void_p
    lib.otf_batch_stream.argtypes = [c_void_p]
    lib.otf_misfit_scratch_bytes.restype = c_longlong
    lib.otf_misfit_scratch_bytes.argtypes = [c_int, c_int, c_int]
    lib._batch_declared = True
    return lib


def _is_torch(a):
    return type(a).__module__.startswith("torch")


def _ptr(a):
    """(pointer, on_device) of a numpy array or torch CUDA tensor. A CUDA
    tensor's pending work on torch's current stream is waited for first: the
    library reads and writes it on the batch's own stream."""
    if a is None:
        return None, 0
    if _is_torch(a):
        assert a.is_contiguous()
        if a.is_cuda:
            import torch
            torch.cuda.current_stream(a.device).synchronize()
        return ctypes.c_void_p(a.data_ptr()), int(a.is_cuda)
    return ctypes.c_void_p(a.ctypes.data), 0


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32).ravel())


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel())


def fmc_shots(n):
    """Full-matrix capture shot table: shot s fires source s alone."""
    return np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32)


class ShotBatch:
    """All shots of one acquisition on one GPU.

    Parameters follow ``Cuda_interface_PML`` (cuda_interface_pml.py:34) plus
    the ring width of ``init_regression`` (``prec_deriv``), the shot table
    (default: full-matrix capture, one shot per source) and the numerics
    (``precision`` 0 = faithful to the reference, 1 = fast FP32 sums)."""

    def __init__(self, X, Z, T, PML_size, src_mask, rec_mask, source, prec_deriv=4, shots=None,
                 max_shots=None, precision=0, tile=0, constvec=(1.0, 1.0, 1.0), d_x=None, d_z=None,
                 kernel=-1, lib=None):
        self._lib = _declare(_lib.load(lib))
        self.X, self.Z, self.T, self.PML = X, Z, T, PML_size
        pz, px = np.where(src_mask)
        mz, mx = np.where(rec_mask)
        self.n_src, self.n_rec = len(px), len(mx)
        if d_x is None:
            d_x, d_z = pml_damping(X, Z, PML_size)
        rz, rx = np.where(ring_mask(X, Z, PML_size, np.where(src_mask), prec_deriv))
        ptr, srcs = shots if shots is not None else fmc_shots(self.n_src)
        self.n_shots = len(ptr) - 1
        ms = max_shots or self.n_shots
        k = [_f32(constvec), _f32(d_x), _f32(d_z), _i32(px), _i32(pz), _f32(source), _i32(mx), _i32(mz),
             _i32(rx), _i32(rz)]
        fp = lambda a: a.ctypes.data_as(POINTER(c_float))
        ip = lambda a: a.ctypes.data_as(POINTER(c_int))
        h = self._lib.otf_batch_create(X, Z, T, fp(k[0]), fp(k[1]), fp(k[2]), self.n_src, ip(k[3]),
                                       ip(k[4]), fp(k[5]), self.n_rec, ip(k[6]), ip(k[7]), len(rx),
                                       ip(k[8]), ip(k[9]), ms, precision, tile)
        if not h:
            _lib.check(self._lib)
            raise _lib.OtfwiError("otf_batch_create failed")
        self._h = c_void_p(h)
        self.set_kernel(kernel)
        self.set_shots(ptr, srcs)

    def _ok(self, rc):
        if rc != 0:
            _lib.check(self._lib)
            raise _lib.OtfwiError("batched call failed")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.otf_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_shots(self, ptr, srcs):
        ptr, srcs = _i32(ptr), _i32(srcs)
        self.n_shots = len(ptr) - 1
        self._ok(self._lib.otf_batch_set_shots(self._h, self.n_shots, ptr.ctypes.data_as(POINTER(c_int)),
                                               srcs.ctypes.data_as(POINTER(c_int))))

    def set_model(self, c=None, cquad=None):
        """Nondimensional velocity c (or c^2 directly), [Z, X]."""
        if cquad is None:
            cquad = c * c if _is_torch(c) else np.asarray(c, np.float64) ** 2
        if not _is_torch(cquad):
            cquad = _f32(cquad)
        else:
            cquad = cquad.float().contiguous()
        p, dev = _ptr(cquad)
        self._ok(self._lib.otf_batch_set_model(self._h, p, dev))
        if dev:
            self.sync()  # the library reads the tensor on its own stream
        self._keep_model = cquad

    def set_observed(self, obs):
        if not _is_torch(obs):
            obs = _f32(obs)
        p, dev = _ptr(obs)
        self._ok(self._lib.otf_batch_set_observed(self._h, p, dev))
        if dev:
            self.sync()
        self._keep_obs = obs

    def set_precision(self, precision):
        self._ok(self._lib.otf_batch_set_precision(self._h, precision))

    def set_tile(self, tile):
        self._ok(self._lib.otf_batch_set_tile(self._h, tile))

    def set_kernel(self, variant):
        """-1: automatic; 0: one tile per CTA per step; 1: persistent
        TMA-pipelined CTAs; 2: persistent strip-split kernels (fast numerics);
        3: z-streaming strips (fast numerics); 4: unfused streaming
        half-steps (fast numerics); 5: paired half-steps, one launch per
        step (fast numerics); 6: row-lag fused half-steps, one pass per step
        (fast numerics)."""
        self._ok(self._lib.otf_batch_set_kernel(self._h, variant))

    def set_lanes(self, lanes):
        """Shot groups run as parallel launch chains by the unfused kernels
        (0: automatic, one per 16 shots up to 4; 1: one chain)."""
        self._ok(self._lib.otf_batch_set_lanes(self._h, int(lanes)))

    def lanes(self):
        """Lanes (parallel launch chains) of this batch's time loops."""
        return int(self._lib.otf_batch_lanes(self._h))

    def set_fused_rows(self, rows):
        """Rows per chunk of the row-lag fused kernels (variant 6, >= 8)."""
        self._ok(self._lib.otf_batch_set_fused_rows(self._h, int(rows)))

    def set_paired_lead(self, lead):
        """P items issued before the first A item by the paired kernels
        (variant 5); 0 = one generation of resident CTAs."""
        self._ok(self._lib.otf_batch_set_paired_lead(self._h, int(lead)))

    def set_stream_rows(self, rows):
        """Rows per segment of the z-streaming kernels (variant 3)."""
        self._ok(self._lib.otf_batch_set_stream_rows(self._h, int(rows)))

    def sync(self):
        self._ok(self._lib.otf_batch_sync(self._h))

    def stream(self):
        return self._lib.otf_batch_stream(self._h)

    def forward(self, out=None, ring=False):
        """Traces of every shot [n_shots, n_rec, T] (numpy unless ``out`` is a tensor)."""
        if out is None:
            out = np.zeros((self.n_shots, self.n_rec, self.T), np.float32)
        p, dev = _ptr(out)
        f = self._lib.otf_batch_forward_ring if ring else self._lib.otf_batch_forward
        self._ok(f(self._h, p, dev))
        self.sync()
        return out

    def gradient(self, misfit="wasserstein", grad=None, misfit_out=None):
        """(shot-mean gradient w.r.t. c^2 [Z, X], total misfit) in one graph replay."""
        kind = MISFITS[misfit] if isinstance(misfit, str) else int(misfit)
        if grad is None:
            grad = np.zeros((self.Z, self.X), np.float32)
        gp, dev = _ptr(grad)
        if misfit_out is None:
            misfit_out = np.zeros(1, np.float64) if not dev else None
        mp, _ = _ptr(misfit_out)
        self._ok(self._lib.otf_batch_gradient(self._h, kind, gp, mp, dev))
        self.sync()
        if not dev:
            return grad, float(misfit_out[0])
        return grad, misfit_out

    def objective(self, misfit="wasserstein", out=None):
        """Total misfit of a forward of every shot (no reverse phase): a
        line-search evaluation, one graph replay. ``out``: optional float64
        device tensor of one element."""
        kind = MISFITS[misfit] if isinstance(misfit, str) else int(misfit)
        host = out is None
        if host:
            out = np.zeros(1, np.float64)
        p, dev = _ptr(out)
        self._ok(self._lib.otf_batch_objective(self._h, kind, p, dev))
        self.sync()
        return float(out[0]) if host else out

    def illumination(self, every=8, out=None):
        """Sum over shots and every ``every``-th forward step of P^2, [Z, X]."""
        if out is None:
            out = np.zeros((self.Z, self.X), np.float32)
        p, dev = _ptr(out)
        self._ok(self._lib.otf_batch_illumination(self._h, int(every), p, dev))
        self.sync()
        return out

    def frames(self, every=1, shot=0):
        """Headless video of one forward modelling (the reference's
        ``simulate(output=True)`` frames): uint8 [(T-1)//every, Z, X], the
        total pressure of shot ``shot`` at steps every, 2 every, ... mapped
        from the frame's [min, max] onto 0..255, receivers 255. Traces of
        every shot are recorded as by ``forward``."""
        n = (self.T - 1) // int(every)
        out = np.zeros((n, self.Z, self.X), np.uint8)
        self._ok(self._lib.otf_batch_frames(self._h, int(every), int(shot), ctypes.c_void_p(out.ctypes.data)))
        self.sync()
        return out

    def misfit(self, misfit="wasserstein"):
        kind = MISFITS[misfit] if isinstance(misfit, str) else int(misfit)
        out = np.zeros(self.n_shots * self.n_rec, np.float64)
        self._ok(self._lib.otf_batch_misfit(self._h, kind, ctypes.c_void_p(out.ctypes.data), 0))
        adj = np.zeros((self.n_shots, self.n_rec, self.T), np.float32)
        self._ok(self._lib.otf_batch_adjoint(self._h, ctypes.c_void_p(adj.ctypes.data), 0))
        self.sync()
        return out.reshape(self.n_shots, self.n_rec), adj

    def reverse(self, adj=None, grad=None, scale=1.0):
        """Reverse phase after forward(ring=True) with adjoint sources
        [n_shots, n_rec, T] (None: those of the last misfit()); returns
        scale * sum over shots of the gradients."""
        if adj is not None and not _is_torch(adj):
            adj = _f32(adj)
        ap, adev = _ptr(adj)
        if grad is None:
            grad = np.zeros((self.Z, self.X), np.float32)
        gp, gdev = _ptr(grad)
        self._ok(self._lib.otf_batch_reverse(self._h, ap, adev, gp, float(scale), gdev))
        self.sync()
        return grad

    def shot_gradient(self, shot):
        g = np.zeros((self.Z, self.X), np.float32)
        self._ok(self._lib.otf_batch_shot_grad(self._h, shot, ctypes.c_void_p(g.ctypes.data), 0))
        self.sync()
        return g


def device_misfit(sim, obs, misfit="wasserstein", lib=None):
    """Misfit + adjoint source of host traces [n, T] on the GPU (test helper)."""
    import torch
    L = _declare(_lib.load(lib))
    kind = MISFITS[misfit]
    s = torch.as_tensor(np.asarray(sim, np.float32)).cuda().contiguous()
    o = torch.as_tensor(np.asarray(obs, np.float32)).cuda().contiguous()
    n, T = s.shape
    adj = torch.empty_like(s)
    mis = torch.empty(n, dtype=torch.float64, device=s.device)
    nb = int(L.otf_misfit_scratch_bytes(kind, n, T))
    scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device=s.device)
    st = torch.cuda.current_stream().cuda_stream
    rc = L.otf_misfit(kind, c_void_p(s.data_ptr()), c_void_p(o.data_ptr()), c_void_p(adj.data_ptr()),
                      c_void_p(mis.data_ptr()), n, T, c_void_p(scratch.data_ptr()), nb, c_void_p(st))
    if rc != 0:
        _lib.check(L)
        raise _lib.OtfwiError("otf_misfit failed")
    torch.cuda.synchronize()
    return mis.cpu().numpy(), adj.cpu().numpy()


class MultiBatch:
    """Independent inversions (different grids, shot counts and T) whose
    gradients run as parallel branches of one CUDA graph (otf_multi_*): one
    launch for all of them. The ShotBatch instances stay owned by the caller."""

    def __init__(self, batches):
        self.batches = list(batches)
        L = self._lib = self.batches[0]._lib
        if not getattr(L, "_multi_declared", False):
            L.otf_multi_create.restype = c_void_p
            L.otf_multi_create.argtypes = [c_int, ctypes.c_void_p]
            L.otf_multi_destroy.restype = None
            L.otf_multi_destroy.argtypes = [c_void_p]
            for name in ("otf_multi_gradient",):
                getattr(L, name).restype = c_int
                getattr(L, name).argtypes = [c_void_p, c_int]
            L.otf_multi_sync.restype = c_int
            L.otf_multi_sync.argtypes = [c_void_p]
            L.otf_batch_last_gradient.restype = c_int
            L.otf_batch_last_gradient.argtypes = [c_void_p, c_void_p, c_void_p, c_int]
            L._multi_declared = True
        arr = (c_void_p * len(self.batches))(*[b._h.value for b in self.batches])
        h = L.otf_multi_create(len(self.batches), arr)
        if not h:
            _lib.check(L)
            raise _lib.OtfwiError("otf_multi_create failed")
        self._h = c_void_p(h)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.otf_multi_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def gradient(self, misfit="wasserstein"):
        """[(grad [Z, X], misfit)] of every instance from one graph launch."""
        kind = MISFITS[misfit] if isinstance(misfit, str) else int(misfit)
        L = self._lib
        if L.otf_multi_gradient(self._h, kind) != 0 or L.otf_multi_sync(self._h) != 0:
            _lib.check(L)
            raise _lib.OtfwiError("multi-instance gradient failed")
        out = []
        for b in self.batches:
            g = np.zeros((b.Z, b.X), np.float32)
            m = np.zeros(1, np.float64)
            b._ok(L.otf_batch_last_gradient(b._h, ctypes.c_void_p(g.ctypes.data),
                                            ctypes.c_void_p(m.ctypes.data), 0))
            b.sync()
            out.append((g, float(m[0])))
        return out
