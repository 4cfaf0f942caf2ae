"""Trace misfits with the reference's call signature, computed on the GPU.

Each function takes (sim [n_traces, T], obs [n_traces, T]) and returns
(misfit, adjoint source [n_traces, T]) like the reference's
adjoint_functions.py, so it can be handed to ``Cuda_interface_PML.
init_regression`` as the adjoint callback:

  L2                    adjoint_functions.py:8-11
  wasserstein           adjoint_functions.py:25-67
  wasserstein_softplus  Wasserstein on softplus-normalised traces (no
                        reference counterpart; definition in misfit.cu)
  wasserstein_quad      adjoint_functions.py:70-108
  quad_envelope         adjoint_functions.py:14-22
  wasserstein_pm        adjoint_functions.py:144-223, its negative-part CDFs
                        built from the negative parts (lines 179-180 of the
                        reference take the positive ones)

The arithmetic runs in the library's misfit kernels (otf_misfit); device
memory comes from PyTorch. No CPU fallback: without a GPU these raise.
"""
import ctypes

import numpy as np

from . import _lib
from .batch import MISFITS, _declare


def _device_misfit(kind, sim, obs):
    import torch
    if not torch.cuda.is_available():
        raise _lib.OtfwiError("the misfit kernels need a CUDA device")
    lib = _declare(_lib.load())
    s = torch.as_tensor(np.ascontiguousarray(sim, dtype=np.float32)).cuda()
    o = torch.as_tensor(np.ascontiguousarray(obs, dtype=np.float32)).cuda()
    if s.ndim == 1:
        s, o = s[None], o[None]
    n, T = s.shape
    adj = torch.empty_like(s)
    mis = torch.empty(n, dtype=torch.float64, device=s.device)
    nb = int(lib.otf_misfit_scratch_bytes(kind, n, T))
    scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device=s.device)
    st = torch.cuda.current_stream().cuda_stream
    rc = lib.otf_misfit(kind, ctypes.c_void_p(s.data_ptr()), ctypes.c_void_p(o.data_ptr()),
                        ctypes.c_void_p(adj.data_ptr()), ctypes.c_void_p(mis.data_ptr()), n, T,
                        ctypes.c_void_p(scratch.data_ptr()), nb, ctypes.c_void_p(st))
    if rc != 0:
        _lib.check(lib)
        raise _lib.OtfwiError("otf_misfit failed")
    torch.cuda.current_stream().synchronize()
    return float(mis.sum().item()), adj.cpu().numpy().astype(np.float64)


def L2(sim, obs):
    return _device_misfit(MISFITS["l2"], sim, obs)


def wasserstein(sim, obs):
    return _device_misfit(MISFITS["wasserstein"], sim, obs)


def wasserstein_softplus(sim, obs):
    return _device_misfit(MISFITS["wasserstein_softplus"], sim, obs)


def wasserstein_quad(sim, obs):
    return _device_misfit(MISFITS["wasserstein_quad"], sim, obs)


def quad_envelope(sim, obs):
    return _device_misfit(MISFITS["quad_envelope"], sim, obs)


def wasserstein_pm(sim, obs):
    return _device_misfit(MISFITS["wasserstein_pm"], sim, obs)
