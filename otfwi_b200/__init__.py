"""Otfwi on B200: the inversion hot path of lassip-utfpr/Otfwi (2D acoustic
split-field PML forward / adjoint, source injection and receiver recording,
cross-correlation gradient, Wasserstein trace misfit) as hand-written sm_100a
CUDA behind the reference's own C ABI.

  otfwi_b200.cuda_interface_pml  host mirror of the reference's ctypes wrapper
  otfwi_b200.adjoint_functions   misfits with the reference's call signature
  otfwi_b200.batch               all shots of an acquisition in one launch stream
  otfwi_b200.scenarios           seeded synthetic NDT scenarios
"""
__all__ = ["cuda_interface_pml", "batch", "scenarios"]
