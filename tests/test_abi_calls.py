"""The mirror wrapper (otfwi_b200/cuda_interface_pml.py) drives the C ABI
exactly as the reference's unchanged cuda_interface_pml.py does.

Both wrappers run the same session -- construction (init_memory_sim),
simulate over every shot and for one shot, init_regression, calc_grad over
every shot and for one shot with a model update (setCquad), the misfit
callback -- against a recording stand-in library (tests/abi_stub/
abi_recorder.c, built here with gcc) that logs each call with digests of its
array arguments and returns deterministic traces and gradients. Identical
logs and identical wrapper outputs mean that the GPU parity tests, which
drive libotfwi.so through the mirror, stand for the reference's own wrapper
driving it: the reference's Python stays in the reference tree (it is not
carried to the GPU machine), so this check runs here, on CPU, wherever that
tree is present.

The wrappers' one deliberate difference is not exercised: _set_source
(cuda_interface_pml.py:163-183) takes positions from the mask it is given
(pos_source[1], pos_source[0]) where the mirror uses np.where of it, as the
constructor does; the reference library does not export set_source at all.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import misfit_oracle as mo
from conftest import ROOT
from test_abi import _load_reference_wrapper

STUB = os.path.join(ROOT, "tests", "abi_stub", "abi_recorder.c")


def _build_stub(tmp_path):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    out = tmp_path / "abi_recorder.so"
    subprocess.run(["gcc", "-O1", "-fPIC", "-shared", "-o", str(out), STUB], check=True)
    return str(out)


def _session(cls, sc, log, **kw):
    os.environ["OTFWI_ABI_LOG"] = str(log)
    try:
        out = {}
        cp = cls(sc.X, sc.Z, sc.T, sc.PML, sc.c_true, sc.n_src, sc.src_mask, sc.n_rec, sc.rec_mask, sc.source,
                 multishot=True, **kw)
        cp.simulate()
        out["recording"] = cp.recording.copy()
        obs = (0.9 * cp.recording).astype(np.float32)
        cp.init_regression(obs, mo.L2, prec_deriv=4)
        cp.calc_grad(c=sc.c_start)
        out["grad"], out["mse"] = cp.grad.copy(), cp.mse.copy()
        one = cls(sc.X, sc.Z, sc.T, sc.PML, sc.c_true, sc.n_src, sc.src_mask, sc.n_rec, sc.rec_mask, sc.source,
                  multishot=False, **kw)
        one.simulate(idx_source=1)
        out["recording1"] = one.recording.copy()
        one.init_regression(obs[1], mo.wasserstein, prec_deriv=8)
        one.calc_grad(c=0.98 * sc.c_start, idx_source=1)
        out["grad1"], out["mse1"] = one.grad.copy(), one.mse.copy()
        return out, open(log).read().splitlines()
    finally:
        os.environ.pop("OTFWI_ABI_LOG", None)


def test_mirror_makes_the_reference_wrappers_calls(tmp_path):
    from otfwi_b200 import scenarios
    from otfwi_b200.cuda_interface_pml import Cuda_interface_PML
    stub = _build_stub(tmp_path)
    ref = _load_reference_wrapper(tmp_path, stub)  # binds simulator/bin/... = the stub
    sc = scenarios.small(X=80, Z=72, T=60, n_src=3, n_rec=5, seed=2, f0=0.08)
    sc.c_start = sc.c_start * 1.01
    a, log_a = _session(ref.Cuda_interface_PML, sc, tmp_path / "ref.log")
    b, log_b = _session(Cuda_interface_PML, sc, tmp_path / "mirror.log", lib=stub)
    assert len(log_a) == len(log_b) > 10
    for i, (la, lb) in enumerate(zip(log_a, log_b)):
        assert la == lb, (i, la, lb)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
