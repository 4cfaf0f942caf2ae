"""CPU tests of the C-ABI boundary: the library loads and exports every
symbol include/otfwi.h declares; the reference's own ctypes wrapper binds to
it unchanged; host-side set-up logic matches the reference. No compute calls
(no GPU here)."""
import importlib.util
import os
import shutil

import numpy as np
import pytest

from conftest import REFERENCE, ROOT


def test_library_exports_header_symbols(lib):
    from otfwi_b200 import _lib
    names = _lib.exported_symbols_from_header(os.path.join(ROOT, "include", "otfwi.h"))
    # the reference ABI (regression_PML_single.cu / hilbert.cpp) is all there
    for ref_name in ("init_memory_sim", "init_memory_reg", "setCquad", "cuda_simulate",
                     "cuda_grad_ext", "def_python_adj", "hilbert"):
        assert ref_name in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_dropin_file_name_exists(lib):
    from otfwi_b200 import _lib
    assert os.path.exists(_lib.DROPIN)


def test_calls_before_init_report_errors_without_gpu(lib):
    from otfwi_b200 import _lib
    lib.otf_release()
    lib.otf_clear_error()
    lib.cuda_simulate(0, -1)
    assert lib.otf_last_status() != 0
    assert b"before init_memory_sim" in lib.otf_last_error()
    with pytest.raises(_lib.OtfwiError):
        lib.cuda_simulate(0, -1)
        _lib.check(lib)


def test_oversized_grid_is_refused_before_any_input_is_read(lib):
    """A 46400 x 46400 grid pads to more than 2^31 cells per field, past the
    32-bit cell offsets of the point tables: init_memory_sim records an error
    before it reads an input array (one-element arrays stand in for them)."""
    import ctypes
    from ctypes import POINTER, c_float, c_int
    lib.otf_release()
    lib.otf_clear_error()
    one_f = (c_float * 3)(1.0, 1.0, 1.0)
    one_i = (c_int * 1)(20)
    rec = POINTER(c_float)()
    lib.init_memory_sim(46400, 46400, 100, one_f, one_f, one_f, one_f, 1, one_i, one_i, 1, one_i, one_i,
                        one_f, None, ctypes.byref(rec))
    assert lib.otf_last_status() != 0
    assert b"grid too large" in lib.otf_last_error()
    lib.otf_release()
    lib.otf_clear_error()


def test_product_entry_points_fail_loudly_without_a_gpu(lib):
    """There is no CPU fallback: without a CUDA device every public entry
    point (the reference wrapper's mirror, the batched shots, the
    reference-signature misfits, the CPML simulator) raises OtfwiError."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from otfwi_b200 import _lib, adjoint_functions, scenarios
    from otfwi_b200.batch import ShotBatch
    from otfwi_b200.cpml import CPMLSimulator
    from otfwi_b200.cuda_interface_pml import Cuda_interface_PML
    sc = scenarios.small(X=96, Z=80, T=50, n_src=1, n_rec=4, seed=1)
    calls = [
        lambda: Cuda_interface_PML(sc.X, sc.Z, sc.T, sc.PML, sc.c_true, sc.n_src, sc.src_mask, sc.n_rec,
                                   sc.rec_mask, sc.source, multishot=True).simulate(),
        lambda: ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source).forward(),
        lambda: CPMLSimulator(sc.X, sc.Z, sc.T, sc.PML, sc.c_true, sc.src_mask, sc.rec_mask, sc.source,
                              f0=0.04).simulate(-1),
    ]
    tr = np.zeros((2, 16), np.float32)
    for name in ("L2", "wasserstein", "wasserstein_softplus", "wasserstein_quad", "quad_envelope",
                 "wasserstein_pm"):
        calls.append(lambda f=getattr(adjoint_functions, name): f(tr, tr))
    for call in calls:
        with pytest.raises(_lib.OtfwiError):
            call()
    lib.otf_release()
    lib.otf_clear_error()


def _load_reference_wrapper(tmp_path, libpath):
    """Import the reference's unchanged cuda_interface_pml.py with CWD set so
    its relative 'simulator/bin/cuda_regression_PML_single.so' is this library."""
    src = os.path.join(REFERENCE, "cuda_interface_pml.py")
    if not os.path.exists(src):
        pytest.skip("reference tree not present")
    os.makedirs(tmp_path / "simulator" / "bin", exist_ok=True)
    shutil.copyfile(libpath, tmp_path / "simulator" / "bin" / "cuda_regression_PML_single.so")
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        spec = importlib.util.spec_from_file_location("ref_cuda_interface_pml", src)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        os.chdir(cwd)
    return mod


def test_unchanged_reference_wrapper_binds(tmp_path, lib):
    from otfwi_b200 import _lib
    mod = _load_reference_wrapper(tmp_path, _lib.LIB)
    # module-level bindings of cuda_interface_pml.py:17-30 resolved against us
    for name in ("cuda_init_sim", "cuda_init_reg", "cuda_set_cquad", "cuda_simulate_c", "cuda_grad_c"):
        assert getattr(mod, name) is not None
    assert hasattr(mod.clib, "set_source")  # what _set_source (:183) calls


def test_damping_and_ring_match_reference_wrapper(tmp_path, lib):
    from otfwi_b200 import _lib
    from otfwi_b200.cuda_interface_pml import pml_damping, ring_mask
    mod = _load_reference_wrapper(tmp_path, _lib.LIB)

    class Fake:
        pass

    f = Fake()
    f.X, f.Z, f.PML_size = 96, 80, 20
    dx_ref, dz_ref = mod.Cuda_interface_PML._calcPML(f)
    dx, dz = pml_damping(96, 80, 20)
    assert np.array_equal(dx, dx_ref) and np.array_equal(dz, dz_ref)

    # init_regression builds the ring before calling into C; capture the mask
    f.pos_source = (np.array([26, 30]), np.array([40, 50]))
    captured = {}
    orig = mod.cuda_init_reg
    mod.cuda_init_reg = lambda obs, gp, rx, rz, n: captured.update(rx=list(rx), rz=list(rz), n=n.value)
    try:
        mod.Cuda_interface_PML.init_regression(f, np.zeros((2, 3, 4), np.float32), None, prec_deriv=4)
    finally:
        mod.cuda_init_reg = orig
    m = ring_mask(96, 80, 20, f.pos_source, 4)
    rz, rx = np.where(m)
    assert captured["n"] == m.sum()
    assert captured["rx"] == list(rx) and captured["rz"] == list(rz)
