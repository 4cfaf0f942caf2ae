"""GPU tests of the headless video frames (cuda_simulate with en_out = 1 and
otf_batch_frames): with faithful numerics the device's 8-bit frames equal the
oracle's byte for byte (the oracle's are pinned to the reference's traces and
to a numpy restatement of writeFramePipe by tests/test_frames.py); with the
fast numerics they differ by at most one grey level."""
import os
import sys

import numpy as np
import pytest

import pml_oracle as po
from abi_driver import _f32, _fp, _i32, _ip
from conftest import GOLDEN, ROOT

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

pytestmark = pytest.mark.gpu


def _oracle_frames(d, every, idx_source=-1):
    return po.frames(np.asarray(d["c_true"], np.float32) ** 2, d["constvec"], d["d_x"], d["d_z"], d["src_x"],
                     d["src_z"], d["source"], d["rec_x"], d["rec_z"], every=every, idx_source=idx_source)[0]


@pytest.mark.parametrize("name", ["small", "general"])
def test_dropin_en_out_writes_reference_frames(lib, tmp_path, name):
    from otfwi_b200 import _lib
    from otfwi_b200._lib import c_float_p, c_float_pp
    d = dict(np.load(os.path.join(GOLDEN, f"sim_{name}.npz")))
    X, Z, T = int(d["X"]), int(d["Z"]), int(d["T"])
    nm = len(d["rec_x"])
    k = dict(cq=_f32(np.asarray(d["c_true"], np.float32) ** 2), cv=_f32(d["constvec"]), dx=_f32(d["d_x"]),
             dz=_f32(d["d_z"]), sx=_i32(d["src_x"]), sz=_i32(d["src_z"]), mx=_i32(d["rec_x"]),
             mz=_i32(d["rec_z"]), src=_f32(d["source"]), init=_f32(np.zeros((Z, X, 2))))
    recptr = c_float_pp(c_float_p())
    lib.init_memory_sim(X, Z, T, _fp(k["cq"]), _fp(k["cv"]), _fp(k["dx"]), _fp(k["dz"]), len(d["src_x"]),
                        _ip(k["sx"]), _ip(k["sz"]), nm, _ip(k["mx"]), _ip(k["mz"]), _fp(k["src"]),
                        _fp(k["init"]), recptr)
    _lib.check(lib)
    path = tmp_path / "video" / "frames.gray"
    os.environ["OTFWI_FRAMES_PATH"] = str(path)
    try:
        lib.cuda_simulate(1, -1)
        _lib.check(lib)
    finally:
        os.environ.pop("OTFWI_FRAMES_PATH", None)
    got = np.fromfile(path, np.uint8)
    assert got.size == (T - 1) * Z * X
    ref = _oracle_frames(d, 1)
    nd = int(np.sum(got.reshape(ref.shape) != ref))
    assert nd == 0, (name, nd)
    # the traces of the same call are those of the plain forward (the reference's)
    tr = np.ctypeslib.as_array(recptr[0], shape=(nm * T,)).copy().reshape(nm, T)
    assert np.array_equal(tr[:, 1:], d["traces_all"][:, 1:])
    lib.otf_release()


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_frames_of_one_shot(lib, precision):
    import make_sim_golden
    from otfwi_b200 import scenarios
    from otfwi_b200.batch import ShotBatch
    from otfwi_b200.cuda_interface_pml import pml_damping
    sc = scenarios.small(X=128, Z=96, T=300, n_src=3, n_rec=10, seed=21, f0=0.035)
    inp = make_sim_golden.case_inputs(sc, *pml_damping(sc.X, sc.Z, sc.PML), np.ones(3))
    b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, precision=precision)
    b.set_model(inp["c_true"])  # the FP32 model the oracle squares
    got = b.frames(every=5, shot=1)
    ref = _oracle_frames(inp, 5, idx_source=1)
    assert got.shape == ref.shape
    diff = np.abs(got.astype(np.int16) - ref.astype(np.int16))
    if precision == 0:
        assert int(np.sum(diff != 0)) == 0
    else:
        assert diff.max() <= 1 and np.mean(diff != 0) < 0.05, (diff.max(), np.mean(diff != 0))
    # traces were recorded as by the plain forward
    tr = b.forward()
    fr2 = b.frames(every=5, shot=1)
    assert np.array_equal(fr2, got)
    assert np.array_equal(b.forward(), tr)
    b.close()
