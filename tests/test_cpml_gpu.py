"""GPU tests of the second-order CPML library (lib/cuda_regression_CPML.so)
against the reference's own CPML library outputs (tests/golden/cpml_*.npz,
made by tests/golden/make_cpml_golden.py) and the CPU oracle.

Tolerances: faithful numerics bit-identical to the reference library and to
the oracle's reference-arithmetic mode; against the FP64 oracle max|d| /
max|ref| <= 1e-5 (faithful) and 1e-4 (fast FP32 staggered sums)."""
import glob
import os
import subprocess
import sys

import numpy as np
import pytest

import cpml_oracle as co
from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

sys.path.insert(0, GOLDEN)


def _ours(name, precision=0):
    """Traces of this package's CPML library for a golden case, in a child
    process (the drop-in keeps process-global state)."""
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r); sys.path.insert(0, %r);"
        "import make_cpml_golden as m; sim, idx, ppe = m.case_sim(%r, None);"
        "np.save(sys.argv[1], sim.simulate(idx))" % (ROOT, GOLDEN, name))
    out = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"cpml_{name}_{precision}_{os.getpid()}.npy")
    env = dict(os.environ, OTFWI_PRECISION=str(precision))
    subprocess.run([sys.executable, "-c", code, out], check=True, env=env)
    r = np.load(out)
    os.remove(out)
    return r


def _rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / np.abs(b).max())


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "cpml_*.npz"))), ids=os.path.basename)
def test_cpml_matches_reference_library_and_oracle(path):
    d = np.load(path)
    name = os.path.basename(path)[:-4]
    X, Z, T, idx, ppe = (int(d[k]) for k in ("X", "Z", "T", "idx", "ppe"))
    inp = {k: d[k] for k in d.files}
    ours = _ours(name)
    nd = int(np.sum(ours != d["traces"]))
    print(name, "differing samples vs reference library:", nd, "max rel", _rel(ours, d["traces"]))
    assert nd == 0
    o32 = co.simulate(inp, X, Z, T, idx_source=idx, ppe=ppe)
    assert np.array_equal(o32, d["traces"])  # the oracle pinned to the reference
    o64 = co.simulate(inp, X, Z, T, idx_source=idx, ppe=ppe, mode="f64")
    assert _rel(ours, o64) <= 1e-5
    fast = _ours(name, precision=1)
    print(name, "fast vs FP64 oracle", _rel(fast, o64))
    assert _rel(fast, o64) <= 1e-4


def test_cpml_repeated_calls_replay_one_graph():
    """The forward loop is one captured graph replayed with idx_source read on
    the device: a sequence of calls with different sources (and a call after
    set_source changes the source count) gives what fresh calls give."""
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r); sys.path.insert(0, %r);"
        "import make_cpml_golden as m; sim, idx, ppe = m.case_sim('cpml_shot1', None);"
        "a = [sim.simulate(i) for i in (1, -1, 0, 1)];"
        "import ctypes; from ctypes import POINTER, c_int;"
        "x = np.ascontiguousarray(sim.inputs['ps_x'][:2]); z = np.ascontiguousarray(sim.inputs['ps_z'][:2]);"
        "sim.L.set_source(2, x.ctypes.data_as(POINTER(c_int)), z.ctypes.data_as(POINTER(c_int))); sim._check();"
        "a.append(sim.simulate(-1)); np.save(sys.argv[1], np.stack(a))" % (ROOT, GOLDEN))
    out = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"cpml_seq_{os.getpid()}.npy")
    subprocess.run([sys.executable, "-c", code, out], check=True)
    seq = np.load(out)
    os.remove(out)
    d = np.load(os.path.join(GOLDEN, "cpml_shot1.npz"))
    X, Z, T, ppe = (int(d[k]) for k in ("X", "Z", "T", "ppe"))
    inp = {k: d[k] for k in d.files}
    assert np.array_equal(seq[0], d["traces"]) and np.array_equal(seq[3], d["traces"])
    for i, idx in ((1, -1), (2, 0)):
        assert np.array_equal(seq[i], co.simulate(inp, X, Z, T, idx_source=idx, ppe=ppe)), idx
    two = dict(inp, ps_x=inp["ps_x"][:2], ps_z=inp["ps_z"][:2])
    assert np.array_equal(seq[4], co.simulate(two, X, Z, T, idx_source=-1, ppe=ppe))


def test_cpml_all_sources_batch_matches_per_source_calls():
    """otf_cpml_simulate_all (every source its own shot, one launch per step)
    against cuda_simulate2 per source: identical traces, twice in a row (the
    captured graph replayed) and after set_source drops a source."""
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r); sys.path.insert(0, %r);"
        "import make_cpml_golden as m; sim, idx, ppe = m.case_sim('cpml_shot1', None);"
        "b1 = sim.simulate_all(); b2 = sim.simulate_all();"
        "one = np.stack([sim.simulate(s) for s in range(sim.n_src)]);"
        "from ctypes import POINTER, c_int;"
        "x = np.ascontiguousarray(sim.inputs['ps_x'][:2]); z = np.ascontiguousarray(sim.inputs['ps_z'][:2]);"
        "sim.L.set_source(2, x.ctypes.data_as(POINTER(c_int)), z.ctypes.data_as(POINTER(c_int))); sim._check();"
        "sim.n_src = 2; b3 = sim.simulate_all(); two = np.stack([sim.simulate(s) for s in range(2)]);"
        "np.savez(sys.argv[1], b1=b1, b2=b2, one=one, b3=b3, two=two)" % (ROOT, GOLDEN))
    out = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"cpml_all_{os.getpid()}.npz")
    subprocess.run([sys.executable, "-c", code, out], check=True)
    d = dict(np.load(out))
    os.remove(out)
    assert d["one"].shape[0] == 3
    assert np.array_equal(d["b1"], d["one"]) and np.array_equal(d["b2"], d["one"])
    assert np.array_equal(d["b3"], d["two"])
    g = np.load(os.path.join(GOLDEN, "cpml_shot1.npz"))
    assert np.array_equal(d["one"][1], g["traces"])


def test_cpml_general_spacing_and_stretching_bit_exact():
    """A spacing that is not a power of two and K profiles that are not 1
    (the step divides by both) against the oracle's reference arithmetic,
    which is pinned bit for bit to the reference library: identical traces."""
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r);"
        "from otfwi_b200 import scenarios; from otfwi_b200.cpml import CPMLSimulator;"
        "sc = scenarios.small(X=112, Z=90, T=300, n_src=2, n_rec=8, seed=8, f0=0.04);"
        "rho = 1.0 + 0.5 * np.random.default_rng(8).random((sc.Z, sc.X));"
        "sim = CPMLSimulator(sc.X, sc.Z, sc.T, sc.PML, sc.c_true, sc.src_mask, sc.rec_mask, sc.source, rho=rho,"
        " f0=0.04, dx=0.7, dt=0.7, k_max=2.0);"
        "np.savez(sys.argv[1], traces=sim.simulate(-1), **sim.inputs)" % ROOT)
    out = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"cpml_gen_{os.getpid()}.npz")
    subprocess.run([sys.executable, "-c", code, out], check=True)
    d = dict(np.load(out))
    os.remove(out)
    assert not np.all(d["K_x"] == 1.0)
    ref = co.simulate(d, 112, 90, 300, idx_source=-1, ppe=1, dx=0.7, dt=0.7)
    assert np.array_equal(d["traces"], ref)


def test_cpml_errors_are_reported():
    from otfwi_b200 import _lib
    from otfwi_b200.cpml import CPMLSimulator
    from otfwi_b200 import scenarios
    sc = scenarios.small(X=64, Z=64, T=50, n_src=1, n_rec=2, seed=1)
    sc.src_mask[:] = False
    sc.src_mask[2, 30] = True  # z = 2: outside the update region
    with pytest.raises(_lib.OtfwiError):
        CPMLSimulator(sc.X, sc.Z, sc.T, sc.PML, sc.c_true, sc.src_mask, sc.rec_mask, sc.source)


def test_cpml_gradient_matches_fp64_adjoint_and_is_checkpoint_invariant():
    """dL/dkappa of this library (checkpointed recompute, FP32) against the
    FP64 exact adjoint oracle (relative L2 <= 1e-4), identical for every
    checkpoint interval."""
    code = r'''
import sys, numpy as np
sys.path.insert(0, %r); sys.path.insert(0, %r)
import make_cpml_golden as m
sim, idx, ppe = m.case_sim("cpml_small", None)
rec = sim.simulate(idx).astype(np.float64)
obs = 0.9 * rec + 0.01 * np.roll(rec, 3, axis=1)
g = rec - obs
outs = [sim.gradient(g, idx_source=idx, checkpoint_every=k) for k in (1, 7, None, sim.T)]
np.savez(sys.argv[1], g=g, rec=rec, grads=np.stack(outs), **sim.inputs)
''' % (ROOT, GOLDEN)
    out = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"cpml_grad_{os.getpid()}.npz")
    subprocess.run([sys.executable, "-c", code, out], check=True)
    d = np.load(out)
    os.remove(out)
    grads = d["grads"]
    for k in range(1, len(grads)):
        assert np.array_equal(grads[k], grads[0])
    import make_cpml_golden as m
    X, Z, T, ns, nr, seed, idx, ppe, _ = m.CASES["cpml_small"]
    inp = {k: d[k] for k in d.files if k not in ("g", "rec", "grads")}
    ref, _ = co.adjoint(inp, X, Z, T, d["g"], idx_source=idx, ppe=ppe)
    rel = float(np.linalg.norm(grads[0] - ref) / np.linalg.norm(ref))
    print("CPML gradient vs FP64 adjoint rel L2", rel)
    assert rel <= 1e-4
