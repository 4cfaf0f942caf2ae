"""CPU tests of the CPML path: the library exports every symbol its header
declares, the profiles are the convolutional-PML recursion coefficients,
the oracle's reference-arithmetic mode is bit-identical to the reference's
own CPML library on the committed golden cases, and it agrees with its FP64
mode."""
import ctypes
import glob
import os

import numpy as np
import pytest

import cpml_oracle as co
from conftest import GOLDEN, ROOT


def test_cpml_library_exports_header_symbols():
    from otfwi_b200 import _lib
    from otfwi_b200.cpml import CPML_LIB
    if not os.path.exists(CPML_LIB):
        pytest.skip("CPML library not built")
    L = ctypes.CDLL(CPML_LIB)
    names = _lib.exported_symbols_from_header(os.path.join(ROOT, "include", "otfwi_cpml.h"))
    for ref_name in ("init_memory_sim", "setCquad", "set_source", "cuda_simulate2", "def_python_adj"):
        assert ref_name in names
    assert not [n for n in names if not hasattr(L, n)]


def test_profiles_are_the_cpml_recursion():
    from otfwi_b200.cpml import cpml_profiles
    (d, K, al, a, b), (dh, Kh, alh, ah, bh) = cpml_profiles(100, 20, 1.0, 0.5, 0.4, 0.05)
    inner = slice(21, 79)
    assert np.all(d[inner] == 0) and np.all(a[inner] == 0) and np.all(b[inner] == 1)
    assert d[0] > d[10] > 0 and d[-1] > d[-10] > 0
    assert np.allclose(b, np.exp(-(d / K + al) * 0.5), rtol=1e-6)
    m = d > 0
    assert np.allclose(a[m], d[m] * (b[m] - 1) / (K[m] * (d[m] + K[m] * al[m])), rtol=1e-5)
    assert np.all(dh[:19] > 0) and dh[50] == 0


def _inputs(X=72, Z=64, T=250):
    """Arrays as CPMLSimulator passes them, built without a library."""
    from otfwi_b200 import scenarios
    from otfwi_b200.cpml import cpml_profiles
    sc = scenarios.small(X=X, Z=Z, T=T, n_src=2, n_rec=5, seed=11, f0=0.05)
    c = sc.c_true.astype(np.float64)
    f32 = lambda a: np.ascontiguousarray(np.asarray(a, np.float32).ravel())
    i32 = lambda a: np.ascontiguousarray(np.asarray(a, np.int32).ravel())
    sz, sx = np.where(sc.src_mask)
    mz, mx = np.where(sc.rec_mask)
    inp = {"ps_x": i32(sx), "ps_z": i32(sz), "pm_x": i32(mx), "pm_z": i32(mz), "cq": f32(c * c),
           "kappa": f32(c * c), "rhx": f32(np.ones((Z, X))), "rhz": f32(np.ones((Z, X))), "src": f32(sc.source),
           "init": f32(np.zeros((2, Z, X)))}
    for name, prof in zip(("x", "xh"), cpml_profiles(X, sc.PML, 1.0, 1.0, float(c.max()), 0.05)):
        for k, v in zip(("d", "K", "alpha", "a", "b"), prof):
            inp[f"{k}_{name}"] = f32(v)
    for name, prof in zip(("z", "zh"), cpml_profiles(Z, sc.PML, 1.0, 1.0, float(c.max()), 0.05)):
        for k, v in zip(("d", "K", "alpha", "a", "b"), prof):
            inp[f"{k}_{name}"] = f32(v)
    return inp, X, Z, T


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "cpml_*.npz"))), ids=os.path.basename)
def test_cpml_oracle_pinned_to_reference(path):
    """The oracle's reference-arithmetic mode gives every trace sample of the
    reference's own CPML library (tests/golden/make_cpml_golden.py ran it on
    a GPU): one shot, all sources together, odd grid sizes, two points per
    element and an initial field; the FP64 mode stays within 1e-5."""
    d = np.load(path)
    X, Z, T, idx, ppe = (int(d[k]) for k in ("X", "Z", "T", "idx", "ppe"))
    inp = {k: d[k] for k in d.files}
    o32 = co.simulate(inp, X, Z, T, idx_source=idx, ppe=ppe)
    assert np.array_equal(o32, d["traces"])
    o64 = co.simulate(inp, X, Z, T, idx_source=idx, ppe=ppe, mode="f64")
    err = float(np.abs(o64 - d["traces"]).max() / np.abs(o64).max())
    assert err <= 1e-5, err


def test_cpml_oracle_modes_agree_and_absorb():
    inp, X, Z, T = _inputs()
    r32 = co.simulate(inp, X, Z, T)
    r64 = co.simulate(inp, X, Z, T, mode="f64")
    assert np.abs(r64).max() > 0
    assert np.abs(r32 - r64).max() <= 1e-5 * np.abs(r64).max()
    # the layers absorb: the late traces are far below the direct arrival
    late = np.abs(r64[:, -40:]).max()
    assert late < 0.05 * np.abs(r64).max()


def test_cpml_adjoint_oracle_matches_finite_differences():
    """The FP64 exact adjoint of the CPML scheme w.r.t. kappa (the
    reference has no CPML adjoint) against central differences of the FP64
    forward, along seeded directions; the perturbation is the exact
    difference of the FP32-stored kappas, so storage rounding does not enter."""
    inp, X, Z, T = _inputs()
    r0 = co.simulate(inp, X, Z, T, mode="f64")
    obs = 0.9 * r0 + 0.01 * np.roll(r0, 3, axis=1)
    grad, rec = co.adjoint(inp, X, Z, T, r0 - obs)
    assert np.abs(rec - r0).max() <= 1e-12 * np.abs(r0).max()
    k0 = inp["kappa"].astype(np.float64)
    rng = np.random.default_rng(0)

    def loss(kap32):
        inp2 = dict(inp)
        inp2["kappa"] = kap32
        return 0.5 * np.sum((co.simulate(inp2, X, Z, T, mode="f64") - obs) ** 2)

    for _ in range(4):
        v = rng.standard_normal(Z * X)
        kp = np.ascontiguousarray((k0 * (1 + 1e-5 * v)).astype(np.float32))
        km = np.ascontiguousarray((k0 * (1 - 1e-5 * v)).astype(np.float32))
        fd = loss(kp) - loss(km)
        an = float(np.sum(grad.ravel() * (kp.astype(np.float64) - km.astype(np.float64))))
        assert abs(fd - an) <= 1e-5 * abs(fd), (fd, an)


def test_cpml_caller_declares_every_abi_argument():
    """The Python caller's init_memory_sim declaration has exactly the
    header's (and the reference's) 43 parameters, in the same kinds."""
    import re
    from otfwi_b200 import cpml
    text = open(os.path.join(ROOT, "include", "otfwi_cpml.h")).read()
    sig = re.search(r"void init_memory_sim\((.*?)\);", text, re.S).group(1)
    params = [p.strip() for p in sig.split(",")]
    L = ctypes.CDLL(cpml.CPML_LIB)
    cpml._declare(L)
    assert len(L.init_memory_sim.argtypes) == len(params) == 43
    kinds = ["float**" if "**" in p else ("int*" if p.startswith("int") else "float*") if "*" in p else
             ("int" if p.startswith("int") else "float") for p in params]
    for t, k in zip(L.init_memory_sim.argtypes, kinds):
        name = getattr(t, "__name__", str(t))
        assert {"int": "c_int", "float": "c_float", "int*": "LP_c_int", "float*": "LP_c_float",
                "float**": "LP_LP_c_float"}[k] == name, (k, name)
