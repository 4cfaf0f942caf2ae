"""CPU tests of the oracle itself: pinned against the reference's own outputs.

* misfit oracle vs tests/golden/misfit_*.npz (the reference's
  adjoint_functions.wasserstein / L2 / wasserstein_quad, run unchanged):
  bit-exact; quad_envelope within single-precision FFT rounding;
* simulator oracle ("f32" mode) vs tests/golden/sim_*.npz (the reference's
  regression_PML_single.cu run on a GPU): traces and gradients;
* "f32" vs "f64" mode agreement on the same inputs.
"""
import glob
import os

import numpy as np
import pytest

import misfit_oracle as mo
import pml_oracle as po
from conftest import GOLDEN


def _misfit_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "misfit_*.npz")))


@pytest.mark.parametrize("path", _misfit_cases(), ids=os.path.basename)
def test_misfit_oracle_matches_reference_bit_exact(path):
    d = np.load(path)
    sim = d["sim"].astype(np.float64)
    w2, adj = mo.wasserstein(sim, d["obs"])
    assert w2 == d["w2"]
    assert np.array_equal(adj, d["w2_adj"])
    l2, r = mo.L2(sim, d["obs"])
    assert l2 == d["l2"]
    assert np.array_equal(r, d["l2_adj"])
    w2q, adjq = mo.wasserstein_quad(sim, d["obs"])
    assert w2q == d["w2q"]
    assert np.array_equal(adjq, d["w2q_adj"])


@pytest.mark.parametrize("path", _misfit_cases(), ids=os.path.basename)
def test_wasserstein_pm_oracle_matches_reference_bit_exact(path):
    """The oracle of adjoint_functions.wasserstein_pm as written (its G_n / F_n
    built from the positive parts) reproduces the reference bit for bit; the
    fixed form differs from it only through the negative parts."""
    d = np.load(path)
    sim = d["sim"].astype(np.float64)
    w2, adj = mo.wasserstein_pm(sim, d["obs"], fixed=False)
    assert w2 == d["w2pm"]
    assert np.array_equal(adj, d["w2pm_adj"])
    w2f, adjf = mo.wasserstein_pm(sim, d["obs"], fixed=True)
    assert w2f != w2 and np.all(np.isfinite(adjf))


@pytest.mark.parametrize("path", _misfit_cases(), ids=os.path.basename)
def test_quad_envelope_oracle_vs_reference(path):
    """The reference's analytic signal of the float32 observed trace goes
    through scipy.fft in single precision; the oracle's is FP64, so the two
    agree to single-precision FFT rounding, not bit for bit."""
    d = np.load(path)
    e, adj = mo.quad_envelope(d["sim"].astype(np.float64), d["obs"])
    assert abs(e - d["env"]) <= 1e-6 * abs(d["env"])
    assert np.max(np.abs(adj - d["env_adj"])) <= 1e-5 * np.max(np.abs(d["env_adj"]))


def test_misfit_golden_covers_nonmonotone_cdf():
    # the "nonmono" case must exercise interp1d's sort of a non-monotone CDF
    d = np.load(os.path.join(GOLDEN, "misfit_nonmono.npz"))
    T = d["sim"].shape[1]
    t = np.linspace(0, 1, T)
    found = False
    for s in range(d["sim"].shape[0]):
        g = d["obs"][s].astype(np.float64)
        c = max(-1.1 * g.min(), 0.1 * g.max())
        f = d["sim"][s].astype(np.float64) + c
        F = mo.cumtrapz0(f / np.sum(f * (t[1] - t[0])), t)
        found |= bool(np.any(np.diff(F) < 0))
    assert found


def _sim_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "sim_*.npz")))


def rel_trace_err(a, b):
    """max over receivers of max_{t>=1} |a-b| / max_t |b|."""
    a = np.asarray(a, np.float64)[..., 1:]
    b = np.asarray(b, np.float64)[..., 1:]
    den = np.abs(b).max(axis=-1)
    den[den == 0] = 1.0
    return float((np.abs(a - b).max(axis=-1) / den).max())


def rel_l2(a, b):
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def oracle_case(d, mode, shots=None):
    """Run the oracle on a golden case's inputs: traces per shot and grads."""
    args = (np.asarray(d["c_true"], np.float32) ** 2, d["constvec"], d["d_x"], d["d_z"], d["src_x"],
            d["src_z"], d["source"], d["rec_x"], d["rec_z"])
    out = {"traces_all": po.simulate(*args, idx_source=-1, mode=mode)}
    ns = len(d["src_x"])
    for s in range(ns):
        out[f"traces_s{s}"] = po.simulate(*args, idx_source=s, mode=mode)
    obs = np.stack([np.asarray(d[f"traces_s{s}"]) for s in range(ns)]) if "traces_s0" in d else None
    gargs = (np.asarray(d["c_start"], np.float32) ** 2,) + args[1:]
    for s in (range(ns) if shots is None else shots):
        o = obs[s] if obs is not None else out[f"traces_s{s}"]

        def adj(sim, o=o):
            r = sim - o
            r[:, 0] = 0.0
            return float(np.sum(r ** 2)), r

        g, rec, _ = po.grad(*gargs, d["ring_x"], d["ring_z"], adj, idx_source=s, mode=mode)
        out[f"grad_s{s}"] = g
        out[f"sim_s{s}"] = rec
    return out


@pytest.mark.parametrize("path", _sim_cases(), ids=os.path.basename)
def test_sim_oracle_pinned_to_reference(path):
    """The f32 oracle restates the reference's arithmetic operation by
    operation: its traces (t >= 1) and gradients are bit-identical to the
    reference library's (run on a GPU by tests/golden/make_sim_golden.py)."""
    d = dict(np.load(path))
    o = oracle_case(d, "f32")
    for k in [k for k in d if k.startswith(("traces_", "sim_s"))]:
        assert np.array_equal(o[k][:, 1:], d[k][:, 1:]), k
    for k in [k for k in d if k.startswith("grad_s")]:
        assert np.array_equal(o[k], d[k]), k
    # and the FP64 oracle stays within FP32 accumulation error of both
    o64 = oracle_case(d, "f64", shots=[0])
    assert rel_trace_err(o64["traces_all"], d["traces_all"]) <= 1e-5
    assert rel_l2(o64["grad_s0"], d["grad_s0"]) <= 1e-4


def test_oracle_f32_vs_f64_small():
    from otfwi_b200 import scenarios
    from otfwi_b200.cuda_interface_pml import pml_damping
    sc = scenarios.small(T=300)
    dxp, dzp = pml_damping(sc.X, sc.Z, sc.PML)
    sx, sz = sc.src_xz()
    mx, mz = sc.rec_xz()
    args = (sc.c_true ** 2, np.ones(3), dxp, dzp, sx, sz, sc.source, mx, mz)
    r32 = po.simulate(*args, mode="f32")
    r64 = po.simulate(*args, mode="f64")
    assert np.abs(r64).max() > 1e-3
    assert rel_trace_err(r32, r64) < 1e-5
