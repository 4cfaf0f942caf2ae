"""GPU misfit kernels against the reference's adjoint_functions outputs
(tests/golden/misfit_*.npz) and the numpy oracle.

Tolerances: L2 adjoint bit-identical, L2 misfit rel 1e-12; Wasserstein and
wasserstein_quad misfit rel 1e-5 and adjoint max|d| / max|ref| <= 1e-5
(compensated FP32 scans against the reference's FP64 numpy); softplus
variant the same against the oracle's FP64 definition.
"""
import glob
import os

import numpy as np
import pytest

import misfit_oracle as mo
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _rel_max(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "misfit_*.npz"))),
                         ids=os.path.basename)
def test_device_misfits_match_reference(lib, path):
    from otfwi_b200.batch import device_misfit
    d = np.load(path)
    m, adj = device_misfit(d["sim"], d["obs"], "l2")
    assert np.array_equal(adj, d["l2_adj"].astype(np.float32))
    assert abs(m.sum() - d["l2"]) <= 1e-12 * abs(d["l2"])
    m, adj = device_misfit(d["sim"], d["obs"], "wasserstein")
    assert abs(m.sum() - d["w2"]) <= 1e-5 * abs(d["w2"]), (m.sum(), d["w2"])
    assert _rel_max(adj, d["w2_adj"]) <= 1e-5
    m, adj = device_misfit(d["sim"], d["obs"], "wasserstein_quad")
    assert abs(m.sum() - d["w2q"]) <= 1e-5 * abs(d["w2q"]), (m.sum(), d["w2q"])
    assert _rel_max(adj, d["w2q_adj"]) <= 1e-5


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "misfit_*.npz"))),
                         ids=os.path.basename)
def test_device_softplus_wasserstein_matches_oracle(lib, path):
    from otfwi_b200.batch import device_misfit
    d = np.load(path)
    w2, ref = mo.wasserstein_softplus(d["sim"].astype(np.float64), d["obs"])
    m, adj = device_misfit(d["sim"], d["obs"], "wasserstein_softplus")
    assert abs(m.sum() - w2) <= 1e-5 * abs(w2)
    assert _rel_max(adj, ref) <= 1e-5


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "misfit_*.npz"))),
                         ids=os.path.basename)
def test_device_quad_envelope(lib, path):
    """quad_envelope through batched cuFFT in FP64: against the FP64 oracle
    (misfit rel 1e-9, adjoint 1e-6: FP32 output) and against the reference
    itself (1e-5: its analytic signal of the float32 observed trace is a
    single-precision FFT)."""
    from otfwi_b200.batch import device_misfit
    d = np.load(path)
    e, ref = mo.quad_envelope(d["sim"].astype(np.float64), d["obs"])
    m, adj = device_misfit(d["sim"], d["obs"], "quad_envelope")
    assert abs(m.sum() - e) <= 1e-9 * abs(e)
    assert _rel_max(adj, ref) <= 1e-6
    assert abs(m.sum() - d["env"]) <= 1e-5 * abs(d["env"])
    assert _rel_max(adj, d["env_adj"]) <= 1e-5


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "misfit_*.npz"))),
                         ids=os.path.basename)
def test_device_wasserstein_pm(lib, path):
    """wasserstein_pm with its negative-part CDFs from the negative parts,
    against the oracle of that form (whose as-written form reproduces the
    reference bit for bit, tests/test_oracle.py), to the Wasserstein kinds'
    tolerance; and through the batched gradient graph (kind 5)."""
    from otfwi_b200.batch import device_misfit
    d = np.load(path)
    w2, ref = mo.wasserstein_pm(d["sim"].astype(np.float64), d["obs"], fixed=True)
    m, adj = device_misfit(d["sim"], d["obs"], "wasserstein_pm")
    assert abs(m.sum() - w2) <= 1e-5 * abs(w2), (m.sum(), w2)
    assert _rel_max(adj, ref) <= 1e-5


def test_batched_gradient_with_wasserstein_pm(lib):
    """The gradient graph with misfit kind 5: the misfit it reports equals the
    stand-alone device misfit of the same traces."""
    from otfwi_b200 import scenarios
    from otfwi_b200.batch import ShotBatch, device_misfit
    sc = scenarios.small(X=128, Z=96, T=300, n_src=3, n_rec=10, seed=21, f0=0.035)
    b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, precision=1)
    b.set_model(sc.c_true)
    obs = b.forward()
    b.set_observed(obs)
    b.set_model(sc.c_start)
    sim = b.forward()
    g, mis = b.gradient("wasserstein_pm")
    m, _ = device_misfit(sim.reshape(-1, sc.T), obs.reshape(-1, sc.T), "wasserstein_pm")
    assert np.isfinite(g).all() and np.abs(g).max() > 0
    assert abs(mis - m.sum()) <= 1e-12 * abs(m.sum())
    b.close()


def test_wasserstein_long_traces_and_many(lib):
    """T = 4000 traces (the FMC length), many traces in one launch."""
    from otfwi_b200.batch import device_misfit
    rng = np.random.default_rng(3)
    T, n = 4000, 48
    t = np.arange(T)
    obs = np.stack([np.exp(-((t - rng.uniform(800, 3000)) / 60.0) ** 2) * np.cos(0.1 * t)
                    for _ in range(n)]).astype(np.float32)
    sim = (np.roll(obs, 7, axis=1) + rng.normal(0, 1e-3, obs.shape)).astype(np.float32)
    w2, ref = mo.wasserstein(sim.astype(np.float64), obs)
    m, adj = device_misfit(sim, obs, "wasserstein")
    assert abs(m.sum() - w2) <= 1e-5 * abs(w2)
    assert _rel_max(adj, ref) <= 1e-5
    w2s, refs = mo.wasserstein_softplus(sim.astype(np.float64), obs)
    ms, adjs = device_misfit(sim, obs, "wasserstein_softplus")
    assert abs(ms.sum() - w2s) <= 1e-5 * abs(w2s)
    assert _rel_max(adjs, refs) <= 1e-5
    w2q, refq = mo.wasserstein_quad(sim.astype(np.float64), obs)
    mq, adjq = device_misfit(sim, obs, "wasserstein_quad")
    assert abs(mq.sum() - w2q) <= 1e-5 * abs(w2q)
    assert _rel_max(adjq, refq) <= 1e-5
