"""GPU tests of the batched multi-shot path (otf_batch_*): every shot in the
same launches must give exactly what the drop-in per-shot calls give
(bit-identical traces, per-shot gradients and the wrapper's shot mean), and
the device-misfit gradient must match the host-callback gradient."""
import os
import sys

import numpy as np
import pytest

import misfit_oracle as mo
from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

pytestmark = pytest.mark.gpu


def _scenario(n_src=4, T=300):
    from otfwi_b200 import scenarios
    sc = scenarios.small(X=128, Z=96, T=T, n_src=n_src, n_rec=10, seed=21, f0=0.035)
    return sc


def _wrapper(sc, precision=0):
    from otfwi_b200.cuda_interface_pml import Cuda_interface_PML
    os.environ["OTFWI_PRECISION"] = str(precision)
    try:
        cp = Cuda_interface_PML(sc.X, sc.Z, sc.T, sc.PML, sc.c_true, sc.n_src, sc.src_mask, sc.n_rec,
                                sc.rec_mask, sc.source, multishot=True)
    finally:
        os.environ.pop("OTFWI_PRECISION", None)
    return cp


@pytest.mark.parametrize("precision", [0, 1])
def test_batched_equals_per_shot_dropin(lib, precision):
    from otfwi_b200.batch import ShotBatch
    sc = _scenario()
    cp = _wrapper(sc, precision)
    cp.simulate()
    obs = cp.recording.copy()
    cp.init_regression(obs, mo.L2, prec_deriv=4)
    per_shot = []
    for s in range(sc.n_src):
        cp.calc_grad(c=sc.c_start, idx_source=None)  # multishot: loops and averages
        break
    mean_ref = cp.grad.copy()
    mse_ref = cp.mse[0]

    b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, prec_deriv=4,
                  precision=precision)
    b.set_model(sc.c_true)
    tr = b.forward()
    assert np.array_equal(tr[:, :, 1:], obs[:, :, 1:])
    b.set_observed(obs)
    b.set_model(sc.c_start)
    g, mis = b.gradient("l2")
    assert np.array_equal(g, mean_ref)
    # the wrapper's mse is the shot mean of each shot's sum of squares
    assert abs(mis / sc.n_src - mse_ref) <= 1e-9 * abs(mse_ref)


def test_batched_wasserstein_matches_host_callback(lib):
    """Device Wasserstein adjoint vs the reference's recipe on the host
    (oracle), through the full gradient."""
    from otfwi_b200.batch import ShotBatch
    sc = _scenario(n_src=3)
    b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, prec_deriv=4)
    b.set_model(sc.c_true)
    obs = b.forward()
    b.set_observed(obs)
    b.set_model(sc.c_start)
    g_dev, mis = b.gradient("wasserstein")
    # host path: drop-in per shot with the oracle's wasserstein as callback
    cp = _wrapper(sc)
    cp.init_regression(obs, mo.wasserstein, prec_deriv=4)
    cp.calc_grad(c=sc.c_start)
    rel = np.linalg.norm(g_dev - cp.grad) / np.linalg.norm(cp.grad)
    assert rel <= 1e-4, rel
    assert abs(mis / sc.n_src - cp.mse[0]) <= 1e-5 * abs(cp.mse[0])


@pytest.mark.parametrize("tile", [0, 1, 4])
def test_batched_kernel_variants_identical_many_shots(lib, tile):
    """Persistent TMA kernels vs one-tile-per-CTA kernels on a batch whose
    item count is not a multiple of the persistent grid, fast precision."""
    from otfwi_b200 import scenarios
    from otfwi_b200.batch import ShotBatch
    sc = scenarios.fmc(X=200, Z=168, T=160, n_elem=24, pitch=5, x_first=40)
    out = []
    for kernel in (0, 1):
        b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, prec_deriv=4,
                      precision=1, tile=tile, kernel=kernel)
        b.set_model(sc.c_true)
        obs = b.forward()
        b.set_observed(obs)
        b.set_model(sc.c_start)
        g, m = b.gradient("wasserstein_softplus")
        out.append((obs, g, m))
        b.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]


def test_batched_reverse_with_external_adjoint(lib):
    from otfwi_b200.batch import ShotBatch
    sc = _scenario(n_src=2, T=200)
    b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, prec_deriv=4)
    b.set_model(sc.c_true)
    obs = b.forward()
    b.set_observed(obs)
    b.set_model(sc.c_start)
    g_ref, _ = b.gradient("l2")
    b.forward(ring=True)
    mis, adj = b.misfit("l2")
    g = b.reverse(adj=adj, scale=0.0)
    assert np.array_equal(g, g_ref)
    g1 = b.shot_gradient(1)
    assert np.abs(g1).max() > 0


def test_unfused_kernels_identical_to_strip_split_many_shots(lib):
    """The unfused half-steps (kernel 4) against the strip-split kernels on an
    FMC batch (sources and receivers on one row, 24 shots, full gradient with
    the device Wasserstein misfit): identical traces, gradient and misfit."""
    from otfwi_b200 import scenarios
    from otfwi_b200.batch import ShotBatch
    sc = scenarios.fmc(X=200, Z=168, T=160, n_elem=24, pitch=5, x_first=40)
    out = []
    for kernel in (2, 4):
        b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, prec_deriv=4,
                      precision=1, tile=4, kernel=kernel)
        b.set_model(sc.c_true)
        obs = b.forward()
        b.set_observed(obs)
        b.set_model(sc.c_start)
        g, m = b.gradient("wasserstein_softplus")
        out.append((obs, g, m))
        b.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]
