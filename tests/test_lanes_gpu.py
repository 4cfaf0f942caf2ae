"""Shot lanes of the unfused kernels (otf_batch_set_lanes): the shots split
into groups whose time loops run as parallel launch chains inside the
captured graphs. Every output -- observed and simulated traces, gradient,
misfit, illumination -- is bit-identical for one chain, the automatic choice
(2 lanes for 37 shots), 2 lanes and an uneven split (5 lanes requested,
capped at 4: groups of 9 and 10 shots), and the launch-count check of every
time loop passes (an error otherwise)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(sc, lanes):
    from otfwi_b200.batch import ShotBatch
    b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, prec_deriv=4, precision=1,
                  kernel=4)
    try:
        b.set_lanes(lanes)
        b.set_model(sc.c_true)
        obs = b.forward().copy()
        b.set_observed(obs)
        b.set_model(sc.c_start)
        sim = b.forward().copy()
        g, m = b.gradient("l2")
        illum = b.illumination(5).copy()
        return obs, sim, g.copy(), m, illum
    finally:
        b.close()


def test_lanes_bit_identical(lib):
    from otfwi_b200 import scenarios
    sc = scenarios.fmc(X=200, Z=120, T=180, n_elem=37, pitch=4, x_first=30, seed=9)
    ref = _run(sc, 1)
    assert np.abs(ref[2]).max() > 0
    for lanes in (0, 2, 5):
        out = _run(sc, lanes)
        for name, a, b in zip(("obs", "sim", "grad", "misfit", "illum"), out, ref):
            assert np.array_equal(np.asarray(a), np.asarray(b)), (lanes, name)
