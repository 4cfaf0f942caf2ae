"""GPU tests of the FWI outer loop: the forward-only objective equals the
gradient graph's misfit, illumination is additive over shots and quadratic
in the source amplitude, the reference-style objective (regression.py:45-49)
is consistent with the batched gradient, and plain descent with line search
decreases the misfit at every accepted step and the velocity error overall."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(T=700, iters=3):
    from otfwi_b200 import fwi
    from otfwi_b200.learned import defect_scenario
    sc = defect_scenario(128, 128, T, 3, 16, 6, 3, n_src=4, amin=4, amax=9)
    return sc, fwi.Problem(sc, [fwi.Band(2.5e6, iters), fwi.Band(5e6, iters)], misfit="wasserstein")


def test_objective_equals_gradient_misfit(lib):
    import torch
    sc, prob = _problem()
    c = torch.as_tensor(sc.c_start, dtype=torch.float32).cuda()
    for b in range(2):
        _, J = prob.gradient(b, c)
        assert prob.objective(b, c) == J
    # at the true model the misfit vanishes
    assert prob.objective(0, prob.c_true) == 0.0


def test_illumination_additive_and_quadratic(lib):
    from otfwi_b200.batch import ShotBatch
    sc, _ = _problem()
    args = (sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask)
    full = ShotBatch(*args, sc.source, precision=1)
    full.set_model(sc.c_true)
    i_all = full.illumination(4).astype(np.float64)
    parts = np.zeros_like(i_all)
    for s in range(sc.n_src):
        one = ShotBatch(*args, sc.source, shots=(np.array([0, 1]), np.array([s])), precision=1)
        one.set_model(sc.c_true)
        parts += one.illumination(4)
        one.close()
    assert np.max(np.abs(parts - i_all)) <= 1e-5 * i_all.max()
    twice = ShotBatch(*args, 2 * sc.source, precision=1)
    twice.set_model(sc.c_true)
    assert np.allclose(twice.illumination(4), 4 * i_all, rtol=1e-5, atol=1e-6 * i_all.max())
    assert i_all.min() >= 0 and i_all.max() > 0


def test_reference_objective_consistent_with_batch(lib):
    import torch
    from otfwi_b200 import fwi
    sc, prob = _problem()
    f, g = fwi.objfun(prob, 0, sc.c_start.ravel(), grad_scale=1e-2)
    g0, J = prob.gradient(0, torch.as_tensor(sc.c_start, dtype=torch.float32).cuda())
    assert f == pytest.approx(1e3 * J / prob.batch(0).n_shots, rel=1e-12)
    assert np.allclose(g, (1e-2 * prob.gmask * g0).double().cpu().numpy().ravel())


def test_plain_descent_decreases_misfit_and_error(lib):
    from otfwi_b200 import fwi
    sc, prob = _problem()
    c, h = fwi.descent(prob, sc.c_start)
    print("rms", h.rms, "misfit", h.misfit)
    assert len(h.rms) >= 4
    for b in (0, 1):
        m = [v for v, bb in zip(h.misfit[1:], h.band[1:]) if bb == b]
        assert all(x > y for x, y in zip(m, m[1:]))
    assert h.rms[-1] < h.rms[0]
    assert float(c.min()) >= prob.vmin - 1e-7 and float(c.max()) <= prob.vmax + 1e-7


def test_lbfgsb_result_file(lib, tmp_path):
    """The reference's L-BFGS-B driver (regression.py:82-96) end to end: a
    few iterations over the batched GPU objective, then the closing
    re-simulation, L2 misfit and result pickle."""
    from otfwi_b200 import fwi, results
    sc, prob = _problem(iters=2)
    r, mm = fwi.lbfgsb(prob, sc.c_start, b=0, maxiter=2)
    assert r.fun < fwi.objfun(prob, 0, sc.c_start.ravel())[0]
    path = tmp_path / "output" / "regression_small.pickle"
    out = results.finish(prob, r.x, r.fun, mm, str(path), b=0)
    d = results.load(str(path))
    sb = prob.batch(0)
    assert d["recording"].shape == (sb.n_shots, sb.n_rec, sc.T) and d["recording"].dtype == np.float32
    assert np.array_equal(d["model"], r.x.reshape(sc.Z, sc.X))
    assert d["mseL2"] == results.l2(d["recording"], sb._obs_dev.cpu().numpy()) == out["mseL2"]
    assert d["model_misfit"] == mm and len(mm) >= 1
    assert d["vmin"] == prob.vmin and d["fun"] == r.fun
