"""CPU property tests of what the parity cases and the inversion are built
from: the seeded scenario builders (geometry and wavelet of the benchmark's
plain single-shot and full-matrix-capture cases, and the preconditioner's
two-array inversion case), the misfit oracle (a trace compared with itself
has zero misfit and a zero adjoint source, for every recipe), and the
preconditioner's input features and proposal."""
import numpy as np
import pytest

import misfit_oracle as mo


def test_ricker_wavelet_closed_form():
    """Peak 1 at t0, symmetric about it, zero where (pi f0 (t - t0))^2 = 1/2."""
    from otfwi_b200.scenarios import ricker
    f0, t0 = 1.0 / 59.0, 70
    w = ricker(200, f0, t0)
    assert w[t0] == 1.0 and np.argmax(w) == t0
    k = np.arange(1, 60)
    assert np.allclose(w[t0 - k], w[t0 + k], rtol=0, atol=1e-15)
    tz = t0 + 1.0 / (np.pi * f0 * np.sqrt(2.0))
    i = int(np.floor(tz))
    assert w[i] > 0 > w[i + 1]  # the first zero crossing after the peak


def test_plain_single_shot_geometry():
    """256^2, T = 1500, one source at (x = 128, z = 26), 32 receivers at z = 26,
    x = 4 + 8i; nondimensional velocities 0.4 for 5900 m/s and 0.2034 for the
    3000 m/s defects; a 5 MHz Ricker at about 59 samples per period."""
    from otfwi_b200 import scenarios
    sc = scenarios.plain_single_shot()
    assert (sc.X, sc.Z, sc.T, sc.PML) == (256, 256, 1500, 20)
    zs, xs = np.where(sc.src_mask)
    assert list(zs) == [26] and list(xs) == [128]
    zr, xr = np.where(sc.rec_mask)
    assert np.all(zr == 26) and list(xr) == list(4 + 8 * np.arange(32))
    assert set(np.unique(np.round(sc.c_true, 4))) == {0.2034, 0.4}
    assert np.all(sc.c_start == 0.4)
    dt = 0.4 * sc.dx / sc.c_max
    assert abs(1.0 / (5e6 * dt) - 59.0) < 0.01
    assert sc.source.shape == (1, 1500) and sc.source.dtype == np.float32


def test_fmc_geometry():
    """512^2, T = 4000, 64 elements at x = 67 + 6i, z = 26, each element both a
    source (one shot each) and a receiver, the same wavelet on every element."""
    from otfwi_b200 import scenarios
    sc = scenarios.fmc()
    assert (sc.X, sc.Z, sc.T) == (512, 512, 4000)
    xs = 67 + 6 * np.arange(64)
    for m in (sc.src_mask, sc.rec_mask):
        z, x = np.where(m)
        assert np.all(z == 26) and list(x) == list(xs)
    assert sc.n_src == 64 and sc.n_rec == 64
    assert sc.source.shape == (64, 4000) and np.all(sc.source == sc.source[0])


@pytest.mark.parametrize("name", ["L2", "wasserstein", "wasserstein_softplus", "wasserstein_quad",
                                  "quad_envelope", "wasserstein_pm"])
def test_misfit_oracle_of_a_trace_with_itself_is_zero(name):
    """sim = obs: exactly zero misfit and an exactly zero adjoint source for
    every misfit the library offers (identical CDFs invert to identical
    quantiles, so no round-off survives)."""
    from otfwi_b200 import scenarios
    sc = scenarios.small(X=96, Z=80, T=300, n_src=2, n_rec=4, seed=2)
    rng = np.random.default_rng(0)
    tr = np.stack([np.roll(sc.source[i % 2], 15 * i) for i in range(4)]).astype(np.float32)
    tr += (1e-3 * rng.standard_normal(tr.shape)).astype(np.float32)
    mis, adj = getattr(mo, name)(tr, tr)
    assert mis == 0.0
    assert not np.any(np.asarray(adj, np.float64))


def test_misfit_oracle_grows_with_a_time_shift():
    """A trace against a delayed copy of itself: the Wasserstein misfit grows
    with the delay (transport cost), which is why it is the benchmark's
    misfit for cycle-skipping-prone data."""
    from otfwi_b200.scenarios import ricker
    T = 400
    obs = ricker(T, 1.0 / 40.0, 100).astype(np.float32)[None]
    w = [mo.wasserstein(ricker(T, 1.0 / 40.0, 100 + d).astype(np.float32)[None], obs)[0] for d in (0, 5, 10, 20)]
    assert w[0] <= 1e-12 and w[0] < w[1] < w[2] < w[3]


class _FakeProblem:
    """fwi.Problem's interface for the preconditioner's input features, on CPU
    tensors: a gradient mask and an illumination map."""

    def __init__(self, Z, X, seed):
        import torch
        self.torch = torch
        g = np.random.default_rng(seed)
        self.gmask = torch.zeros(Z, X)
        self.gmask[Z // 4:Z - Z // 4, X // 4:X - X // 4] = 1.0
        self._illum = torch.as_tensor(10.0 ** g.uniform(-6, 2, (Z, X)), dtype=torch.float32)

    def illumination(self, b, c):
        return self._illum


def test_preconditioner_features_and_proposal():
    """Network input [1, Z, X, 3]: the masked negative gradient scaled to max
    |.| = 1, log-scaled illumination in [0, 1.0002], the model's offset from the
    background over the velocity span; the proposal is the network's output
    times the span, zero outside the gradient mask."""
    import torch
    from otfwi_b200 import learned
    Z, X = 48, 64
    prob = _FakeProblem(Z, X, 3)
    rng = np.random.default_rng(4)
    g = torch.as_tensor(rng.standard_normal((Z, X)), dtype=torch.float32)
    c = torch.full((Z, X), float(learned.C_BG)) + 0.01 * torch.as_tensor(rng.standard_normal((Z, X)),
                                                                         dtype=torch.float32)
    f = learned.features(prob, 0, c, g)
    assert f.shape == (1, Z, X, 3) and f.dtype == torch.float32
    gm, il, cn = f[0, ..., 0], f[0, ..., 1], f[0, ..., 2]
    assert float(gm.abs().max()) == 1.0 and not torch.any(gm[prob.gmask == 0])
    assert torch.equal(torch.sign(gm[prob.gmask == 1]), torch.sign(-g[prob.gmask == 1]))
    # log10(i / max + 1e-3) / 3 + 1 maps (0, max] onto (0, 1 + log10(1.001) / 3]
    assert float(il.min()) >= 0.0 and abs(float(il.max()) - (1.0 + np.log10(1.001) / 3.0)) < 1e-6
    assert torch.allclose(cn, (c - learned.C_BG) / learned.SPAN)

    class Net:
        def forward(self, x):
            return torch.ones(1, Z, X)

    dc = learned.Proposer(Net())(prob, 0, c, g, 0.0)
    assert torch.equal(dc, learned.SPAN * prob.gmask)


def test_inversion_scenario_geometry():
    """Two centred linear arrays at rows PML + 6 and Z - 1 - (PML + 6), every
    element receiving, n_src elements firing (half per array), velocities
    within the defect family's range, the homogeneous background as start."""
    from otfwi_b200 import learned
    sc = learned.defect_scenario(256, 256, 1500, seed=7, n_elem=32, pitch=6, n_def=4, n_src=16)
    rows = (26, 256 - 1 - 26)
    zr, xr = np.where(sc.rec_mask)
    assert set(zr) == set(rows) and sc.n_rec == 64
    xs = np.unique(xr)
    assert len(xs) == 32 and np.all(np.diff(xs) == 6) and xs[0] + xs[-1] in (255, 256)
    zs, _ = np.where(sc.src_mask)
    assert sc.n_src == 16 and sum(zs == rows[0]) == 8 and sum(zs == rows[1]) == 8
    assert np.all(sc.src_mask <= sc.rec_mask)
    v = sc.c_true * learned.C_MAX / 0.4
    assert v.min() >= learned.V_LO - 1e-3 and v.max() <= learned.V_HI + 1e-3
    assert np.all(sc.c_start == learned.C_BG)
