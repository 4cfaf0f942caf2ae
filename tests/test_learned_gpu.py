"""GPU test of the trained learned preconditioner (otfwi_b200/weights/
precond_unet.npz, produced by ``python -m otfwi_b200.learned``): on a seeded
256^2 inversion of the training distribution (a seed the training runs did
not use), learned-preconditioned FWI reaches the plain method's final RMS
velocity error in at most half of the plain method's wall time (graphs
captured and observed data modelled before either clock starts; the
learned run's time includes the network's inference), with fewer
forward-modelling equivalents (a gradient counts 92/28 forward modellings, a
line-search or proposal trial one) than plain FWI spends, and ends with a
lower error; every accepted learned step lowered the misfit
(accept-if-decrease)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_learned_preconditioner_beats_plain_fwi(lib):
    from otfwi_b200 import fwi, learned
    from otfwi_b200.unet import UNet
    sc = learned.defect_scenario(256, 256, 1500, 99, 32, 6, 5, n_src=16)
    bands = [fwi.Band(2.5e6, 4), fwi.Band(5e6, 4)]
    net = UNet.load(learned.WEIGHTS)
    hist = {}
    for name, prop in (("plain", None), ("learned", learned.Proposer(net))):
        prob = fwi.Problem(sc, bands, misfit="wasserstein")
        c0 = prob.torch.as_tensor(sc.c_start, dtype=prob.torch.float32).cuda()
        for b in range(len(bands)):  # observed data and graph captures outside the timed run
            prob.gradient(b, c0)
            prob.objective(b, c0)
        if prop is not None:
            prop(prob, 0, c0, prob.gradient(0, c0)[0], 0.0)  # network buffers allocated once
        _, hist[name] = fwi.descent(prob, sc.c_start, proposer=prop)
    hp, hl = hist["plain"], hist["learned"]
    target = hp.rms[-1]
    print("plain rms", hp.rms[0], "->", target, "evals", hp.evals[-1], "time", hp.time_to(target))
    print("learned rms", hl.rms, "evals", hl.evals, "learned steps", sum(hl.learned), "time", hl.time_to(target))
    reach = next(e for e, r in zip(hl.evals, hl.rms) if r <= target)
    assert reach < hp.evals[-1]
    assert hl.time_to(target) <= 0.5 * hp.time_to(target)
    assert hl.rms[-1] < target
    assert sum(hl.learned) >= 1
    for b in range(2):
        m = [v for v, bb in zip(hl.misfit[1:], hl.band[1:]) if bb == b]
        assert all(x > y for x, y in zip(m, m[1:]))
