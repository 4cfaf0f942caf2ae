"""Generate tests/golden/misfit_*.npz from the reference's own misfit code.

Run in a checkout that has the reference project (default location given by
--ref). It imports the reference's ``adjoint_functions.py`` unchanged, with two
import shims the installed environment needs:
  * ``matplotlib`` is absent: a stub module satisfies ``utils.py:3,6``;
  * scipy 1.18 removed ``scipy.integrate.cumtrapz``: it is aliased to
    ``scipy.integrate.cumulative_trapezoid`` (the function it was renamed to).
Inputs are seeded synthetic traces with the shape of recorded ultrasonic
A-scans (Ricker-like pulses with travel-time shifts and noise), stored as
float32 like the simulator's recordings. The outputs are the reference's
(W2, adjoint source), (L2, residual), wasserstein_quad's (W2, adjoint),
quad_envelope's (misfit, adjoint) and wasserstein_pm's (W2, adjoint), the
last as written (its negative-part CDFs are built from the positive parts).

    python tests/golden/make_misfit_golden.py --ref /path/to/Otfwi
"""
import argparse
import subprocess
import os
import sys
import types

import numpy as np


def _install_shims():
    import scipy.integrate as integ

    if not hasattr(integ, "cumtrapz"):
        integ.cumtrapz = integ.cumulative_trapezoid
    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = plt
    mpl.use = lambda *a, **k: None
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", plt)


def pulse(t, t0, f0):
    a = (np.pi * f0 * (t - t0)) ** 2
    return (1 - 2 * a) * np.exp(-a)


def make_case(rng, n_tr, T, f0, neg_excursion=False):
    t = np.arange(T, dtype=np.float64)
    obs = np.zeros((n_tr, T))
    sim = np.zeros((n_tr, T))
    for i in range(n_tr):
        t1 = rng.uniform(0.15, 0.35) * T
        t2 = rng.uniform(0.5, 0.8) * T
        a1, a2 = rng.uniform(0.5, 1.5, size=2)
        obs[i] = a1 * pulse(t, t1, f0) + 0.4 * a2 * pulse(t, t2, f0)
        d1, d2 = rng.normal(0, 0.01 * T, size=2)
        sim[i] = (a1 * (1 + rng.normal(0, 0.05)) * pulse(t, t1 + d1, f0)
                  + 0.4 * a2 * pulse(t, t2 + d2, f0))
        sim[i] += rng.normal(0, 0.002, size=T)
        if neg_excursion and i % 2 == 0:
            # drive the shifted simulated density below zero: F is then not
            # monotone and interp1d's sort path is exercised
            sim[i] -= 3.0 * pulse(t, 0.9 * T, f0)
    return sim.astype(np.float32), obs.astype(np.float32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="reference tree (default: the oracle recipe's REF)")
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    args = ap.parse_args()
    if args.ref is None:
        root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
        args.ref = subprocess.run(["make", "-s", "-C", os.path.join(root, "oracle"), "print-ref"],
                                  capture_output=True, text=True, check=True).stdout.strip()
    _install_shims()
    sys.path.insert(0, args.ref)
    import adjoint_functions as adj  # the reference module, unchanged

    rng = np.random.default_rng(20261203)
    cases = {
        "basic": make_case(rng, 6, 500, 0.02),
        "long": make_case(rng, 3, 1500, 0.01),
        "nonmono": make_case(rng, 4, 400, 0.03, neg_excursion=True),
    }
    for name, (sim, obs) in cases.items():
        # the reference callback hands the misfit float64 copies of the
        # float32 recording (cuda_interface_pml.py:239) and float32 observed
        w2, s_w2 = adj.wasserstein(sim.astype(np.float64), obs)
        l2, resid = adj.L2(sim.astype(np.float64), obs)
        w2q, s_w2q = adj.wasserstein_quad(sim.astype(np.float64), obs)
        env, env_adj = adj.quad_envelope(sim.astype(np.float64), obs)
        w2pm, s_w2pm = adj.wasserstein_pm(sim.astype(np.float64), obs)
        path = os.path.join(args.out, f"misfit_{name}.npz")
        np.savez_compressed(path, sim=sim, obs=obs, w2=np.float64(w2), w2_adj=s_w2,
                            l2=np.float64(l2), l2_adj=resid, w2q=np.float64(w2q), w2q_adj=s_w2q,
                            env=np.float64(env), env_adj=env_adj, w2pm=np.float64(w2pm), w2pm_adj=s_w2pm)
        print(path, sim.shape, float(w2), float(l2))


if __name__ == "__main__":
    main()
