"""Full-size check of the differentiable path (1024^2 velocity model, 32
shots, T=6000, sqrt(T) checkpoints).

The model has a 5900 m/s background with +-3% Gaussian-smoothed
heterogeneity (sigma 4 cells) and 8 elliptical 4000-6300 m/s defects
(scenarios.heterogeneous_defects); two linear arrays of 64 elements (top and
bottom, pitch 12), 16 firing per array. The model of the check is the true
model smoothed (sigma 8 cells). Reported:

- the exact adjoint gradient of L = 1/2 sum_{t>=1} (traces - obs)^2 through
  ``PMLPropagator`` (torch.autograd) and its wall time;
- central finite differences of L (forward only, FP32 traces, the loss summed
  in FP64) along the gradient's own direction and 16 seeded smooth random
  directions, each as a Richardson pair: D(e) and D(e/2) combined as
  (4 D(e/2) - D(e)) / 3, which cancels the e^2 truncation term, so that e can
  be large enough for the FP32 rounding noise of the losses (divided by e) to
  stay small; the relative error of each against <grad, v> must stay within
  the stated tolerance (``fd_tolerance``);
- the cosine, over the cells at least PML away from the edge, with the
  gradient of the reference's algorithm (cuda_grad_ext: cross-correlation
  of the reconstructed field with the adjoint of the L2 residual), computed
  by this library's faithful numerics, bit-identical to the reference
  library.

    python -m otfwi_b200.gradcheck --report out.json
"""
import argparse
import json
import time

import numpy as np

from .batch import ShotBatch
from .learned import defect_scenario
from .scenarios import gaussian_smooth


FD_TOLERANCE = 1e-2  # relative, Richardson-combined central differences of an FP32 forward


def run(X=1024, T=6000, n_elem=64, pitch=12, shots=32, n_dir=16, eps=8e-3, seed=3, log=print):
    import torch
    from .autograd import PMLPropagator
    sc = defect_scenario(X, X, T, seed, n_elem, pitch, 8, n_src=shots)
    rep = {"grid": [X, X], "nt": T, "shots": sc.n_src, "receivers": sc.n_rec, "directions": n_dir, "eps": eps}
    prop = PMLPropagator(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, precision=1)
    rep["checkpoint_every"] = prop.every
    c_true = torch.as_tensor(sc.c_true, dtype=torch.float32, device="cuda")
    c0 = torch.as_tensor(gaussian_smooth(sc.c_true, 8.0), dtype=torch.float32, device="cuda")
    with torch.no_grad():
        obs = prop(c_true).clone()

    def loss_of(tr):
        d = (tr[:, :, 1:] - obs[:, :, 1:]).double()
        return 0.5 * (d * d).sum()

    c = c0.clone().requires_grad_(True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L = loss_of(prop(c))
    L.backward()
    torch.cuda.synchronize()
    rep["gradient_s"] = time.perf_counter() - t0
    g = c.grad.double()
    rep["loss"] = float(L.item())
    log(f"exact gradient in {rep['gradient_s']:.1f} s (loss {rep['loss']:.4e}, checkpoint every {prop.every})")
    rng = np.random.default_rng(seed + 100)
    fd = []

    def central(v, e):
        with torch.no_grad():
            lp = float(loss_of(prop(c0 + e * v)).item())
            lm = float(loss_of(prop(c0 - e * v)).item())
        return (lp - lm) / (2 * e)

    dirs = [("gradient", g.float() / g.abs().max().float() * float(c0.mean()))]
    for k in range(n_dir):
        v = gaussian_smooth(rng.standard_normal((sc.Z, sc.X)), 6.0)
        dirs.append((f"random {k}", torch.as_tensor(v / np.abs(v).max(), dtype=torch.float32, device="cuda")
                     * float(c0.mean())))
    for name, v in dirs:
        d1 = central(v, eps)
        d2 = central(v, eps / 2)
        r = (4 * d2 - d1) / 3
        a = float((g * v.double()).sum().item())
        rel = lambda f: abs(f - a) / max(abs(f), 1e-300)
        fd.append({"direction": name, "fd_eps": d1, "fd_half_eps": d2, "fd_richardson": r, "adjoint": a,
                   "rel_eps": rel(d1), "rel_half_eps": rel(d2), "rel": rel(r)})
        log(f"{name}: FD(e) {d1:.6e} FD(e/2) {d2:.6e} Richardson {r:.6e} adjoint {a:.6e} "
            f"rel {fd[-1]['rel']:.2e} (single e/2: {fd[-1]['rel_half_eps']:.2e})")
    rep["fd"] = fd
    rep["fd_tolerance"] = FD_TOLERANCE
    rep["fd_rel_median"] = float(np.median([d["rel"] for d in fd]))
    rep["fd_rel_max"] = float(np.max([d["rel"] for d in fd]))
    rep["fd_pass"] = bool(rep["fd_rel_max"] <= FD_TOLERANCE)
    prop.batch.close()
    del prop
    torch.cuda.empty_cache()
    # the reference's algorithm (faithful numerics, bit-identical to the reference library)
    b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, precision=0)
    b.set_model(c_true)
    b.set_observed(b.forward())
    b.set_model(c0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    gref, _ = b.gradient("l2")
    rep["reference_algorithm_gradient_s"] = time.perf_counter() - t0
    b.close()
    P = sc.PML
    ge = (g / (2 * c0.double())).cpu().numpy()[P:-P, P:-P]  # dL/dc^2
    gr = gref.astype(np.float64)[P:-P, P:-P]
    rep["cosine_vs_reference_algorithm"] = float(np.sum(ge * gr) / (np.linalg.norm(ge) * np.linalg.norm(gr)))
    log(f"cosine(exact, reference algorithm) {rep['cosine_vs_reference_algorithm']:.4f}")
    return rep


def main(argv=None):
    ap = argparse.ArgumentParser(description="full-size gradient check of the differentiable path")
    ap.add_argument("--grid", type=int, default=1024)
    ap.add_argument("--nt", type=int, default=6000)
    ap.add_argument("--shots", type=int, default=32)
    ap.add_argument("--directions", type=int, default=16)
    ap.add_argument("--eps", type=float, default=8e-3, help="larger step of the Richardson pair (e, e/2)")
    ap.add_argument("--report", default=None)
    a = ap.parse_args(argv)
    rep = run(X=a.grid, T=a.nt, shots=a.shots, n_dir=a.directions, eps=a.eps)
    print(json.dumps({k: v for k, v in rep.items() if k != "fd"}))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(rep, f)


if __name__ == "__main__":
    main()
