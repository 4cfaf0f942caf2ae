"""Learned-preconditioned FWI: training pairs from plain FWI runs, U-Net
training on the GPU, and the learned proposal inside the FWI loop.

No reference counterpart (the reference's inversion is plain L-BFGS-B,
regression.py:82-88). The design:

- data: plain FWI (``fwi.descent``, bracketing line search, band by band) on
  seeded defect models (elliptical 4000-6300 m/s defects in a 5900 m/s
  background with +-3% smoothed heterogeneity) between two linear arrays,
  top and bottom, as in the reference's inversion setups. Every
  iterate k of a run gives one pair: features (gradient, illumination,
  current model) -> the update the plain method accepted from k to the end
  of the run, c_final - c_k (the sum of its accepted updates);
- features, per cell: -gmask*g / max|gmask*g|, log-scaled illumination in
  [0, 1], (c - c_bg) / span; target (c_final - c_k) / span, with c_bg the
  background and span the defect contrast (nondimensional units);
- training: weighted MSE (weight = gradient mask), Adam, random horizontal
  flips (the arrays are centred), all on the GPU by the library's kernels;
- inference: the network's update is tried first at every iteration and
  accepted only if the misfit decreases; otherwise the plain line-search step
  is taken (``fwi.descent(proposer=...)``).
"""
import argparse
import json
import math
import os
import time

import numpy as np

from . import fwi
from .scenarios import Scenario, heterogeneous_defects, ricker

C_MAX, C_BG_MPS, V_LO, V_HI = 6300.0, 5900.0, 4000.0, 6300.0
C_BG = 0.4 * C_BG_MPS / C_MAX
SPAN = 0.4 * (C_BG_MPS - V_LO) / C_MAX
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "precond_unet.npz")


def defect_scenario(X, Z, T, seed, n_elem, pitch, n_def, n_src=None, PML=20, f0_hz=5e6, amin=4, amax=14):
    """Seeded inversion case: 5900 m/s background with +-3% smoothed
    heterogeneity and n_def elliptical defects of 4000-6300 m/s centred in
    the central half of the grid (scenarios.heterogeneous_defects), between
    two centred linear arrays of n_elem elements near the top and the bottom,
    as in the reference's inversion setups (setups/setup1_OCNDT.py:56-77:
    sources and receivers at rows p1a and -p1a). Every element receives;
    n_src elements fire, half on each array, evenly spaced. Velocities are
    nondimensionalised with CFL 0.4 at 6300 m/s; the start is the homogeneous
    background."""
    rng = np.random.default_rng(seed)
    dx = 5e-5
    dt = 0.4 * dx / C_MAX
    c = heterogeneous_defects(X, Z, rng, n_def=n_def, c_bg=C_BG_MPS, v_lo=V_LO, v_hi=V_HI, amin=amin, amax=amax,
                              lo=0.25 * min(X, Z) + 4, hi=0.75 * min(X, Z) - 4)
    rows = (PML + 6, Z - 1 - (PML + 6))
    x_first = (X - (n_elem - 1) * pitch) // 2
    xs = x_first + pitch * np.arange(n_elem)
    rec = np.zeros((Z, X), dtype=bool)
    src = np.zeros((Z, X), dtype=bool)
    n_src = 2 * n_elem if n_src is None else n_src
    fire = xs[np.round(np.linspace(0, n_elem - 1, n_src // 2)).astype(int)]
    for z in rows:
        rec[z, xs] = True
        src[z, fire] = True
    f0 = f0_hz * dt
    w = ricker(T, f0, 1.2 / f0).astype(np.float32)
    return Scenario(X, Z, T, PML, 0.4 * c / C_MAX, np.full((Z, X), C_BG), src, rec,
                    np.repeat(w[None, :], int(src.sum()), axis=0), dx, C_MAX, f"defects{X}x{Z}_s{seed}")


def features(prob, b, c, g):
    """[1, Z, X, 3] FP32 network input at model c with gradient g."""
    torch = prob.torch
    gm = -g * prob.gmask
    gm = gm / torch.clamp(gm.abs().max(), min=1e-30)
    il = prob.illumination(b, c)
    il = torch.log10(il / torch.clamp(il.max(), min=1e-30) + 1e-3) / 3.0 + 1.0
    cn = (c - C_BG) / SPAN
    return torch.stack([gm, il, cn], dim=-1)[None].contiguous()


class Proposer:
    """fwi.descent proposer: the network's update (nondimensional) at c."""

    def __init__(self, net):
        self.net = net

    def __call__(self, prob, b, c, g, J):
        out = self.net.forward(features(prob, b, c, g))
        return (out[0] * SPAN * prob.gmask).clone()


def _bands(f_lo, f_hi, iters):
    return [fwi.Band(f_lo, iters), fwi.Band(f_hi, iters)]


def _plain_run(r, seed0, X, Z, T, n_elem, pitch, n_src, iters, bands_hz, misfit):
    """One plain FWI run of the training set: its (features, target) pairs
    (FP16, on the GPU), the gradient mask and the run's statistics."""
    rng = np.random.default_rng(seed0 + r)
    sc = defect_scenario(X, Z, T, seed0 + r, n_elem, pitch, int(rng.integers(3, 9)), n_src=n_src)
    prob = fwi.Problem(sc, _bands(bands_hz[0], bands_hz[1], iters), misfit=misfit)
    feats, models, pending = [], [], {}

    def on_step(b, it, c, g, J0):
        pending["p"] = (features(prob, b, c, g)[0].half(), c.clone())

    def on_iter(b, it, c_new, g, J0, J_new):
        f, ck = pending.pop("p")
        feats.append(f)
        models.append(ck)

    c_fin, h = fwi.descent(prob, sc.c_start, on_step=on_step, on_iter=on_iter)
    ys = [((c_fin - ck) / SPAN * prob.gmask).half() for ck in models]
    stat = {"seed": seed0 + r, "rms0": h.rms[0], "rms_final": h.rms[-1], "iters": len(h.rms) - 1,
            "wall_s": h.t[-1], "pairs": len(feats)}
    gmask = prob.gmask.clone()
    for sb in prob._batches.values():
        sb.close()
    return feats, ys, gmask, stat


def generate(n_runs, seed0=1000, X=256, Z=256, T=1500, n_elem=32, pitch=6, n_src=16, iters=8,
             bands_hz=(2.5e6, 5e6), misfit="wasserstein", log=None, workers=1):
    """Training pairs from n_runs plain FWI runs: (inputs [M, Z, X, 3],
    targets [M, Z, X], weight [Z, X]) on the GPU, and per-run statistics.

    ``workers`` > 1 runs that many inversions at once, each in its own host
    thread with its own CUDA streams (the library's calls release the
    interpreter lock while they wait): one small inversion leaves most of the
    GPU idle between its short launches, several fill it. Pairs are returned
    in run order whatever the worker count."""
    import threading
    import torch
    from concurrent.futures import ThreadPoolExecutor
    t0 = time.perf_counter()
    results = [None] * n_runs
    lock = threading.Lock()
    dev = torch.cuda.current_device()
    args = (seed0, X, Z, T, n_elem, pitch, n_src, iters, bands_hz, misfit)

    def note(r):
        if log:
            st = results[r][3]
            with lock:
                log(f"run {r}: rms {st['rms0']:.1f} -> {st['rms_final']:.1f} m/s in {st['wall_s']:.2f} s "
                    f"({st['pairs']} pairs, {time.perf_counter() - t0:.0f} s total)")

    def work(w):
        torch.cuda.set_device(dev)
        with torch.cuda.stream(torch.cuda.Stream()):
            for r in range(w, n_runs, workers):
                out = _plain_run(r, *args)
                torch.cuda.current_stream().synchronize()
                results[r] = out
                note(r)

    if workers <= 1:
        for r in range(n_runs):
            results[r] = _plain_run(r, *args)
            note(r)
    else:
        with ThreadPoolExecutor(max_workers=workers) as ex:
            for f in [ex.submit(work, w) for w in range(workers)]:
                f.result()
        torch.cuda.synchronize()
    xs = [x for res in results for x in res[0]]
    ys = [y for res in results for y in res[1]]
    return torch.stack(xs), torch.stack(ys), results[0][2], [res[3] for res in results]


def train(net, X, Y, weight, steps=4000, batch=16, lr=1e-3, seed=0, log=None, group=None):
    """Adam on the weighted MSE with cosine learning-rate decay and random
    horizontal flips; returns the loss history (host floats, every step).

    Data parallel when a process group is initialised (one process per GPU):
    rank 0's parameters are broadcast first, every rank draws its own
    micro-batch of ``batch`` pairs (global batch = batch x world), and the
    flat parameter gradient is averaged over ranks by one all-reduce before
    each Adam step, so every rank keeps identical parameters. The loss
    history is the mean over ranks."""
    import torch
    from .distributed import broadcast_params_, dp_average_, world_of
    world, rank = world_of(group)
    dev = net.params.device
    if world > 1:
        broadcast_params_(net.params, group)
        net.pack()
    g = torch.Generator(device=dev)
    g.manual_seed(seed + 7919 * rank)
    M = X.shape[0]
    w = weight[None].expand(batch, -1, -1).contiguous()
    inv = 1.0 / float(w.sum().item())
    losses = []
    for s in range(steps):
        idx = torch.randint(0, M, (batch,), device=dev, generator=g)
        xb = X[idx].float()
        yb = Y[idx].float()
        flip = torch.rand(batch, device=dev, generator=g) < 0.5
        xb = torch.where(flip[:, None, None, None], xb.flip(2), xb).contiguous()
        yb = torch.where(flip[:, None, None], yb.flip(2), yb).contiguous()
        wb = torch.where(flip[:, None, None], w.flip(2), w).contiguous()
        lr_s = lr * 0.5 * (1 + math.cos(math.pi * s / steps))
        net.forward(xb)
        loss = net.loss_grad(yb, wb, inv_norm=inv).clone()
        net.backward(net._buffers(*yb.shape)["dout"])
        if world > 1:
            dp_average_(net.grads, group)
            dp_average_(loss, group)
        net.adam(lr_s)
        losses.append(loss)
        if log and (s % 500 == 0 or s == steps - 1):
            log(f"step {s}: loss {float(loss.item()):.5f}")
    return [float(l.item()) for l in losses]


def validation_loss(net, X, Y, weight, batch=16):
    """Weighted MSE of the network over held-out pairs (no flips, forward
    only), normalised as the training loss is."""
    M = X.shape[0]
    tot, n = 0.0, 0
    for i in range(0, M, batch):
        xb = X[i:i + batch].float().contiguous()
        yb = Y[i:i + batch].float().contiguous()
        k = xb.shape[0]
        wb = weight[None].expand(k, -1, -1).contiguous()
        net.forward(xb)
        loss = net.loss_grad(yb, wb, inv_norm=1.0 / float(wb.sum().item()))
        tot += float(loss.item()) * k
        n += k
    return tot / max(n, 1)


def learning_curve(X, Y, w, stats, n_val, sizes, steps, batch, lr, log=None):
    """Validation loss on the pairs of the last n_val runs for networks
    trained (same seed, steps, batch, lr) on the pairs of the first k runs,
    for each k in sizes: whether more plain-FWI runs still help."""
    from .unet import UNet
    ends = np.cumsum([0] + [st["pairs"] for st in stats])
    n_train = len(stats) - n_val
    Xv, Yv = X[ends[n_train]:], Y[ends[n_train]:]
    out = []
    for k in sizes:
        k = min(int(k), n_train)
        net = UNet(base=32, in_ch=3, seed=0)
        losses = train(net, X[:ends[k]], Y[:ends[k]], w, steps=steps, batch=batch, lr=lr)
        vl = validation_loss(net, Xv, Yv, w)
        out.append({"runs": k, "pairs": int(ends[k]), "train_loss_last_100": float(np.mean(losses[-100:])),
                    "validation_loss": vl})
        if log:
            log(f"learning curve: {k} runs ({int(ends[k])} pairs): validation loss {vl:.5f}")
    return out


def evaluate(net, X=512, Z=512, T=4000, n_elem=64, pitch=6, n_src=64, iters=15, seed=7, n_def=8,
             bands_hz=(2.5e6, 5e6), misfit="wasserstein", log=None):
    """Plain vs learned FWI on one seeded model: time for the learned method
    to reach the plain method's final RMS velocity error."""
    sc = defect_scenario(X, Z, T, seed, n_elem, pitch, n_def, n_src=n_src)
    out = {"grid": [X, Z], "nt": T, "shots": sc.n_src, "receivers": sc.n_rec, "bands_hz": list(bands_hz),
           "iters_per_band": iters, "misfit": misfit, "seed": seed}
    hist = {}
    for name, prop in (("plain", None), ("learned", Proposer(net))):
        prob = fwi.Problem(sc, _bands(bands_hz[0], bands_hz[1], iters), misfit=misfit)
        c0 = prob.torch.as_tensor(sc.c_start, dtype=prob.torch.float32).cuda()
        for b in range(len(prob.bands)):  # observed data and graph captures outside the timed runs
            prob.gradient(b, c0)
            prob.objective(b, c0)
        _, h = fwi.descent(prob, sc.c_start, proposer=prop)
        hist[name] = h
        if log:
            log(f"{name}: rms {h.rms[0]:.1f} -> {h.rms[-1]:.1f} m/s in {h.t[-1]:.2f} s, "
                f"{sum(h.learned)} learned steps")
        del prob
    target = hist["plain"].rms[-1]
    t_plain = hist["plain"].time_to(target)
    t_learned = hist["learned"].time_to(target)
    out.update({
        "rms_start_mps": hist["plain"].rms[0],
        "plain_final_rms_mps": target,
        "learned_final_rms_mps": hist["learned"].rms[-1],
        "plain_time_s": hist["plain"].t[-1],
        "plain_time_to_final_rms_s": t_plain,
        "learned_time_to_plain_final_rms_s": t_learned,
        "time_ratio": (t_learned / t_plain) if (t_learned is not None and t_plain) else None,
        "learned_steps_accepted": int(sum(hist["learned"].learned)),
        "history": {k: {"t": v.t, "rms": v.rms, "misfit": v.misfit, "learned": v.learned, "band": v.band}
                    for k, v in hist.items()},
    })
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description="learned-preconditioned FWI: data, training, evaluation")
    ap.add_argument("--runs", type=int, default=256, help="plain FWI runs that generate training pairs")
    ap.add_argument("--workers", type=int, default=1, help="plain FWI runs in flight at once (host threads)")
    ap.add_argument("--val-runs", type=int, default=0,
                    help="further plain runs held out for a learning curve (validation loss only)")
    ap.add_argument("--curve", default="", help="comma-separated training-set sizes (runs) of the learning curve")
    ap.add_argument("--train-iters", type=int, default=10, help="plain iterations per band in data runs")
    ap.add_argument("--steps", type=int, default=4000, help="training steps")
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--eval-grid", type=int, default=512)
    ap.add_argument("--eval-nt", type=int, default=4000)
    ap.add_argument("--eval-elements", type=int, default=64, help="elements per array (top and bottom)")
    ap.add_argument("--eval-shots", type=int, default=64)
    ap.add_argument("--eval-iters", type=int, default=15, help="iterations per band in the evaluation")
    ap.add_argument("--eval-seeds", default="7", help="comma-separated model seeds of the evaluation")
    ap.add_argument("--weights", default=WEIGHTS, help="where to save / load the trained network")
    ap.add_argument("--skip-train", action="store_true", help="evaluate the saved network")
    ap.add_argument("--report", default=None, help="JSON report path")
    a = ap.parse_args(argv)
    from .unet import UNet

    def log(m):
        print(m, flush=True)

    rep = {}
    if not a.skip_train:
        t0 = time.perf_counter()
        X, Y, w, stats = generate(a.runs + a.val_runs, iters=a.train_iters, log=log, workers=a.workers)
        data_s = time.perf_counter() - t0
        if a.curve and a.val_runs:
            rep["learning_curve"] = learning_curve(X, Y, w, stats, a.val_runs,
                                                   [int(v) for v in a.curve.split(",")], a.steps, a.batch,
                                                   a.lr, log=log)
        if a.val_runs:
            n_keep = int(np.sum([st["pairs"] for st in stats[:a.runs]]))
            X, Y, stats = X[:n_keep], Y[:n_keep], stats[:a.runs]
        rep["data"] = {"runs": a.runs, "workers": a.workers, "pairs": int(X.shape[0]),
                       "held_out_runs": a.val_runs, "wall_s": data_s,
                       "grid": [256, 256], "iters_per_band": a.train_iters,
                       "mean_rms_start": float(np.mean([s["rms0"] for s in stats])),
                       "mean_rms_final": float(np.mean([s["rms_final"] for s in stats]))}
        net = UNet(base=32, in_ch=3, seed=0)
        t0 = time.perf_counter()
        losses = train(net, X, Y, w, steps=a.steps, batch=a.batch, lr=a.lr, log=log)
        rep["train"] = {"steps": a.steps, "batch": a.batch, "lr": a.lr, "wall_s": time.perf_counter() - t0,
                        "loss_first": losses[0], "loss_last_100": float(np.mean(losses[-100:]))}
        os.makedirs(os.path.dirname(a.weights), exist_ok=True)
        net.save(a.weights)
        del X, Y
    else:
        net = UNet.load(a.weights)
    rep["eval"] = []
    for seed in [int(x) for x in a.eval_seeds.split(",")]:
        ev = evaluate(net, X=a.eval_grid, Z=a.eval_grid, T=a.eval_nt, n_elem=a.eval_elements, n_src=a.eval_shots,
                      iters=a.eval_iters, seed=seed, log=log)
        rep["eval"].append(ev)
        log(json.dumps({k: v for k, v in ev.items() if k != "history"}))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(rep, f)
    return rep


if __name__ == "__main__":
    main()
