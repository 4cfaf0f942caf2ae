"""Uneven multi-instance batch: many independent inversions of different
grid sizes, shot counts and T, their complete gradients run as parallel
branches of one CUDA graph per wave (otf_multi_*).

No reference counterpart: the reference computes one shot of one problem per
cuda_grad_ext call (cuda_interface_pml.py:225-236). Instances are seeded
defect models (scenarios.heterogeneous_defects) between a top and a bottom
linear array; each instance's kernel variant and tile shape come from the
autotuner; instances are packed into waves whose device memory fits a
budget, one graph launch per wave. Reported: whole-batch Gcell-steps/s
(2 X Z (T-1) shots per instance, forward + adjoint) and the same instances
run one graph at a time. The per-instance gradient error against the FP64
oracle is checked on the smallest instances by tests/test_uneven_gpu.py.

    python -m otfwi_b200.uneven --instances 48 --report out.json
"""
import argparse
import json
import time

import numpy as np

from .batch import MultiBatch, ShotBatch
from .learned import C_BG, defect_scenario


def min_steps(Z, PML=20):
    """Steps for a transmission record between the two arrays (rows PML + 6
    and Z - 1 - (PML + 6)): 1.2 times the background travel time plus the
    wavelet. Shorter records leave the far array's traces empty, and the
    Wasserstein misfit of an all-zero observed trace is 0/0 (NaN), as in the
    reference's adjoint_functions.py:25-67."""
    return int(1.2 * (Z - 1 - 2 * (PML + 6)) / C_BG) + 300


def instance_specs(n, seed=2024, grid=(192, 768), shots=(8, 64), nt=(1500, 5000)):
    """Seeded (X, Z, T, shots, n_elem, seed) per instance; grids multiples of 32."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        X = int(rng.integers(grid[0] // 32, grid[1] // 32 + 1)) * 32
        Z = int(rng.integers(grid[0] // 32, grid[1] // 32 + 1)) * 32
        T = max(int(rng.integers(nt[0], nt[1] + 1)), min_steps(Z))
        n_elem = min(64, (X - 2 * 40) // 6 + 1)
        ns = int(rng.integers(shots[0] // 2, min(shots[1], 2 * n_elem) // 2 + 1)) * 2
        out.append({"X": X, "Z": Z, "T": T, "shots": ns, "n_elem": n_elem, "seed": int(seed + i)})
    return out


def scenario(spec):
    rng = np.random.default_rng(spec["seed"])
    return defect_scenario(spec["X"], spec["Z"], spec["T"], spec["seed"], spec["n_elem"], 6,
                           int(rng.integers(3, 9)), n_src=spec["shots"])


def device_bytes(spec, n_ring_per_shot=None):
    """Estimate of one instance's device memory (fields, ring, traces)."""
    X, Z, T, S = spec["X"], spec["Z"], spec["T"], spec["shots"]
    slot = (Z + 16) * ((X + 16 + 31) // 32 * 32) * 4
    fields = 2 * 4 * 2 * S * slot + S * slot  # two field sets, ping-pong, gradient
    ring = n_ring_per_shot if n_ring_per_shot is not None else 2 * 5 * (X + Z) + 16
    n_rec = 2 * spec["n_elem"]
    return fields + 4 * T * S * ring + 4 * 4 * S * n_rec * T


def waves(specs, budget):
    """Greedy packing (largest first) of instances into waves within budget bytes."""
    order = sorted(range(len(specs)), key=lambda i: -device_bytes(specs[i]))
    out, cur, used = [], [], 0
    for i in order:
        b = device_bytes(specs[i])
        if cur and used + b > budget:
            out.append(cur)
            cur, used = [], 0
        cur.append(i)
        used += b
    if cur:
        out.append(cur)
    return out


def build(spec, sc, misfit, tune):
    from .autotune import autotune
    kernel, tile = -1, 4
    if tune:
        kernel, tile, _ = autotune(sc, precision=1, misfit=misfit, T_proxy=150,
                                  cands=[(4, 4), (2, 0), (2, 1), (2, 4)])
    b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, precision=1, tile=tile,
                  kernel=kernel)
    b.set_model(sc.c_true)
    obs = b.forward()
    b.set_observed(obs)
    b.set_model(sc.c_start)
    return b, kernel, tile


def run(n=48, budget_gb=120.0, misfit="wasserstein", tune=True, log=print):
    import torch
    specs = instance_specs(n)
    plan = waves(specs, budget_gb * 1e9)
    cells = [2.0 * s["X"] * s["Z"] * (s["T"] - 1) * s["shots"] for s in specs]
    rep = {"instances": specs, "waves": plan, "budget_gb": budget_gb, "misfit": misfit}
    t_multi, t_single = 0.0, 0.0
    for w, idx in enumerate(plan):
        scs = {i: scenario(specs[i]) for i in idx}
        bs = {}
        for i in idx:
            bs[i], specs[i]["kernel"], specs[i]["tile"] = build(specs[i], scs[i], misfit, tune)
        m = MultiBatch([bs[i] for i in idx])
        m.gradient(misfit)  # capture and warm
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = m.gradient(misfit)
        torch.cuda.synchronize()
        dt_m = time.perf_counter() - t0
        t_multi += dt_m
        # the same instances one graph at a time
        for i in idx:
            bs[i].gradient(misfit)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in idx:
            bs[i].gradient(misfit)
        torch.cuda.synchronize()
        dt_s = time.perf_counter() - t0
        t_single += dt_s
        for i, (g, mis) in zip(idx, res):
            specs[i]["misfit"] = mis
            specs[i]["grad_norm"] = float(np.linalg.norm(g))
        log(f"wave {w}: {len(idx)} instances, {sum(cells[i] for i in idx) / 1e9:.0f} Gcell-steps, "
            f"one graph {dt_m:.2f} s, one by one {dt_s:.2f} s")
        m.close()
        for b in bs.values():
            b.close()
        del bs
        torch.cuda.empty_cache()
    total = sum(cells)
    rep["all_finite"] = bool(all(np.isfinite(s["misfit"]) and np.isfinite(s["grad_norm"]) for s in specs))
    rep.update({"gcell_steps": total / 1e9, "multi_s": t_multi, "single_s": t_single,
                "multi_gcell_steps_per_s": total / t_multi / 1e9,
                "single_gcell_steps_per_s": total / t_single / 1e9})
    return rep


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--instances", type=int, default=48)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--misfit", default="wasserstein")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--report", default=None)
    a = ap.parse_args(argv)
    rep = run(a.instances, a.budget_gb, a.misfit, not a.no_tune)
    print(json.dumps({k: v for k, v in rep.items() if k not in ("instances", "waves")}))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(rep, f)


if __name__ == "__main__":
    main()
