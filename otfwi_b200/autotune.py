"""Autotuner for the step kernels: picks the kernel variant and tile shape.

For a problem (grid, shot count, numerics) every compiled candidate is timed
on a short proxy of the real run -- the same grid and shots, a few hundred
time steps of the full gradient (forward, misfit, reverse) replayed as the
same CUDA graph -- with CUDA events on the library's stream. The winner is
cached in a JSON file keyed by (X, Z, shots, receivers, precision, GPU name)
so the search runs once per configuration.

Candidates: tile shapes 0 (56x56), 1 (120x24), 4 (56x24) with the persistent
TMA kernels (variant 1) and, for the fast numerics, the strip-split kernels
(variant 2), the unfused streaming half-steps (variant 4, no tiles) and the
paired half-steps (variant 5, both in one launch, no tiles);
shapes 2 (120x56) and 3 (248x24) with the one-tile-per-CTA kernels
(variant 0).
"""
import json
import os
import time

import numpy as np

TILES = {0: (56, 56), 1: (120, 24), 2: (120, 56), 3: (248, 24), 4: (56, 24)}


def candidates(precision):
    """(kernel variant, tile) pairs timed by `tune`. The paired (5) and
    row-lag fused (6) variants are left out: bit-identical to the unfused
    kernels (4) and measured slower on the 64-shot 512^2 gradient (0.47 and
    0.84 ms per step against 0.39)."""
    c = [(1, 0), (1, 1), (1, 4), (0, 2), (0, 3)]
    if precision == 1:
        c = [(4, 4), (2, 0), (2, 1), (2, 4)] + c
    return c


def cache_path():
    return os.environ.get("OTFWI_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "otfwi_b200", "tune.json"))


def _key(X, Z, shots, n_rec, precision, gpu, cands):
    tried = ",".join(f"{k}/{t}" for k, t in cands)
    return f"{gpu}|{X}x{Z}|shots{shots}|rx{n_rec}|prec{precision}|{tried}"


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(d):
    """Write the cache through a per-process temporary file and an atomic
    rename, so ranks tuning at the same time never leave a torn file."""
    p = cache_path()
    tmp = f"{p}.{os.getpid()}.tmp"
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, p)
    except OSError:
        try:
            os.remove(tmp)
        except OSError:
            pass


def time_config(sc, kernel, tile, precision, T_proxy, misfit, reps=2):
    """ms per proxy gradient of one candidate (ShotBatch on a truncated T)."""
    import torch
    from .batch import ShotBatch
    T = min(sc.T, T_proxy)
    b = ShotBatch(sc.X, sc.Z, T, sc.PML, sc.src_mask, sc.rec_mask, np.ascontiguousarray(sc.source[:, :T]),
                  prec_deriv=4, precision=precision, tile=tile, kernel=kernel)
    try:
        b.set_model(sc.c_start)
        dev = torch.device("cuda", torch.cuda.current_device())
        obs = torch.zeros((b.n_shots, b.n_rec, T), dtype=torch.float32, device=dev)
        b.set_observed(obs)
        grad = torch.empty((sc.Z, sc.X), dtype=torch.float32, device=dev)
        mis = torch.empty(1, dtype=torch.float64, device=dev)
        stream = torch.cuda.ExternalStream(b.stream(), device=dev)
        b.gradient(misfit, grad=grad, misfit_out=mis)  # capture + warm
        b.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            b.gradient(misfit, grad=grad, misfit_out=mis)
        e1.record(stream)
        e1.synchronize()
        b.sync()
        return e0.elapsed_time(e1) / reps
    finally:
        b.close()


def autotune(sc, precision=1, misfit="wasserstein_softplus", T_proxy=300, use_cache=True, verbose=False,
             cands=None):
    """Best (kernel, tile) for a scenario; returns (kernel, tile, table).
    ``cands``: [(kernel, tile)] to try instead of every compiled candidate."""
    import torch
    gpu = torch.cuda.get_device_name()
    cands = cands if cands is not None else candidates(precision)
    key = _key(sc.X, sc.Z, sc.n_src, sc.n_rec, precision, gpu, cands)
    cache = _load() if use_cache else {}
    if key in cache:
        e = cache[key]
        return e["kernel"], e["tile"], e.get("table", {})
    table = {}
    for kernel, tile in cands:
        t0 = time.perf_counter()
        try:
            ms = time_config(sc, kernel, tile, precision, T_proxy, misfit)
        except Exception as ex:  # a candidate that cannot run here is skipped
            ms = float("inf")
            if verbose:
                print(f"autotune: kernel {kernel} tile {tile} skipped: {ex}")
        table[f"k{kernel}_t{tile}"] = ms
        if verbose:
            print(f"autotune: kernel {kernel} tile {TILES[tile]} {ms:.2f} ms ({time.perf_counter() - t0:.1f} s)")
    best = min(table, key=table.get)
    kernel, tile = int(best.split("_")[0][1:]), int(best.split("_")[1][1:])
    cache[key] = {"kernel": kernel, "tile": tile, "table": table}
    if use_cache:
        _store(cache)
    return kernel, tile, table
