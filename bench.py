"""Benchmark: batched full-matrix-capture forward + adjoint gradient.

Workload (one "step"): one complete FWI gradient of a 64-element
full-matrix-capture acquisition on a 512 x 512 grid, T = 4000 time steps,
20-cell PML, 64 shots x 64 receivers, quadratic Wasserstein misfit on
softplus-normalised traces: forward modelling of all 64 shots with boundary
ring recording, device misfit and adjoint sources, adjoint + reconstruction
+ imaging condition for all shots, shot mean of the gradient. Synthetic,
seeded model (5900 m/s with three 3000 m/s circular defects) and 5 MHz
Ricker source; the gradient is taken at the homogeneous starting model
against data simulated from the true model.

Metric: fwd+adj Gcell-steps/s = 2 * X * Z * (T-1) * shots / step time
(whole job over all ranks). Run: python bench.py [--gpus N --steps K --warmup W]
or --impl reference for the reference library's per-shot loop.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+adj Gcell-steps/s"
UNIT = "Gcell-steps/s"
# algorithmic HBM bytes per cell per time step (one shot): forward 28
# (P, Ax, Az read + write, c^2 read), adjoint 28, reconstruction 28, gradient
# read + write 8 -> 92; the reverse step kernel carries 64 of them, the forward 28
BYTES_FWD = 28
BYTES_REV = 64
BYTES_STEP = 92
BYTES_AREV = 52  # k_unfused_a_rev_sets: both sets' P, Ax, Az, the adjoint P again (the imaging CTA's
#                  own cells) and grad read; four A fields and grad written


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", type=int, default=int(os.environ.get("OTFWI_BENCH_PRECISION", "1")))
    ap.add_argument("--tile", type=int, default=int(os.environ.get("OTFWI_BENCH_TILE", "-1")),
                    help="tile shape index; -1 = chosen by the autotuner (otfwi_b200.autotune)")
    ap.add_argument("--kernel", type=int, default=int(os.environ.get("OTFWI_BENCH_KERNEL", "-1")),
                    help="-1 automatic, 0 per-tile, 1 persistent TMA, 2 persistent strip-split")
    ap.add_argument("--stream-rows", type=int, default=64, help="segment rows of the z-streaming kernels")
    ap.add_argument("--X", type=int, default=512)
    ap.add_argument("--T", type=int, default=4000)
    ap.add_argument("--shots", type=int, default=64)
    ap.add_argument("--misfit", default="wasserstein_softplus")
    ap.add_argument("--mode", default="weak", choices=["weak", "strong"],
                    help="weak: every rank inverts its own 64-shot acquisition (default); strong: the shots "
                         "of ONE acquisition split over the ranks (distributed.ShardedShots' partition)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-shots", type=int, default=2, help="shots per reference-arm step")
    ap.add_argument("--leg", default="gradient", choices=["gradient", "cpml", "misfits"],
                    help="gradient: the headline FMC gradient (default); cpml: the second-order CPML "
                         "path, this library against the reference's; misfits: the device trace misfits "
                         "against the CPU restatement")
    ap.add_argument("--cpml-impl", default=None, help=argparse.SUPPRESS)
    return ap.parse_args()


def workload(args, rank=0):
    """The FMC acquisition of one rank: rank r's array sits 2r cells to the
    right (each rank inverts its own acquisition of the same specimen)."""
    from otfwi_b200 import scenarios
    return scenarios.fmc(X=args.X, Z=args.X, T=args.T, n_elem=args.shots,
                         x_first=max(24, args.X // 2 - 3 * args.shots + 3) + 2 * rank)


def config_block(args, sc, world=1):
    """The workload's description, identical for both arms at the same N."""
    return {"workload": f"fmc{sc.X}x{sc.Z}_T{sc.T}_{sc.n_src}shots_{sc.n_rec}rx_{args.misfit}",
            "grid": [sc.X, sc.Z], "nt": sc.T, "pml": sc.PML, "shots": sc.n_src, "receivers": sc.n_rec,
            "misfit": args.misfit, "precision": ["faithful", "fast"][args.precision],
            "l2": "working set (fields of 64 shots, about 1.2 GB) larger than the 126 MB L2; no flush needed",
            "parallelism": (f"shots of one acquisition over {world} GPU(s)" if args.mode == "strong"
                            else f"one acquisition per GPU, {world} GPU(s)")}


class Clocks:
    """Samples nvidia-smi during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(kernel):
    """DRAM bytes per cell of one reverse step from the committed ncu summary
    of the kernel variant in use (line 'dram_bytes_per_cell: N'):
    profiles/reverse_step_fmc.md for the fused strip-split step (one
    launch), profiles/reverse_step_unfused_fmc.md for the unfused one (its
    three launches summed)."""
    return profile_value(kernel, "dram_bytes_per_cell")


def profile_value(kernel, key):
    """A 'key: N' line of the committed ncu summary of the reverse step of
    this kernel variant (None when absent)."""
    name = {4: "reverse_step_unfused_fmc.md", 5: "reverse_step_paired_fmc.md",
            6: "reverse_step_fused_fmc.md"}.get(kernel, "reverse_step_fmc.md")
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith(key + ":"):
            return float(line.split(":")[1])
    return None


def cpu_baseline(args, sc):
    """FP64 oracle (C, OpenMP, all host threads) on a bounded sample: one shot
    of the same FMC problem, the first T_s time steps, forward + misfit +
    adjoint gradient; rate in the metric's unit."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pml_oracle as po
    import misfit_oracle as mo
    from otfwi_b200.cuda_interface_pml import pml_damping, ring_mask
    Ts = 1200
    dxp, dzp = pml_damping(sc.X, sc.Z, sc.PML)
    sx, sz = sc.src_xz()
    mx, mz = sc.rec_xz()
    rz, rx = np.where(ring_mask(sc.X, sc.Z, sc.PML, np.where(sc.src_mask), 4))
    src = sc.source[:1, :Ts]
    args0 = (sc.c_true ** 2, np.ones(3), dxp, dzp, sx[:1], sz[:1], src, mx, mz)
    obs = po.simulate(*args0, mode="f32")
    t0 = time.perf_counter()
    g64, rec64, _ = po.grad(sc.c_start ** 2, np.ones(3), dxp, dzp, sx[:1], sz[:1], src, mx, mz, rx, rz,
                            lambda s: mo.wasserstein_softplus(s, obs), mode="f64")
    dt = time.perf_counter() - t0
    v = 2 * sc.X * sc.Z * (Ts - 1) / dt / 1e9
    base = {"value": v, "unit": UNIT, "cores": po.num_threads(), "kind": "port",
            "sample": f"FP64 oracle (oracle/pml_oracle.c, OpenMP) + numpy softplus-W2 misfit: 1 shot, "
                      f"{sc.X}x{sc.Z}, first {Ts} of {sc.T} steps, forward + adjoint gradient, {dt:.1f} s"}
    return base, {"Ts": Ts, "obs": obs, "g64": g64, "rec64": rec64}


def err_vs_fp64(args, sc, sample):
    """The benched numerics (same kernel variant and tile, fast or faithful)
    on the baseline's sample -- shot 0, the first Ts steps, the same observed
    traces and misfit -- against the FP64 oracle's traces and gradient:
    max over receivers of max_t|d| / max_t|ref| and relative L2."""
    from otfwi_b200.batch import ShotBatch
    Ts = sample["Ts"]
    b = ShotBatch(sc.X, sc.Z, Ts, sc.PML, sc.src_mask, sc.rec_mask, np.ascontiguousarray(sc.source[:, :Ts]),
                  prec_deriv=4, precision=args.precision, tile=max(args.tile, 0), kernel=args.kernel,
                  shots=(np.array([0, 1]), np.array([0])))
    b.set_observed(sample["obs"][None])
    b.set_model(sc.c_start)
    sim = b.forward()[0]
    g, _ = b.gradient(args.misfit)
    b.close()
    ref, rg = np.asarray(sample["rec64"])[:, 1:], np.asarray(sample["g64"])
    den = np.abs(ref).max(axis=1)
    den[den == 0] = 1.0
    et = float((np.abs(sim[:, 1:] - ref).max(axis=1) / den).max())
    eg = float(np.linalg.norm(g - rg) / np.linalg.norm(rg))
    return {"trace_max_rel": et, "grad_rel_l2": eg,
            "sample": f"shot 0, first {Ts} steps, benched kernels vs FP64 oracle (oracle/pml_oracle.c)",
            "full_size_check": "tests/test_benchmark_configs_gpu.py (T = 4000, shots 0 and 63)"}


def run_ours(args):
    import torch
    import torch.distributed as dist
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    from otfwi_b200.batch import ShotBatch
    from otfwi_b200.distributed import allreduce_sum_, shard_block
    strong = args.mode == "strong"
    sc = workload(args, 0 if strong else rank)
    shots, n_local = None, sc.n_src
    if strong:
        # this rank's contiguous block of the acquisition's shots
        lo, hi = shard_block(sc.n_src, world, rank)
        if hi <= lo:
            raise SystemExit(f"rank {rank}: no shots left for it ({sc.n_src} shots over {world} ranks)")
        shots, n_local = (np.arange(hi - lo + 1), np.arange(lo, hi)), hi - lo
    tuned = None
    if args.tile < 0:
        from otfwi_b200.autotune import autotune, TILES
        k, t, table = autotune(sc, precision=args.precision, misfit=args.misfit)
        if world > 1:
            # every rank tunes (the GPUs stay in step); all run rank 0's choice
            from otfwi_b200.distributed import agree_ints
            k, t = agree_ints([k, t], device=torch.device("cuda", local))
        if args.kernel < 0:
            args.kernel = k
        args.tile = t
        tuned = {"kernel": k, "tile": list(TILES[t]), "candidates_ms_T300": table}
    b = ShotBatch(sc.X, sc.Z, sc.T, sc.PML, sc.src_mask, sc.rec_mask, sc.source, prec_deriv=4,
                  precision=args.precision, tile=args.tile, kernel=args.kernel, shots=shots)
    b.set_stream_rows(args.stream_rows)
    lanes = b.lanes()
    dev = torch.device("cuda", local)
    stream = torch.cuda.ExternalStream(b.stream(), device=dev)
    c_true = torch.tensor(sc.c_true, dtype=torch.float32, device=dev)
    c0 = torch.tensor(sc.c_start, dtype=torch.float32, device=dev)
    obs = torch.empty((n_local, sc.n_rec, sc.T), dtype=torch.float32, device=dev)
    b.set_model(cquad=(c_true * c_true).contiguous())
    b.forward(out=obs)
    b.set_observed(obs)
    b.set_model(cquad=(c0 * c0).contiguous())
    grad = torch.empty((sc.Z, sc.X), dtype=torch.float32, device=dev)
    mis = torch.empty(1, dtype=torch.float64, device=dev)

    def step():
        b.gradient(args.misfit, grad=grad, misfit_out=mis)
        if world > 1:
            # weak: the FWI gradient is the sum over every rank's acquisition;
            # strong: the shot mean of one acquisition (local means weighted
            # by their shot counts). One NCCL all-reduce of the X*Z gradient
            # and the misfit per step either way.
            with torch.cuda.stream(stream):
                if strong:
                    grad.mul_(n_local / sc.n_src)
                allreduce_sum_([grad, mis])

    for _ in range(args.warmup):
        step()
    b.sync()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    job_cells = 2 * sc.X * sc.Z * (sc.T - 1) * (sc.n_src if strong else sc.n_src * world)
    value = job_cells / (ms / 1e3) / 1e9

    # per-kernel live timing of the two step kernels (graphs of T-1 launches
    # each), for the roofline of the dominant kernel
    def time_graph(fn, reps=2):
        fn()
        b.sync()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(reps):
            fn()
        f1.record(stream)
        f1.synchronize()
        return f0.elapsed_time(f1) / reps / (sc.T - 1)

    ms_fwd = time_graph(lambda: b._lib.otf_batch_forward_ring(b._h, None, 0))
    b._lib.otf_batch_misfit(b._h, 2, None, 0)
    ms_rev = time_graph(lambda: b._lib.otf_batch_reverse(b._h, None, 0, None, 1.0, 0))
    peak, peak_kind = measured_peak()
    per_launch_cells = sc.X * sc.Z * n_local
    ach_rev = BYTES_REV * per_launch_cells / (ms_rev / 1e3) / 1e9
    ach_fwd = BYTES_FWD * per_launch_cells / (ms_fwd / 1e3) / 1e9
    tr = profile_traffic(args.kernel)
    if args.kernel == 6:
        rev_name = ("k_fused_rev (reverse step in one pass: adjoint + reconstruction + imaging "
                    "condition, all shots)")
    elif args.kernel == 5:
        rev_name = ("k_paired_rev (reverse step in one launch: adjoint + reconstruction + imaging "
                    "condition, all shots)")
    elif args.kernel == 4:
        rev_name = ("reverse step (k_unfused_p_rev + k_unfused_a_rev_sets: adjoint + reconstruction + "
                    "imaging condition, all shots; 92 B/cell moved)")
    else:
        rev_name = "k_reverse_split (adjoint + reconstruction + imaging condition, all shots)"
    roof = {"kernel": rev_name,
            "bound": "hbm", "achieved": round(ach_rev, 1), "peak": peak, "unit": "GB/s",
            "frac": round(ach_rev / peak, 4), "peak_kind": peak_kind,
            "traffic": (tr * per_launch_cells if tr else None),
            "algorithmic_bytes_per_launch": BYTES_REV * per_launch_cells,
            "launch_ms": round(ms_rev, 4),
            "forward_kernel": {"achieved": round(ach_fwd, 1), "frac": round(ach_fwd / peak, 4),
                               "launch_ms": round(ms_fwd, 4),
                               "algorithmic_bytes_per_launch": BYTES_FWD * per_launch_cells},
            "whole_step_frac": round(BYTES_STEP * sc.X * sc.Z * (sc.T - 1) * n_local
                                     / (ms / 1e3) / 1e9 / peak, 4)}
    share = profile_value(args.kernel, "a_rev_share_of_step") if args.kernel == 4 else None
    if share:
        # the largest single kernel of the unfused reverse step; its time is the
        # step's live CUDA-event time times its share of the step in the
        # committed launch list (a graph's kernels cannot be timed one by one)
        ms_a = ms_rev * share
        ach_a = BYTES_AREV * per_launch_cells / (ms_a / 1e3) / 1e9
        roof["dominant_kernel"] = {"name": "k_unfused_a_rev_sets", "algorithmic_bytes_per_launch":
                                   BYTES_AREV * per_launch_cells, "launch_ms_est": round(ms_a, 4),
                                   "share_of_step": share, "achieved": round(ach_a, 1),
                                   "frac": round(ach_a / peak, 4)}

    # end to end through the public API with host buffers: model and
    # observed traces from pinned host memory, gradient and misfit back
    h_cq = torch.tensor(sc.c_start.astype(np.float32) ** 2).pin_memory()
    h_obs = obs.cpu().pin_memory()
    h_grad = torch.empty((sc.Z, sc.X), dtype=torch.float32).pin_memory()
    h_mis = torch.empty(1, dtype=torch.float64).pin_memory()

    def e2e_step():
        b.set_model(cquad=h_cq.numpy())
        b.set_observed(h_obs.numpy())
        step()  # gradient on the device (and, with several ranks, its all-reduce)
        stream.synchronize()
        # blocking copies on torch's own stream: pinned buffers used on the
        # library's stream would be tracked by torch's host allocator, which
        # records events on that stream when they are freed -- after the
        # library has destroyed it
        h_grad.copy_(grad)
        h_mis.copy_(mis)

    for _ in range(max(1, args.warmup // 2)):
        e2e_step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    n_e2e = max(2, args.steps // 2)
    for _ in range(n_e2e):
        e2e_step()
    g1.record(stream)
    g1.synchronize()
    ms_e2e = g0.elapsed_time(g1) / n_e2e
    if world > 1:
        t = torch.tensor([ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e = {"value": job_cells / (ms_e2e / 1e3) / 1e9, "unit": UNIT,
           "h2d_bytes_per_step": int(h_cq.numel() * 4 + h_obs.numel() * 4),
           "d2h_bytes_per_step": int(h_grad.numel() * 4 + 8), "ms_per_step": round(ms_e2e, 3)}

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
                "higher_is_better": True, "scaling": args.mode, "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded model, Ricker source; no external dataset)",
                "config": config_block(args, sc, world),
                "tuning": {"kernel_variant": args.kernel, "tile": args.tile, "autotune": tuned,
                           "stream_rows": args.stream_rows if args.kernel == 3 else None},
                "roofline": roof, "e2e": e2e,
                # per time step one fused launch forward and one reverse (the
                # unfused variant 4: a P and an A launch in each, per shot
                # lane); per gradient the misfit, its sum, the running
                # integral, shot mean, and for variants 4 and 5 one check
                # kernel after each time loop (launch count, tickets)
                "gpu_launches": args.steps * ((4 * lanes if args.kernel == 4 else 2) * (sc.T - 1) + 4
                                              + (2 if args.kernel in (4, 5) else 0)),
                "clocks": clk.summary(),
                "misfit_value": float(mis.item())}
        if not args.no_cpu_baseline and world == 1:
            # the host-core baseline is one figure for the job, taken at N = 1
            # only (the other ranks would wait for it at the closing barrier)
            line["cpu_baseline"], sample = cpu_baseline(args, sc)
            line["err_vs_fp64"] = err_vs_fp64(args, sc, sample)
        print(json.dumps(line), flush=True)
    b.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args):
    """The reference's own CUDA library (oracle/_ref, compiled from
    regression_PML_single.cu) driven as cuda_interface_pml.py drives it: one
    cuda_grad_ext per shot with the host misfit callback (the reference's
    wasserstein recipe, restated in oracle/misfit_oracle.py). Runs in this
    process only; it must not share a CUDA context (the library resets the
    device on init). Each step is a bounded sample of the FMC workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import ctypes
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import misfit_oracle as mo
    from otfwi_b200.cuda_interface_pml import Cuda_interface_PML
    path = os.path.join(ROOT, "oracle", "_ref", "cuda_regression_PML_single.so")
    sc = workload(args)
    cfg = config_block(args, sc)
    if not os.path.exists(path):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref library not built"}))
        return
    cp = Cuda_interface_PML(sc.X, sc.Z, sc.T, sc.PML, sc.c_true, sc.n_src, sc.src_mask, sc.n_rec,
                            sc.rec_mask, sc.source, multishot=True, lib=path)
    ns = args.ref_shots
    obs = np.zeros((sc.n_src, sc.n_rec, sc.T), np.float32)
    buf = np.zeros((sc.n_rec, sc.T), np.float32)
    for s in range(ns):
        cp._lib.cuda_simulate(0, s)
        ctypes.memmove(buf.ctypes.data, cp.recptr[0], buf.nbytes)
        obs[s] = buf
    # the same trace misfit as this library's arm: the reference recipe
    # (adjoint_functions.wasserstein, restated) or, for the softplus variant
    # the reference lacks, its numpy definition -- a host callback either way,
    # as the reference wrapper runs its misfits
    host_misfit = {"wasserstein": mo.wasserstein, "wasserstein_softplus": mo.wasserstein_softplus,
                   "l2": mo.L2, "wasserstein_quad": mo.wasserstein_quad}[args.misfit]
    cp.init_regression(obs, host_misfit, prec_deriv=4)
    cp._set_c_quad(sc.c_start ** 2)

    def step():
        for s in range(ns):
            cp.idx_source = s
            mse = (ctypes.c_float * 1)(0.0)
            cp._lib.cuda_grad_ext(mse, cp.adj_wrapper_ptr, s)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    value = 2 * sc.X * sc.Z * (sc.T - 1) * ns / dt / 1e9
    sample = (f"reference CUDA library (regression_PML_single.cu built by oracle/Makefile) on the GPU, "
              f"per-shot cuda_grad_ext with the host {args.misfit} callback (numpy; the reference's "
              f"wrapper runs its misfits on the host): {ns} of {sc.n_src} shots per step")
    print(json.dumps({"metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": 1,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 2),
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                      "data": "synthetic", "config": cfg, "impl": "reference",
                      "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": 1,
                                       "kind": "reference", "sample": sample},
                      "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}), flush=True)


def cpml_case(args):
    """The CPML leg's workload: a 512x512 seeded model (scenarios.small's
    layered velocity with density 1-1.5), 8 sources firing together, 64
    receivers, T steps; the CPML profiles built by otfwi_b200.cpml."""
    from otfwi_b200 import scenarios
    sc = scenarios.small(X=args.X, Z=args.X, T=args.T, n_src=8, n_rec=64, seed=31, f0=0.02)
    rho = 1.0 + 0.5 * np.random.default_rng(31).random((sc.Z, sc.X))
    return sc, rho


def run_cpml_impl(args):
    """One library's CPML forward (and, for this library, its exact adjoint)
    timed in this process; prints a JSON fragment. The reference's library
    resets the device on init, so each library runs in its own process."""
    from otfwi_b200.cpml import CPML_LIB, CPMLSimulator
    sc, rho = cpml_case(args)
    lib = CPML_LIB if args.cpml_impl == "ours" else os.path.join(ROOT, "oracle", "_ref", "cuda_regression_CPML.so")
    if not os.path.exists(lib):
        print(json.dumps({"unavailable": f"{os.path.relpath(lib, ROOT)} not built"}))
        return
    sim = CPMLSimulator(sc.X, sc.Z, sc.T, sc.PML, sc.c_true, sc.src_mask, sc.rec_mask, sc.source, rho=rho,
                        f0=0.02, lib=lib)
    for _ in range(args.warmup):
        rec = sim.simulate(-1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rec = sim.simulate(-1)
    dt = (time.perf_counter() - t0) / args.steps
    out = {"forward_s": dt, "forward_gcell_steps_per_s": sc.X * sc.Z * (sc.T - 1) / dt / 1e9,
           "traces_max": float(np.abs(rec).max())}
    # every source fired alone: the reference loops cuda_simulate2 over the
    # sources; this library also has one batched call for all of them
    ns = int(sc.n_src)
    t0 = time.perf_counter()
    for s in range(ns):
        sim.simulate(s)
    dt = time.perf_counter() - t0
    out["per_source_loop_s"] = dt
    out["per_source_loop_gcell_steps_per_s"] = ns * sc.X * sc.Z * (sc.T - 1) / dt / 1e9
    if args.cpml_impl == "ours":
        sim.simulate_all()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            sim.simulate_all()
        dt = (time.perf_counter() - t0) / args.steps
        out["all_sources_batched_s"] = dt
        out["all_sources_batched_gcell_steps_per_s"] = ns * sc.X * sc.Z * (sc.T - 1) / dt / 1e9
        g = np.asarray(rec, np.float32) * 1e-3
        sim.gradient(g)
        t0 = time.perf_counter()
        sim.gradient(g)
        out["gradient_s"] = time.perf_counter() - t0
    print(json.dumps(out), flush=True)


def run_cpml_leg(args):
    """CPML path (regression_CPML.cu): this library's forward against the
    reference's own library on the same inputs, each through its C ABI and
    timed around cuda_simulate2 (traces copied back, as the ABI returns
    them); the exact adjoint of this library beside it (the reference has
    none)."""
    import subprocess
    res = {}
    for impl in ("ours", "reference"):
        cmd = [sys.executable, os.path.abspath(__file__), "--leg", "cpml", "--cpml-impl", impl, "--X",
               str(args.X), "--T", str(args.T), "--steps", str(args.steps), "--warmup", str(args.warmup)]
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=1800)
        lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
        res[impl] = json.loads(lines[-1]) if lines else {"unavailable": out.stderr.strip()[-300:]}
    ours = res["ours"].get("forward_gcell_steps_per_s")
    ref = res["reference"].get("forward_gcell_steps_per_s")
    print(json.dumps({"metric": "CPML forward Gcell-steps/s", "value": ours, "unit": "Gcell-steps/s",
                      "leg": "cpml", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                      "higher_is_better": True, "data": "synthetic",
                      "config": {"workload": f"cpml{args.X}x{args.X}_T{args.T}_8src_64rx"},
                      "reference_value": ref, "speedup": (ours / ref) if ours and ref else None,
                      "all_sources": {"ours_batched": res["ours"].get("all_sources_batched_gcell_steps_per_s"),
                                      "reference_loop": res["reference"].get("per_source_loop_gcell_steps_per_s")},
                      "ours": res["ours"], "reference": res["reference"]}), flush=True)


def run_misfit_leg(args):
    """Device trace misfits: every kind on the FMC workload's trace count
    (shots x receivers x T), timed with CUDA events, against the CPU
    restatement (oracle/misfit_oracle.py, the reference's numpy recipes)
    timed on a sample of traces."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import misfit_oracle as mo
    from otfwi_b200.batch import MISFITS, _declare
    from otfwi_b200 import _lib
    L = _declare(_lib.load())
    rng = np.random.default_rng(7)
    n, T = args.shots * args.shots, args.T
    t = np.arange(T)
    sim = np.zeros((n, T), np.float32)
    obs = np.zeros((n, T), np.float32)
    for i in range(n):
        t1 = rng.uniform(0.2, 0.6) * T
        a = (np.pi * 0.01 * (t - t1)) ** 2
        obs[i] = (1 - 2 * a) * np.exp(-a)
        a = (np.pi * 0.01 * (t - t1 - rng.normal(0, 3))) ** 2
        sim[i] = (1 - 2 * a) * np.exp(-a) + rng.normal(0, 1e-3, T)
    s = torch.as_tensor(sim).cuda()
    o = torch.as_tensor(obs).cuda()
    adj = torch.empty_like(s)
    mis = torch.empty(n, dtype=torch.float64, device="cuda")
    cpu = {"wasserstein": mo.wasserstein, "wasserstein_quad": mo.wasserstein_quad, "l2": mo.L2,
           "quad_envelope": mo.quad_envelope, "wasserstein_pm": mo.wasserstein_pm,
           "wasserstein_softplus": mo.wasserstein_softplus}
    out = {}
    for name, kind in MISFITS.items():
        nb = int(L.otf_misfit_scratch_bytes(kind, n, T))
        scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device="cuda")
        st = torch.cuda.current_stream()

        def call():
            rc = L.otf_misfit(kind, ctypes.c_void_p(s.data_ptr()), ctypes.c_void_p(o.data_ptr()),
                              ctypes.c_void_p(adj.data_ptr()), ctypes.c_void_p(mis.data_ptr()), n, T,
                              ctypes.c_void_p(scratch.data_ptr()), nb, ctypes.c_void_p(st.cuda_stream))
            if rc:
                _lib.check(L)
        for _ in range(args.warmup):
            call()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            call()
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        rec = {"ms": round(ms, 3), "traces_per_s": round(n / (ms / 1e3), 1)}
        if name in cpu:
            k = 16
            t0 = time.perf_counter()
            cpu[name](sim[:k].astype(np.float64), obs[:k])
            dt = time.perf_counter() - t0
            rec["cpu_traces_per_s"] = round(k / dt, 1)
            rec["speedup"] = round(rec["traces_per_s"] / rec["cpu_traces_per_s"], 1)
        out[name] = rec
    print(json.dumps({"metric": "device misfit traces/s", "leg": "misfits", "unit": "traces/s",
                      "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "data": "synthetic",
                      "config": {"workload": f"{n} traces x {T} samples"},
                      "cpu_baseline": {"kind": "port", "cores": 1,
                                       "sample": "oracle/misfit_oracle.py (the reference's numpy recipes), 16 traces"},
                      "kinds": out}), flush=True)


def main():
    args = parse()
    if args.leg == "cpml":
        run_cpml_impl(args) if args.cpml_impl else run_cpml_leg(args)
    elif args.leg == "misfits":
        run_misfit_leg(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
